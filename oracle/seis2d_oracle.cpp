// seis2d_oracle.cpp - CPU restatement of the reference 2-D P-SV solver (TEST INFRASTRUCTURE).
//
// Only the tests, the smoke check and the CPU-baseline leg of the benchmark use this file; it
// is the checker of the CUDA solver, never part of it.  It restates, in plain C++ loops, the
// update order of runGpuSimulationStep (CUDA_Kernels/Cuda_Check.cu:1027-1085):
//
//   stress (Type 1 :224-266 | Type 2 :315-365 | Type 3 :416-487) -> free-surface mirror
//   (:491-508) -> velocity (Type 1 :270-311 | Type 2 :368-412 | Type 3 :512-563) -> point or
//   multi source (:567-640, :822-834) -> outer-ring clear (:643-667)
//
// with receivers as extractReceiverSamplesKernel (:793-818).  Every loop reads the previous
// pass's arrays in place, which is what the race-free reference kernels compute.  The solver
// is templated on the arithmetic type: float (IEEE operations, no contraction: the build uses
// -ffp-contract=off) and double (the FP64 run of the same scheme: the FP32 inputs promoted).
#include "../include/seis2d_capi.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Base {
    virtual ~Base() = default;
    virtual void step(int it, const seis2d_context& c, int numActive, bool advance) = 0;
    virtual void field(int which, float* out) const = 0;
    virtual void setField(int which, const float* in) = 0;
    virtual void record(const int* idx, int n, float* vx, float* vz) const = 0;
    virtual void wavefield(float* vz) const = 0;
    std::vector<seis2d_source> sources;
    std::vector<char> dropped;
};

template <class T> struct Solver : Base {
    int NX, NZ, total, npml, fs, flag, up;
    T dt, inv_dt, c1, c2, c3, c4;
    std::vector<T> vx1, vx2, vz1, vz2, sxx1, sxx2, szz1, szz2, sxz1, sxz2;
    std::vector<T> vx, vz, sxx, szz, sxz;
    std::vector<T> rho, mu, lambda, l2m, muX, lambdaX, l2mX, muZ, rhoXZ, rhoOrig;
    std::vector<T> dx, dxh, dz, dzh, dp;

    static std::vector<T> promote(const seis2d_float_view& v, std::size_t n) {
        std::vector<T> out(n, T(0));
        for (std::size_t k = 0; k < n && k < std::size_t(v.size); ++k) out[k] = T(v.data[k]);
        return out;
    }

    explicit Solver(const seis2d_context& c) {
        NX = c.NX; NZ = c.NZ; total = c.total_grid; npml = c.npml; fs = c.npml; flag = c.flag_type; up = c.upFlag;
        dt = T(c.dt);
        // GPUSimData::inv_dt = 1.0f / ctx.dt (Cuda_Check.cu:893) in the solver's arithmetic.
        inv_dt = T(1) / T(c.dt);
        c1 = T(c.c1_h); c2 = T(c.c2_h); c3 = T(c.c3_h); c4 = T(c.c4_h);
        const std::size_t n = std::size_t(total);
        for (auto* a : {&vx1, &vx2, &vz1, &vz2, &sxx1, &sxx2, &szz1, &szz2, &sxz1, &sxz2}) a->assign(n, T(0));
        rho = promote(c.rho, n); mu = promote(c.mu, n); lambda = promote(c.lambda, n); l2m = promote(c.lambda2mu, n);
        dx = promote(c.dx, NX); dxh = promote(c.dx_half, NX); dz = promote(c.dz, NZ); dzh = promote(c.dz_half, NZ);
        if (flag == 3) dp = promote(c.dp_flat, NX);
        if (flag == 2) {
            for (auto* a : {&vx, &vz, &sxx, &szz, &sxz}) a->assign(n, T(0));
            for (auto* a : {&muX, &lambdaX, &l2mX, &muZ, &rhoXZ, &rhoOrig}) a->assign(n, T(0));
            // Staggered averages of initializeGpuSimulation (Cuda_Check.cu:922-939), in FP32 there;
            // computed from the same FP32 inputs here.
            for (int i = 0; i < NZ; ++i)
                for (int j = 0; j < NX; ++j) {
                    const std::size_t k = std::size_t(i) * NX + j;
                    const std::size_t kx = j < NX - 1 ? k + 1 : k, kz = i < NZ - 1 ? k + NX : k;
                    const std::size_t kd = (i < NZ - 1 && j < NX - 1) ? k + NX + 1 : k;
                    const float* m = c.mu.data;
                    const float* la = c.lambda.data;
                    const float* lm = c.lambda2mu.data;
                    const float* r = c.rho.data;
                    rhoOrig[k] = T(r[k]);
                    muX[k] = T(0.5f * (m[k] + m[kx]));
                    lambdaX[k] = T(0.5f * (la[k] + la[kx]));
                    l2mX[k] = T(0.5f * (lm[k] + lm[kx]));
                    muZ[k] = T(0.5f * (m[k] + m[kz]));
                    rhoXZ[k] = T(0.25f * (r[k] + r[kx] + r[kz] + r[kd]));
                }
        }
        sources.assign(SEIS2D_MAX_ACTIVE_SOURCES, seis2d_source{});
        dropped.assign(SEIS2D_MAX_ACTIVE_SOURCES, 0);
    }

    // Split and total derivative taps in the reference's operand order.
    static T tap(const T* a, const T* b, std::size_t u, std::size_t l) { return a[u] + b[u] - a[l] - b[l]; }
    T sum4(T t1, T t2, T t3, T t4) const { return c1 * t1 + c2 * t2 + c3 * t3 + c4 * t4; }

    T dxF(const T* a, const T* b, std::size_t k) const {
        return sum4(tap(a, b, k + 1, k), tap(a, b, k + 2, k - 1), tap(a, b, k + 3, k - 2), tap(a, b, k + 4, k - 3));
    }
    T dxB(const T* a, const T* b, std::size_t k) const {
        return sum4(tap(a, b, k, k - 1), tap(a, b, k + 1, k - 2), tap(a, b, k + 2, k - 3), tap(a, b, k + 3, k - 4));
    }
    T dzF(const T* a, const T* b, std::size_t k) const {
        const std::size_t w = NX;
        return sum4(tap(a, b, k + w, k), tap(a, b, k + 2 * w, k - w), tap(a, b, k + 3 * w, k - 2 * w),
                    tap(a, b, k + 4 * w, k - 3 * w));
    }
    T dzB(const T* a, const T* b, std::size_t k) const {
        const std::size_t w = NX;
        return sum4(tap(a, b, k, k - w), tap(a, b, k + w, k - 2 * w), tap(a, b, k + 2 * w, k - 3 * w),
                    tap(a, b, k + 3 * w, k - 4 * w));
    }
    T dxF(const T* a, std::size_t k) const { return sum4(a[k + 1] - a[k], a[k + 2] - a[k - 1], a[k + 3] - a[k - 2], a[k + 4] - a[k - 3]); }
    T dxB(const T* a, std::size_t k) const { return sum4(a[k] - a[k - 1], a[k + 1] - a[k - 2], a[k + 2] - a[k - 3], a[k + 3] - a[k - 4]); }
    T dzF(const T* a, std::size_t k) const {
        const std::size_t w = NX;
        return sum4(a[k + w] - a[k], a[k + 2 * w] - a[k - w], a[k + 3 * w] - a[k - 2 * w], a[k + 4 * w] - a[k - 3 * w]);
    }
    T dzB(const T* a, std::size_t k) const {
        const std::size_t w = NX;
        return sum4(a[k] - a[k - w], a[k + w] - a[k - 2 * w], a[k + 2 * w] - a[k - 3 * w], a[k + 3 * w] - a[k - 4 * w]);
    }

    bool typeOne() const { return flag == 1 || (flag == 3 && !up); }

    // Type 1 stress (Cuda_Check.cu:224-266).
    void stress1() {
#pragma omp parallel for schedule(static)
        for (int i = 4; i < NZ - 4; ++i)
            for (int j = 4; j < NX - 4; ++j) {
                const std::size_t k = std::size_t(i) * NX + j;
                const T d_z = dz[i], d_z_h = dzh[i], d_x = dx[j], d_x_h = dxh[j];
                const T dvx_dx = dxF(vx1.data(), vx2.data(), k);
                const T dvz_dz = dzB(vz1.data(), vz2.data(), k);
                sxx1[k] = (sxx1[k] * (inv_dt - d_x_h) + T(0.5) * (l2m[k] + l2m[k + 1]) * dvx_dx) / (inv_dt + d_x_h);
                sxx2[k] = (sxx2[k] * (inv_dt - d_z) + T(0.5) * (lambda[k] + lambda[k + 1]) * dvz_dz) / (inv_dt + d_z);
                szz1[k] = (szz1[k] * (inv_dt - d_x_h) + T(0.5) * (lambda[k] + lambda[k + 1]) * dvx_dx) / (inv_dt + d_x_h);
                szz2[k] = (szz2[k] * (inv_dt - d_z) + T(0.5) * (l2m[k] + l2m[k + 1]) * dvz_dz) / (inv_dt + d_z);
                const T dvz_dx = dxB(vz1.data(), vz2.data(), k);
                const T dvx_dz = dzF(vx1.data(), vx2.data(), k);
                sxz1[k] = (sxz1[k] * (inv_dt - d_x) + T(0.5) * (mu[k] + mu[k + NX]) * dvz_dx) / (inv_dt + d_x);
                sxz2[k] = (sxz2[k] * (inv_dt - d_z_h) + T(0.5) * (mu[k] + mu[k + NX]) * dvx_dz) / (inv_dt + d_z_h);
            }
    }

    // Type 1 velocity (Cuda_Check.cu:270-311).
    void velocity1() {
#pragma omp parallel for schedule(static)
        for (int i = 4; i < NZ - 4; ++i)
            for (int j = 4; j < NX - 4; ++j) {
                const std::size_t k = std::size_t(i) * NX + j;
                const T d_z = dz[i], d_z_h = dzh[i], d_x = dx[j], d_x_h = dxh[j];
                const T cur_rho = rho[k];
                const T dsigxx_dx = dxB(sxx1.data(), sxx2.data(), k);
                const T dsigxz_dz = dzB(sxz1.data(), sxz2.data(), k);
                vx1[k] = (vx1[k] * (inv_dt - d_x) + dsigxx_dx / cur_rho) / (inv_dt + d_x);
                vx2[k] = (vx2[k] * (inv_dt - d_z) + dsigxz_dz / cur_rho) / (inv_dt + d_z);
                const T dsigxz_dx = dxF(sxz1.data(), sxz2.data(), k);
                const T dsigzz_dz = dzF(szz1.data(), szz2.data(), k);
                const T rho_avg = T(0.25) * (rho[k] + rho[k + 1] + rho[k + NX] + rho[k + NX + 1]);
                vz1[k] = (vz1[k] * (inv_dt - d_x_h) + dsigxz_dx / rho_avg) / (inv_dt + d_x_h);
                vz2[k] = (vz2[k] * (inv_dt - d_z_h) + dsigzz_dz / rho_avg) / (inv_dt + d_z_h);
            }
    }

    bool pml(int i, int j) const { return i < npml || i >= NZ - npml || j < npml || j >= NX - npml; }

    // Type 2 stress (Cuda_Check.cu:315-365).
    void stress2() {
#pragma omp parallel for schedule(static)
        for (int i = 4; i < NZ - 4; ++i)
            for (int j = 4; j < NX - 4; ++j) {
                const std::size_t k = std::size_t(i) * NX + j;
                const T dvz_dx = dxB(vz.data(), k), dvx_dz = dzF(vx.data(), k);
                const T dvx_dx = dxF(vx.data(), k), dvz_dz = dzB(vz.data(), k);
                if (!pml(i, j)) {
                    sxz[k] += dt * muZ[k] * (dvz_dx + dvx_dz);
                    sxx[k] += dt * (l2mX[k] * dvx_dx + lambdaX[k] * dvz_dz);
                    szz[k] += dt * (lambdaX[k] * dvx_dx + l2mX[k] * dvz_dz);
                } else {
                    const T d_z = dz[i], d_z_h = dzh[i], d_x = dx[j], d_x_h = dxh[j];
                    sxz1[k] = (sxz1[k] * (inv_dt - d_x) + muZ[k] * dvz_dx) / (inv_dt + d_x);
                    sxz2[k] = (sxz2[k] * (inv_dt - d_z_h) + muZ[k] * dvx_dz) / (inv_dt + d_z_h);
                    sxx1[k] = (sxx1[k] * (inv_dt - d_x_h) + l2mX[k] * dvx_dx) / (inv_dt + d_x_h);
                    szz1[k] = (szz1[k] * (inv_dt - d_x_h) + lambdaX[k] * dvx_dx) / (inv_dt + d_x_h);
                    sxx2[k] = (sxx2[k] * (inv_dt - d_z) + lambdaX[k] * dvz_dz) / (inv_dt + d_z);
                    szz2[k] = (szz2[k] * (inv_dt - d_z) + l2mX[k] * dvz_dz) / (inv_dt + d_z);
                    sxz[k] = sxz1[k] + sxz2[k];
                    sxx[k] = sxx1[k] + sxx2[k];
                    szz[k] = szz1[k] + szz2[k];
                }
            }
    }

    // Type 2 velocity (Cuda_Check.cu:368-412).
    void velocity2() {
#pragma omp parallel for schedule(static)
        for (int i = 4; i < NZ - 4; ++i)
            for (int j = 4; j < NX - 4; ++j) {
                const std::size_t k = std::size_t(i) * NX + j;
                const T dsigxz_dx = dxF(sxz.data(), k), dsigzz_dz = dzF(szz.data(), k);
                const T dsigxx_dx = dxB(sxx.data(), k), dsigxz_dz = dzB(sxz.data(), k);
                if (!pml(i, j)) {
                    vz[k] += dt * (dsigxz_dx + dsigzz_dz) / rhoXZ[k];
                    vx[k] += dt * (dsigxx_dx + dsigxz_dz) / rhoOrig[k];
                } else {
                    const T d_z = dz[i], d_z_h = dzh[i], d_x = dx[j], d_x_h = dxh[j];
                    vz1[k] = (vz1[k] * (inv_dt - d_x_h) + dsigxz_dx / rhoXZ[k]) / (inv_dt + d_x_h);
                    vz2[k] = (vz2[k] * (inv_dt - d_z_h) + dsigzz_dz / rhoXZ[k]) / (inv_dt + d_z_h);
                    vx1[k] = (vx1[k] * (inv_dt - d_x) + dsigxx_dx / rhoOrig[k]) / (inv_dt + d_x);
                    vx2[k] = (vx2[k] * (inv_dt - d_z) + dsigxz_dz / rhoOrig[k]) / (inv_dt + d_z);
                    vx[k] = vx1[k] + vx2[k];
                    vz[k] = vz1[k] + vz2[k];
                }
            }
    }

    // Type 3 stress (Cuda_Check.cu:416-487) followed by the mirror (:491-508).
    void stress3() {
#pragma omp parallel for schedule(static)
        for (int i = fs; i < NZ - 4; ++i)
            for (int j = 4; j < NX - 4; ++j) {
                const std::size_t k = std::size_t(i) * NX + j;
                const bool nearSurface = i <= fs + 5;
                const T d_z = nearSurface ? T(0) : dz[i], d_z_h = nearSurface ? T(0) : dzh[i];
                const T d_x = dx[j], d_x_h = dxh[j];
                const T muAvg = T(0.5) * (mu[k] + mu[k + NX]);
                if (i == fs) {
                    szz1[k] = T(0); szz2[k] = T(0);
                    const T dvx_dx = dxF(vx1.data(), vx2.data(), k);
                    sxx1[k] = (sxx1[k] * (inv_dt - d_x_h) + dp[j] * dvx_dx) / (inv_dt + d_x_h);
                    sxx2[k] = T(0);
                    const T dvz_dx = c1 * tap(vz1.data(), vz2.data(), k, k - 1) + c2 * tap(vz1.data(), vz2.data(), k + 1, k - 2);
                    const T dvx_dz = c1 * tap(vx1.data(), vx2.data(), k + NX, k) +
                                     c2 * tap(vx1.data(), vx2.data(), k + 2 * NX, k - NX);
                    sxz1[k] = (sxz1[k] * (inv_dt - d_x) + muAvg * dvz_dx) / (inv_dt + d_x);
                    sxz2[k] = (sxz2[k] * (inv_dt - d_z_h) + muAvg * dvx_dz) / (inv_dt + d_z_h);
                } else {
                    const T dvx_dx = dxF(vx1.data(), vx2.data(), k);
                    const T dvz_dz = dzB(vz1.data(), vz2.data(), k);
                    sxx1[k] = (sxx1[k] * (inv_dt - d_x_h) + T(0.5) * (l2m[k] + l2m[k + 1]) * dvx_dx) / (inv_dt + d_x_h);
                    sxx2[k] = (sxx2[k] * (inv_dt - d_z) + T(0.5) * (lambda[k] + lambda[k + 1]) * dvz_dz) / (inv_dt + d_z);
                    szz1[k] = (szz1[k] * (inv_dt - d_x_h) + T(0.5) * (lambda[k] + lambda[k + 1]) * dvx_dx) / (inv_dt + d_x_h);
                    szz2[k] = (szz2[k] * (inv_dt - d_z) + T(0.5) * (l2m[k] + l2m[k + 1]) * dvz_dz) / (inv_dt + d_z);
                    const T dvz_dx = dxB(vz1.data(), vz2.data(), k);
                    const T dvx_dz = dzF(vx1.data(), vx2.data(), k);
                    sxz1[k] = (sxz1[k] * (inv_dt - d_x) + muAvg * dvz_dx) / (inv_dt + d_x);
                    sxz2[k] = (sxz2[k] * (inv_dt - d_z_h) + muAvg * dvx_dz) / (inv_dt + d_z_h);
                }
            }
        for (int j = 4; j < NX - 4; ++j)
            for (int l = 1; l <= 4; ++l) {
                const long above = long(fs - l) * NX + j, below = long(fs + l) * NX + j;
                if (above >= 0 && below < total) {
                    szz1[above] = -szz1[below];
                    szz2[above] = -szz2[below];
                    const long belowShear = long(fs + l - 1) * NX + j;
                    sxz1[above] = -sxz1[belowShear];
                    sxz2[above] = -sxz2[belowShear];
                }
            }
    }

    // Type 3 velocity (Cuda_Check.cu:512-563).
    void velocity3() {
#pragma omp parallel for schedule(static)
        for (int i = 4; i < NZ - 4; ++i)
            for (int j = 4; j < NX - 4; ++j) {
                const std::size_t k = std::size_t(i) * NX + j;
                if (i < fs) {
                    vx1[k] = vx2[k] = vz1[k] = vz2[k] = T(0);
                    continue;
                }
                const bool nearSurface = i <= fs + 5;
                const T d_z = nearSurface ? T(0) : dz[i], d_z_h = nearSurface ? T(0) : dzh[i];
                const T d_x = dx[j], d_x_h = dxh[j];
                const T cur_rho = rho[k];
                const T dsigxx_dx = dxB(sxx1.data(), sxx2.data(), k);
                const T dsigxz_dz = dzB(sxz1.data(), sxz2.data(), k);
                vx1[k] = (vx1[k] * (inv_dt - d_x) + dsigxx_dx / cur_rho) / (inv_dt + d_x);
                vx2[k] = (vx2[k] * (inv_dt - d_z) + dsigxz_dz / cur_rho) / (inv_dt + d_z);
                const T dsigxz_dx = dxF(sxz1.data(), sxz2.data(), k);
                const T dsigzz_dz = dzF(szz1.data(), szz2.data(), k);
                const T rho_avg = T(0.25) * (rho[k] + rho[k + 1] + rho[k + NX] + rho[k + NX + 1]);
                vz1[k] = (vz1[k] * (inv_dt - d_x_h) + dsigxz_dx / rho_avg) / (inv_dt + d_x_h);
                vz2[k] = (vz2[k] * (inv_dt - d_z_h) + dsigzz_dz / rho_avg) / (inv_dt + d_z_h);
            }
    }

    // applyPointSource (Cuda_Check.cu:567-634).
    void applySource(T w, long idx, int type, float angle) {
        if (idx < 0 || idx >= total || !std::isfinite(double(w))) return;
        const int x = int(idx % NX), z = int(idx / NX);
        if (x < 4 || x >= NX - 4 || z < 4 || z >= NZ - 4 || (flag == 3 && up && z <= fs)) return;
        const std::size_t k = std::size_t(idx);
        const bool split = flag == 1 || flag == 3;
        const T sinA = T(std::sin(float(double(angle) * kPi / 180.0f)));
        const T cosA = T(std::cos(float(double(angle) * kPi / 180.0f)));
        if (type == SEIS2D_VERTICAL_FORCE || type == SEIS2D_ROTATED_FORCE) {
            const T fz = type == SEIS2D_ROTATED_FORCE ? cosA * w : w;
            if (split) {
                const T rho_avg = T(0.25) * (rho[k] + rho[k + 1] + rho[k + NX] + rho[k + NX + 1]);
                vz1[k] += fz * dt / rho_avg;
            } else {
                vz[k] += fz * dt / rhoXZ[k];
            }
        }
        if (type == SEIS2D_HORIZONTAL_FORCE || type == SEIS2D_ROTATED_FORCE) {
            const T fx = type == SEIS2D_ROTATED_FORCE ? sinA * w : w;
            if (split) vx1[k] += fx * dt / rho[k];
            else vx[k] += fx * dt / rhoOrig[k];
        }
        if (type == SEIS2D_EXPLOSIVE) {
            if (split) { sxx1[k] += w * T(0.5); sxx2[k] += w * T(0.5); szz1[k] += w * T(0.5); szz2[k] += w * T(0.5); }
            else { sxx[k] += w; szz[k] += w; }
        } else if (type == SEIS2D_SHEAR) {
            if (split) { sxz1[k] += w * T(0.5); sxz2[k] += w * T(0.5); }
            else sxz[k] += w;
        }
    }

    void zeroRing() {
        const bool split = flag == 1 || flag == 3;
        auto clear = [&](std::size_t k) {
            if (split) vx1[k] = vx2[k] = vz1[k] = vz2[k] = T(0);
            else vx[k] = vz[k] = T(0);
        };
        for (int j = 0; j < NX; ++j) { clear(std::size_t(j)); clear(std::size_t(NZ - 1) * NX + j); }
        for (int i = 0; i < NZ; ++i) { clear(std::size_t(i) * NX); clear(std::size_t(i) * NX + NX - 1); }
    }

    void step(int it, const seis2d_context& c, int numActive, bool advance) override {
        if (typeOne()) stress1();
        else if (flag == 2) stress2();
        else stress3();
        if (typeOne()) velocity1();
        else if (flag == 2) velocity2();
        else velocity3();
        if (numActive >= 0) {
            // injectMultipleSourcesKernel (Cuda_Check.cu:822-834); with `advance`, the host loop
            // of src/Seis2D/Workflow2D.inc:300-312 first moves each source by dt and drops the
            // ones past 2.5 / f_peak.
            for (int r = 0; r < numActive; ++r) {
                seis2d_source& s = sources[r];
                if (advance) {
                    if (dropped[r]) continue;
                    s.t = s.t + c.dt;
                    if (s.t > 2.5f * (1.0f / s.f_peak)) { dropped[r] = 1; continue; }
                }
                if (!std::isfinite(s.f_peak) || s.f_peak <= 0.0f || !std::isfinite(s.t)) continue;
                T val;
                if (sizeof(T) == sizeof(float)) {
                    const float t_peak = 1.0f / s.f_peak;
                    const float x = kPi * s.f_peak * (s.t - t_peak);
                    val = T(s.amp * (1.0f - 2.0f * x * x) * std::exp(-x * x));
                } else {
                    const double t_peak = 1.0 / double(s.f_peak);
                    const double x = kPi * double(s.f_peak) * (double(s.t) - t_peak);
                    val = T(double(s.amp) * (1.0 - 2.0 * x * x) * std::exp(-x * x));
                }
                applySource(val * T(SEIS2D_SOURCE_INJECTION_SCALE), s.idx, c.src_type, c.src_angle);
            }
        } else if (it < c.nt && it < c.wavelet.size) {
            // runGpuSimulationStep single source (Cuda_Check.cu:1068-1078).
            T w;
            if (sizeof(T) == sizeof(float)) w = T(c.wavelet.data[it] * c.src_amp * SEIS2D_SOURCE_INJECTION_SCALE);
            else w = T(c.wavelet.data[it]) * T(c.src_amp) * T(SEIS2D_SOURCE_INJECTION_SCALE);
            const long z = (flag == 3 && up) ? std::max(c.src_z_idx, fs + 1) : c.src_z_idx;
            const long idx = z * NX + (c.src_idx % NX);
            applySource(w, idx, c.src_type, c.src_angle);
        }
        zeroRing();
    }

    std::vector<T>* fieldVector(int which) {
        std::vector<T>* table[SEIS2D_FIELD_COUNT] = {&vx1, &vx2, &vz1, &vz2, &sxx1, &sxx2, &szz1, &szz2, &sxz1, &sxz2,
                                                     &vx, &vz, &sxx, &szz, &sxz, &rho, &mu, &lambda, &l2m,
                                                     &muX, &lambdaX, &l2mX, &muZ, &rhoXZ, &rhoOrig};
        return which >= 0 && which < SEIS2D_FIELD_COUNT ? table[which] : nullptr;
    }
    void field(int which, float* out) const override {
        auto* v = const_cast<Solver*>(this)->fieldVector(which);
        for (std::size_t k = 0; v && k < v->size(); ++k) out[k] = float((*v)[k]);
    }
    void setField(int which, const float* in) override {
        auto* v = fieldVector(which);
        for (std::size_t k = 0; v && k < v->size(); ++k) (*v)[k] = T(in[k]);
    }
    void record(const int* idx, int n, float* outVx, float* outVz) const override {
        const bool split = flag == 1 || flag == 3;
        for (int r = 0; r < n; ++r) {
            const int k = idx[r];
            if (k < 0 || k >= total) { outVx[r] = outVz[r] = 0.0f; continue; }
            outVx[r] = float(split ? vx1[k] + vx2[k] : vx[k]);
            outVz[r] = float(split ? vz1[k] + vz2[k] : vz[k]);
        }
    }
    void wavefield(float* out) const override {
        const bool split = flag == 1 || flag == 3;
        for (int k = 0; k < total; ++k) out[k] = float(split ? vz1[k] + vz2[k] : vz[k]);
    }
};

}  // namespace

extern "C" {

void* oracle2d_create(const seis2d_context* c, int precision) {
    if (!c) return nullptr;
    if (precision == 64) return new Solver<double>(*c);
    return new Solver<float>(*c);
}

void oracle2d_destroy(void* h) { delete static_cast<Base*>(h); }

void oracle2d_set_sources(void* h, const seis2d_source* sources, int count) {
    auto* b = static_cast<Base*>(h);
    for (int r = 0; r < count && r < SEIS2D_MAX_ACTIVE_SOURCES; ++r) {
        b->sources[r] = sources[r];
        b->dropped[r] = 0;
    }
}

void oracle2d_get_sources(void* h, seis2d_source* sources, int count) {
    auto* b = static_cast<Base*>(h);
    for (int r = 0; r < count && r < SEIS2D_MAX_ACTIVE_SOURCES; ++r) sources[r] = b->sources[r];
}

// Steps first..first+count-1; when rec_vx is given, records [r][count] after every step.
void oracle2d_run(void* h, int first, int count, const seis2d_context* c, int numActive, int advance, const int* rcv,
                  int nrcv, float* rec_vx, float* rec_vz) {
    auto* b = static_cast<Base*>(h);
    std::vector<float> vx(std::max(nrcv, 0)), vz(std::max(nrcv, 0));
    for (int q = 0; q < count; ++q) {
        b->step(first + q, *c, numActive, advance != 0);
        if (rec_vx && nrcv > 0) {
            b->record(rcv, nrcv, vx.data(), vz.data());
            for (int r = 0; r < nrcv; ++r) {
                rec_vx[std::size_t(r) * count + q] = vx[r];
                rec_vz[std::size_t(r) * count + q] = vz[r];
            }
        }
    }
}

void oracle2d_field(void* h, int which, float* out) { static_cast<Base*>(h)->field(which, out); }
void oracle2d_set_field(void* h, int which, const float* in) { static_cast<Base*>(h)->setField(which, in); }
void oracle2d_record(void* h, const int* idx, int n, float* vx, float* vz) { static_cast<Base*>(h)->record(idx, n, vx, vz); }
void oracle2d_wavefield(void* h, float* vz) { static_cast<Base*>(h)->wavefield(vz); }

}  // extern "C"
