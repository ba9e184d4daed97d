// seis3d_kernels.cuh - sm_100a kernels of the 3-D elastic velocity-stress solver.
//
// The time step is two z-marching passes (velocity, then stress).  Each CTA owns a
// 32 x TY column tile of the xy plane and walks a chunk of z planes:
//   * z derivatives come from per-thread register rings of 8 planes (no re-reads);
//   * x/y derivatives come from shared-memory plane tiles with 4-cell halos, filled
//     with coalesced row loads (rows are 128-byte aligned, see seis3d_device.cuh);
//   * the CPML recurrences run only for threads inside a slab and touch psi with
//     unit stride along x on every axis;
//   * the Ricker source is injected by the threads that own its 27 nodes, inside the
//     pass that the reference follows with sourceKernel3D (force: velocity pass,
//     explosion: stress pass);
//   * the non-finite check is reduced per warp to one atomic.
// Arithmetic per node follows the reference expression by expression so that FP32
// results agree to rounding (cuda/Cuda_Seis3D.cu:78-111, :222-245, :275-310, :313-332).
#pragma once

#include "seis3d_device.cuh"

namespace seis3d {

// Eighth-order staggered weights (cuda/Cuda_Seis3D.cu:72-75).
#define SEIS3D_W0 (1225.0f / 1024.0f)
#define SEIS3D_W1 (-245.0f / 3072.0f)
#define SEIS3D_W2 (49.0f / 5120.0f)
#define SEIS3D_W3 (-5.0f / 7168.0f)

// First derivative from an 8-sample window s[0..7]: for D- the window starts at i-4,
// for D+ at i-3; both reduce to sum_r w_r (s[4+r] - s[3-r]) accumulated r = 0..3, then
// scaled by 1/h (cuda/Cuda_Seis3D.cu:78-89).
__device__ __forceinline__ float diff8(float s0, float s1, float s2, float s3, float s4, float s5, float s6,
                                       float s7, float inv) {
    float r = 0.0f;
    r += SEIS3D_W0 * (s4 - s3);
    r += SEIS3D_W1 * (s5 - s2);
    r += SEIS3D_W2 * (s6 - s1);
    r += SEIS3D_W3 * (s7 - s0);
    return r * inv;
}

__device__ __forceinline__ float diffRing(const float (&s)[8], float inv) {
    return diff8(s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], inv);
}

// Row window of a shared tile (x derivative).
template <int W> __device__ __forceinline__ float diffRow(const float* row, float inv) {
    return diff8(row[0], row[1], row[2], row[3], row[4], row[5], row[6], row[7], inv);
}

// Column window of a shared tile (y derivative), `W` = row length.
template <int W> __device__ __forceinline__ float diffCol(const float* col, float inv) {
    return diff8(col[0], col[W], col[2 * W], col[3 * W], col[4 * W], col[5 * W], col[6 * W], col[7 * W], inv);
}

// One CPML memory update: psi = b psi + a d; returns d/kappa + psi (cuda/Cuda_Seis3D.cu:109-110).
__device__ __forceinline__ float cpmlUpdate(float d, float* psi, float a, float b, float ik) {
    float m = *psi;
    m = b * m + a * d;
    *psi = m;
    return ik * d + m;
}

// Slab index along one axis or -1 outside the slab (cuda/Cuda_Seis3D.cu:97-102).
__device__ __forceinline__ int slabIndex(int coord, int n, int pml, bool topFree) {
    if (!topFree && coord < kRadius + pml) return coord - kRadius;
    if (coord >= n - kRadius - pml) return (topFree ? 0 : pml) + coord - (n - kRadius - pml);
    return -1;
}

// Ricker amplitude of the 3x3x3 source at node offset (dx,dy,dz) and time t
// (cuda/Cuda_Seis3D.cu:319-322): FP64 phase, FP32 spatial weight.
__device__ __forceinline__ float sourceValue(const Geometry& G, const SourceParams& S, int dx, int dy, int dz,
                                             double time) {
    const double phase = 3.141592653589793 * G.frequency * (time - 1.2 / G.frequency);
    const float ricker = float((1 - 2 * phase * phase) * exp(-phase * phase));
    const float norm = 10.8387785335f;  // (1 + 2 exp(-1/2))^3
    return G.dt * S.amplitude * ricker * expf(-0.5f * float(dx * dx + dy * dy + dz * dz)) / norm;
}

__device__ __forceinline__ void flagNonFinite(const Fields& F, bool bad) {
    const unsigned any = __ballot_sync(0xffffffffu, bad);
    if (any && (threadIdx.x & 31) == 0) atomicExch(F.status, 1u);
}

// ---------------------------------------------------------------------------------------
// Velocity pass: v(n+1/2) = v(n-1/2) + dt * 2ab/(a+b) * sum_axis CPML(D sigma)
// (cuda/Cuda_Seis3D.cu:222-245) with the force source fused (:313-332).
// ---------------------------------------------------------------------------------------
template <int TY>
__global__ void __launch_bounds__(32 * TY) velocityPass(Geometry G, Fields F, SourceParams S, int zChunk) {
    constexpr int TX = 32, HX = TX + 8, HY = TY + 8;
    __shared__ float sXX[TY][HX];      // sigma_xx, x halo
    __shared__ float sXY[HY][HX];      // sigma_xy, x and y halo
    __shared__ float sXZ[TY][HX];      // sigma_xz, x halo
    __shared__ float sYY[HY][TX];      // sigma_yy, y halo
    __shared__ float sYZ[HY][TX];      // sigma_yz, y halo
    __shared__ float sB[TY + 1][TX + 1];  // 1/rho with +1 halo

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int x0 = kRadius + blockIdx.x * TX, y0 = kRadius + blockIdx.y * TY;
    const int x = x0 + tx, y = y0 + ty;
    const bool active = x < G.gx - kRadius && y < G.gy - kRadius;
    const int zBegin = kRadius + blockIdx.z * zChunk;
    const int zEnd = min(zBegin + zChunk, G.gz - kRadius);
    if (zBegin >= zEnd) return;
    const int64_t P = G.pitch, PL = G.plane;
    const int64_t col = int64_t(min(y, G.gy - 1)) * P + min(x, G.gx - 1);
    const float inv = G.invH;

    // CPML slab membership: x and y are fixed per thread, z per plane.
    const bool cp = !G.reflecting;
    const int qx = cp ? slabIndex(x, G.gx, G.pml, false) : -1;
    const int qy = cp ? slabIndex(y, G.gy, G.pml, false) : -1;
    float kx[6] = {0, 0, 0, 0, 0, 0}, ky[6] = {0, 0, 0, 0, 0, 0};
    if (qx >= 0 && active)
        for (int h = 0; h < 2; ++h)
            for (int j = 0; j < 3; ++j) kx[3 * h + j] = F.coef[0][(int64_t(h) * G.gx + x) * 3 + j];
    if (qy >= 0 && active)
        for (int h = 0; h < 2; ++h)
            for (int j = 0; j < 3; ++j) ky[3 * h + j] = F.coef[1][(int64_t(h) * G.gy + y) * 3 + j];

    float* const vx = F.f[0];
    float* const vy = F.f[1];
    float* const vz = F.f[2];
    const float* const gXX = F.f[3];
    const float* const gYY = F.f[4];
    const float* const gZZ = F.f[5];
    const float* const gXY = F.f[6];
    const float* const gYZ = F.f[7];
    const float* const gXZ = F.f[8];

    // z rings: rXZ/rYZ hold planes z-4..z+3 (D-), rZZ planes z-3..z+4 (D+).
    float rXZ[8], rYZ[8], rZZ[8];
    if (active) {
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            rXZ[k] = gXZ[int64_t(zBegin - 4 + k) * PL + col];
            rYZ[k] = gYZ[int64_t(zBegin - 4 + k) * PL + col];
            rZZ[k] = gZZ[int64_t(zBegin - 3 + k) * PL + col];
        }
    }
    const unsigned long long step = F.clock->step;
    const bool forceHere = S.kind == 1 && active && abs(x - S.gxs) <= 1 && abs(y - S.gys) <= 1;
    bool bad = false;

    for (int z = zBegin; z < zEnd; ++z) {
        const int64_t base = int64_t(z) * PL;
        if (active) {
            rXZ[7] = gXZ[base + 3 * PL + col];
            rYZ[7] = gYZ[base + 3 * PL + col];
            rZZ[7] = gZZ[base + 4 * PL + col];
        }
        __syncthreads();
        // Plane tiles with halos.
        for (int e = tid; e < TY * HX; e += TX * TY) {
            const int r = e / HX, c = e - r * HX;
            const int gxc = x0 - 4 + c, gyc = y0 + r;
            const bool in = gxc < G.gx && gyc < G.gy;
            const int64_t o = base + int64_t(gyc) * P + gxc;
            sXX[r][c] = in ? gXX[o] : 0.0f;
            sXZ[r][c] = in ? gXZ[o] : 0.0f;
        }
        for (int e = tid; e < HY * HX; e += TX * TY) {
            const int r = e / HX, c = e - r * HX;
            const int gxc = x0 - 4 + c, gyc = y0 - 4 + r;
            const bool in = gxc < G.gx && gyc < G.gy;
            sXY[r][c] = in ? gXY[base + int64_t(gyc) * P + gxc] : 0.0f;
        }
        for (int e = tid; e < HY * TX; e += TX * TY) {
            const int r = e / TX, c = e - r * TX;
            const int gxc = x0 + c, gyc = y0 - 4 + r;
            const bool in = gxc < G.gx && gyc < G.gy;
            const int64_t o = base + int64_t(gyc) * P + gxc;
            sYY[r][c] = in ? gYY[o] : 0.0f;
            sYZ[r][c] = in ? gYZ[o] : 0.0f;
        }
        for (int e = tid; e < (TY + 1) * (TX + 1); e += TX * TY) {
            const int r = e / (TX + 1), c = e - r * (TX + 1);
            const int gxc = x0 + c, gyc = y0 + r;
            const bool in = gxc < G.gx && gyc < G.gy;
            sB[r][c] = in ? F.invRho[base + int64_t(gyc) * P + gxc] : 1.0f;
        }
        __syncthreads();

        if (active) {
            const int64_t i = base + col;
            const int qz = cp ? slabIndex(z, G.gz, G.pml, G.freeSurface != 0) : -1;
            float kz[6] = {0, 0, 0, 0, 0, 0};
            if (qz >= 0)
                for (int h = 0; h < 2; ++h)
                    for (int j = 0; j < 3; ++j) kz[3 * h + j] = F.coef[2][(int64_t(h) * G.gz + z) * 3 + j];

            // Raw derivatives.  vx: D+x sxx, D-y sxy, D-z sxz.  vy: D-x sxy, D+y syy, D-z syz.
            // vz: D-x sxz, D-y syz, D+z szz.
            float dx0 = diffRow<HX>(&sXX[ty][tx + 1], inv);
            float dy0 = diffCol<HX>(&sXY[ty][tx + 4], inv);
            float dz0 = diffRing(rXZ, inv);
            float dx1 = diffRow<HX>(&sXY[ty + 4][tx], inv);
            float dy1 = diffCol<TX>(&sYY[ty + 1][tx], inv);
            float dz1 = diffRing(rYZ, inv);
            float dx2 = diffRow<HX>(&sXZ[ty][tx], inv);
            float dy2 = diffCol<TX>(&sYZ[ty][tx], inv);
            float dz2 = diffRing(rZZ, inv);

            if (qx >= 0) {
                float* p = F.psi[0] + (int64_t(z) * G.gy + y) * G.thick[0] + qx;
                const int64_t slot = int64_t(G.gz) * G.gy * G.thick[0];
                dx0 = cpmlUpdate(dx0, p, kx[3], kx[4], kx[5]);
                dx1 = cpmlUpdate(dx1, p + slot, kx[0], kx[1], kx[2]);
                dx2 = cpmlUpdate(dx2, p + 2 * slot, kx[0], kx[1], kx[2]);
            }
            if (qy >= 0) {
                float* p = F.psi[1] + (int64_t(z) * G.thick[1] + qy) * P + x;
                const int64_t slot = int64_t(G.gz) * G.thick[1] * P;
                dy0 = cpmlUpdate(dy0, p, ky[0], ky[1], ky[2]);
                dy1 = cpmlUpdate(dy1, p + slot, ky[3], ky[4], ky[5]);
                dy2 = cpmlUpdate(dy2, p + 2 * slot, ky[0], ky[1], ky[2]);
            }
            if (qz >= 0) {
                float* p = F.psi[2] + (int64_t(qz) * G.gy + y) * P + x;
                const int64_t slot = int64_t(G.thick[2]) * G.gy * P;
                dz0 = cpmlUpdate(dz0, p, kz[0], kz[1], kz[2]);
                dz1 = cpmlUpdate(dz1, p + slot, kz[0], kz[1], kz[2]);
                dz2 = cpmlUpdate(dz2, p + 2 * slot, kz[3], kz[4], kz[5]);
            }

            float div0 = 0.0f; div0 += dx0; div0 += dy0; div0 += dz0;
            float div1 = 0.0f; div1 += dx1; div1 += dy1; div1 += dz1;
            float div2 = 0.0f; div2 += dx2; div2 += dy2; div2 += dz2;

            const float a = sB[ty][tx];
            const float bx = sB[ty][tx + 1], by = sB[ty + 1][tx], bz = F.invRho[i + PL];
            const float cx = 2 * a * bx / (a + bx);
            const float cy = 2 * a * by / (a + by);
            const float cz = 2 * a * bz / (a + bz);
            float v0 = vx[i] + G.dt * cx * div0;
            float v1 = vy[i] + G.dt * cy * div1;
            float v2 = vz[i] + G.dt * cz * div2;
            if (forceHere && abs(z - S.gzs) <= 1) {
                const float value = sourceValue(G, S, x - S.gxs, y - S.gys, z - S.gzs, double(step) * G.dt);
                v0 += value * S.direction[0] * cx;
                v1 += value * S.direction[1] * cy;
                v2 += value * S.direction[2] * cz;
            }
            vx[i] = v0; vy[i] = v1; vz[i] = v2;
            bad |= !isfinite(v0) || !isfinite(v1) || !isfinite(v2);
        }
#pragma unroll
        for (int k = 0; k < 7; ++k) { rXZ[k] = rXZ[k + 1]; rYZ[k] = rYZ[k + 1]; rZZ[k] = rZZ[k + 1]; }
    }
    flagNonFinite(F, bad);
}

// ---------------------------------------------------------------------------------------
// Stress pass: sigma(n+1) from CPML-filtered velocity derivatives (cuda/Cuda_Seis3D.cu:281-310),
// harmonic shear moduli from shared reciprocals (:275-278), free-surface closure at z=4
// (:299, :303) and the explosion source fused (:313-332).
// ---------------------------------------------------------------------------------------
template <int TY>
__global__ void __launch_bounds__(32 * TY) stressPass(Geometry G, Fields F, SourceParams S, int zChunk) {
    constexpr int TX = 32, HX = TX + 8, HY = TY + 8;
    __shared__ float sVX[HY][HX];
    __shared__ float sVY[HY][HX];
    __shared__ float sVZ[HY][HX];
    __shared__ float sR[2][TY + 1][TX + 1];  // 1/mu on planes z (parity) and z+1

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int x0 = kRadius + blockIdx.x * TX, y0 = kRadius + blockIdx.y * TY;
    const int x = x0 + tx, y = y0 + ty;
    const bool active = x < G.gx - kRadius && y < G.gy - kRadius;
    const int zBegin = kRadius + blockIdx.z * zChunk;
    const int zEnd = min(zBegin + zChunk, G.gz - kRadius);
    if (zBegin >= zEnd) return;
    const int64_t P = G.pitch, PL = G.plane;
    const int64_t col = int64_t(min(y, G.gy - 1)) * P + min(x, G.gx - 1);
    const float inv = G.invH;

    const bool cp = !G.reflecting;
    const int qx = cp ? slabIndex(x, G.gx, G.pml, false) : -1;
    const int qy = cp ? slabIndex(y, G.gy, G.pml, false) : -1;
    float kx[6] = {0, 0, 0, 0, 0, 0}, ky[6] = {0, 0, 0, 0, 0, 0};
    if (qx >= 0 && active)
        for (int h = 0; h < 2; ++h)
            for (int j = 0; j < 3; ++j) kx[3 * h + j] = F.coef[0][(int64_t(h) * G.gx + x) * 3 + j];
    if (qy >= 0 && active)
        for (int h = 0; h < 2; ++h)
            for (int j = 0; j < 3; ++j) ky[3 * h + j] = F.coef[1][(int64_t(h) * G.gy + y) * 3 + j];

    const float* const gVX = F.f[0];
    const float* const gVY = F.f[1];
    const float* const gVZ = F.f[2];
    const float* const mu = F.mu;

    // Reciprocal shear modulus of one tile cell of a plane (IEEE division, as the
    // reference's 1/m): mu == 0 gives +inf so the harmonic mean below is exactly 0.
    auto loadRecip = [&](int z, int buf) {
        for (int e = tid; e < (TY + 1) * (TX + 1); e += TX * TY) {
            const int r = e / (TX + 1), c = e - r * (TX + 1);
            const int gxc = x0 + c, gyc = y0 + r;
            const bool in = gxc < G.gx && gyc < G.gy;
            sR[buf][r][c] = in ? 1.0f / mu[int64_t(z) * PL + int64_t(gyc) * P + gxc] : 0.0f;
        }
    };

    // z rings: rVX/rVY planes z-3..z+4 (D+), rVZ planes z-4..z+3 (D-).
    float rVX[8], rVY[8], rVZ[8];
    if (active) {
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            rVX[k] = gVX[int64_t(zBegin - 3 + k) * PL + col];
            rVY[k] = gVY[int64_t(zBegin - 3 + k) * PL + col];
            rVZ[k] = gVZ[int64_t(zBegin - 4 + k) * PL + col];
        }
    }
    loadRecip(zBegin, zBegin & 1);
    const unsigned long long step = F.clock->step;
    const bool blastHere = S.kind == 0 && active && abs(x - S.gxs) <= 1 && abs(y - S.gys) <= 1;
    bool bad = false;

    for (int z = zBegin; z < zEnd; ++z) {
        const int64_t base = int64_t(z) * PL;
        if (active) {
            rVX[7] = gVX[base + 4 * PL + col];
            rVY[7] = gVY[base + 4 * PL + col];
            rVZ[7] = gVZ[base + 3 * PL + col];
        }
        __syncthreads();
        for (int e = tid; e < HY * HX; e += TX * TY) {
            const int r = e / HX, c = e - r * HX;
            const int gxc = x0 - 4 + c, gyc = y0 - 4 + r;
            const bool in = gxc < G.gx && gyc < G.gy;
            const int64_t o = base + int64_t(gyc) * P + gxc;
            sVX[r][c] = in ? gVX[o] : 0.0f;
            sVY[r][c] = in ? gVY[o] : 0.0f;
            sVZ[r][c] = in ? gVZ[o] : 0.0f;
        }
        loadRecip(z + 1, (z + 1) & 1);
        __syncthreads();

        if (active) {
            const int64_t i = base + col;
            const int qz = cp ? slabIndex(z, G.gz, G.pml, G.freeSurface != 0) : -1;
            float kz[6] = {0, 0, 0, 0, 0, 0};
            if (qz >= 0)
                for (int h = 0; h < 2; ++h)
                    for (int j = 0; j < 3; ++j) kz[3 * h + j] = F.coef[2][(int64_t(h) * G.gz + z) * 3 + j];

            // d[v][a]: D- along its own axis, D+ across (cuda/Cuda_Seis3D.cu:293-295).
            float d00 = diffRow<HX>(&sVX[ty + 4][tx], inv);
            float d01 = diffCol<HX>(&sVX[ty + 1][tx + 4], inv);
            float d02 = diffRing(rVX, inv);
            float d10 = diffRow<HX>(&sVY[ty + 4][tx + 1], inv);
            float d11 = diffCol<HX>(&sVY[ty][tx + 4], inv);
            float d12 = diffRing(rVY, inv);
            float d20 = diffRow<HX>(&sVZ[ty + 4][tx + 1], inv);
            float d21 = diffCol<HX>(&sVZ[ty + 1][tx + 4], inv);
            float d22 = diffRing(rVZ, inv);

            if (qx >= 0) {
                float* p = F.psi[0] + (3 * int64_t(G.gz) + z) * G.gy * G.thick[0] + int64_t(y) * G.thick[0] + qx;
                const int64_t slot = int64_t(G.gz) * G.gy * G.thick[0];
                d00 = cpmlUpdate(d00, p, kx[0], kx[1], kx[2]);
                d10 = cpmlUpdate(d10, p + slot, kx[3], kx[4], kx[5]);
                d20 = cpmlUpdate(d20, p + 2 * slot, kx[3], kx[4], kx[5]);
            }
            if (qy >= 0) {
                float* p = F.psi[1] + ((3 * int64_t(G.gz) + z) * G.thick[1] + qy) * P + x;
                const int64_t slot = int64_t(G.gz) * G.thick[1] * P;
                d01 = cpmlUpdate(d01, p, ky[3], ky[4], ky[5]);
                d11 = cpmlUpdate(d11, p + slot, ky[0], ky[1], ky[2]);
                d21 = cpmlUpdate(d21, p + 2 * slot, ky[3], ky[4], ky[5]);
            }
            if (qz >= 0) {
                float* p = F.psi[2] + ((3 * int64_t(G.thick[2]) + qz) * G.gy + y) * P + x;
                const int64_t slot = int64_t(G.thick[2]) * G.gy * P;
                d02 = cpmlUpdate(d02, p, kz[3], kz[4], kz[5]);
                d12 = cpmlUpdate(d12, p + slot, kz[3], kz[4], kz[5]);
                d22 = cpmlUpdate(d22, p + 2 * slot, kz[0], kz[1], kz[2]);
            }

            const float lambda = F.lambda[i], m = mu[i];
            const bool top = G.freeSurface && z == kRadius;
            if (top) d22 = -lambda / (lambda + 2 * m) * (d00 + d11);
            const float trace = d00 + d11 + d22;
            const int b0 = z & 1, b1 = b0 ^ 1;
            const float r000 = sR[b0][ty][tx], r100 = sR[b0][ty][tx + 1], r010 = sR[b0][ty + 1][tx],
                        r110 = sR[b0][ty + 1][tx + 1];
            const float r001 = sR[b1][ty][tx], r101 = sR[b1][ty][tx + 1], r011 = sR[b1][ty + 1][tx];
            const float muXY = 4.0f / (r000 + r100 + r010 + r110);
            const float muYZ = 4.0f / (r000 + r010 + r001 + r011);
            const float muXZ = 4.0f / (r000 + r100 + r001 + r101);

            float sxx = F.f[3][i] + G.dt * (lambda * trace + 2 * m * d00);
            float syy = F.f[4][i] + G.dt * (lambda * trace + 2 * m * d11);
            float szz = top ? 0.0f : F.f[5][i] + G.dt * (lambda * trace + 2 * m * d22);
            float sxy = F.f[6][i] + G.dt * muXY * (d01 + d10);
            float syz = F.f[7][i] + G.dt * muYZ * (d12 + d21);
            float sxz = F.f[8][i] + G.dt * muXZ * (d02 + d20);
            bad |= !isfinite(sxx) || !isfinite(syy) || !isfinite(szz) || !isfinite(sxy) || !isfinite(syz) ||
                   !isfinite(sxz);
            if (blastHere && abs(z - S.gzs) <= 1) {
                const float value = sourceValue(G, S, x - S.gxs, y - S.gys, z - S.gzs, (double(step) + 0.5) * G.dt);
                sxx += value; syy += value; szz += value;
            }
            F.f[3][i] = sxx; F.f[4][i] = syy; F.f[5][i] = szz;
            F.f[6][i] = sxy; F.f[7][i] = syz; F.f[8][i] = sxz;
        }
#pragma unroll
        for (int k = 0; k < 7; ++k) { rVX[k] = rVX[k + 1]; rVY[k] = rVY[k + 1]; rVZ[k] = rVZ[k + 1]; }
    }
    flagNonFinite(F, bad);
}

// ---------------------------------------------------------------------------------------
// Free surface (planar, z = 4): traction images of the stresses (cuda/Cuda_Seis3D.cu:203-219)
// and velocity images from the zero-traction constraints (:249-272).
// ---------------------------------------------------------------------------------------
__global__ void stressImages(Geometry G, Fields F) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + kRadius;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + kRadius;
    if (x >= G.gx - kRadius || y >= G.gy - kRadius) return;
    const int64_t c = int64_t(y) * G.pitch + x, PL = G.plane;
    F.f[5][4 * PL + c] = 0.0f;
#pragma unroll
    for (int k = 1; k <= 4; ++k) {
        const int64_t g = (4 - k) * PL + c, m = (4 + k) * PL + c, sm = (3 + k) * PL + c;
        F.f[5][g] = -F.f[5][m];
        F.f[8][g] = -F.f[8][sm];
        F.f[7][g] = -F.f[7][sm];
        F.f[3][g] = F.f[3][m];
        F.f[4][g] = F.f[4][m];
        F.f[6][g] = F.f[6][m];
    }
}

__global__ void velocityImages(Geometry G, Fields F) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + kRadius;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + kRadius;
    if (x >= G.gx - kRadius || y >= G.gy - kRadius) return;
    const int64_t P = G.pitch, PL = G.plane;
    const int64_t i = 4 * PL + int64_t(y) * P + x, n = i + PL;
    const float inv = G.invH;
    const float* vx = F.f[0];
    const float* vy = F.f[1];
    const float* vz = F.f[2];
    const float ex = diff8(vx[i - 4], vx[i - 3], vx[i - 2], vx[i - 1], vx[i], vx[i + 1], vx[i + 2], vx[i + 3], inv);
    const float ey = diff8(vy[i - 4 * P], vy[i - 3 * P], vy[i - 2 * P], vy[i - P], vy[i], vy[i + P], vy[i + 2 * P],
                           vy[i + 3 * P], inv);
    const float zx0 = diff8(vz[i - 3], vz[i - 2], vz[i - 1], vz[i], vz[i + 1], vz[i + 2], vz[i + 3], vz[i + 4], inv);
    const float zx1 = diff8(vz[n - 3], vz[n - 2], vz[n - 1], vz[n], vz[n + 1], vz[n + 2], vz[n + 3], vz[n + 4], inv);
    const float zy0 = diff8(vz[i - 3 * P], vz[i - 2 * P], vz[i - P], vz[i], vz[i + P], vz[i + 2 * P], vz[i + 3 * P],
                            vz[i + 4 * P], inv);
    const float zy1 = diff8(vz[n - 3 * P], vz[n - 2 * P], vz[n - P], vz[n], vz[n + P], vz[n + 2 * P], vz[n + 3 * P],
                            vz[n + 4 * P], inv);
    const float dzVx = -(1.5f * zx0 - 0.5f * zx1);
    const float dzVy = -(1.5f * zy0 - 0.5f * zy1);
    const float dzVz = -F.lambda[i] / (F.lambda[i] + 2 * F.mu[i]) * (ex + ey);
    const int64_t c = int64_t(y) * P + x;
#pragma unroll
    for (int k = 1; k <= 4; ++k) {
        const int64_t g = (4 - k) * PL + c, m = (4 + k) * PL + c;
        F.f[0][g] = F.f[0][m] - 2 * k * G.h * dzVx;
        F.f[1][g] = F.f[1][m] - 2 * k * G.h * dzVy;
        F.f[2][g] = F.f[2][(3 + k) * PL + c] - (2 * k - 1) * G.h * dzVz;
    }
}

// Slip-wall images of one axis pair (cuda/Cuda_Seis3D.cu:152-175).
__global__ void reflectingImages(Geometry G, Fields F, int axis, int velocities) {
    const int len[3] = {G.gx, G.gy, G.gz};
    const int ua = (axis + 1) % 3, va = (axis + 2) % 3;
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    if (u >= len[ua] || v >= len[va]) return;
    const int high = len[axis] - kRadius - 1;
    int p[3] = {0, 0, 0};
    p[ua] = u; p[va] = v;
    auto at = [&](const int* q) { return int64_t(q[2]) * G.plane + int64_t(q[1]) * G.pitch + q[0]; };
    for (int f = velocities ? 0 : 3; f < (velocities ? 3 : 9); ++f) {
        const bool half = f < 3 ? f == axis : f == 6 ? axis != 2 : f == 7 ? axis != 0 : f == 8 ? axis != 1 : false;
        float* field = F.f[f];
        for (int side = 0; side < 2; ++side)
            for (int depth = 1; depth <= kRadius; ++depth) {
                p[axis] = side ? high + depth : kRadius - depth;
                const int64_t dst = at(p);
                if (half && !side && depth == 1) { field[dst] = 0.0f; continue; }
                p[axis] = side ? high + 1 - depth - int(half) : kRadius + depth - 1 - int(half);
                const float value = field[at(p)];
                field[dst] = half ? -value : value;
            }
        if (half) { p[axis] = high; field[at(p)] = 0.0f; }
    }
}

// ---------------------------------------------------------------------------------------
// Receivers: collocated [vx, vy, vz] (cuda/Cuda_Seis3D.cu:335-352, :421-428).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void collocate(const Geometry& G, const Fields& F, int4 r, float* out) {
    const int64_t i = int64_t(r.z) * G.plane + int64_t(r.y) * G.pitch + r.x;
    out[0] = 0.5f * (F.f[0][i] + F.f[0][i - 1]);
    out[1] = 0.5f * (F.f[1][i] + F.f[1][i - G.pitch]);
    out[2] = 0.5f * (F.f[2][i] + F.f[2][i - G.plane]);
}

// Receivers are passed as grid coordinates (x+ox, y+oy, z+oz, 0).
__global__ void sampleReceivers(Geometry G, Fields F, const int4* receivers, int count, float* out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < count) collocate(G, F, receivers[r], out + 3 * r);
}

// End of a step: record a gather sample when (step+1) % stride == 0, advance the clock
// (src/Seis3D_Sim.cpp:127-132 cadence).  One block.
__global__ void stepTail(Geometry G, Fields F, const int4* receivers, int count, float* gather) {
    Clock* clk = F.clock;
    const unsigned long long next = clk->step + 1;
    const int stride = clk->stride, sample = clk->sample;
    const bool record = stride > 0 && gather && next % (unsigned long long)stride == 0 && sample < clk->target;
    if (record)
        for (int r = threadIdx.x; r < count; r += blockDim.x)
            collocate(G, F, receivers[r], gather + (int64_t(sample) * count + r) * 3);
    __syncthreads();
    if (threadIdx.x == 0) {
        clk->step = next;
        if (record) clk->sample = sample + 1;
    }
}

__global__ void setClock(Clock* clk, unsigned long long step) { clk->step = step; }

// ---------------------------------------------------------------------------------------
// Materials.
// ---------------------------------------------------------------------------------------
struct ModelParams {
    int kind;
    float vp, vs, rho, layerVp, layerVs, layerRho;
    float interfaceDepth, layerDip, layerThickness, faultThrow, anomalyRadius;
};

// Procedural model with the nearest physical cell extended into padding
// (cuda/Cuda_Seis3D.cu:114-147).
__global__ void generateMaterials(Geometry G, Fields F, ModelParams M) {
    const int64_t cells = int64_t(G.gx) * G.gy * G.gz;
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    const int gxI = int(i % G.gx), gyI = int((i / G.gx) % G.gy), gzI = int(i / (int64_t(G.gx) * G.gy));
    const int x = max(0, min(G.nx - 1, gxI - G.ox));
    const int y = max(0, min(G.ny - 1, gyI - G.oy));
    const int z = max(0, min(G.nz - 1, gzI - G.oz));
    const float dx = (x - G.nx * 0.5f) / G.nx;
    const float dy = (y - G.ny * 0.5f) / G.ny;
    const float dz = (z - G.nz * 0.55f) / G.nz;
    const float depth = float(z) / float(G.nz - 1), horizontal = float(x) / float(G.nx - 1) - 0.5f;
    float blend = 0;
    switch (M.kind) {
    case 1: blend = depth >= M.interfaceDepth; break;
    case 2: blend = dx * dx + dy * dy + dz * dz < M.anomalyRadius * M.anomalyRadius; break;
    case 4: blend = depth < 1.0f / 3 ? 0 : depth < 2.0f / 3 ? 0.5f : 1; break;
    case 5: blend = depth >= M.interfaceDepth + M.layerDip * horizontal; break;
    case 6: blend = fabsf(depth - M.interfaceDepth) <= 0.5f * M.layerThickness; break;
    case 7: blend = depth >= M.interfaceDepth + M.layerDip * horizontal + (horizontal > 0 ? M.faultThrow : 0); break;
    case 8: blend = depth; break;
    case 9: {
        const float v = (depth - 0.78f) / 0.52f;
        blend = (dx * dx + dy * dy) / (M.anomalyRadius * M.anomalyRadius) + v * v < 1;
        break;
    }
    default: break;
    }
    const float vp = M.vp + blend * (M.layerVp - M.vp), vs = M.vs + blend * (M.layerVs - M.vs);
    const float rho = M.rho + blend * (M.layerRho - M.rho);
    const int64_t o = int64_t(gzI) * G.plane + int64_t(gyI) * G.pitch + gxI;
    F.invRho[o] = 1.0f / rho;
    F.mu[o] = rho * vs * vs;
    F.lambda[o] = rho * (vp * vp - 2.0f * vs * vs);
}

// Extend imported physical materials into CPML and ghost cells (cuda/Cuda_Seis3D.cu:188-200).
__global__ void extendMaterials(Geometry G, Fields F) {
    const int64_t cells = int64_t(G.gx) * G.gy * G.gz;
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    const int x = int(i % G.gx), y = int((i / G.gx) % G.gy), z = int(i / (int64_t(G.gx) * G.gy));
    const int px = max(G.ox, min(x, G.ox + G.nx - 1));
    const int py = max(G.oy, min(y, G.oy + G.ny - 1));
    const int pz = max(G.oz, min(z, G.oz + G.nz - 1));
    if (x == px && y == py && z == pz) return;
    const int64_t d = int64_t(z) * G.plane + int64_t(y) * G.pitch + x;
    const int64_t s = int64_t(pz) * G.plane + int64_t(py) * G.pitch + px;
    F.invRho[d] = F.invRho[s];
    F.mu[d] = F.mu[s];
    F.lambda[d] = F.lambda[s];
}

}  // namespace seis3d
