// seis3d_oracle.cpp - CPU oracle of the SeisWave Lab 3-D elastic solver.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, on the CPU, the algorithm of the
// reference's GPU solver cuda/Cuda_Seis3D.cu so that the B200 kernels can be checked
// against it.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
// it; the product library never does.
//
// Parity pinning: the validation and memory-budget functions are checked against the
// reference's own known answers (tests/Seis3DBoundaryRegression.cpp:70-82 and the BUDGET
// lines it prints), the CPML tables bit-for-bit against the reference's
// makeCoefficients3D compiled from its own source (oracle/ref3d_shim.cu), and the time
// stepping against traces of the reference CUDA solver run on a B200
// (tests/golden/ref3d_*.npz, generated by tests/golden/make_ref3d_golden.py).
//
// Two precisions share one template: FP32 (float state and arithmetic, the reference's
// own precision) and FP64 (the same scheme in double, used as the error reference of
// every storage precision).  Arithmetic is compiled without contraction
// (-ffp-contract=off) so the FP32 path is plain IEEE single precision.
//
// Storage emulation (oracle3d_set_storage): every value written to the wavefields and/or the
// materials can be rounded to FP16 or BF16 with a per-field power-of-two scale, the state a
// 16-bit storage kernel would keep while computing in FP32.  It measures what a storage
// precision costs in trace error before any kernel is written for it.
#include "../include/seis3d_capi.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <new>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kRadius = 4;  // include/Common3D.h:9

// Staggered 8th-order weights (cuda/Cuda_Seis3D.cu:72-75).
template <class T> inline T weight(int r) {
    return r == 0 ? T(1225.0f / 1024.0f) : r == 1 ? T(-245.0f / 3072.0f)
         : r == 2 ? T(49.0f / 5120.0f) : T(-5.0f / 7168.0f);
}
template <> inline double weight<double>(int r) {
    return r == 0 ? 1225.0 / 1024.0 : r == 1 ? -245.0 / 3072.0 : r == 2 ? 49.0 / 5120.0 : -5.0 / 7168.0;
}

// Material admissibility (cuda/Cuda_Seis3D.cu:30-34).
bool admissible(float vp, float vs, float rho) {
    return std::isfinite(vp) && std::isfinite(vs) && std::isfinite(rho) && vp > 0 && vp <= 30000 &&
           vs >= 0 && vs < vp && vp * vp > (4.0f / 3.0f) * vs * vs && rho > 0 && rho <= 50000;
}

int activePml(const seis3d_context& c) { return c.reflecting3D ? 0 : c.pml3D; }  // Common3D.h:63-65

// Slab extent per axis, cross-axis corners included (cuda/Cuda_Seis3D.cu:37-42).
std::size_t slabCells(const seis3d_context& c, int axis) {
    if (c.reflecting3D) return 0;
    if (axis == 0) return std::size_t(2 * c.pml3D) * c.gy3D * c.gz3D;
    if (axis == 1) return std::size_t(2 * c.pml3D) * c.gx3D * c.gz3D;
    return std::size_t((c.freeSurface3D ? 1 : 2) * c.pml3D) * c.gx3D * c.gy3D;
}

// Thinnest CPML the validation accepts: the reference's 8 (cuda/Cuda_Seis3D.cu:448), or 4 for
// the thin layers of the learned-boundary mode (oracle3d_set_min_pml).
int g_minPml = 8;

// Derivation and validation of a context (cuda/Cuda_Seis3D.cu:433-483).  Returns "" on
// success, else the rejection message.
std::string validate(seis3d_context& c) {
    if (c.reflecting3D) c.freeSurface3D = 0;
    if (c.modelKind3D < 0 || c.modelKind3D > SEIS3D_MODEL_SALT_DOME || !std::isfinite(c.interfaceDepth3D) ||
        c.interfaceDepth3D < .1f || c.interfaceDepth3D > .9f || !std::isfinite(c.layerDip3D) ||
        std::abs(c.layerDip3D) > .6f || !std::isfinite(c.layerThickness3D) || c.layerThickness3D < .03f ||
        c.layerThickness3D > .5f || !std::isfinite(c.faultThrow3D) || std::abs(c.faultThrow3D) > .4f ||
        !std::isfinite(c.anomalyRadius3D) || c.anomalyRadius3D < .05f || c.anomalyRadius3D > .4f)
        return "invalid procedural model geometry";
    if (c.nx3D < 16 || c.ny3D < 16 || c.nz3D < 16) return "every physical dimension must be at least 16";
    const std::size_t cap = SEIS3D_MAX_PHYSICAL_NODES;
    if (std::size_t(c.nx3D) > cap / std::size_t(c.ny3D) ||
        std::size_t(c.nx3D) * std::size_t(c.ny3D) > cap / std::size_t(c.nz3D))
        return "physical node count exceeds 36,000,000";
    if (c.pml3D < g_minPml || c.pml3D > 40 || !std::isfinite(c.spacing3D) || c.spacing3D <= 0 ||
        !std::isfinite(c.frequency3D) || c.frequency3D <= 0 || c.frequency3D > 10000 ||
        !std::isfinite(c.cfl3D) || c.cfl3D <= 0 || c.cfl3D > 0.9f)
        return "invalid CPML, spacing, frequency or CFL";
    if (!admissible(c.vp3D, c.vs3D, c.density3D) || !admissible(c.layerVp3D, c.layerVs3D, c.layerDensity3D))
        return "invalid material";
    if (c.modelKind3D != SEIS3D_MODEL_IMPORTED)
        c.maxVp3D = c.modelKind3D == SEIS3D_MODEL_UNIFORM ? c.vp3D : std::max(c.vp3D, c.layerVp3D);
    if (!std::isfinite(c.maxVp3D) || c.maxVp3D <= 0 || c.maxVp3D > 30000) return "invalid maximum vp";
    const int p = activePml(c);
    c.ox3D = c.oy3D = p + 4;
    c.oz3D = c.freeSurface3D ? 4 : p + 4;
    c.gx3D = c.nx3D + 2 * p + 8;
    c.gy3D = c.ny3D + 2 * p + 8;
    c.gz3D = c.nz3D + (c.freeSurface3D ? 1 : 2) * p + 8;
    c.cells3D = uint64_t(c.gx3D) * c.gy3D * c.gz3D;
    const double sumW = 1225.0 / 1024 + 245.0 / 3072 + 49.0 / 5120 + 5.0 / 7168;
    const double safe = c.cfl3D * c.spacing3D / (std::sqrt(3.0) * c.maxVp3D * sumW);
    const double us = std::floor(safe * 1.0e6);
    if (us < 1 || us > 65535) return "safe dt outside 1..65535 us";
    c.safeDt3D = float(us * 1.0e-6);
    c.dt3D = c.safeDt3D;
    if (c.manualTimeStep3D) {
        const double req = double(c.requestedDtMs3D) * 1000;
        const double rounded = std::round(req);
        if (!std::isfinite(req) || rounded < 1 || rounded > 65535) return "manual dt out of range";
        if (std::abs(req - rounded) > 0.05) return "manual dt must be whole microseconds";
        if (rounded > us) return "manual dt exceeds the CFL ceiling";
        c.dt3D = float(rounded * 1.0e-6);
    }
    return "";
}

// View layout (cuda/Cuda_Seis3D.cu:486-501), needed by the memory budget.
seis3d_view_layout viewLayout(const seis3d_context& c) {
    seis3d_view_layout l{};
    const int p = activePml(c);
    const int nx = c.nx3D + 2 * p, ny = c.ny3D + 2 * p, nz = c.nz3D + (c.freeSurface3D ? 1 : 2) * p;
    l.domainSize3D[0] = nx; l.domainSize3D[1] = ny; l.domainSize3D[2] = nz;
    l.domainOrigin3D[0] = -p; l.domainOrigin3D[1] = -p; l.domainOrigin3D[2] = c.freeSurface3D ? 0 : -p;
    l.sliceWidth3D[0] = nx; l.sliceHeight3D[0] = nz;
    l.sliceWidth3D[1] = ny; l.sliceHeight3D[1] = nz;
    l.sliceWidth3D[2] = nx; l.sliceHeight3D[2] = ny;
    l.sliceOffset3D[1] = uint64_t(nx) * nz;
    l.sliceOffset3D[2] = l.sliceOffset3D[1] + uint64_t(ny) * nz;
    l.volumeOffset3D = l.sliceOffset3D[2] + uint64_t(nx) * ny;
    l.volumeX3D = std::min(SEIS3D_MAX_VOLUME_AXIS, nx);
    l.volumeY3D = std::min(SEIS3D_MAX_VOLUME_AXIS, ny);
    l.volumeZ3D = std::min(SEIS3D_MAX_VOLUME_AXIS, nz);
    l.totalSamples3D = l.volumeOffset3D + uint64_t(l.volumeX3D) * l.volumeY3D * l.volumeZ3D;
    return l;
}

// CPML a/b/(1/kappa) per node at centre (half=0) and half-grid (half=1) positions
// (cuda/Cuda_Seis3D.cu:45-64), kept in double for the FP64 oracle.
std::vector<double> profile(const seis3d_context& c, int axis) {
    const int n = axis == 0 ? c.gx3D : axis == 1 ? c.gy3D : c.gz3D;
    std::vector<double> out(std::size_t(n) * 6);
    const double sigmaMax = -4.0 * c.maxVp3D * std::log(1.0e-6) / (2.0 * c.pml3D * c.spacing3D);
    const bool topFree = axis == 2 && c.freeSurface3D;
    for (int half = 0; half < 2; ++half)
        for (int i = 0; i < n; ++i) {
            const double at = i + 0.5 * half;
            double d = (at - (n - kRadius - c.pml3D - 0.5)) / c.pml3D;          // far face
            if (!topFree) d = std::max(d, (kRadius + c.pml3D - 0.5 - at) / c.pml3D);  // near face
            d = std::clamp(d, 0.0, 1.0);
            const double cube = d * d * d;
            const double sigma = sigmaMax * cube, kappa = 1.0 + 2.0 * cube;
            const double alpha = d > 0 ? 3.141592653589793 * c.frequency3D * (1.0 - d) : 0.0;
            const double b = std::exp(-(sigma / kappa + alpha) * c.dt3D);
            const double a = sigma > 0 ? sigma * (b - 1.0) / (kappa * (sigma + kappa * alpha)) : 0.0;
            double* slot = out.data() + (std::size_t(half) * n + i) * 3;
            slot[0] = a; slot[1] = b; slot[2] = 1.0 / kappa;
        }
    return out;
}

// Whole state of one oracle run in precision T.

// Storage emulation: 0 none, 1 FP16, 2 BF16; mask 1 velocities, 2 stresses, 4 materials.
int g_storage = 0;
int g_storageMask = 7;

// FP32 -> BF16 -> FP32, round to nearest even (finite inputs).
inline float bf16Round(float x) {
    std::uint32_t b;
    std::memcpy(&b, &x, 4);
    b = (b + 0x7FFFu + ((b >> 16) & 1u)) & 0xFFFF0000u;
    float y;
    std::memcpy(&y, &b, 4);
    return y;
}

inline float storageRound(float x) {
    if (g_storage == 1) return float(_Float16(x));
    if (g_storage == 2) return bf16Round(x);
    return x;
}

// CPML-memory storage emulation: 0 FP32, 1 FP16, 2 BF16 (round to nearest even, no scaling).
int g_psiStorage = 0;

// Reads only g_psiStorage, which is set between runs: the memory updates run in parallel.
inline float psiRound(float x) { return g_psiStorage == 1 ? float(_Float16(x)) : bf16Round(x); }

// Rounds a whole field as 16-bit storage with a power-of-two scale that maps its largest
// magnitude just below 2^15 (inside the FP16 range).
template <class T> void storeRounded(std::vector<T>& f) {
    double m = 0;
    for (const T v : f) m = std::max(m, std::abs(double(v)));
    if (m == 0 || !std::isfinite(m)) return;
    const double scale = std::exp2(std::ceil(std::log2(m / 16384.0)));
    for (T& v : f) v = T(double(storageRound(float(double(v) / scale))) * scale);
}

template <class T> struct State {
    seis3d_context c{};
    std::size_t cells = 0, sx = 1, sy = 0, sz = 0;
    std::vector<T> field[9];
    std::vector<T> invRho, lambda, mu;
    std::vector<T> psi[3];      // 6 slots per axis, reference slab indexing
    std::size_t slab[3]{};
    std::vector<T> coef[3];     // {a,b,1/kappa} per (half, node)
    bool nonFinite = false;

    std::size_t at(int x, int y, int z) const { return (std::size_t(z) * c.gy3D + y) * c.gx3D + x; }

    explicit State(const seis3d_context& ctx) : c(ctx) {
        cells = std::size_t(c.cells3D);
        sy = std::size_t(c.gx3D);
        sz = std::size_t(c.gx3D) * c.gy3D;
        for (auto& f : field) f.assign(cells, T(0));
        invRho.assign(cells, T(0)); lambda.assign(cells, T(0)); mu.assign(cells, T(0));
        for (int a = 0; a < 3; ++a) {
            slab[a] = slabCells(c, a);
            psi[a].assign(slab[a] * 6, T(0));
            if (!c.reflecting3D) {
                const auto p = profile(c, a);
                coef[a].resize(p.size());
                // FP32: the reference rounds the FP64 profile to float (:61); FP64 keeps it.
                for (std::size_t i = 0; i < p.size(); ++i) coef[a][i] = T(sizeof(T) == 4 ? double(float(p[i])) : p[i]);
            }
        }
    }

    void reset() {
        for (auto& f : field) std::fill(f.begin(), f.end(), T(0));
        for (auto& p : psi) std::fill(p.begin(), p.end(), T(0));
        nonFinite = false;
    }

    // Procedural materials (cuda/Cuda_Seis3D.cu:114-147), nearest physical cell in padding.
    void generate() {
        for (std::size_t i = 0; i < cells; ++i) {
            const int x = std::max(0, std::min(c.nx3D - 1, int(i % c.gx3D) - c.ox3D));
            const int y = std::max(0, std::min(c.ny3D - 1, int((i / c.gx3D) % c.gy3D) - c.oy3D));
            const int z = std::max(0, std::min(c.nz3D - 1, int(i / (std::size_t(c.gx3D) * c.gy3D)) - c.oz3D));
            const float dx = (x - c.nx3D * 0.5f) / c.nx3D;
            const float dy = (y - c.ny3D * 0.5f) / c.ny3D;
            const float dz = (z - c.nz3D * 0.55f) / c.nz3D;
            const float depth = float(z) / float(c.nz3D - 1), horizontal = float(x) / float(c.nx3D - 1) - 0.5f;
            float blend = 0;
            const float r2 = c.anomalyRadius3D * c.anomalyRadius3D;
            switch (c.modelKind3D) {
            case SEIS3D_MODEL_TWO_LAYER: blend = depth >= c.interfaceDepth3D; break;
            case SEIS3D_MODEL_SPHERE: blend = dx * dx + dy * dy + dz * dz < r2; break;
            case SEIS3D_MODEL_THREE_LAYER: blend = depth < 1.0f / 3 ? 0 : depth < 2.0f / 3 ? 0.5f : 1; break;
            case SEIS3D_MODEL_DIPPING_LAYER: blend = depth >= c.interfaceDepth3D + c.layerDip3D * horizontal; break;
            case SEIS3D_MODEL_LOW_VELOCITY_LAYER: blend = std::fabs(depth - c.interfaceDepth3D) <= 0.5f * c.layerThickness3D; break;
            case SEIS3D_MODEL_FAULT:
                blend = depth >= c.interfaceDepth3D + c.layerDip3D * horizontal + (horizontal > 0 ? c.faultThrow3D : 0);
                break;
            case SEIS3D_MODEL_GRADIENT: blend = depth; break;
            case SEIS3D_MODEL_SALT_DOME: {
                const float v = (depth - 0.78f) / 0.52f;
                blend = (dx * dx + dy * dy) / r2 + v * v < 1;
                break;
            }
            default: break;
            }
            const float vp = c.vp3D + blend * (c.layerVp3D - c.vp3D), vs = c.vs3D + blend * (c.layerVs3D - c.vs3D);
            const float rho = c.density3D + blend * (c.layerDensity3D - c.density3D);
            setMaterial(i, vp, vs, rho);
        }
    }

    // SI -> 1/rho, lambda, mu (cuda/Cuda_Seis3D.cu:144-146 and :704).  FP32 evaluates in
    // float as the reference does; FP64 evaluates the same formulas in double.
    void setMaterial(std::size_t i, float vp, float vs, float rho) {
        if (sizeof(T) == 4) {
            invRho[i] = T(1.0f / rho); mu[i] = T(rho * vs * vs); lambda[i] = T(rho * (vp * vp - 2.0f * vs * vs));
        } else {
            const double P = vp, S = vs, R = rho;
            invRho[i] = T(1.0 / R); mu[i] = T(R * S * S); lambda[i] = T(R * (P * P - 2.0 * S * S));
        }
    }

    // uploadModelPlane3D (cuda/Cuda_Seis3D.cu:696-711).
    std::string uploadPlane(int z, const float* values) {
        if (z < 0 || z >= c.nz3D || !values) return "invalid model plane";
        const std::size_t n = std::size_t(c.nx3D) * c.ny3D;
        for (std::size_t k = 0; k < n; ++k) {
            const float vp = values[3 * k], vs = values[3 * k + 1], rho = values[3 * k + 2];
            if (!admissible(vp, vs, rho) || vp > c.maxVp3D * (1 + 1.0e-6f)) return "invalid or changed imported material";
        }
        for (int y = 0; y < c.ny3D; ++y)
            for (int x = 0; x < c.nx3D; ++x) {
                const std::size_t k = std::size_t(y) * c.nx3D + x;
                setMaterial(at(x + c.ox3D, y + c.oy3D, z + c.oz3D), values[3 * k], values[3 * k + 1], values[3 * k + 2]);
            }
        return "";
    }

    // extendMaterialsKernel3D (cuda/Cuda_Seis3D.cu:188-200).
    void finishUpload() {
        for (int z = 0; z < c.gz3D; ++z)
            for (int y = 0; y < c.gy3D; ++y)
                for (int x = 0; x < c.gx3D; ++x) {
                    const int px = std::max(c.ox3D, std::min(x, c.ox3D + c.nx3D - 1));
                    const int py = std::max(c.oy3D, std::min(y, c.oy3D + c.ny3D - 1));
                    const int pz = std::max(c.oz3D, std::min(z, c.oz3D + c.nz3D - 1));
                    if (x == px && y == py && z == pz) continue;
                    const std::size_t i = at(x, y, z), j = at(px, py, pz);
                    invRho[i] = invRho[j]; mu[i] = mu[j]; lambda[i] = lambda[j];
                }
    }

    // D+ (plus) at i+1/2 or D- at i along one stride (cuda/Cuda_Seis3D.cu:78-89).
    template <bool plus> T diff(const std::vector<T>& f, std::size_t i, std::size_t stride, T inv) const {
        T sum = 0;
        for (int r = 0; r < 4; ++r) {
            const std::size_t hi = i + std::size_t(r + (plus ? 1 : 0)) * stride;
            const std::size_t lo = i - std::size_t(r + (plus ? 0 : 1)) * stride;
            sum += weight<T>(r) * (f[hi] - f[lo]);
        }
        return sum * inv;
    }

    // CPML memory recurrence of one derivative (cuda/Cuda_Seis3D.cu:92-111).
    T cpml(int x, int y, int z, int axis, int slot, bool half, T d) {
        if (c.reflecting3D) return d;
        const int n = axis == 0 ? c.gx3D : axis == 1 ? c.gy3D : c.gz3D;
        const int coord = axis == 0 ? x : axis == 1 ? y : z;
        const bool topFree = axis == 2 && c.freeSurface3D;
        int q = -1;
        if (!topFree && coord < kRadius + c.pml3D) q = coord - kRadius;
        else if (coord >= n - kRadius - c.pml3D) q = (topFree ? 0 : c.pml3D) + coord - (n - kRadius - c.pml3D);
        if (q < 0) return d;
        const int thick = (topFree ? 1 : 2) * c.pml3D;
        const std::size_t s = axis == 0 ? (std::size_t(z) * c.gy3D + y) * thick + q
                            : axis == 1 ? (std::size_t(z) * c.gx3D + x) * thick + q
                                        : (std::size_t(y) * c.gx3D + x) * thick + q;
        T& m = psi[axis][std::size_t(slot) * slab[axis] + s];
        const T* k = coef[axis].data() + (std::size_t(half) * n + coord) * 3;
        const T updated = k[1] * m + k[0] * d;
        // 16-bit CPML-memory storage (oracle3d_set_psi_storage): the update is used in full
        // precision and only the stored memory is rounded.
        m = g_psiStorage ? T(psiRound(float(updated))) : updated;
        return k[2] * d + updated;
    }

    // Free-surface stress images (cuda/Cuda_Seis3D.cu:203-219).
    void stressGhosts() {
        for (int y = 4; y < c.gy3D - 4; ++y)
            for (int x = 4; x < c.gx3D - 4; ++x) {
                field[5][at(x, y, 4)] = 0;
                for (int k = 1; k <= 4; ++k) {
                    const std::size_t g = at(x, y, 4 - k), m = at(x, y, 4 + k), sm = at(x, y, 3 + k);
                    field[5][g] = -field[5][m];
                    field[8][g] = -field[8][sm];
                    field[7][g] = -field[7][sm];
                    field[3][g] = field[3][m];
                    field[4][g] = field[4][m];
                    field[6][g] = field[6][m];
                }
            }
    }

    // Velocity update v(n+1/2) (cuda/Cuda_Seis3D.cu:222-245).
    void velocity() {
        const T inv = T(1) / T(c.spacing3D);
        const T dt = T(c.dt3D);
        const std::size_t st[3] = {1, sy, sz};
        static const int S[3][3] = {{3, 6, 8}, {6, 4, 7}, {8, 7, 5}};
        bool bad = false;
#pragma omp parallel for schedule(static) reduction(|| : bad)
        for (int z = 4; z < c.gz3D - 4; ++z)
            for (int y = 4; y < c.gy3D - 4; ++y)
                for (int x = 4; x < c.gx3D - 4; ++x) {
                    const std::size_t i = at(x, y, z);
                    for (int v = 0; v < 3; ++v) {
                        T div = 0;
                        for (int a = 0; a < 3; ++a) {
                            const auto& f = field[S[v][a]];
                            const T d = a == v ? diff<true>(f, i, st[a], inv) : diff<false>(f, i, st[a], inv);
                            div += cpml(x, y, z, a, v, a == v, d);
                        }
                        const T A = invRho[i], B = invRho[i + st[v]];
                        const T value = field[v][i] + dt * (2 * A * B / (A + B)) * div;
                        field[v][i] = value;
                        if (!std::isfinite(double(value))) bad = true;
                    }
                }
        nonFinite = nonFinite || bad;
    }

    // Free-surface velocity images from the zero-traction constraints (cuda/Cuda_Seis3D.cu:249-272).
    void velocityGhosts() {
        const T inv = T(1) / T(c.spacing3D);
        const T h = T(c.spacing3D);
        for (int y = 4; y < c.gy3D - 4; ++y)
            for (int x = 4; x < c.gx3D - 4; ++x) {
                const std::size_t i = at(x, y, 4), next = i + sz;
                const T ex = diff<false>(field[0], i, 1, inv);
                const T ey = diff<false>(field[1], i, sy, inv);
                const T dzVx = -(T(1.5) * diff<true>(field[2], i, 1, inv) - T(0.5) * diff<true>(field[2], next, 1, inv));
                const T dzVy = -(T(1.5) * diff<true>(field[2], i, sy, inv) - T(0.5) * diff<true>(field[2], next, sy, inv));
                const T dzVz = -lambda[i] / (lambda[i] + 2 * mu[i]) * (ex + ey);
                for (int k = 1; k <= 4; ++k) {
                    const std::size_t g = at(x, y, 4 - k), m = at(x, y, 4 + k);
                    field[0][g] = field[0][m] - T(2 * k) * h * dzVx;
                    field[1][g] = field[1][m] - T(2 * k) * h * dzVy;
                    field[2][g] = field[2][at(x, y, 3 + k)] - T(2 * k - 1) * h * dzVz;
                }
            }
    }

    // Harmonic 4-cell shear modulus (cuda/Cuda_Seis3D.cu:275-278).
    T shearMu(std::size_t i, std::size_t a, std::size_t b) const {
        const T m0 = mu[i], m1 = mu[i + a], m2 = mu[i + b], m3 = mu[i + a + b];
        return (m0 > 0 && m1 > 0 && m2 > 0 && m3 > 0) ? 4 / (1 / m0 + 1 / m1 + 1 / m2 + 1 / m3) : T(0);
    }

    // Stress update sigma(n+1) (cuda/Cuda_Seis3D.cu:281-310).
    void stress() {
        const T inv = T(1) / T(c.spacing3D);
        const T dt = T(c.dt3D);
        const std::size_t st[3] = {1, sy, sz};
        bool bad = false;
#pragma omp parallel for schedule(static) reduction(|| : bad)
        for (int z = 4; z < c.gz3D - 4; ++z)
            for (int y = 4; y < c.gy3D - 4; ++y)
                for (int x = 4; x < c.gx3D - 4; ++x) {
                    const std::size_t i = at(x, y, z);
                    T d[3][3];
                    for (int v = 0; v < 3; ++v)
                        for (int a = 0; a < 3; ++a) {
                            const T raw = a == v ? diff<false>(field[v], i, st[a], inv) : diff<true>(field[v], i, st[a], inv);
                            d[v][a] = cpml(x, y, z, a, 3 + v, a != v, raw);
                        }
                    const T L = lambda[i], M = mu[i];
                    const bool top = c.freeSurface3D && z == 4;
                    if (top) d[2][2] = -L / (L + 2 * M) * (d[0][0] + d[1][1]);
                    const T tr = d[0][0] + d[1][1] + d[2][2];
                    field[3][i] += dt * (L * tr + 2 * M * d[0][0]);
                    field[4][i] += dt * (L * tr + 2 * M * d[1][1]);
                    field[5][i] = top ? T(0) : field[5][i] + dt * (L * tr + 2 * M * d[2][2]);
                    field[6][i] += dt * shearMu(i, st[0], st[1]) * (d[0][1] + d[1][0]);
                    field[7][i] += dt * shearMu(i, st[1], st[2]) * (d[1][2] + d[2][1]);
                    field[8][i] += dt * shearMu(i, st[0], st[2]) * (d[0][2] + d[2][0]);
                    for (int f = 3; f < 9; ++f)
                        if (!std::isfinite(double(field[f][i]))) bad = true;
                }
        nonFinite = nonFinite || bad;
    }

    // 3x3x3 Gaussian-weighted Ricker source (cuda/Cuda_Seis3D.cu:313-332).
    void source(const seis3d_source& s, double time) {
        const double phase = 3.141592653589793 * c.frequency3D * (time - 1.2 / c.frequency3D);
        const double rickerD = (1 - 2 * phase * phase) * std::exp(-phase * phase);
        for (int a = 0; a < 27; ++a) {
            const int dx = a % 3 - 1, dy = (a / 3) % 3 - 1, dz = a / 9 - 1;
            const std::size_t i = at(s.x3D + c.ox3D + dx, s.y3D + c.oy3D + dy, s.z3D + c.oz3D + dz);
            const int r2 = dx * dx + dy * dy + dz * dz;
            T value;
            if (sizeof(T) == 4) {
                const float ricker = float(rickerD);
                value = T(c.dt3D * s.amplitude3D * ricker * std::exp(-0.5f * float(r2)) / 10.8387785335f);
            } else {
                const double norm = std::pow(1.0 + 2.0 * std::exp(-0.5), 3.0);
                value = T(double(c.dt3D) * double(s.amplitude3D) * rickerD * std::exp(-0.5 * r2) / norm);
            }
            if (s.kind3D == SEIS3D_SOURCE_EXPLOSION) {
                field[3][i] += value; field[4][i] += value; field[5][i] += value;
            } else {
                const std::size_t st[3] = {1, sy, sz};
                for (int v = 0; v < 3; ++v) {
                    const T A = invRho[i], B = invRho[i + st[v]];
                    field[v][i] += value * T(s.direction3D[v]) * (2 * A * B / (A + B));
                }
            }
        }
    }

    // Slip-wall images per axis with stagger parity (cuda/Cuda_Seis3D.cu:152-185).
    void reflectingWalls(bool velocities) {
        const int len[3] = {c.gx3D, c.gy3D, c.gz3D};
        for (int axis = 0; axis < 3; ++axis) {
            const int ua = (axis + 1) % 3, va = (axis + 2) % 3;
            const int high = len[axis] - kRadius - 1;
            for (int v = 0; v < len[va]; ++v)
                for (int u = 0; u < len[ua]; ++u) {
                    int p[3] = {0, 0, 0};
                    p[ua] = u; p[va] = v;
                    for (int f = velocities ? 0 : 3; f < (velocities ? 3 : 9); ++f) {
                        const bool half = f < 3 ? f == axis : f == 6 ? axis != 2 : f == 7 ? axis != 0 : f == 8 ? axis != 1 : false;
                        for (int side = 0; side < 2; ++side)
                            for (int depth = 1; depth <= kRadius; ++depth) {
                                p[axis] = side ? high + depth : kRadius - depth;
                                const std::size_t dst = at(p[0], p[1], p[2]);
                                if (half && !side && depth == 1) { field[f][dst] = 0; continue; }
                                p[axis] = side ? high + 1 - depth - int(half) : kRadius + depth - 1 - int(half);
                                const T value = field[f][at(p[0], p[1], p[2])];
                                field[f][dst] = half ? -value : value;
                            }
                        if (half) { p[axis] = high; field[f][at(p[0], p[1], p[2])] = 0; }
                    }
                }
        }
    }

    // One leapfrog step in the launch order of runStep3D (cuda/Cuda_Seis3D.cu:602-624).
    void step(const seis3d_source& s, uint64_t n) {
        if (g_storage && (g_storageMask & 4) && !roundedMaterials) {
            storeRounded(invRho); storeRounded(lambda); storeRounded(mu);
            roundedMaterials = true;
        }
        if (c.freeSurface3D) stressGhosts();
        if (c.reflecting3D) reflectingWalls(false);
        velocity();
        if (s.kind3D == SEIS3D_SOURCE_FORCE) source(s, double(n) * double(c.dt3D));
        if (g_storage && (g_storageMask & 1)) for (int k = 0; k < 3; ++k) storeRounded(field[k]);
        if (c.freeSurface3D) velocityGhosts();
        if (c.reflecting3D) reflectingWalls(true);
        if (g_storage && (g_storageMask & 1)) for (int k = 0; k < 3; ++k) storeRounded(field[k]);
        stress();
        if (s.kind3D == SEIS3D_SOURCE_EXPLOSION) source(s, (double(n) + 0.5) * double(c.dt3D));
        if (c.freeSurface3D) stressGhosts();
        if (c.reflecting3D) reflectingWalls(false);
        if (g_storage && (g_storageMask & 2)) for (int k = 3; k < 9; ++k) storeRounded(field[k]);
    }
    bool roundedMaterials = false;

    // Collocated receiver velocities (cuda/Cuda_Seis3D.cu:335-352, 421-428): [vx, vy, vz].
    void sample(const seis3d_receiver* r, int count, double* out) const {
        for (int k = 0; k < count; ++k) {
            const std::size_t i = at(r[k].x3D + c.ox3D, r[k].y3D + c.oy3D, r[k].z3D + c.oz3D);
            const T h = T(0.5);
            out[3 * k + 0] = double(h * (field[0][i] + field[0][i - 1]));
            out[3 * k + 1] = double(h * (field[1][i] + field[1][i - sy]));
            out[3 * k + 2] = double(h * (field[2][i] + field[2][i - sz]));
        }
    }
};

struct Handle {
    int precision = 32;
    std::unique_ptr<State<float>> f32;
    std::unique_ptr<State<double>> f64;
};

thread_local std::string lastMessage;

}  // namespace

// seis3d_oracle_gpu.cu includes this file for its host pieces (validation, CPML profiles) and
// defines its own C API.
#ifndef SEIS3D_ORACLE_HOST_ONLY
extern "C" {

const char* oracle3d_last_error(void) { return lastMessage.c_str(); }

// Storage emulation of later steps: precision 0 none, 1 FP16, 2 BF16; mask of the arrays
// (1 velocities, 2 stresses, 4 materials).
void oracle3d_set_psi_storage(int precision) { g_psiStorage = precision; }

void oracle3d_set_min_pml(int cells) { g_minPml = cells >= 4 && cells <= 8 ? cells : 8; }

void oracle3d_set_storage(int precision, int mask) {
    g_storage = precision;
    g_storageMask = mask;
}

void oracle3d_set_threads(int threads) {
#ifdef _OPENMP
    omp_set_num_threads(threads > 0 ? threads : omp_get_num_procs());
#else
    (void)threads;
#endif
}

int oracle3d_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// 0 = accepted (context derived in place), 1 = rejected.
int oracle3d_validate(seis3d_context* c) {
    lastMessage = validate(*c);
    return lastMessage.empty() ? 0 : 1;
}

int oracle3d_estimate_memory(const seis3d_context* context, seis3d_memory_budget* b) {
    seis3d_context c = *context;
    lastMessage = validate(c);
    if (!lastMessage.empty()) return 1;
    *b = seis3d_memory_budget{};
    b->fieldBytes3D = c.cells3D * 12 * sizeof(float);
    for (int a = 0; a < 3; ++a) b->cpmlBytes3D += slabCells(c, a) * 6 * sizeof(float);
    const auto l = viewLayout(c);
    b->viewBytes3D = l.totalSamples3D * 4 * sizeof(float) + l.volumeOffset3D * 4 +
                     uint64_t(SEIS3D_MAX_VOLUME_OUTPUT) * SEIS3D_MAX_VOLUME_OUTPUT * 4;
    b->totalBytes3D = b->fieldBytes3D + b->cpmlBytes3D + b->viewBytes3D +
                      uint64_t(c.gx3D + c.gy3D + c.gz3D) * 6 * sizeof(float) +
                      uint64_t(SEIS3D_MAX_RECEIVERS) * (sizeof(seis3d_receiver) + 3 * sizeof(float)) + 2 * 1024 * 1024;
    return 0;
}

// FP32 coefficient table exactly as the reference stores it (n*6 floats).
int oracle3d_make_coefficients(const seis3d_context* c, int axis, float* out) {
    const auto p = profile(*c, axis);
    for (std::size_t i = 0; i < p.size(); ++i) out[i] = float(p[i]);
    return int(p.size());
}

void* oracle3d_create(const seis3d_context* c, int precision) {
    try {
        auto h = new Handle;
        h->precision = precision == 64 ? 64 : 32;
        if (h->precision == 64) h->f64.reset(new State<double>(*c));
        else h->f32.reset(new State<float>(*c));
        return h;
    } catch (const std::exception& e) {
        lastMessage = e.what();
        return nullptr;
    }
}

void oracle3d_destroy(void* handle) { delete static_cast<Handle*>(handle); }

#define ORACLE_DISPATCH(h, call) \
    (static_cast<Handle*>(h)->precision == 64 ? static_cast<Handle*>(h)->f64->call : static_cast<Handle*>(h)->f32->call)

void oracle3d_generate_materials(void* h) { ORACLE_DISPATCH(h, generate()); }
void oracle3d_reset(void* h) { ORACLE_DISPATCH(h, reset()); }

int oracle3d_upload_plane(void* h, int z, const float* values) {
    lastMessage = ORACLE_DISPATCH(h, uploadPlane(z, values));
    return lastMessage.empty() ? 0 : 1;
}

void oracle3d_finish_upload(void* h) { ORACLE_DISPATCH(h, finishUpload()); }

void oracle3d_step(void* h, const seis3d_source* s, uint64_t step) { ORACLE_DISPATCH(h, step(*s, step)); }

void oracle3d_run(void* h, const seis3d_source* s, uint64_t first, int count) {
    for (int k = 0; k < count; ++k) ORACLE_DISPATCH(h, step(*s, first + uint64_t(k)));
}

// Run `count` steps from `first`, sampling the receivers after every step whose
// (step+1) % stride == 0 (src/Seis3D_Sim.cpp:127-132) into out[sample][r][3].
int oracle3d_run_gather(void* h, const seis3d_source* s, uint64_t first, int count,
                        const seis3d_receiver* r, int nr, int stride, double* out, int capacity) {
    int taken = 0;
    for (int k = 0; k < count; ++k) {
        const uint64_t n = first + uint64_t(k);
        ORACLE_DISPATCH(h, step(*s, n));
        if (stride > 0 && (n + 1) % uint64_t(stride) == 0 && taken < capacity) {
            ORACLE_DISPATCH(h, sample(r, nr, out + std::size_t(taken) * nr * 3));
            ++taken;
        }
    }
    return taken;
}

void oracle3d_sample(void* h, const seis3d_receiver* r, int count, double* out) { ORACLE_DISPATCH(h, sample(r, count, out)); }

// Copy one field (0-8 wavefields, 9 = 1/rho, 10 = lambda, 11 = mu) as double, reference layout.
void oracle3d_get_field(void* handle, int f, double* out) {
    auto* h = static_cast<Handle*>(handle);
    auto copy = [&](auto& st) {
        const auto& src = f < 9 ? st.field[f] : f == 9 ? st.invRho : f == 10 ? st.lambda : st.mu;
        for (std::size_t i = 0; i < src.size(); ++i) out[i] = double(src[i]);
    };
    if (h->precision == 64) copy(*h->f64); else copy(*h->f32);
}

// Overwrite one field from double values (reference layout), e.g. to seed a test state.
void oracle3d_set_field(void* handle, int f, const double* in) {
    auto* h = static_cast<Handle*>(handle);
    auto put = [&](auto& st) {
        using T = typename std::remove_reference<decltype(st.invRho)>::type::value_type;
        auto& dst = f < 9 ? st.field[f] : f == 9 ? st.invRho : f == 10 ? st.lambda : st.mu;
        for (std::size_t i = 0; i < dst.size(); ++i) dst[i] = T(in[i]);
    };
    if (h->precision == 64) put(*h->f64); else put(*h->f32);
}

int oracle3d_non_finite(void* h) { return ORACLE_DISPATCH(h, nonFinite) ? 1 : 0; }

}  // extern "C"
#endif  // SEIS3D_ORACLE_HOST_ONLY
