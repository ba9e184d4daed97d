// seis3d_kernels.cuh - sm_100a kernels of the 3-D elastic velocity-stress solver.
//
// The time step is two z-marching passes (velocity, then stress).  Each CTA owns a
// 32 x 8 column tile of the xy plane and walks a chunk of z planes:
//   * every plane of the tile arrives through a 3-deep ring of shared-memory stages
//     filled by TMA tile copies (halo tiles for the x/y derivatives, centre tiles for
//     the read-modify-write and for the z rings), so HBM latency overlaps compute;
//   * z derivatives come from per-thread register rings of 8 planes (no re-reads);
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
#include "seis3d_tma.cuh"

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
// Shared pieces of the two z-marching passes.  A CTA is 8 warps; warp w owns row y0+w of a
// 32 x 8 column tile and marches the tile's z chunk on its own: no block-wide barrier runs
// in the plane loop.  Planes arrive through a ring of TMA stages (seis3d_tma.cuh); a warp
// waits on the stage's mbarrier, computes, then releases the stage, and the last warp to
// release a stage refills it with the plane kStages ahead.  Warps of a CTA therefore drift
// by up to kStages planes, so one warp's CPML memory latency does not stall the others.
// ---------------------------------------------------------------------------------------
constexpr int kTX = 32, kTY = 8, kThreads = kTX * kTY;
#ifndef SEIS3D_MIN_BLOCKS
#define SEIS3D_MIN_BLOCKS 3   // resident CTAs per SM the register allocation is sized for
#endif

struct StageRing {
    uint64_t full[tma::kStages];
    int released[tma::kStages];
    int issued;      // stages issued so far (monotonic)
    int stalled;     // set when a stage did not arrive within the wait bound
};

// Warp-uniform bounded wait for stage j.
__device__ __forceinline__ bool waitFull(StageRing& R, int j) {
    volatile int* stalled = &R.stalled;
    bool ok = !*stalled && tma::waitStage(&R.full[j % tma::kStages], (j / tma::kStages) & 1);
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && threadIdx.x == 0) *stalled = 1;
    return ok;
}

// Release stage j; the last of the kTY warps refills its buffer with stage j + kStages.
template <class Issue> __device__ __forceinline__ void releaseStage(StageRing& R, int j, int nPlanes, Issue&& issue) {
    __syncwarp();
    if (threadIdx.x == 0) {
        __threadfence_block();
        const int b = j % tma::kStages;
        if (atomicAdd(&R.released[b], 1) == kTY - 1) {
            R.released[b] = 0;
            __threadfence_block();
            tma::fenceProxyAsync();
            if (j + tma::kStages < nPlanes) {
                issue(j + tma::kStages);
                R.issued = j + tma::kStages + 1;
            }
        }
    }
}

// After a stall: report it and wait (bounded) for the copies still in flight.
__device__ __forceinline__ void drainAfterStall(const Fields& F, StageRing& R, int consumed) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        atomicOr(F.status + 1, 1u);
        for (int j = consumed; j < R.issued; ++j)
            tma::waitStage(&R.full[j % tma::kStages], (j / tma::kStages) & 1);
    }
}

__device__ __forceinline__ void initRing(StageRing& R) {
    for (int b = 0; b < tma::kStages; ++b) {
        tma::barrierInit(&R.full[b], 1);
        R.released[b] = 0;
    }
    R.issued = 0;
    R.stalled = 0;
    tma::barrierInitFence();
}

// CPML coefficient table of the tile: x nodes of the 32 columns and y nodes of the 8 rows,
// {a, b, 1/kappa} at centre (h = 0) and half grid (h = 1).
struct TileCoefficients {
    float x[2][3][kTX];
    float y[2][3][kTY];
};

__device__ __forceinline__ void loadTileCoefficients(TileCoefficients& T, const Fields& F, const Geometry& G, int x0,
                                                     int y0, int tid) {
    if (G.reflecting) return;
    for (int e = tid; e < 6 * kTX; e += kThreads) {
        const int h = e / (3 * kTX), j = (e / kTX) % 3, c = e % kTX;
        const int x = min(x0 + c, G.gx - 1);
        T.x[h][j][c] = F.coef[0][(int64_t(h) * G.gx + x) * 3 + j];
    }
    for (int e = tid; e < 6 * kTY; e += kThreads) {
        const int h = e / (3 * kTY), j = (e / kTY) % 3, r = e % kTY;
        const int y = min(y0 + r, G.gy - 1);
        T.y[h][j][r] = F.coef[1][(int64_t(h) * G.gy + y) * 3 + j];
    }
}

// psi = b psi + a d; returns d/kappa + psi (cuda/Cuda_Seis3D.cu:109-110).
__device__ __forceinline__ float cpmlApply(float d, float& m, float a, float b, float ik) {
    m = b * m + a * d;
    return ik * d + m;
}

// ---------------------------------------------------------------------------------------
// Velocity pass: v(n+1/2) = v(n-1/2) + dt * 2ab/(a+b) * sum_axis CPML(D sigma)
// (cuda/Cuda_Seis3D.cu:222-245) with the force source fused (:313-332).
// Stage of plane k: sigma halo tiles of plane k, 1/rho tile of k and centre of k+1,
// v centres of k, and the ring feeds sigma_xz/sigma_yz(k+3), sigma_zz(k+4).
// ---------------------------------------------------------------------------------------
struct VelocityStage {
    static constexpr int XX = 0, XY = 320, XZ = 960, YY = 1280, YZ = 1792, B = 2304, B1 = 2656, V = 2912,
                         FXZ = 3680, FYZ = 3936, FZZ = 4192, SIZE = 4448;
    static constexpr uint32_t BYTES = 4u * (320 + 640 + 320 + 512 + 512 + 324 + 256 + 768 + 256 + 256 + 256);
};

__global__ void __launch_bounds__(kThreads, SEIS3D_MIN_BLOCKS) velocityPass(Geometry G, Fields F, SourceParams S, int zChunk) {
    using St = VelocityStage;
    extern __shared__ __align__(128) float smem[];
    __shared__ StageRing R;
    __shared__ TileCoefficients T;

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx;
    const int x0 = kRadius + blockIdx.x * kTX, y0 = kRadius + blockIdx.y * kTY;
    const int x = x0 + tx, y = y0 + ty;
    const bool active = x < G.gx - kRadius && y < G.gy - kRadius;
    const int zBegin = kRadius + blockIdx.z * zChunk;
    const int zEnd = min(zBegin + zChunk, G.gz - kRadius);
    if (zBegin >= zEnd) return;
    const int nPlanes = zEnd - zBegin;
    const int64_t P = G.pitch, PL = G.plane;
    const int64_t col = int64_t(min(y, G.gy - 1)) * P + min(x, G.gx - 1);
    const float inv = G.invH;
    const CUtensorMap* M = F.maps;

    auto issue = [&](int j) {
        float* st = smem + (j % tma::kStages) * St::SIZE;
        uint64_t* bar = &R.full[j % tma::kStages];
        const int k = zBegin + j;
        tma::arriveExpectTx(bar, St::BYTES);
        tma::load3d(st + St::XX, M + tma::kSxxX, x0 - 4, y0, k, bar);
        tma::load3d(st + St::XY, M + tma::kSxyXY, x0 - 4, y0 - 4, k, bar);
        tma::load3d(st + St::XZ, M + tma::kSxzX, x0 - 4, y0, k, bar);
        tma::load3d(st + St::YY, M + tma::kSyyY, x0, y0 - 4, k, bar);
        tma::load3d(st + St::YZ, M + tma::kSyzY, x0, y0 - 4, k, bar);
        tma::load3d(st + St::B, M + tma::kRhoT, x0, y0, k, bar);
        tma::load3d(st + St::B1, M + tma::kCenter0 + 9, x0, y0, k + 1, bar);
        tma::load3d(st + St::V, M + tma::kCenter0 + 0, x0, y0, k, bar);
        tma::load3d(st + St::V + 256, M + tma::kCenter0 + 1, x0, y0, k, bar);
        tma::load3d(st + St::V + 512, M + tma::kCenter0 + 2, x0, y0, k, bar);
        tma::load3d(st + St::FXZ, M + tma::kCenter0 + 8, x0, y0, k + 3, bar);
        tma::load3d(st + St::FYZ, M + tma::kCenter0 + 7, x0, y0, k + 3, bar);
        tma::load3d(st + St::FZZ, M + tma::kCenter0 + 5, x0, y0, k + 4, bar);
    };

    if (tid == 0) initRing(R);
    loadTileCoefficients(T, F, G, x0, y0, tid);
    __syncthreads();
    if (tid == 0) {
        const int first = min(tma::kStages, nPlanes);
        for (int j = 0; j < first; ++j) issue(j);
        R.issued = first;
    }

    // CPML slab membership: x and y are fixed per thread, z per plane.
    const bool cp = !G.reflecting;
    const int qx = cp && active ? slabIndex(x, G.gx, G.pml, false) : -1;
    const int qy = cp && active ? slabIndex(y, G.gy, G.pml, false) : -1;
    const bool topFree = G.freeSurface != 0;
    const int64_t slotX = int64_t(G.gz) * G.gy * G.thick[0];
    const int64_t slotY = int64_t(G.gz) * G.thick[1] * P;
    const int64_t slotZ = int64_t(G.thick[2]) * G.gy * P;
    float* px = qx >= 0 ? F.psi[0] + (int64_t(zBegin) * G.gy + y) * G.thick[0] + qx : nullptr;
    float* py = qy >= 0 ? F.psi[1] + (int64_t(zBegin) * G.thick[1] + qy) * P + x : nullptr;
    auto zSlab = [&](int z) -> float* {
        const int qz = cp && active ? slabIndex(z, G.gz, G.pml, topFree) : -1;
        return qz >= 0 ? F.psi[2] + (int64_t(qz) * G.gy + y) * P + x : nullptr;
    };
    float* pz = zSlab(zBegin);
    // psi of the current plane, loaded one plane ahead.
    float mx[3] = {0, 0, 0}, my[3] = {0, 0, 0}, mz[3] = {0, 0, 0};
#pragma unroll
    for (int s3 = 0; s3 < 3; ++s3) {
        if (px) mx[s3] = px[s3 * slotX];
        if (py) my[s3] = py[s3 * slotY];
        if (pz) mz[s3] = pz[s3 * slotZ];
    }

    float* const vx = F.f[0];
    float* const vy = F.f[1];
    float* const vz = F.f[2];

    // z rings: rXZ/rYZ hold planes z-4..z+3 (D-), rZZ planes z-3..z+4 (D+); the leading
    // element of each arrives with the stage.
    float rXZ[8], rYZ[8], rZZ[8];
    if (active) {
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            rXZ[k] = F.f[8][int64_t(zBegin - 4 + k) * PL + col];
            rYZ[k] = F.f[7][int64_t(zBegin - 4 + k) * PL + col];
            rZZ[k] = F.f[5][int64_t(zBegin - 3 + k) * PL + col];
        }
    }
    const unsigned long long step = F.clock->step;
    const bool forceHere = S.kind == 1 && active && abs(x - S.gxs) <= 1 && abs(y - S.gys) <= 1;
    bool bad = false;
    int consumed = 0;

    for (int j = 0; j < nPlanes; ++j) {
        const int z = zBegin + j;
        if (!waitFull(R, j)) break;
        if (active) {
            const float* st = smem + (j % tma::kStages) * St::SIZE;
            const int c = ty * kTX + tx;
            rXZ[7] = st[St::FXZ + c];
            rYZ[7] = st[St::FYZ + c];
            rZZ[7] = st[St::FZZ + c];
            const int64_t i = int64_t(z) * PL + col;

            // vx: D+x sxx, D-y sxy, D-z sxz.  vy: D-x sxy, D+y syy, D-z syz.  vz: D-x sxz, D-y syz, D+z szz.
            float dx0 = diffRow<40>(st + St::XX + ty * 40 + tx + 1, inv);
            float dy0 = diffCol<40>(st + St::XY + ty * 40 + tx + 4, inv);
            float dz0 = diffRing(rXZ, inv);
            float dx1 = diffRow<40>(st + St::XY + (ty + 4) * 40 + tx, inv);
            float dy1 = diffCol<32>(st + St::YY + (ty + 1) * 32 + tx, inv);
            float dz1 = diffRing(rYZ, inv);
            float dx2 = diffRow<40>(st + St::XZ + ty * 40 + tx, inv);
            float dy2 = diffCol<32>(st + St::YZ + ty * 32 + tx, inv);
            float dz2 = diffRing(rZZ, inv);

            if (px) {
                dx0 = cpmlApply(dx0, mx[0], T.x[1][0][tx], T.x[1][1][tx], T.x[1][2][tx]);
                dx1 = cpmlApply(dx1, mx[1], T.x[0][0][tx], T.x[0][1][tx], T.x[0][2][tx]);
                dx2 = cpmlApply(dx2, mx[2], T.x[0][0][tx], T.x[0][1][tx], T.x[0][2][tx]);
                px[0] = mx[0]; px[slotX] = mx[1]; px[2 * slotX] = mx[2];
            }
            if (py) {
                dy0 = cpmlApply(dy0, my[0], T.y[0][0][ty], T.y[0][1][ty], T.y[0][2][ty]);
                dy1 = cpmlApply(dy1, my[1], T.y[1][0][ty], T.y[1][1][ty], T.y[1][2][ty]);
                dy2 = cpmlApply(dy2, my[2], T.y[0][0][ty], T.y[0][1][ty], T.y[0][2][ty]);
                py[0] = my[0]; py[slotY] = my[1]; py[2 * slotY] = my[2];
            }
            if (pz) {
                const float* kz = F.coef[2] + int64_t(z) * 3;
                const float* kh = F.coef[2] + (int64_t(G.gz) + z) * 3;
                dz0 = cpmlApply(dz0, mz[0], kz[0], kz[1], kz[2]);
                dz1 = cpmlApply(dz1, mz[1], kz[0], kz[1], kz[2]);
                dz2 = cpmlApply(dz2, mz[2], kh[0], kh[1], kh[2]);
                pz[0] = mz[0]; pz[slotZ] = mz[1]; pz[2 * slotZ] = mz[2];
            }

            float div0 = 0.0f; div0 += dx0; div0 += dy0; div0 += dz0;
            float div1 = 0.0f; div1 += dx1; div1 += dy1; div1 += dz1;
            float div2 = 0.0f; div2 += dx2; div2 += dy2; div2 += dz2;

            const float* sb = st + St::B + ty * 36 + tx;
            const float a = sb[0], bx = sb[1], by = sb[36], bz = st[St::B1 + c];
            const float cx = 2 * a * bx / (a + bx);
            const float cy = 2 * a * by / (a + by);
            const float cz = 2 * a * bz / (a + bz);
            float v0 = st[St::V + c] + G.dt * cx * div0;
            float v1 = st[St::V + 256 + c] + G.dt * cy * div1;
            float v2 = st[St::V + 512 + c] + G.dt * cz * div2;
            if (forceHere && abs(z - S.gzs) <= 1) {
                const float value = sourceValue(G, S, x - S.gxs, y - S.gys, z - S.gzs, double(step) * G.dt);
                v0 += value * S.direction[0] * cx;
                v1 += value * S.direction[1] * cy;
                v2 += value * S.direction[2] * cz;
            }
            vx[i] = v0; vy[i] = v1; vz[i] = v2;
            bad |= !isfinite(v0) || !isfinite(v1) || !isfinite(v2);
#pragma unroll
            for (int k = 0; k < 7; ++k) { rXZ[k] = rXZ[k + 1]; rYZ[k] = rYZ[k + 1]; rZZ[k] = rZZ[k + 1]; }

            // Prefetch the CPML memories of the next plane.
            if (j + 1 < nPlanes) {
                if (px) {
                    px += int64_t(G.gy) * G.thick[0];
#pragma unroll
                    for (int s3 = 0; s3 < 3; ++s3) mx[s3] = px[s3 * slotX];
                }
                if (py) {
                    py += int64_t(G.thick[1]) * P;
#pragma unroll
                    for (int s3 = 0; s3 < 3; ++s3) my[s3] = py[s3 * slotY];
                }
                pz = zSlab(z + 1);
                if (pz) {
#pragma unroll
                    for (int s3 = 0; s3 < 3; ++s3) mz[s3] = pz[s3 * slotZ];
                }
            }
        }
        releaseStage(R, j, nPlanes, issue);
        consumed = j + 1;
    }
    if (R.stalled) drainAfterStall(F, R, consumed);
    flagNonFinite(F, bad);
}

// ---------------------------------------------------------------------------------------
// Stress pass: sigma(n+1) from CPML-filtered velocity derivatives (cuda/Cuda_Seis3D.cu:281-310),
// harmonic shear moduli (:275-278) from reciprocals carried plane to plane in registers,
// free-surface closure at z=4 (:299, :303) and the explosion source fused (:313-332).
// Stage of plane k: velocity cross tiles of k, mu tiles of k and k+1, lambda and the six
// stresses of k, and the ring feeds vx/vy(k+4), vz(k+3).
// ---------------------------------------------------------------------------------------
struct StressStage {
    static constexpr int VX = 0, VY = 640, VZ = 1280, M0 = 1920, M1 = 2272, L = 2624, S = 2880, FVX = 4416,
                         FVY = 4672, FVZ = 4928, SIZE = 5184;
    static constexpr uint32_t BYTES = 4u * (3 * 640 + 2 * 324 + 256 + 6 * 256 + 3 * 256);
};

__global__ void __launch_bounds__(kThreads, SEIS3D_MIN_BLOCKS) stressPass(Geometry G, Fields F, SourceParams S, int zChunk) {
    using St = StressStage;
    extern __shared__ __align__(128) float smem[];
    __shared__ StageRing R;
    __shared__ TileCoefficients T;

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx;
    const int x0 = kRadius + blockIdx.x * kTX, y0 = kRadius + blockIdx.y * kTY;
    const int x = x0 + tx, y = y0 + ty;
    const bool active = x < G.gx - kRadius && y < G.gy - kRadius;
    const int zBegin = kRadius + blockIdx.z * zChunk;
    const int zEnd = min(zBegin + zChunk, G.gz - kRadius);
    if (zBegin >= zEnd) return;
    const int nPlanes = zEnd - zBegin;
    const int64_t P = G.pitch, PL = G.plane;
    const int64_t col = int64_t(min(y, G.gy - 1)) * P + min(x, G.gx - 1);
    const float inv = G.invH;
    const CUtensorMap* M = F.maps;

    auto issue = [&](int j) {
        float* st = smem + (j % tma::kStages) * St::SIZE;
        uint64_t* bar = &R.full[j % tma::kStages];
        const int k = zBegin + j;
        tma::arriveExpectTx(bar, St::BYTES);
        tma::load3d(st + St::VX, M + tma::kVxXY, x0 - 4, y0 - 4, k, bar);
        tma::load3d(st + St::VY, M + tma::kVyXY, x0 - 4, y0 - 4, k, bar);
        tma::load3d(st + St::VZ, M + tma::kVzXY, x0 - 4, y0 - 4, k, bar);
        tma::load3d(st + St::M0, M + tma::kMuT, x0, y0, k, bar);
        tma::load3d(st + St::M1, M + tma::kMuT, x0, y0, k + 1, bar);
        tma::load3d(st + St::L, M + tma::kCenter0 + 10, x0, y0, k, bar);
#pragma unroll
        for (int f = 0; f < 6; ++f) tma::load3d(st + St::S + 256 * f, M + tma::kCenter0 + 3 + f, x0, y0, k, bar);
        tma::load3d(st + St::FVX, M + tma::kCenter0 + 0, x0, y0, k + 4, bar);
        tma::load3d(st + St::FVY, M + tma::kCenter0 + 1, x0, y0, k + 4, bar);
        tma::load3d(st + St::FVZ, M + tma::kCenter0 + 2, x0, y0, k + 3, bar);
    };

    if (tid == 0) initRing(R);
    loadTileCoefficients(T, F, G, x0, y0, tid);
    __syncthreads();
    if (tid == 0) {
        const int first = min(tma::kStages, nPlanes);
        for (int j = 0; j < first; ++j) issue(j);
        R.issued = first;
    }

    const bool cp = !G.reflecting;
    const int qx = cp && active ? slabIndex(x, G.gx, G.pml, false) : -1;
    const int qy = cp && active ? slabIndex(y, G.gy, G.pml, false) : -1;
    const bool topFree = G.freeSurface != 0;
    const int64_t slotX = int64_t(G.gz) * G.gy * G.thick[0];
    const int64_t slotY = int64_t(G.gz) * G.thick[1] * P;
    const int64_t slotZ = int64_t(G.thick[2]) * G.gy * P;
    float* px = qx >= 0 ? F.psi[0] + 3 * slotX + (int64_t(zBegin) * G.gy + y) * G.thick[0] + qx : nullptr;
    float* py = qy >= 0 ? F.psi[1] + 3 * slotY + (int64_t(zBegin) * G.thick[1] + qy) * P + x : nullptr;
    auto zSlab = [&](int z) -> float* {
        const int qz = cp && active ? slabIndex(z, G.gz, G.pml, topFree) : -1;
        return qz >= 0 ? F.psi[2] + 3 * slotZ + (int64_t(qz) * G.gy + y) * P + x : nullptr;
    };
    float* pz = zSlab(zBegin);
    float mx[3] = {0, 0, 0}, my[3] = {0, 0, 0}, mz[3] = {0, 0, 0};
#pragma unroll
    for (int s3 = 0; s3 < 3; ++s3) {
        if (px) mx[s3] = px[s3 * slotX];
        if (py) my[s3] = py[s3 * slotY];
        if (pz) mz[s3] = pz[s3 * slotZ];
    }

    // Reciprocal shear moduli 1/mu at (x,y), (x+1,y), (x,y+1), (x+1,y+1) of the current
    // plane (IEEE division, as the reference's 1/m): mu == 0 gives +inf, so the harmonic
    // means below are exactly 0 there, as the reference's fluid branch returns.
    float r00 = 0, r10 = 0, r01 = 0, r11 = 0;
    if (active) {
        const float* m = F.mu + int64_t(zBegin) * PL + col;
        r00 = 1.0f / m[0]; r10 = 1.0f / m[1]; r01 = 1.0f / m[P]; r11 = 1.0f / m[P + 1];
    }

    // z rings: rVX/rVY planes z-3..z+4 (D+), rVZ planes z-4..z+3 (D-).
    float rVX[8], rVY[8], rVZ[8];
    if (active) {
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            rVX[k] = F.f[0][int64_t(zBegin - 3 + k) * PL + col];
            rVY[k] = F.f[1][int64_t(zBegin - 3 + k) * PL + col];
            rVZ[k] = F.f[2][int64_t(zBegin - 4 + k) * PL + col];
        }
    }
    const unsigned long long step = F.clock->step;
    const bool blastHere = S.kind == 0 && active && abs(x - S.gxs) <= 1 && abs(y - S.gys) <= 1;
    bool bad = false;
    int consumed = 0;

    for (int j = 0; j < nPlanes; ++j) {
        const int z = zBegin + j;
        if (!waitFull(R, j)) break;
        if (active) {
            const float* st = smem + (j % tma::kStages) * St::SIZE;
            const int c = ty * kTX + tx;
            rVX[7] = st[St::FVX + c];
            rVY[7] = st[St::FVY + c];
            rVZ[7] = st[St::FVZ + c];
            const int64_t i = int64_t(z) * PL + col;

            // d[v][a]: D- along its own axis, D+ across (cuda/Cuda_Seis3D.cu:293-295).
            float d00 = diffRow<40>(st + St::VX + (ty + 4) * 40 + tx, inv);
            float d01 = diffCol<40>(st + St::VX + (ty + 1) * 40 + tx + 4, inv);
            float d02 = diffRing(rVX, inv);
            float d10 = diffRow<40>(st + St::VY + (ty + 4) * 40 + tx + 1, inv);
            float d11 = diffCol<40>(st + St::VY + ty * 40 + tx + 4, inv);
            float d12 = diffRing(rVY, inv);
            float d20 = diffRow<40>(st + St::VZ + (ty + 4) * 40 + tx + 1, inv);
            float d21 = diffCol<40>(st + St::VZ + (ty + 1) * 40 + tx + 4, inv);
            float d22 = diffRing(rVZ, inv);

            if (px) {
                d00 = cpmlApply(d00, mx[0], T.x[0][0][tx], T.x[0][1][tx], T.x[0][2][tx]);
                d10 = cpmlApply(d10, mx[1], T.x[1][0][tx], T.x[1][1][tx], T.x[1][2][tx]);
                d20 = cpmlApply(d20, mx[2], T.x[1][0][tx], T.x[1][1][tx], T.x[1][2][tx]);
                px[0] = mx[0]; px[slotX] = mx[1]; px[2 * slotX] = mx[2];
            }
            if (py) {
                d01 = cpmlApply(d01, my[0], T.y[1][0][ty], T.y[1][1][ty], T.y[1][2][ty]);
                d11 = cpmlApply(d11, my[1], T.y[0][0][ty], T.y[0][1][ty], T.y[0][2][ty]);
                d21 = cpmlApply(d21, my[2], T.y[1][0][ty], T.y[1][1][ty], T.y[1][2][ty]);
                py[0] = my[0]; py[slotY] = my[1]; py[2 * slotY] = my[2];
            }
            if (pz) {
                const float* kz = F.coef[2] + int64_t(z) * 3;
                const float* kh = F.coef[2] + (int64_t(G.gz) + z) * 3;
                d02 = cpmlApply(d02, mz[0], kh[0], kh[1], kh[2]);
                d12 = cpmlApply(d12, mz[1], kh[0], kh[1], kh[2]);
                d22 = cpmlApply(d22, mz[2], kz[0], kz[1], kz[2]);
                pz[0] = mz[0]; pz[slotZ] = mz[1]; pz[2 * slotZ] = mz[2];
            }

            const float* m0 = st + St::M0 + ty * 36 + tx;
            const float* m1 = st + St::M1 + ty * 36 + tx;
            const float lambda = st[St::L + c], m = m0[0];
            const bool top = G.freeSurface && z == kRadius;
            if (top) d22 = -lambda / (lambda + 2 * m) * (d00 + d11);
            const float trace = d00 + d11 + d22;
            const float n00 = 1.0f / m1[0], n10 = 1.0f / m1[1], n01 = 1.0f / m1[36], n11 = 1.0f / m1[37];
            const float muXY = 4.0f / (r00 + r10 + r01 + r11);
            const float muYZ = 4.0f / (r00 + r01 + n00 + n01);
            const float muXZ = 4.0f / (r00 + r10 + n00 + n10);
            r00 = n00; r10 = n10; r01 = n01; r11 = n11;

            const float* so = st + St::S + c;
            float sxx = so[0] + G.dt * (lambda * trace + 2 * m * d00);
            float syy = so[256] + G.dt * (lambda * trace + 2 * m * d11);
            float szz = top ? 0.0f : so[512] + G.dt * (lambda * trace + 2 * m * d22);
            float sxy = so[768] + G.dt * muXY * (d01 + d10);
            float syz = so[1024] + G.dt * muYZ * (d12 + d21);
            float sxz = so[1280] + G.dt * muXZ * (d02 + d20);
            bad |= !isfinite(sxx) || !isfinite(syy) || !isfinite(szz) || !isfinite(sxy) || !isfinite(syz) ||
                   !isfinite(sxz);
            if (blastHere && abs(z - S.gzs) <= 1) {
                const float value = sourceValue(G, S, x - S.gxs, y - S.gys, z - S.gzs, (double(step) + 0.5) * G.dt);
                sxx += value; syy += value; szz += value;
            }
            F.f[3][i] = sxx; F.f[4][i] = syy; F.f[5][i] = szz;
            F.f[6][i] = sxy; F.f[7][i] = syz; F.f[8][i] = sxz;
#pragma unroll
            for (int k = 0; k < 7; ++k) { rVX[k] = rVX[k + 1]; rVY[k] = rVY[k + 1]; rVZ[k] = rVZ[k + 1]; }

            if (j + 1 < nPlanes) {
                if (px) {
                    px += int64_t(G.gy) * G.thick[0];
#pragma unroll
                    for (int s3 = 0; s3 < 3; ++s3) mx[s3] = px[s3 * slotX];
                }
                if (py) {
                    py += int64_t(G.thick[1]) * P;
#pragma unroll
                    for (int s3 = 0; s3 < 3; ++s3) my[s3] = py[s3 * slotY];
                }
                pz = zSlab(z + 1);
                if (pz) {
#pragma unroll
                    for (int s3 = 0; s3 < 3; ++s3) mz[s3] = pz[s3 * slotZ];
                }
            }
        }
        releaseStage(R, j, nPlanes, issue);
        consumed = j + 1;
    }
    if (R.stalled) drainAfterStall(F, R, consumed);
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
