// seis3d_kernels.cuh - sm_100a kernels of the 3-D elastic velocity-stress solver.
//
// The time step is two z-marching passes (velocity, then stress).  Each CTA owns a
// 32 x 16 column tile of the xy plane and walks a chunk of z planes:
//   * every plane of the tile arrives through a 3-deep ring of shared-memory stages
//     filled by TMA tile copies (halo tiles for the x/y derivatives, centre tiles for
//     the read-modify-write and for the z rings), so HBM latency overlaps compute;
//   * z derivatives come from per-thread register rings of 8 planes (no re-reads);
//   * the CPML recurrences run only for threads inside a slab and touch psi with
//     unit stride along x on every axis; each pass body is compiled twice, with and
//     without the CPML code, and a CTA whose tile and z chunk touch no slab runs the
//     CPML-free copy (the same arithmetic for its cells, 5 % off the step);
//   * the Ricker source is injected by the threads that own its 27 nodes, inside the
//     pass that the reference follows with sourceKernel3D (force: velocity pass,
//     explosion: stress pass);
//   * with a free surface the first z chunk of each pass writes the ghost-plane images its
//     z rings read, each thread for its own columns (velocity pass: stress images, stress
//     pass: velocity images);
//   * a second instantiation of each pass keeps the CPML memories in BF16
//     (SEIS3D_STORAGE_BF16_CPML), everything else unchanged;
//   * the non-finite check is a running FP32 sum of every output of the thread (a NaN or an
//     infinity anywhere makes it non-finite; finite values would have to exceed 3e38 to
//     raise it falsely), tested once per thread and reduced per warp to one atomic.
// Arithmetic per node follows the reference expression by expression so that FP32
// results agree to rounding (cuda/Cuda_Seis3D.cu:78-111, :222-245, :275-310, :313-332).
#pragma once

#include <cuda_bf16.h>

#include <type_traits>

#include "seis3d_device.cuh"
#include "seis3d_tma.cuh"

namespace seis3d {

// Eighth-order staggered weights (cuda/Cuda_Seis3D.cu:72-75).
#define SEIS3D_W0 (1225.0f / 1024.0f)
#define SEIS3D_W1 (-245.0f / 3072.0f)
#define SEIS3D_W2 (49.0f / 5120.0f)
#define SEIS3D_W3 (-5.0f / 7168.0f)

// First derivative from an 8-sample window s[0..7]: for D- the window starts at i-4,
// for D+ at i-3; both reduce to (sum_r w_r (s[4+r] - s[3-r])) / h accumulated r = 0..3
// (cuda/Cuda_Seis3D.cu:78-89).  `w` holds the four weights and 1/h (Geometry::w), and the
// sum is scaled after it as the reference does.  Weights pre-divided by h save the multiply
// but round each weight separately: a fixed perturbation of the stencil that, measured
// against an FP64 run of the 300x50x300 layered shot (2000 steps), doubled the gather's
// distance to FP64 for 0.3 % of the step time.  The scale is an explicit IEEE multiply so
// that no caller's addition absorbs it into a fused multiply-add: the pass bodies with and
// without the CPML code then round every derivative alike, and results do not depend on the
// launch shape.
__device__ __forceinline__ float diff8(float s0, float s1, float s2, float s3, float s4, float s5, float s6,
                                       float s7, const float* w) {
    float r = w[0] * (s4 - s3);
    r += w[1] * (s5 - s2);
    r += w[2] * (s6 - s1);
    r += w[3] * (s7 - s0);
    return __fmul_rn(r, w[4]);
}

__device__ __forceinline__ float diffRing(const float (&s)[8], const float* inv) {
    return diff8(s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], inv);
}

// Row window of a shared tile (x derivative).
template <int W> __device__ __forceinline__ float diffRow(const float* row, const float* inv) {
    return diff8(row[0], row[1], row[2], row[3], row[4], row[5], row[6], row[7], inv);
}

// Column window of a shared tile (y derivative), `W` = row length.
template <int W> __device__ __forceinline__ float diffCol(const float* col, const float* inv) {
    return diff8(col[0], col[W], col[2 * W], col[3 * W], col[4 * W], col[5 * W], col[6 * W], col[7 * W], inv);
}

// Stored CPML memories: FP32, or BF16 in the 16-bit memory mode (SEIS3D_STORAGE_BF16_CPML).
// Threads hold a memory in its storage type from its load to its update, so a memory loaded a
// plane ahead is not waited for until the plane that uses it (converting at the load would
// wait at once: measured 13 % slower passes).
template <typename Mem> __device__ __forceinline__ Mem memZero();
template <> __device__ __forceinline__ float memZero<float>() { return 0.0f; }
template <> __device__ __forceinline__ __nv_bfloat16 memZero<__nv_bfloat16>() { return __ushort_as_bfloat16(0); }

// Slab index along one axis or -1 outside the slab (cuda/Cuda_Seis3D.cu:97-102).
__device__ __forceinline__ int slabIndex(int coord, int n, int pml, bool topFree) {
    if (!topFree && coord < kRadius + pml) return coord - kRadius;
    if (coord >= n - kRadius - pml) return (topFree ? 0 : pml) + coord - (n - kRadius - pml);
    return -1;
}

// Ricker amplitude of the 3x3x3 source at node offset (dx,dy,dz) and time t
// (cuda/Cuda_Seis3D.cu:319-322): FP64 phase, FP32 spatial weight.
__device__ __noinline__ float sourceValue(const Geometry& G, const SourceParams& S, int dx, int dy, int dz,
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
// Shared pieces of the two z-marching passes.
//
// A CTA owns a 32 (x) x 16 (y) column tile and marches a chunk of z planes.  It has 8 warps;
// warp w owns rows 2w and 2w+1 of the tile, one x column per lane, so each thread updates
// two cells per plane and the y-derivative windows of its two rows share 9 of their 16
// loads.  No block-wide barrier runs in the plane loop: planes arrive through a ring of
// TMA stages (seis3d_tma.cuh); a warp waits on the stage's mbarrier, computes, then
// releases the stage, and the last warp to release a stage refills it with the plane
// kStages ahead, so warps of a CTA drift by up to kStages planes and one warp's CPML
// memory latency does not stall the others.  The stage ring is a plain (non-template)
// type on purpose: a templated form compiled to a schedule 30 % slower on B200.  The z rings
// shift by one register per plane: unrolling the plane loop eight times so that they rotate by
// renaming instead measured 45 % slower (1.09 vs 0.75 ms velocity pass on the 300x300x400
// grid), the eight copies of the plane body costing more than the moves they remove.
// ---------------------------------------------------------------------------------------
constexpr int kTX = 32, kTY = 16, kWarps = 8, kThreads = kTX * kWarps;
#ifndef SEIS3D_MIN_BLOCKS
#define SEIS3D_MIN_BLOCKS 2   // resident CTAs per SM the register allocation is sized for
#endif

template <int N> using Int = std::integral_constant<int, N>;

struct StageRing {
    uint64_t full[tma::kStages];
    int released[tma::kStages];
    int issued;      // stages issued so far (monotonic)
    int stalled;     // set when a stage did not arrive within the wait bound
};

// Warp-uniform bounded wait for the stage in buffer b with phase parity `phase`.
__device__ __forceinline__ bool waitFull(StageRing& R, int b, uint32_t phase, long long limit) {
    volatile int* stalled = &R.stalled;
    bool ok = !*stalled && tma::waitStage(&R.full[b], phase, limit);
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && threadIdx.x == 0) *stalled = 1;
    return ok;
}

// Release stage j (buffer b); the last of the warps refills the buffer with stage
// j + kStages.
template <class Issue>
__device__ __forceinline__ void releaseStage(StageRing& R, int j, int b, int nPlanes, Issue&& issue) {
    __syncwarp();
    if (threadIdx.x == 0) {
        __threadfence_block();
        if (atomicAdd(&R.released[b], 1) == kWarps - 1) {
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
__device__ __forceinline__ void drainAfterStall(const Fields& F, StageRing& R, int consumed, long long limit) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        atomicOr(F.status + 1, 1u);
        for (int j = consumed; j < R.issued; ++j)
            tma::waitStage(&R.full[j % tma::kStages], (j / tma::kStages) & 1, limit);
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

// CPML coefficient table of the tile's 16 rows: {a, b, 1/kappa} at centre (h = 0) and half
// grid (h = 1).
struct RowCoefficients {
    float y[2][3][kTY];
    float x[2][3][kTX];   // the tile's 32 columns, same layout (loaded and read by the stress pass)
};

__device__ __forceinline__ void loadRowCoefficients(RowCoefficients& T, const Fields& F, const Geometry& G, int x0,
                                                    int y0, int tid, bool columns) {
    if (G.reflecting) return;
    for (int e = tid; e < 6 * kTY; e += kThreads) {
        const int h = e / (3 * kTY), j = (e / kTY) % 3, r = e % kTY;
        T.y[h][j][r] = F.coef[1][(h * G.gy + min(y0 + r, G.gy - 1)) * 3 + j];
    }
    if (!columns) return;
    for (int e = tid; e < 6 * kTX; e += kThreads) {
        const int h = e / (3 * kTX), j = (e / kTX) % 3, c = e % kTX;
        T.x[h][j][c] = F.coef[0][(h * G.gx + min(x0 + c, G.gx - 1)) * 3 + j];
    }
}

// psi = b psi + a d; returns d/kappa + psi (cuda/Cuda_Seis3D.cu:109-110).
__device__ __forceinline__ float cpmlApply(float d, float& m, float a, float b, float ik) {
    m = b * m + a * d;
    return ik * d + m;
}

// The same with a BF16 memory: the update runs in FP32 and the step uses it in full; only the
// memory kept for the next step is rounded (to nearest even).
__device__ __forceinline__ float cpmlApply(float d, __nv_bfloat16& m, float a, float b, float ik) {
    const float u = b * __bfloat162float(m) + a * d;
    m = __float2bfloat16_rn(u);
    return ik * d + u;
}

// Two y derivatives of adjacent rows from one 9-row column window (W = row length).
template <int W> __device__ __forceinline__ void diffColPair(const float* col, const float* inv, float& da, float& db) {
    const float v0 = col[0], v1 = col[W], v2 = col[2 * W], v3 = col[3 * W], v4 = col[4 * W], v5 = col[5 * W],
                v6 = col[6 * W], v7 = col[7 * W], v8 = col[8 * W];
    da = diff8(v0, v1, v2, v3, v4, v5, v6, v7, inv);
    db = diff8(v1, v2, v3, v4, v5, v6, v7, v8, inv);
}

// z derivative of an 8-plane register ring whose oldest element sits at index U.
template <int U> __device__ __forceinline__ float diffRingAt(const float (&r)[8], const float* inv) {
    return diff8(r[U & 7], r[(U + 1) & 7], r[(U + 2) & 7], r[(U + 3) & 7], r[(U + 4) & 7], r[(U + 5) & 7],
                 r[(U + 6) & 7], r[(U + 7) & 7], inv);
}

// Pulls the z-slab memories (three slots, rows a and b) of the next plane into L2, so that
// their loads in that plane wait on L2 rather than DRAM; no register is written.  Used by the
// stress pass (1.2 % faster); the velocity pass measured 0.5 % slower with it.
template <typename Mem>
__device__ __forceinline__ void prefetchZSlab(const Mem* p, unsigned slot, unsigned pitch, bool rowB) {
#pragma unroll
    for (int s3 = 0; s3 < 3; ++s3) {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(p + s3 * slot));
        if (rowB) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + pitch + s3 * slot));
    }
}

// Per-thread CPML bookkeeping of one axis for the thread's two rows: 32-bit offsets of
// slot 0 (row a, row b) into that axis's psi array and the prefetched memories.
template <typename Mem> struct SlabRows {
    bool a, b;           // row a / row b inside the slab
    unsigned oa, ob;     // slot-0 offsets of the current plane
    Mem ma[3], mb[3];    // memories of the current plane (slots s, s+1, s+2)
};

// Stores the three slots of one row's memories.
template <typename Mem>
__device__ __forceinline__ void storeSlots(Mem* base, unsigned o, unsigned slot, const Mem (&m)[3]) {
    base[o] = m[0]; base[o + slot] = m[1]; base[o + 2 * slot] = m[2];
}

// ---------------------------------------------------------------------------------------
// Free surface (planar, z = 4): traction images of the stresses (cuda/Cuda_Seis3D.cu:203-219)
// and velocity images from the zero-traction constraints (:249-272), one column at a time.
// In a step the first z chunk of each pass writes the images its z rings read, each column's
// by the thread that owns it: the velocity pass the stress images (at the start of the step,
// where the reference runs stressGhostKernel3D) and the stress pass the velocity images.  The
// standalone kernels serve z chunks shorter than 4 planes, the end of each stepping call, and
// the learned boundary's corrections.
// ---------------------------------------------------------------------------------------
// Stress images of one column (x, y): traction-free surface plane, odd/even images above it.
__device__ __forceinline__ void stressImageColumn(const Geometry& G, const Fields& F, int x, int y) {
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

// Velocity images of one column (x, y) from the final velocities of planes 4-8 of the column
// and of its x/y neighbours on planes 4-5.  Every operation is an explicit round-to-nearest
// one (a - b c as one fused multiply-add, rounded once), so the images are the same bits
// wherever this is inlined (the stress pass's first z chunk, or the standalone kernel).
__device__ __forceinline__ void velocityImageColumn(const Geometry& G, const Fields& F, int x, int y) {
    const int64_t P = G.pitch, PL = G.plane;
    const int64_t i = 4 * PL + int64_t(y) * P + x, n = i + PL;
    const float* inv = G.w;
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
    // -(1.5 a - 0.5 b) and -lambda / (lambda + 2 mu) * (ex + ey) (cuda/Cuda_Seis3D.cu:258-266).
    const float dzVx = -__fmaf_rn(1.5f, zx0, __fmul_rn(-0.5f, zx1));
    const float dzVy = -__fmaf_rn(1.5f, zy0, __fmul_rn(-0.5f, zy1));
    const float lambda = F.lambda[i], mu = F.mu[i];
    const float dzVz = __fmul_rn(__fdiv_rn(-lambda, __fadd_rn(lambda, __fmul_rn(2.0f, mu))), __fadd_rn(ex, ey));
    const int64_t c = int64_t(y) * P + x;
#pragma unroll
    for (int k = 1; k <= 4; ++k) {
        const int64_t g = (4 - k) * PL + c, m = (4 + k) * PL + c;
        F.f[0][g] = __fmaf_rn(-__fmul_rn(float(2 * k), G.h), dzVx, F.f[0][m]);
        F.f[1][g] = __fmaf_rn(-__fmul_rn(float(2 * k), G.h), dzVy, F.f[1][m]);
        F.f[2][g] = __fmaf_rn(-__fmul_rn(float(2 * k - 1), G.h), dzVz, F.f[2][(3 + k) * PL + c]);
    }
}

// ---------------------------------------------------------------------------------------
// Velocity pass: v(n+1/2) = v(n-1/2) + dt * 2ab/(a+b) * sum_axis CPML(D sigma)
// (cuda/Cuda_Seis3D.cu:222-245) with the force source fused (:313-332).
// Stage of plane k: sigma halo tiles of plane k, 1/rho tile of k and centre of k+1,
// v centres of k, and the ring feeds sigma_xz/sigma_yz(k+3), sigma_zz(k+4).
// ---------------------------------------------------------------------------------------
// True when the CTA's whole tile and z chunk lie outside every CPML slab (or the walls
// reflect): such CTAs run the pass body compiled without the CPML code, which measured 12.6 %
// cheaper per cell than the same body with the CPML code present but never entered.
__device__ __forceinline__ bool interiorTile(const Geometry& G, int zChunk) {
    if (G.reflecting) return true;
    const int x0 = kRadius + blockIdx.x * kTX, y0 = kRadius + blockIdx.y * kTY;
    const int zBegin = kRadius + blockIdx.z * zChunk;
    const int zEnd = min(zBegin + zChunk, G.gz - kRadius);
    const bool topFree = G.freeSurface != 0;
    // Slabs sit at the ends of each axis, so the two ends of each range decide.
    return slabIndex(x0, G.gx, G.pml, false) < 0 && slabIndex(x0 + kTX - 1, G.gx, G.pml, false) < 0 &&
           slabIndex(y0, G.gy, G.pml, false) < 0 && slabIndex(y0 + kTY - 1, G.gy, G.pml, false) < 0 &&
           slabIndex(zBegin, G.gz, G.pml, topFree) < 0 && slabIndex(max(zEnd - 1, zBegin), G.gz, G.pml, topFree) < 0;
}

struct VelocityStage {
    static constexpr int XX = 0, XY = 640, XZ = 1600, YY = 2240, YZ = 3008, B = 3776, B1 = 4416, V = 4928,
                         FXZ = 6464, FYZ = 6976, FZZ = 7488, SIZE = 8000;
    static constexpr uint32_t BYTES = 4u * (640 + 960 + 640 + 768 + 768 + 612 + 512 + 3 * 512 + 3 * 512);
};

template <bool kCpml, typename Mem>
__device__ __forceinline__ void velocityBody(const Geometry& G, const Fields& F, const SourceParams& S, int zChunk) {
    using St = VelocityStage;
    extern __shared__ __align__(128) float smem[];
    __shared__ StageRing R;
    __shared__ RowCoefficients T;

    const int tx = threadIdx.x, w = threadIdx.y, tid = w * kTX + tx;
    const int ra = 2 * w, rb = ra + 1;
    const int x0 = kRadius + blockIdx.x * kTX, y0 = kRadius + blockIdx.y * kTY;
    const int x = x0 + tx, ya = y0 + ra, yb = ya + 1;
    const bool activeA = x < G.gx - kRadius && ya < G.gy - kRadius;
    const bool activeB = activeA && yb < G.gy - kRadius;
    const int zBegin = kRadius + blockIdx.z * zChunk;
    const int zEnd = min(zBegin + zChunk, G.gz - kRadius);
    if (zBegin >= zEnd) return;
    const int nPlanes = zEnd - zBegin;
    const unsigned P = unsigned(G.pitch), PL = unsigned(G.plane);
    const float* inv = G.w;
    const CUtensorMap* M = F.maps;

    auto issue = [&](int j) {
        float* st = smem + (j % tma::kStages) * St::SIZE;
        uint64_t* bar = &R.full[j % tma::kStages];
        const int k = zBegin + j;
        if (j == G.withheldStage) return;   // test hook: this stage never arrives
        tma::arriveExpectTx(bar, St::BYTES);
        tma::load3d(st + St::XX, M + tma::kSxxX, x0 - 4, y0, k, bar);
        tma::load3d(st + St::XY, M + tma::kSxyXY, x0 - 4, y0 - 4, k, bar);
        tma::load3d(st + St::XZ, M + tma::kSxzX, x0 - 4, y0, k, bar);
        tma::load3d(st + St::YY, M + tma::kSyyY, x0, y0 - 4, k, bar);
        tma::load3d(st + St::YZ, M + tma::kSyzY, x0, y0 - 4, k, bar);
        tma::load3d(st + St::B, M + tma::kRhoT, x0, y0, k, bar);
        tma::load3d(st + St::B1, M + tma::kCenter0 + 9, x0, y0, k + 1, bar);
        tma::load3d(st + St::V, M + tma::kCenter0 + 0, x0, y0, k, bar);
        tma::load3d(st + St::V + 512, M + tma::kCenter0 + 1, x0, y0, k, bar);
        tma::load3d(st + St::V + 1024, M + tma::kCenter0 + 2, x0, y0, k, bar);
        tma::load3d(st + St::FXZ, M + tma::kCenter0 + 8, x0, y0, k + 3, bar);
        tma::load3d(st + St::FYZ, M + tma::kCenter0 + 7, x0, y0, k + 3, bar);
        tma::load3d(st + St::FZZ, M + tma::kCenter0 + 5, x0, y0, k + 4, bar);
    };

    if (tid == 0) initRing(R);
    loadRowCoefficients(T, F, G, x0, y0, tid, false);
    __syncthreads();
    if (tid == 0) {
        const int first = min(tma::kStages, nPlanes);
        for (int j = 0; j < first; ++j) issue(j);
        R.issued = first;
    }

    // CPML slab membership: x and y fixed per thread, z per plane (uniform over the CTA).
    const bool cp = kCpml && !G.reflecting;
    const bool topFree = G.freeSurface != 0;
    const int qx = cp && activeA ? slabIndex(x, G.gx, G.pml, false) : -1;
    const int qya = cp && activeA ? slabIndex(ya, G.gy, G.pml, false) : -1;
    const int qyb = cp && activeB ? slabIndex(yb, G.gy, G.pml, false) : -1;
    const unsigned T0 = G.thick[0], T1 = G.thick[1];
    const unsigned slotX = unsigned(G.gz) * G.gy * T0, slotY = unsigned(G.gz) * T1 * P;
    const unsigned slotZ = unsigned(G.thick[2]) * G.gy * P;
    float kx[6] = {0, 0, 0, 0, 0, 0};
    if (qx >= 0)
#pragma unroll
        for (int e = 0; e < 6; ++e) kx[e] = F.coef[0][((e / 3) * G.gx + x) * 3 + e % 3];
    SlabRows<Mem> sx, sy;
    sx.a = qx >= 0; sx.b = qx >= 0 && activeB;
    sx.oa = (unsigned(zBegin) * G.gy + ya) * T0 + unsigned(qx); sx.ob = sx.oa + T0;
    sy.a = qya >= 0; sy.b = qyb >= 0;
    sy.oa = (unsigned(zBegin) * T1 + unsigned(qya)) * P + x; sy.ob = (unsigned(zBegin) * T1 + unsigned(qyb)) * P + x;
    const Mem* psiX = reinterpret_cast<const Mem*>(F.psi[0]);
    const Mem* psiY = reinterpret_cast<const Mem*>(F.psi[1]);
#pragma unroll
    for (int s3 = 0; s3 < 3; ++s3) {
        sx.ma[s3] = sx.a ? psiX[sx.oa + s3 * slotX] : memZero<Mem>();
        sx.mb[s3] = sx.b ? psiX[sx.ob + s3 * slotX] : memZero<Mem>();
        sy.ma[s3] = sy.a ? psiY[sy.oa + s3 * slotY] : memZero<Mem>();
        sy.mb[s3] = sy.b ? psiY[sy.ob + s3 * slotY] : memZero<Mem>();
    }

    // Free surface: the first z chunk writes the stress images of its own columns (ghost planes
    // 0-3, from planes 4-8 of the same column) before its z rings read them.  No other thread
    // reads them in this pass when chunks hold at least 4 planes (the staged tiles start at
    // plane 4 and the next chunk's rings at plane zChunk), and no stress is written here;
    // for shorter chunks the host launches the image kernels instead (foldedImages).
    if (G.freeSurface && zBegin == kRadius && zChunk >= kRadius && activeA) {
        stressImageColumn(G, F, x, ya);
        if (activeB) stressImageColumn(G, F, x, yb);
    }

    // z rings of both rows: rXZ/rYZ hold planes z-4..z+3 (D-), rZZ planes z-3..z+4 (D+).
    float rXZ[2][8], rYZ[2][8], rZZ[2][8];
    const unsigned colA = unsigned(min(ya, G.gy - 1)) * P + unsigned(min(x, G.gx - 1));
    const unsigned colB = unsigned(min(yb, G.gy - 1)) * P + unsigned(min(x, G.gx - 1));
    if (activeA) {
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            rXZ[0][k] = F.f[8][unsigned(zBegin - 4 + k) * PL + colA];
            rYZ[0][k] = F.f[7][unsigned(zBegin - 4 + k) * PL + colA];
            rZZ[0][k] = F.f[5][unsigned(zBegin - 3 + k) * PL + colA];
            rXZ[1][k] = F.f[8][unsigned(zBegin - 4 + k) * PL + colB];
            rYZ[1][k] = F.f[7][unsigned(zBegin - 4 + k) * PL + colB];
            rZZ[1][k] = F.f[5][unsigned(zBegin - 3 + k) * PL + colB];
        }
    }
    const unsigned long long step = F.clock->step;
    const bool forceA = S.kind == 1 && activeA && abs(x - S.gxs) <= 1 && abs(ya - S.gys) <= 1;
    const bool forceB = S.kind == 1 && activeB && abs(x - S.gxs) <= 1 && abs(yb - S.gys) <= 1;
    bool bad = false;
    float check = 0.0f;   // sum of every output: non-finite if any output is
    bool stop = false;
    int j = 0, b = 0;
    uint32_t phase = 0;
    unsigned oa = unsigned(zBegin) * PL + colA;   // field offset of row a at the current plane

    // One plane; U is the ring rotation (j mod 8).
    auto plane = [&](auto rot) {
        constexpr int U = decltype(rot)::value;
        const int z = zBegin + j;
        if (!waitFull(R, b, phase, G.waitCycles)) { stop = true; return; }
        if (activeA) {
            const float* st = smem + b * St::SIZE;
            const int ca = ra * 32 + tx, cb = ca + 32;
            rXZ[0][(U + 7) & 7] = st[St::FXZ + ca]; rXZ[1][(U + 7) & 7] = st[St::FXZ + cb];
            rYZ[0][(U + 7) & 7] = st[St::FYZ + ca]; rYZ[1][(U + 7) & 7] = st[St::FYZ + cb];
            rZZ[0][(U + 7) & 7] = st[St::FZZ + ca]; rZZ[1][(U + 7) & 7] = st[St::FZZ + cb];

            // vx: D+x sxx, D-y sxy, D-z sxz.  vy: D-x sxy, D+y syy, D-z syz.  vz: D-x sxz, D-y syz, D+z szz.
            float dx0a = diffRow<40>(st + St::XX + ra * 40 + tx + 1, inv);
            float dx0b = diffRow<40>(st + St::XX + rb * 40 + tx + 1, inv);
            float dy0a, dy0b;
            diffColPair<40>(st + St::XY + ra * 40 + tx + 4, inv, dy0a, dy0b);
            float dz0a = diffRingAt<U>(rXZ[0], inv), dz0b = diffRingAt<U>(rXZ[1], inv);
            float dx1a = diffRow<40>(st + St::XY + (ra + 4) * 40 + tx, inv);
            float dx1b = diffRow<40>(st + St::XY + (rb + 4) * 40 + tx, inv);
            float dy1a, dy1b;
            diffColPair<32>(st + St::YY + (ra + 1) * 32 + tx, inv, dy1a, dy1b);
            float dz1a = diffRingAt<U>(rYZ[0], inv), dz1b = diffRingAt<U>(rYZ[1], inv);
            float dx2a = diffRow<40>(st + St::XZ + ra * 40 + tx, inv);
            float dx2b = diffRow<40>(st + St::XZ + rb * 40 + tx, inv);
            float dy2a, dy2b;
            diffColPair<32>(st + St::YZ + ra * 32 + tx, inv, dy2a, dy2b);
            float dz2a = diffRingAt<U>(rZZ[0], inv), dz2b = diffRingAt<U>(rZZ[1], inv);

            // CPML: velocity component v uses slot v; its own axis on the half grid.
            Mem* psi0 = reinterpret_cast<Mem*>(F.psi[0]);
            Mem* psi1 = reinterpret_cast<Mem*>(F.psi[1]);
            if (sx.a) {
                dx0a = cpmlApply(dx0a, sx.ma[0], kx[3], kx[4], kx[5]);
                dx1a = cpmlApply(dx1a, sx.ma[1], kx[0], kx[1], kx[2]);
                dx2a = cpmlApply(dx2a, sx.ma[2], kx[0], kx[1], kx[2]);
                storeSlots(psi0, sx.oa, slotX, sx.ma);
                if (sx.b) {
                    dx0b = cpmlApply(dx0b, sx.mb[0], kx[3], kx[4], kx[5]);
                    dx1b = cpmlApply(dx1b, sx.mb[1], kx[0], kx[1], kx[2]);
                    dx2b = cpmlApply(dx2b, sx.mb[2], kx[0], kx[1], kx[2]);
                    storeSlots(psi0, sx.ob, slotX, sx.mb);
                }
            }
            if (sy.a) {
                dy0a = cpmlApply(dy0a, sy.ma[0], T.y[0][0][ra], T.y[0][1][ra], T.y[0][2][ra]);
                dy1a = cpmlApply(dy1a, sy.ma[1], T.y[1][0][ra], T.y[1][1][ra], T.y[1][2][ra]);
                dy2a = cpmlApply(dy2a, sy.ma[2], T.y[0][0][ra], T.y[0][1][ra], T.y[0][2][ra]);
                storeSlots(psi1, sy.oa, slotY, sy.ma);
            }
            if (sy.b) {
                dy0b = cpmlApply(dy0b, sy.mb[0], T.y[0][0][rb], T.y[0][1][rb], T.y[0][2][rb]);
                dy1b = cpmlApply(dy1b, sy.mb[1], T.y[1][0][rb], T.y[1][1][rb], T.y[1][2][rb]);
                dy2b = cpmlApply(dy2b, sy.mb[2], T.y[0][0][rb], T.y[0][1][rb], T.y[0][2][rb]);
                storeSlots(psi1, sy.ob, slotY, sy.mb);
            }
            const int qz = cp ? slabIndex(z, G.gz, G.pml, topFree) : -1;
            if (qz >= 0) {
                const float* kz = F.coef[2] + z * 3;
                const float* kh = F.coef[2] + (G.gz + z) * 3;
                Mem* pz = reinterpret_cast<Mem*>(F.psi[2]) + (unsigned(qz) * G.gy + ya) * P + x;
                Mem m0 = pz[0], m1 = pz[slotZ], m2 = pz[2 * slotZ];
                dz0a = cpmlApply(dz0a, m0, kz[0], kz[1], kz[2]);
                dz1a = cpmlApply(dz1a, m1, kz[0], kz[1], kz[2]);
                dz2a = cpmlApply(dz2a, m2, kh[0], kh[1], kh[2]);
                pz[0] = m0; pz[slotZ] = m1; pz[2 * slotZ] = m2;
                if (activeB) {
                    Mem n0 = pz[P], n1 = pz[P + slotZ], n2 = pz[P + 2 * slotZ];
                    dz0b = cpmlApply(dz0b, n0, kz[0], kz[1], kz[2]);
                    dz1b = cpmlApply(dz1b, n1, kz[0], kz[1], kz[2]);
                    dz2b = cpmlApply(dz2b, n2, kh[0], kh[1], kh[2]);
                    pz[P] = n0; pz[P + slotZ] = n1; pz[P + 2 * slotZ] = n2;
                }
            }

            // Prefetch the x/y memories of the next plane.
            if (j + 1 < nPlanes) {
                sx.oa += G.gy * T0; sx.ob += G.gy * T0;
                sy.oa += T1 * P; sy.ob += T1 * P;
#pragma unroll
                for (int s3 = 0; s3 < 3; ++s3) {
                    if (sx.a) sx.ma[s3] = psiX[sx.oa + s3 * slotX];
                    if (sx.b) sx.mb[s3] = psiX[sx.ob + s3 * slotX];
                    if (sy.a) sy.ma[s3] = psiY[sy.oa + s3 * slotY];
                    if (sy.b) sy.mb[s3] = psiY[sy.ob + s3 * slotY];
                }
            }

            // Row a.
            {
                float div0 = 0.0f; div0 += dx0a; div0 += dy0a; div0 += dz0a;
                float div1 = 0.0f; div1 += dx1a; div1 += dy1a; div1 += dz1a;
                float div2 = 0.0f; div2 += dx2a; div2 += dy2a; div2 += dz2a;
                const float* sb = st + St::B + ra * 36 + tx;
                const float a = sb[0], bx = sb[1], by = sb[36], bz = st[St::B1 + ca];
                // Harmonic buoyancy means in IEEE division, as the reference (2AB/(A+B)).  The
                // hardware reciprocal (2 ulp) perturbs every face coefficient by a fixed amount,
                // which on the layered 300x50x300 shot put the gather 3x further from an FP64
                // run than the reference's; IEEE division here costs 0.04 ms of a 1.52 ms step.
                const float cx = __fdiv_rn(2 * a * bx, a + bx);
                const float cy = __fdiv_rn(2 * a * by, a + by);
                const float cz = __fdiv_rn(2 * a * bz, a + bz);
                float v0 = st[St::V + ca] + G.dt * cx * div0;
                float v1 = st[St::V + 512 + ca] + G.dt * cy * div1;
                float v2 = st[St::V + 1024 + ca] + G.dt * cz * div2;
                if (forceA && abs(z - S.gzs) <= 1) {
                    const float value = sourceValue(G, S, x - S.gxs, ya - S.gys, z - S.gzs, double(step) * G.dt);
                    v0 += value * S.direction[0] * cx;
                    v1 += value * S.direction[1] * cy;
                    v2 += value * S.direction[2] * cz;
                }
                F.f[0][oa] = v0; F.f[1][oa] = v1; F.f[2][oa] = v2;
                check += (v0 + v1) + v2;
            }
            // Row b.
            if (activeB) {
                float div0 = 0.0f; div0 += dx0b; div0 += dy0b; div0 += dz0b;
                float div1 = 0.0f; div1 += dx1b; div1 += dy1b; div1 += dz1b;
                float div2 = 0.0f; div2 += dx2b; div2 += dy2b; div2 += dz2b;
                const float* sb = st + St::B + rb * 36 + tx;
                const float a = sb[0], bx = sb[1], by = sb[36], bz = st[St::B1 + cb];
                const float cx = __fdiv_rn(2 * a * bx, a + bx);
                const float cy = __fdiv_rn(2 * a * by, a + by);
                const float cz = __fdiv_rn(2 * a * bz, a + bz);
                float v0 = st[St::V + cb] + G.dt * cx * div0;
                float v1 = st[St::V + 512 + cb] + G.dt * cy * div1;
                float v2 = st[St::V + 1024 + cb] + G.dt * cz * div2;
                if (forceB && abs(z - S.gzs) <= 1) {
                    const float value = sourceValue(G, S, x - S.gxs, yb - S.gys, z - S.gzs, double(step) * G.dt);
                    v0 += value * S.direction[0] * cx;
                    v1 += value * S.direction[1] * cy;
                    v2 += value * S.direction[2] * cz;
                }
                const unsigned ob = oa + P;
                F.f[0][ob] = v0; F.f[1][ob] = v1; F.f[2][ob] = v2;
                check += (v0 + v1) + v2;
            }
        }
        releaseStage(R, j, b, nPlanes, issue);
        oa += PL;
        ++j;
        if (++b == tma::kStages) { b = 0; phase ^= 1u; }
    };

    while (j < nPlanes) {
        plane(Int<0>{});
        if (stop) break;
#pragma unroll
        for (int k = 0; k < 7; ++k)
#pragma unroll
            for (int r = 0; r < 2; ++r) { rXZ[r][k] = rXZ[r][k + 1]; rYZ[r][k] = rYZ[r][k + 1]; rZZ[r][k] = rZZ[r][k + 1]; }
    }
    if (R.stalled) drainAfterStall(F, R, j, G.waitCycles);
    flagNonFinite(F, bad || !isfinite(check));
}

__global__ void __launch_bounds__(kThreads, SEIS3D_MIN_BLOCKS)
    velocityPass(Geometry G, Fields F, SourceParams S, int zChunk) {
    if (interiorTile(G, zChunk)) velocityBody<false, float>(G, F, S, zChunk);
    else velocityBody<true, float>(G, F, S, zChunk);
}

// The same pass with BF16 CPML memories (SEIS3D_STORAGE_BF16_CPML).
__global__ void __launch_bounds__(kThreads, SEIS3D_MIN_BLOCKS)
    velocityPassBf16Cpml(Geometry G, Fields F, SourceParams S, int zChunk) {
    if (interiorTile(G, zChunk)) velocityBody<false, float>(G, F, S, zChunk);
    else velocityBody<true, __nv_bfloat16>(G, F, S, zChunk);
}

// ---------------------------------------------------------------------------------------
// Stress pass: sigma(n+1) from CPML-filtered velocity derivatives (cuda/Cuda_Seis3D.cu:281-310),
// harmonic shear moduli (:275-278) from reciprocals carried plane to plane in registers,
// free-surface closure at z=4 (:299, :303) and the explosion source fused (:313-332).
// Stage of plane k: velocity cross tiles of k, mu tiles of k and k+1, lambda and the six
// stresses of k, and the ring feeds vx/vy(k+4), vz(k+3).
// ---------------------------------------------------------------------------------------
struct StressStage {
    static constexpr int VX = 0, VY = 960, VZ = 1920, M0 = 2880, M1 = 3520, L = 4160, S = 4672, FVX = 7744,
                         FVY = 8256, FVZ = 8768, SIZE = 9280;
    static constexpr uint32_t BYTES = 4u * (3 * 960 + 2 * 612 + 512 + 6 * 512 + 3 * 512);
};

template <bool kCpml, typename Mem>
__device__ __forceinline__ void stressBody(const Geometry& G, const Fields& F, const SourceParams& S, int zChunk) {
    using St = StressStage;
    extern __shared__ __align__(128) float smem[];
    __shared__ StageRing R;
    __shared__ RowCoefficients T;

    const int tx = threadIdx.x, w = threadIdx.y, tid = w * kTX + tx;
    const int ra = 2 * w, rb = ra + 1;
    const int x0 = kRadius + blockIdx.x * kTX, y0 = kRadius + blockIdx.y * kTY;
    const int x = x0 + tx, ya = y0 + ra, yb = ya + 1;
    const bool activeA = x < G.gx - kRadius && ya < G.gy - kRadius;
    const bool activeB = activeA && yb < G.gy - kRadius;
    const int zBegin = kRadius + blockIdx.z * zChunk;
    const int zEnd = min(zBegin + zChunk, G.gz - kRadius);
    if (zBegin >= zEnd) return;
    const int nPlanes = zEnd - zBegin;
    const unsigned P = unsigned(G.pitch), PL = unsigned(G.plane);
    const float* inv = G.w;
    const CUtensorMap* M = F.maps;

    auto issue = [&](int j) {
        float* st = smem + (j % tma::kStages) * St::SIZE;
        uint64_t* bar = &R.full[j % tma::kStages];
        const int k = zBegin + j;
        if (j == G.withheldStage) return;   // test hook: this stage never arrives
        tma::arriveExpectTx(bar, St::BYTES);
        tma::load3d(st + St::VX, M + tma::kVxXY, x0 - 4, y0 - 4, k, bar);
        tma::load3d(st + St::VY, M + tma::kVyXY, x0 - 4, y0 - 4, k, bar);
        tma::load3d(st + St::VZ, M + tma::kVzXY, x0 - 4, y0 - 4, k, bar);
        tma::load3d(st + St::M0, M + tma::kMuT, x0, y0, k, bar);
        tma::load3d(st + St::M1, M + tma::kMuT, x0, y0, k + 1, bar);
        tma::load3d(st + St::L, M + tma::kCenter0 + 10, x0, y0, k, bar);
#pragma unroll
        for (int f = 0; f < 6; ++f) tma::load3d(st + St::S + 512 * f, M + tma::kCenter0 + 3 + f, x0, y0, k, bar);
        tma::load3d(st + St::FVX, M + tma::kCenter0 + 0, x0, y0, k + 4, bar);
        tma::load3d(st + St::FVY, M + tma::kCenter0 + 1, x0, y0, k + 4, bar);
        tma::load3d(st + St::FVZ, M + tma::kCenter0 + 2, x0, y0, k + 3, bar);
    };

    if (tid == 0) initRing(R);
    loadRowCoefficients(T, F, G, x0, y0, tid, true);
    __syncthreads();
    if (tid == 0) {
        const int first = min(tma::kStages, nPlanes);
        for (int j = 0; j < first; ++j) issue(j);
        R.issued = first;
    }

    const bool cp = kCpml && !G.reflecting;
    const bool topFree = G.freeSurface != 0;
    const int qx = cp && activeA ? slabIndex(x, G.gx, G.pml, false) : -1;
    const int qya = cp && activeA ? slabIndex(ya, G.gy, G.pml, false) : -1;
    const int qyb = cp && activeB ? slabIndex(yb, G.gy, G.pml, false) : -1;
    const unsigned T0 = G.thick[0], T1 = G.thick[1];
    const unsigned slotX = unsigned(G.gz) * G.gy * T0, slotY = unsigned(G.gz) * T1 * P;
    const unsigned slotZ = unsigned(G.thick[2]) * G.gy * P;
    // x-slab coefficients come from the CTA's shared table (T.x) rather than six registers per
    // thread: measured 3.5 % faster for this pass, which runs at its register limit.
    // Stress slots 3..5 start at 3 * slot.
    SlabRows<Mem> sx, sy;
    sx.a = qx >= 0; sx.b = qx >= 0 && activeB;
    sx.oa = 3 * slotX + (unsigned(zBegin) * G.gy + ya) * T0 + unsigned(qx); sx.ob = sx.oa + T0;
    sy.a = qya >= 0; sy.b = qyb >= 0;
    sy.oa = 3 * slotY + (unsigned(zBegin) * T1 + unsigned(qya)) * P + x;
    sy.ob = 3 * slotY + (unsigned(zBegin) * T1 + unsigned(qyb)) * P + x;
    const Mem* psiX = reinterpret_cast<const Mem*>(F.psi[0]);
    const Mem* psiY = reinterpret_cast<const Mem*>(F.psi[1]);
#pragma unroll
    for (int s3 = 0; s3 < 3; ++s3) {
        sx.ma[s3] = sx.a ? psiX[sx.oa + s3 * slotX] : memZero<Mem>();
        sx.mb[s3] = sx.b ? psiX[sx.ob + s3 * slotX] : memZero<Mem>();
        sy.ma[s3] = sy.a ? psiY[sy.oa + s3 * slotY] : memZero<Mem>();
        sy.mb[s3] = sy.b ? psiY[sy.ob + s3 * slotY] : memZero<Mem>();
    }

    // Reciprocal shear moduli 1/mu of the current plane at x and x+1 on rows a, b and b+1,
    // with the hardware reciprocal (2 ulp; the reference divides in IEEE): mu == 0 gives +inf,
    // so the harmonic means below are exactly 0 there, as the reference's fluid branch
    // returns.  Measured against an FP64 run of the layered 300x50x300 shot, IEEE division
    // here and in the harmonic means leaves the gather's and the fields' distance to FP64
    // unchanged, and costs 0.145 ms of a 1.52 ms step, so the stress pass keeps the
    // reciprocal.
    const unsigned colA = unsigned(min(ya, G.gy - 1)) * P + unsigned(min(x, G.gx - 1));
    const unsigned colB = unsigned(min(yb, G.gy - 1)) * P + unsigned(min(x, G.gx - 1));
    float rA0 = 0, rA1 = 0, rB0 = 0, rB1 = 0, rC0 = 0, rC1 = 0;
    if (activeA) {
        const float* m = F.mu + unsigned(zBegin) * PL + colA;
        rA0 = __fdividef(1.0f, m[0]); rA1 = __fdividef(1.0f, m[1]);
        rB0 = __fdividef(1.0f, m[P]); rB1 = __fdividef(1.0f, m[P + 1]);
        rC0 = __fdividef(1.0f, m[2 * P]); rC1 = __fdividef(1.0f, m[2 * P + 1]);
    }

    // Free surface: the first z chunk writes the velocity images of its own columns (ghost planes
    // 0-3) before its z rings read them.  As in the velocity pass, no other thread reads them
    // when chunks hold at least 4 planes, and the final velocities they come from are not
    // written here; shorter chunks leave them to the host's image launches.
    if (G.freeSurface && zBegin == kRadius && zChunk >= kRadius && activeA) {
        velocityImageColumn(G, F, x, ya);
        if (activeB) velocityImageColumn(G, F, x, yb);
    }

    // z rings of both rows: rVX/rVY planes z-3..z+4 (D+), rVZ planes z-4..z+3 (D-).
    float rVX[2][8], rVY[2][8], rVZ[2][8];
    if (activeA) {
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            rVX[0][k] = F.f[0][unsigned(zBegin - 3 + k) * PL + colA];
            rVY[0][k] = F.f[1][unsigned(zBegin - 3 + k) * PL + colA];
            rVZ[0][k] = F.f[2][unsigned(zBegin - 4 + k) * PL + colA];
            rVX[1][k] = F.f[0][unsigned(zBegin - 3 + k) * PL + colB];
            rVY[1][k] = F.f[1][unsigned(zBegin - 3 + k) * PL + colB];
            rVZ[1][k] = F.f[2][unsigned(zBegin - 4 + k) * PL + colB];
        }
    }
    const unsigned long long step = F.clock->step;
    const bool blastA = S.kind == 0 && activeA && abs(x - S.gxs) <= 1 && abs(ya - S.gys) <= 1;
    const bool blastB = S.kind == 0 && activeB && abs(x - S.gxs) <= 1 && abs(yb - S.gys) <= 1;
    bool bad = false;
    float check = 0.0f;   // sum of every output: non-finite if any output is
    bool stop = false;
    int j = 0, b = 0;
    uint32_t phase = 0;
    unsigned oa = unsigned(zBegin) * PL + colA;

    auto plane = [&](auto rot) {
        constexpr int U = decltype(rot)::value;
        const int z = zBegin + j;
        if (!waitFull(R, b, phase, G.waitCycles)) { stop = true; return; }
        if (activeA) {
            const float* st = smem + b * St::SIZE;
            const int ca = ra * 32 + tx, cb = ca + 32;
            rVX[0][(U + 7) & 7] = st[St::FVX + ca]; rVX[1][(U + 7) & 7] = st[St::FVX + cb];
            rVY[0][(U + 7) & 7] = st[St::FVY + ca]; rVY[1][(U + 7) & 7] = st[St::FVY + cb];
            rVZ[0][(U + 7) & 7] = st[St::FVZ + ca]; rVZ[1][(U + 7) & 7] = st[St::FVZ + cb];

            // d[v][a]: D- along its own axis, D+ across (cuda/Cuda_Seis3D.cu:293-295).
            float d00a = diffRow<40>(st + St::VX + (ra + 4) * 40 + tx, inv);
            float d00b = diffRow<40>(st + St::VX + (rb + 4) * 40 + tx, inv);
            float d01a, d01b;
            diffColPair<40>(st + St::VX + (ra + 1) * 40 + tx + 4, inv, d01a, d01b);
            float d02a = diffRingAt<U>(rVX[0], inv), d02b = diffRingAt<U>(rVX[1], inv);
            float d10a = diffRow<40>(st + St::VY + (ra + 4) * 40 + tx + 1, inv);
            float d10b = diffRow<40>(st + St::VY + (rb + 4) * 40 + tx + 1, inv);
            float d11a, d11b;
            diffColPair<40>(st + St::VY + ra * 40 + tx + 4, inv, d11a, d11b);
            float d12a = diffRingAt<U>(rVY[0], inv), d12b = diffRingAt<U>(rVY[1], inv);
            float d20a = diffRow<40>(st + St::VZ + (ra + 4) * 40 + tx + 1, inv);
            float d20b = diffRow<40>(st + St::VZ + (rb + 4) * 40 + tx + 1, inv);
            float d21a, d21b;
            diffColPair<40>(st + St::VZ + (ra + 1) * 40 + tx + 4, inv, d21a, d21b);
            float d22a = diffRingAt<U>(rVZ[0], inv), d22b = diffRingAt<U>(rVZ[1], inv);

            // CPML: velocity component v uses slot 3+v; the half grid across axes.
            Mem* psi0 = reinterpret_cast<Mem*>(F.psi[0]);
            Mem* psi1 = reinterpret_cast<Mem*>(F.psi[1]);
            if (sx.a) {
                d00a = cpmlApply(d00a, sx.ma[0], T.x[0][0][tx], T.x[0][1][tx], T.x[0][2][tx]);
                d10a = cpmlApply(d10a, sx.ma[1], T.x[1][0][tx], T.x[1][1][tx], T.x[1][2][tx]);
                d20a = cpmlApply(d20a, sx.ma[2], T.x[1][0][tx], T.x[1][1][tx], T.x[1][2][tx]);
                storeSlots(psi0, sx.oa, slotX, sx.ma);
                if (sx.b) {
                    d00b = cpmlApply(d00b, sx.mb[0], T.x[0][0][tx], T.x[0][1][tx], T.x[0][2][tx]);
                    d10b = cpmlApply(d10b, sx.mb[1], T.x[1][0][tx], T.x[1][1][tx], T.x[1][2][tx]);
                    d20b = cpmlApply(d20b, sx.mb[2], T.x[1][0][tx], T.x[1][1][tx], T.x[1][2][tx]);
                    storeSlots(psi0, sx.ob, slotX, sx.mb);
                }
            }
            if (sy.a) {
                d01a = cpmlApply(d01a, sy.ma[0], T.y[1][0][ra], T.y[1][1][ra], T.y[1][2][ra]);
                d11a = cpmlApply(d11a, sy.ma[1], T.y[0][0][ra], T.y[0][1][ra], T.y[0][2][ra]);
                d21a = cpmlApply(d21a, sy.ma[2], T.y[1][0][ra], T.y[1][1][ra], T.y[1][2][ra]);
                storeSlots(psi1, sy.oa, slotY, sy.ma);
            }
            if (sy.b) {
                d01b = cpmlApply(d01b, sy.mb[0], T.y[1][0][rb], T.y[1][1][rb], T.y[1][2][rb]);
                d11b = cpmlApply(d11b, sy.mb[1], T.y[0][0][rb], T.y[0][1][rb], T.y[0][2][rb]);
                d21b = cpmlApply(d21b, sy.mb[2], T.y[1][0][rb], T.y[1][1][rb], T.y[1][2][rb]);
                storeSlots(psi1, sy.ob, slotY, sy.mb);
            }
            const int qz = cp ? slabIndex(z, G.gz, G.pml, topFree) : -1;
            if (qz >= 0) {
                const float* kz = F.coef[2] + z * 3;
                const float* kh = F.coef[2] + (G.gz + z) * 3;
                Mem* pz = reinterpret_cast<Mem*>(F.psi[2]) + 3 * slotZ + (unsigned(qz) * G.gy + ya) * P + x;
                Mem m0 = pz[0], m1 = pz[slotZ], m2 = pz[2 * slotZ];
                d02a = cpmlApply(d02a, m0, kh[0], kh[1], kh[2]);
                d12a = cpmlApply(d12a, m1, kh[0], kh[1], kh[2]);
                d22a = cpmlApply(d22a, m2, kz[0], kz[1], kz[2]);
                pz[0] = m0; pz[slotZ] = m1; pz[2 * slotZ] = m2;
                if (activeB) {
                    Mem n0 = pz[P], n1 = pz[P + slotZ], n2 = pz[P + 2 * slotZ];
                    d02b = cpmlApply(d02b, n0, kh[0], kh[1], kh[2]);
                    d12b = cpmlApply(d12b, n1, kh[0], kh[1], kh[2]);
                    d22b = cpmlApply(d22b, n2, kz[0], kz[1], kz[2]);
                    pz[P] = n0; pz[P + slotZ] = n1; pz[P + 2 * slotZ] = n2;
                }
            }

            if (j + 1 < nPlanes) {
                sx.oa += G.gy * T0; sx.ob += G.gy * T0;
                sy.oa += T1 * P; sy.ob += T1 * P;
#pragma unroll
                for (int s3 = 0; s3 < 3; ++s3) {
                    if (sx.a) sx.ma[s3] = psiX[sx.oa + s3 * slotX];
                    if (sx.b) sx.mb[s3] = psiX[sx.ob + s3 * slotX];
                    if (sy.a) sy.ma[s3] = psiY[sy.oa + s3 * slotY];
                    if (sy.b) sy.mb[s3] = psiY[sy.ob + s3 * slotY];
                }
                const int qn = cp ? slabIndex(z + 1, G.gz, G.pml, topFree) : -1;
                if (qn >= 0)
                    prefetchZSlab(reinterpret_cast<const Mem*>(F.psi[2]) + 3 * slotZ + (unsigned(qn) * G.gy + ya) * P + x,
                                  slotZ, P, activeB);
            }

            // Reciprocals of plane z+1 (rows a, b, b+1; columns x, x+1).
            const float* m1 = st + St::M1 + ra * 36 + tx;
            const float nA0 = __fdividef(1.0f, m1[0]), nA1 = __fdividef(1.0f, m1[1]);
            const float nB0 = __fdividef(1.0f, m1[36]), nB1 = __fdividef(1.0f, m1[37]);
            const float nC0 = __fdividef(1.0f, m1[72]), nC1 = __fdividef(1.0f, m1[73]);
            const bool top = G.freeSurface && z == kRadius;
            // Row a.
            {
                const float lambda = st[St::L + ca], m = st[St::M0 + ra * 36 + tx];
                float d22 = d22a;
                if (top) d22 = -lambda / (lambda + 2 * m) * (d00a + d11a);
                const float trace = d00a + d11a + d22;
                const float muXY = __fdividef(4.0f, rA0 + rA1 + rB0 + rB1);
                const float muYZ = __fdividef(4.0f, rA0 + rB0 + nA0 + nB0);
                const float muXZ = __fdividef(4.0f, rA0 + rA1 + nA0 + nA1);
                const float* so = st + St::S + ca;
                float sxx = so[0] + G.dt * (lambda * trace + 2 * m * d00a);
                float syy = so[512] + G.dt * (lambda * trace + 2 * m * d11a);
                float szz = top ? 0.0f : so[1024] + G.dt * (lambda * trace + 2 * m * d22);
                float sxy = so[1536] + G.dt * muXY * (d01a + d10a);
                float syz = so[2048] + G.dt * muYZ * (d12a + d21a);
                float sxz = so[2560] + G.dt * muXZ * (d02a + d20a);
                check += ((sxx + syy) + (szz + sxy)) + (syz + sxz);
                if (blastA && abs(z - S.gzs) <= 1) {
                    const float value = sourceValue(G, S, x - S.gxs, ya - S.gys, z - S.gzs, (double(step) + 0.5) * G.dt);
                    sxx += value; syy += value; szz += value;
                }
                F.f[3][oa] = sxx; F.f[4][oa] = syy; F.f[5][oa] = szz;
                F.f[6][oa] = sxy; F.f[7][oa] = syz; F.f[8][oa] = sxz;
            }
            // Row b.
            if (activeB) {
                const float lambda = st[St::L + cb], m = st[St::M0 + rb * 36 + tx];
                float d22 = d22b;
                if (top) d22 = -lambda / (lambda + 2 * m) * (d00b + d11b);
                const float trace = d00b + d11b + d22;
                const float muXY = __fdividef(4.0f, rB0 + rB1 + rC0 + rC1);
                const float muYZ = __fdividef(4.0f, rB0 + rC0 + nB0 + nC0);
                const float muXZ = __fdividef(4.0f, rB0 + rB1 + nB0 + nB1);
                const float* so = st + St::S + cb;
                float sxx = so[0] + G.dt * (lambda * trace + 2 * m * d00b);
                float syy = so[512] + G.dt * (lambda * trace + 2 * m * d11b);
                float szz = top ? 0.0f : so[1024] + G.dt * (lambda * trace + 2 * m * d22);
                float sxy = so[1536] + G.dt * muXY * (d01b + d10b);
                float syz = so[2048] + G.dt * muYZ * (d12b + d21b);
                float sxz = so[2560] + G.dt * muXZ * (d02b + d20b);
                check += ((sxx + syy) + (szz + sxy)) + (syz + sxz);
                if (blastB && abs(z - S.gzs) <= 1) {
                    const float value = sourceValue(G, S, x - S.gxs, yb - S.gys, z - S.gzs, (double(step) + 0.5) * G.dt);
                    sxx += value; syy += value; szz += value;
                }
                const unsigned ob = oa + P;
                F.f[3][ob] = sxx; F.f[4][ob] = syy; F.f[5][ob] = szz;
                F.f[6][ob] = sxy; F.f[7][ob] = syz; F.f[8][ob] = sxz;
            }
            rA0 = nA0; rA1 = nA1; rB0 = nB0; rB1 = nB1; rC0 = nC0; rC1 = nC1;
        }
        releaseStage(R, j, b, nPlanes, issue);
        oa += PL;
        ++j;
        if (++b == tma::kStages) { b = 0; phase ^= 1u; }
    };

    while (j < nPlanes) {
        plane(Int<0>{});
        if (stop) break;
#pragma unroll
        for (int k = 0; k < 7; ++k)
#pragma unroll
            for (int r = 0; r < 2; ++r) { rVX[r][k] = rVX[r][k + 1]; rVY[r][k] = rVY[r][k + 1]; rVZ[r][k] = rVZ[r][k + 1]; }
    }
    if (R.stalled) drainAfterStall(F, R, j, G.waitCycles);
    flagNonFinite(F, bad || !isfinite(check));
}

__global__ void __launch_bounds__(kThreads, SEIS3D_MIN_BLOCKS)
    stressPass(Geometry G, Fields F, SourceParams S, int zChunk) {
    if (interiorTile(G, zChunk)) stressBody<false, float>(G, F, S, zChunk);
    else stressBody<true, float>(G, F, S, zChunk);
}

// The same pass with BF16 CPML memories (SEIS3D_STORAGE_BF16_CPML).
__global__ void __launch_bounds__(kThreads, SEIS3D_MIN_BLOCKS)
    stressPassBf16Cpml(Geometry G, Fields F, SourceParams S, int zChunk) {
    if (interiorTile(G, zChunk)) stressBody<false, float>(G, F, S, zChunk);
    else stressBody<true, __nv_bfloat16>(G, F, S, zChunk);
}

// Standalone free-surface images (2-D grid of 32 x 8 column tiles).
__global__ void stressImages(Geometry G, Fields F) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + kRadius;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + kRadius;
    if (x < G.gx - kRadius && y < G.gy - kRadius) stressImageColumn(G, F, x, y);
}

__global__ void velocityImages(Geometry G, Fields F) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + kRadius;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + kRadius;
    if (x < G.gx - kRadius && y < G.gy - kRadius) velocityImageColumn(G, F, x, y);
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

// Materials of `planes` physical z planes from raw SI vp, vs, rho volumes ([z][y][x], plane
// z0 first), with the host formula of uploadModelPlane3D (cuda/Cuda_Seis3D.cu:696-711)
// rounded operation by operation (no contraction), so the result is bit-identical to the
// per-plane host conversion.
__global__ void convertMaterials(Geometry G, Fields F, const float* __restrict__ vp, const float* __restrict__ vs,
                                 const float* __restrict__ rho, int z0, int planes) {
    const int64_t n = int64_t(G.nx) * G.ny;
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n * planes) return;
    const int x = int(i % G.nx), y = int((i / G.nx) % G.ny), z = int(i / n) + z0;
    const float p = vp[i], s = vs[i], r = rho[i];
    const int64_t o = int64_t(z + G.oz) * G.plane + int64_t(y + G.oy) * G.pitch + (x + G.ox);
    F.invRho[o] = __fdiv_rn(1.0f, r);
    F.lambda[o] = __fmul_rn(r, __fsub_rn(__fmul_rn(p, p), __fmul_rn(__fmul_rn(2.0f, s), s)));
    F.mu[o] = __fmul_rn(__fmul_rn(r, s), s);
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
