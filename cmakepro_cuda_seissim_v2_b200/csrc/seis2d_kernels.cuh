// seis2d_kernels.cuh - sm_100a kernels of the 2-D P-SV velocity-stress solver.
//
// The reference runs four to five launches per step (CUDA_Kernels/Cuda_Check.cu:1027-1085):
// stress, free-surface mirror, velocity, a one-thread source injection and an edge clear,
// each thread re-reading both halves of every split field from global memory for each of
// its sixteen stencil taps.  Here one step is two kernels:
//
//   stressStep   - stress update of all three schemes; the free-surface mirror is written by
//                  the threads that own the mirrored rows; the stress-type point source of the
//                  previous step is folded into the old value it would have been added to;
//                  an extra row of blocks samples the receivers of the previous step.
//   velocityStep - velocity update; air rows cleared; the force-type point source of this
//                  step is added by the thread that owns the source cell; the outer ring of
//                  velocities is cleared by the threads that own it.
//
// plus, at the end of a batch, finishBatch (stress-type source and receivers of the last
// step) so that the field state between API calls is the reference's.  Every tap is read
// from a shared-memory tile that holds both split halves, so each expression keeps the
// reference's operand order ((a1 + a2 - b1 - b2) per tap, the same tap order and the same
// averaging order) and the arithmetic matches the reference kernels operation for operation.
// The translation unit is compiled with --use_fast_math, the flag the reference builds its
// 2-D solver with (CMakeLists.txt:128-135).
//
// The grid is at most INT_MAX cells (checkedGridElementCount), so 32-bit indices suffice.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/seis2d_capi.h"

namespace seis2d {

constexpr int kBX = 32;               // threads along x per block (one warp per row)
constexpr int kBY = 16;               // rows per block
constexpr int kThreads = kBX * kBY;   // one cell per thread
constexpr int kHalo = 4;              // stencil radius (kStencilRadius, SolverNumerics.h:9)
constexpr int kTW = kBX + 2 * kHalo;  // tile width
constexpr int kTH = kBY + 2 * kHalo;  // tile height
constexpr int kTile = kTW * kTH;

// Scheme ids of the kernels (flag_type, with flag 3 and upFlag off run as flag 1;
// Cuda_Check.cu:1038-1046).
enum Scheme { kSplit = 1, kHybrid = 2, kFree = 3 };

struct Grid2D {
    int NX, NZ, total;
    int npml, fs;
    float dt, inv_dt;
    float c1, c2, c3, c4;
};

// Device buffers of a session (GPUSimData, Cuda_Check.cuh:68-121).
struct Fields2D {
    float *vx1, *vx2, *vz1, *vz2, *sxx1, *sxx2, *szz1, *szz2, *sxz1, *sxz2;
    float *vx, *vz, *sxx, *szz, *sxz;
    const float *rho, *mu, *lambda, *l2m;
    const float *muX, *lambdaX, *l2mX, *muZ, *rhoXZ, *rhoOrig;
    const float *dx, *dxh, *dz, *dzh, *dp;
};

// Per-run control block in device memory, written by configureRun before the steps of a
// run so that one captured graph serves every start step, source and receiver set.
struct Control2D {
    int base;            // step index of graph slot 0; finishBatch advances it
    int srcSingle;       // 1: the context's point source (num_active_sources < 0)
    int srcIdx;          // flat source index after the free-surface clamp
    int srcValid;        // the index passes applyPointSource's bounds checks
    int srcType;
    int srcLength;       // steps that have a wavelet sample: min(nt, wavelet size)
    float srcAngle;
    int multiCount;      // active sources injected after each velocity update
    int multiAdvance;    // advance the active sources' time by dt before each step
    int rcvCount;        // receivers sampled into the gather
    int gatherOn;
    int gatherStart, gatherStride, gatherSamples;
    const float* series; // wavelet * src_amp * 1e7 per step (computed on the host like the reference)
    const int* rcvIdx;
    float* gatherVx;
    float* gatherVz;
    seis2d_source* sources;
};

// ---- shared-memory tiles ----------------------------------------------------------------

// Tile of a field around the block: rows i0-4 .. i0+kBY+3, columns j0-4 .. j0+kBX+3; cells
// outside the grid read 0 (no computed cell uses them).
struct TileRef {
    float (*t)[kTW];
    __device__ __forceinline__ float operator()(int di, int dj) const {
        return t[threadIdx.y + kHalo + di][threadIdx.x + kHalo + dj];
    }
};

__device__ __forceinline__ void loadTiles(const Grid2D& g, int i0, int j0, float* dst, const float* const* src,
                                          int count) {
    const int tid = threadIdx.y * kBX + threadIdx.x;
    for (int t = tid; t < kTile; t += kThreads) {
        const int r = t / kTW, c = t - (t / kTW) * kTW;
        const int i = i0 - kHalo + r, j = j0 - kHalo + c;
        const bool in = i >= 0 && i < g.NZ && j >= 0 && j < g.NX;
        const int k = i * g.NX + j;
        // L2-only loads: in a persistent run other blocks rewrite these fields between the
        // grid barriers, so neither the read-only path nor L1 may hold an old copy.
        for (int a = 0; a < count; ++a) dst[a * kTile + t] = in ? __ldcg(src[a] + k) : 0.0f;
    }
}

// Split-field first derivatives, written exactly as the reference kernels write them
// (Cuda_Check.cu:236-254, 283-304, 434-486, 530-559): for each tap the two halves of the
// upper sample, minus the two halves of the lower sample.
struct Split {
    TileRef a, b;
    __device__ __forceinline__ float tap(int ui, int uj, int li, int lj) const {
        return a(ui, uj) + b(ui, uj) - a(li, lj) - b(li, lj);
    }
};

// Forward x derivative (samples j+1..j+4 minus j..j-3).
__device__ __forceinline__ float dxForward(const Grid2D& g, const Split& f) {
    return g.c1 * f.tap(0, 1, 0, 0) + g.c2 * f.tap(0, 2, 0, -1) + g.c3 * f.tap(0, 3, 0, -2) + g.c4 * f.tap(0, 4, 0, -3);
}
// Backward x derivative (samples j..j+3 minus j-1..j-4).
__device__ __forceinline__ float dxBackward(const Grid2D& g, const Split& f) {
    return g.c1 * f.tap(0, 0, 0, -1) + g.c2 * f.tap(0, 1, 0, -2) + g.c3 * f.tap(0, 2, 0, -3) + g.c4 * f.tap(0, 3, 0, -4);
}
// Forward z derivative (rows i+1..i+4 minus i..i-3).
__device__ __forceinline__ float dzForward(const Grid2D& g, const Split& f) {
    return g.c1 * f.tap(1, 0, 0, 0) + g.c2 * f.tap(2, 0, -1, 0) + g.c3 * f.tap(3, 0, -2, 0) + g.c4 * f.tap(4, 0, -3, 0);
}
// Backward z derivative (rows i..i+3 minus i-1..i-4).
__device__ __forceinline__ float dzBackward(const Grid2D& g, const Split& f) {
    return g.c1 * f.tap(0, 0, -1, 0) + g.c2 * f.tap(1, 0, -2, 0) + g.c3 * f.tap(2, 0, -3, 0) + g.c4 * f.tap(3, 0, -4, 0);
}

// Total-field derivatives of the hybrid scheme (Cuda_Check.cu:324-334, 377-387).
__device__ __forceinline__ float dxForward(const Grid2D& g, const TileRef& f) {
    return g.c1 * (f(0, 1) - f(0, 0)) + g.c2 * (f(0, 2) - f(0, -1)) + g.c3 * (f(0, 3) - f(0, -2)) + g.c4 * (f(0, 4) - f(0, -3));
}
__device__ __forceinline__ float dxBackward(const Grid2D& g, const TileRef& f) {
    return g.c1 * (f(0, 0) - f(0, -1)) + g.c2 * (f(0, 1) - f(0, -2)) + g.c3 * (f(0, 2) - f(0, -3)) + g.c4 * (f(0, 3) - f(0, -4));
}
__device__ __forceinline__ float dzForward(const Grid2D& g, const TileRef& f) {
    return g.c1 * (f(1, 0) - f(0, 0)) + g.c2 * (f(2, 0) - f(-1, 0)) + g.c3 * (f(3, 0) - f(-2, 0)) + g.c4 * (f(4, 0) - f(-3, 0));
}
__device__ __forceinline__ float dzBackward(const Grid2D& g, const TileRef& f) {
    return g.c1 * (f(0, 0) - f(-1, 0)) + g.c2 * (f(1, 0) - f(-2, 0)) + g.c3 * (f(2, 0) - f(-3, 0)) + g.c4 * (f(3, 0) - f(-4, 0));
}

// Receiver sample of the current state (extractReceiverSamplesKernel, Cuda_Check.cu:793-818).
template <int S>
__device__ __forceinline__ void sampleReceiver(const Grid2D& g, const Fields2D& f, int k, float& vx, float& vz) {
    if (k < 0 || k >= g.total) { vx = 0.0f; vz = 0.0f; return; }
    if (S == kHybrid) { vx = __ldcg(f.vx + k); vz = __ldcg(f.vz + k); }
    else { vx = __ldcg(f.vx1 + k) + __ldcg(f.vx2 + k); vz = __ldcg(f.vz1 + k) + __ldcg(f.vz2 + k); }
}

// Gather row of step `step` (the recording rule of src/Seis2D/Workflow2D.inc:320-345).
template <int S>
__device__ void recordStep(const Grid2D& g, const Fields2D& f, const Control2D& c, int step, int tid, int nthreads) {
    if (!c.gatherOn) return;
    const int rs = step - c.gatherStart;
    if (rs < 0 || rs % c.gatherStride != 0) return;
    const int sample = rs / c.gatherStride;
    if (sample >= c.gatherSamples) return;
    for (int r = tid; r < c.rcvCount; r += nthreads) {
        float vx, vz;
        sampleReceiver<S>(g, f, c.rcvIdx[r], vx, vz);
        c.gatherVx[std::size_t(r) * c.gatherSamples + sample] = vx;
        c.gatherVz[std::size_t(r) * c.gatherSamples + sample] = vz;
    }
}

// Stress-type point-source value of `step` (applyPointSource types 2 and 3,
// Cuda_Check.cu:602-621); 0 when that step injects nothing.
__device__ __forceinline__ bool stressSource(const Control2D& c, int step, float& w) {
    if (!c.srcSingle || !c.srcValid || (c.srcType != SEIS2D_EXPLOSIVE && c.srcType != SEIS2D_SHEAR)) return false;
    if (step < 0 || step >= c.srcLength) return false;
    w = c.series[step];
    return isfinite(w);
}

// ---- stress ----------------------------------------------------------------------------

// Split-field stress update of Types 1 and 3 (Cuda_Check.cu:224-266, 416-487) with the
// free-surface mirror of :491-508 written by the owners of the mirrored rows.
// Stress update of tile (bx, by) at `step`; `pendingOk` allows folding in the stress-type
// source of step-1 (false for the first step of a batch, whose source the batch end applied).
// All threads of the block call it; `tiles` holds 4 tiles of shared memory.
template <int S>
__device__ __forceinline__ void stressTile(const Grid2D& g, const Fields2D& f, const Control2D& c, int step,
                                           bool pendingOk, int bx, int by, float* tiles) {
    const int i0 = by * kBY, j0 = bx * kBX;
    if (S == kHybrid) {
        const float* src[2] = {f.vx, f.vz};
        loadTiles(g, i0, j0, tiles, src, 2);
    } else {
        const float* src[4] = {f.vx1, f.vx2, f.vz1, f.vz2};
        loadTiles(g, i0, j0, tiles, src, 4);
    }
    __syncthreads();
    const int i = i0 + threadIdx.y, j = j0 + threadIdx.x;
    const int firstRow = S == kFree ? g.fs : 4;
    if (i < firstRow || i >= g.NZ - 4 || j < 4 || j >= g.NX - 4) return;
    const int k = i * g.NX + j;
    const float inv_dt = g.inv_dt;
    float w = 0.0f;
    const bool pending = pendingOk && k == c.srcIdx && stressSource(c, step - 1, w);

    if (S == kHybrid) {
        const TileRef vx{reinterpret_cast<float(*)[kTW]>(tiles)};
        const TileRef vz{reinterpret_cast<float(*)[kTW]>(tiles + kTile)};
        const float dvz_dx = dxBackward(g, vz);
        const float dvx_dz = dzForward(g, vx);
        const float dvx_dx = dxForward(g, vx);
        const float dvz_dz = dzBackward(g, vz);
        const bool is_pml = (i < g.npml || i >= g.NZ - g.npml || j < g.npml || j >= g.NX - g.npml);
        if (!is_pml) {
            float sxz = f.sxz[k], sxx = f.sxx[k], szz = f.szz[k];
            if (pending) {
                if (c.srcType == SEIS2D_EXPLOSIVE) { sxx = __fadd_rn(sxx, w); szz = __fadd_rn(szz, w); }
                else sxz = __fadd_rn(sxz, w);
            }
            f.sxz[k] = sxz + g.dt * f.muZ[k] * (dvz_dx + dvx_dz);
            f.sxx[k] = sxx + g.dt * (f.l2mX[k] * dvx_dx + f.lambdaX[k] * dvz_dz);
            f.szz[k] = szz + g.dt * (f.lambdaX[k] * dvx_dx + f.l2mX[k] * dvz_dz);
        } else {
            const float d_z_val = f.dz[i], d_z_half_val = f.dzh[i];
            const float d_x_val = f.dx[j], d_x_half_val = f.dxh[j];
            const float sxz1 = (f.sxz1[k] * (inv_dt - d_x_val) + f.muZ[k] * dvz_dx) / (inv_dt + d_x_val);
            const float sxz2 = (f.sxz2[k] * (inv_dt - d_z_half_val) + f.muZ[k] * dvx_dz) / (inv_dt + d_z_half_val);
            const float sxx1 = (f.sxx1[k] * (inv_dt - d_x_half_val) + f.l2mX[k] * dvx_dx) / (inv_dt + d_x_half_val);
            const float szz1 = (f.szz1[k] * (inv_dt - d_x_half_val) + f.lambdaX[k] * dvx_dx) / (inv_dt + d_x_half_val);
            const float sxx2 = (f.sxx2[k] * (inv_dt - d_z_val) + f.lambdaX[k] * dvz_dz) / (inv_dt + d_z_val);
            const float szz2 = (f.szz2[k] * (inv_dt - d_z_val) + f.l2mX[k] * dvz_dz) / (inv_dt + d_z_val);
            f.sxz1[k] = sxz1; f.sxz2[k] = sxz2; f.sxx1[k] = sxx1; f.szz1[k] = szz1; f.sxx2[k] = sxx2; f.szz2[k] = szz2;
            f.sxz[k] = sxz1 + sxz2;
            f.sxx[k] = sxx1 + sxx2;
            f.szz[k] = szz1 + szz2;
        }
        return;
    }

    const Split vx{TileRef{reinterpret_cast<float(*)[kTW]>(tiles)}, TileRef{reinterpret_cast<float(*)[kTW]>(tiles + kTile)}};
    const Split vz{TileRef{reinterpret_cast<float(*)[kTW]>(tiles + 2 * kTile)},
                   TileRef{reinterpret_cast<float(*)[kTW]>(tiles + 3 * kTile)}};
    float d_z = f.dz[i], d_z_h = f.dzh[i];
    if (S == kFree && i <= g.fs + 5) { d_z = 0.0f; d_z_h = 0.0f; }
    const float d_x = f.dx[j], d_x_h = f.dxh[j];
    float sxx1 = f.sxx1[k], sxx2 = f.sxx2[k], szz1 = f.szz1[k], szz2 = f.szz2[k], sxz1 = f.sxz1[k], sxz2 = f.sxz2[k];
    if (pending) {
        const float half = w * 0.5f;
        if (c.srcType == SEIS2D_EXPLOSIVE) {
            sxx1 = __fadd_rn(sxx1, half); sxx2 = __fadd_rn(sxx2, half);
            szz1 = __fadd_rn(szz1, half); szz2 = __fadd_rn(szz2, half);
        } else {
            sxz1 = __fadd_rn(sxz1, half); sxz2 = __fadd_rn(sxz2, half);
        }
    }
    const float muAvg = 0.5f * (f.mu[k] + f.mu[k + g.NX]);
    if (S == kFree && i == g.fs) {
        // Traction-free row (Cuda_Check.cu:431-452).
        const float dvx_dx = dxForward(g, vx);
        sxx1 = (sxx1 * (inv_dt - d_x_h) + f.dp[j] * dvx_dx) / (inv_dt + d_x_h);
        const float dvz_dx = g.c1 * vz.tap(0, 0, 0, -1) + g.c2 * vz.tap(0, 1, 0, -2);
        const float dvx_dz = g.c1 * vx.tap(1, 0, 0, 0) + g.c2 * vx.tap(2, 0, -1, 0);
        sxz1 = (sxz1 * (inv_dt - d_x) + muAvg * dvz_dx) / (inv_dt + d_x);
        sxz2 = (sxz2 * (inv_dt - d_z_h) + muAvg * dvx_dz) / (inv_dt + d_z_h);
        f.szz1[k] = 0.0f; f.szz2[k] = 0.0f;
        f.sxx1[k] = sxx1; f.sxx2[k] = 0.0f;
        f.sxz1[k] = sxz1; f.sxz2[k] = sxz2;
        // Shear image one row up (mirror l = 1 of Cuda_Check.cu:502-505).
        f.sxz1[k - g.NX] = -sxz1; f.sxz2[k - g.NX] = -sxz2;
        return;
    }
    const float dvx_dx = dxForward(g, vx);
    const float dvz_dz = dzBackward(g, vz);
    const float l2mAvg = 0.5f * (f.l2m[k] + f.l2m[k + 1]);
    const float lamAvg = 0.5f * (f.lambda[k] + f.lambda[k + 1]);
    sxx1 = (sxx1 * (inv_dt - d_x_h) + l2mAvg * dvx_dx) / (inv_dt + d_x_h);
    sxx2 = (sxx2 * (inv_dt - d_z) + lamAvg * dvz_dz) / (inv_dt + d_z);
    szz1 = (szz1 * (inv_dt - d_x_h) + lamAvg * dvx_dx) / (inv_dt + d_x_h);
    szz2 = (szz2 * (inv_dt - d_z) + l2mAvg * dvz_dz) / (inv_dt + d_z);
    const float dvz_dx = dxBackward(g, vz);
    const float dvx_dz = dzForward(g, vx);
    sxz1 = (sxz1 * (inv_dt - d_x) + muAvg * dvz_dx) / (inv_dt + d_x);
    sxz2 = (sxz2 * (inv_dt - d_z_h) + muAvg * dvx_dz) / (inv_dt + d_z_h);
    f.sxx1[k] = sxx1; f.sxx2[k] = sxx2; f.szz1[k] = szz1; f.szz2[k] = szz2; f.sxz1[k] = sxz1; f.sxz2[k] = sxz2;
    if (S == kFree) {
        // Odd images above the free surface (Cuda_Check.cu:491-508): szz of row fs+l into
        // row fs-l, sxz of row fs+l-1 into row fs-l, l = 1..4.
        const int l = i - g.fs;
        if (l <= 4) {
            const int above = (g.fs - l) * g.NX + j;
            f.szz1[above] = -szz1; f.szz2[above] = -szz2;
        }
        if (l <= 3) {
            const int above = (g.fs - l - 1) * g.NX + j;
            f.sxz1[above] = -sxz1; f.sxz2[above] = -sxz2;
        }
    }
}

template <int S>
__global__ void __launch_bounds__(kThreads) stressStep(Grid2D g, Fields2D f, const Control2D* __restrict__ ctl, int slot) {
    const Control2D c = *ctl;
    const int step = c.base + slot;
    if (blockIdx.y == gridDim.y - 1) {
        // Receiver row: the velocities of step-1 are final while the stresses update.
        if (slot > 0)
            recordStep<S>(g, f, c, step - 1, blockIdx.x * kThreads + threadIdx.y * kBX + threadIdx.x, kThreads * gridDim.x);
        return;
    }
    __shared__ float tiles[4 * kTile];
    stressTile<S>(g, f, c, step, slot > 0, blockIdx.x, blockIdx.y, tiles);
}

// ---- velocity --------------------------------------------------------------------------

// Force-type point source of `step` added by the owner of the source cell after its update
// (applyPointSource types 0, 1, 4, Cuda_Check.cu:578-600, 622-633).
template <int S>
__device__ __forceinline__ void forceSource(const Grid2D& g, const Fields2D& f, const Control2D& c, int step, int k,
                                            float& vxOut, float& vzOut) {
    if (!c.srcSingle || !c.srcValid || k != c.srcIdx || step < 0 || step >= c.srcLength) return;
    if (c.srcType != SEIS2D_VERTICAL_FORCE && c.srcType != SEIS2D_HORIZONTAL_FORCE && c.srcType != SEIS2D_ROTATED_FORCE)
        return;
    const float w = c.series[step];
    if (!isfinite(w)) return;
    float force_x = w, force_z = w;
    if (c.srcType == SEIS2D_ROTATED_FORCE) {
        // M_PI is a double in the host headers the reference compiles against.
        force_x = sinf(c.srcAngle * 3.14159265358979323846 / 180.0f) * w;
        force_z = cosf(c.srcAngle * 3.14159265358979323846 / 180.0f) * w;
    }
    // The reference adds the force in a separate kernel after the update has been stored, so
    // the sum is rounded on its own: __fadd_rn keeps it from being fused into the update.
    if (S == kHybrid) {
        if (c.srcType != SEIS2D_VERTICAL_FORCE) vxOut = __fadd_rn(vxOut, force_x * g.dt / f.rhoOrig[k]);
        if (c.srcType != SEIS2D_HORIZONTAL_FORCE) vzOut = __fadd_rn(vzOut, force_z * g.dt / f.rhoXZ[k]);
    } else {
        if (c.srcType != SEIS2D_VERTICAL_FORCE) vxOut = __fadd_rn(vxOut, force_x * g.dt / f.rho[k]);
        if (c.srcType != SEIS2D_HORIZONTAL_FORCE) {
            const float rho_avg = 0.25f * (f.rho[k] + f.rho[k + 1] + f.rho[k + g.NX] + f.rho[k + g.NX + 1]);
            vzOut = __fadd_rn(vzOut, force_z * g.dt / rho_avg);
        }
    }
}

// Velocity update of the three schemes (Cuda_Check.cu:270-311, 368-412, 512-563) with the
// outer-ring clear of zeroBoundaryKernel (:643-667) done by the ring's owners.
template <int S>
__device__ __forceinline__ void velocityTile(const Grid2D& g, const Fields2D& f, const Control2D& c, int step, int bx,
                                             int by, float* tiles) {
    const int i0 = by * kBY, j0 = bx * kBX;
    if (S == kHybrid) {
        const float* src[3] = {f.sxx, f.szz, f.sxz};
        loadTiles(g, i0, j0, tiles, src, 3);
    } else {
        const float* src[6] = {f.sxx1, f.sxx2, f.szz1, f.szz2, f.sxz1, f.sxz2};
        loadTiles(g, i0, j0, tiles, src, 6);
    }
    __syncthreads();
    const int i = i0 + threadIdx.y, j = j0 + threadIdx.x;
    if (i >= g.NZ || j >= g.NX) return;
    const int k = i * g.NX + j;
    if (i == 0 || i == g.NZ - 1 || j == 0 || j == g.NX - 1) {
        if (S == kHybrid) { f.vx[k] = 0.0f; f.vz[k] = 0.0f; }
        else { f.vx1[k] = 0.0f; f.vx2[k] = 0.0f; f.vz1[k] = 0.0f; f.vz2[k] = 0.0f; }
        return;
    }
    if (i < 4 || i >= g.NZ - 4 || j < 4 || j >= g.NX - 4) return;
    const float inv_dt = g.inv_dt;

    if (S == kHybrid) {
        const TileRef sxx{reinterpret_cast<float(*)[kTW]>(tiles)};
        const TileRef szz{reinterpret_cast<float(*)[kTW]>(tiles + kTile)};
        const TileRef sxz{reinterpret_cast<float(*)[kTW]>(tiles + 2 * kTile)};
        const float dsigxz_dx = dxForward(g, sxz);
        const float dsigzz_dz = dzForward(g, szz);
        const float dsigxx_dx = dxBackward(g, sxx);
        const float dsigxz_dz = dzBackward(g, sxz);
        const bool is_pml = (i < g.npml || i >= g.NZ - g.npml || j < g.npml || j >= g.NX - g.npml);
        float vxNew, vzNew;
        if (!is_pml) {
            vzNew = f.vz[k] + g.dt * (dsigxz_dx + dsigzz_dz) / f.rhoXZ[k];
            vxNew = f.vx[k] + g.dt * (dsigxx_dx + dsigxz_dz) / f.rhoOrig[k];
        } else {
            const float d_z_val = f.dz[i], d_z_half_val = f.dzh[i];
            const float d_x_val = f.dx[j], d_x_half_val = f.dxh[j];
            const float vz1 = (f.vz1[k] * (inv_dt - d_x_half_val) + dsigxz_dx / f.rhoXZ[k]) / (inv_dt + d_x_half_val);
            const float vz2 = (f.vz2[k] * (inv_dt - d_z_half_val) + dsigzz_dz / f.rhoXZ[k]) / (inv_dt + d_z_half_val);
            const float vx1 = (f.vx1[k] * (inv_dt - d_x_val) + dsigxx_dx / f.rhoOrig[k]) / (inv_dt + d_x_val);
            const float vx2 = (f.vx2[k] * (inv_dt - d_z_val) + dsigxz_dz / f.rhoOrig[k]) / (inv_dt + d_z_val);
            f.vz1[k] = vz1; f.vz2[k] = vz2; f.vx1[k] = vx1; f.vx2[k] = vx2;
            vxNew = vx1 + vx2;
            vzNew = vz1 + vz2;
        }
        forceSource<S>(g, f, c, step, k, vxNew, vzNew);
        f.vx[k] = vxNew; f.vz[k] = vzNew;
        return;
    }

    if (S == kFree && i < g.fs) {
        f.vx1[k] = 0.0f; f.vx2[k] = 0.0f; f.vz1[k] = 0.0f; f.vz2[k] = 0.0f;
        return;
    }
    const Split sxx{TileRef{reinterpret_cast<float(*)[kTW]>(tiles)}, TileRef{reinterpret_cast<float(*)[kTW]>(tiles + kTile)}};
    const Split szz{TileRef{reinterpret_cast<float(*)[kTW]>(tiles + 2 * kTile)},
                    TileRef{reinterpret_cast<float(*)[kTW]>(tiles + 3 * kTile)}};
    const Split sxz{TileRef{reinterpret_cast<float(*)[kTW]>(tiles + 4 * kTile)},
                    TileRef{reinterpret_cast<float(*)[kTW]>(tiles + 5 * kTile)}};
    float d_z = f.dz[i], d_z_h = f.dzh[i];
    if (S == kFree && i <= g.fs + 5) { d_z = 0.0f; d_z_h = 0.0f; }
    const float d_x = f.dx[j], d_x_h = f.dxh[j];
    const float cur_rho = f.rho[k];
    const float dsigxx_dx = dxBackward(g, sxx);
    const float dsigxz_dz = dzBackward(g, sxz);
    float vx1 = (f.vx1[k] * (inv_dt - d_x) + dsigxx_dx / cur_rho) / (inv_dt + d_x);
    const float vx2 = (f.vx2[k] * (inv_dt - d_z) + dsigxz_dz / cur_rho) / (inv_dt + d_z);
    const float dsigxz_dx = dxForward(g, sxz);
    const float dsigzz_dz = dzForward(g, szz);
    const float rho_avg = 0.25f * (f.rho[k] + f.rho[k + 1] + f.rho[k + g.NX] + f.rho[k + g.NX + 1]);
    float vz1 = (f.vz1[k] * (inv_dt - d_x_h) + dsigxz_dx / rho_avg) / (inv_dt + d_x_h);
    const float vz2 = (f.vz2[k] * (inv_dt - d_z_h) + dsigzz_dz / rho_avg) / (inv_dt + d_z_h);
    forceSource<S>(g, f, c, step, k, vx1, vz1);
    f.vx1[k] = vx1; f.vx2[k] = vx2; f.vz1[k] = vz1; f.vz2[k] = vz2;
}

template <int S>
__global__ void __launch_bounds__(kThreads) velocityStep(Grid2D g, Fields2D f, const Control2D* __restrict__ ctl, int slot) {
    const Control2D c = *ctl;
    __shared__ float tiles[6 * kTile];
    velocityTile<S>(g, f, c, c.base + slot, blockIdx.x, blockIdx.y, tiles);
}

// ---- multi-source injection (injectMultipleSourcesKernel, Cuda_Check.cu:822-834) ---------

// Adds one source value through the field the reference's applyPointSource picks
// (Cuda_Check.cu:567-634), with atomics because sources may overlap.
template <int S>
__device__ void applySource(const Grid2D& g, const Fields2D& f, int type, float angle, float w, int idx) {
    if (idx < 0 || idx >= g.total || !isfinite(w)) return;
    const int x = idx % g.NX, z = idx / g.NX;
    if (x < 4 || x >= g.NX - 4 || z < 4 || z >= g.NZ - 4 || (S == kFree && z <= g.fs)) return;
    if (type == SEIS2D_VERTICAL_FORCE || type == SEIS2D_HORIZONTAL_FORCE || type == SEIS2D_ROTATED_FORCE) {
        float force_x = w, force_z = w;
        if (type == SEIS2D_ROTATED_FORCE) {
            force_x = sinf(angle * 3.14159265358979323846 / 180.0f) * w;
            force_z = cosf(angle * 3.14159265358979323846 / 180.0f) * w;
        }
        if (S == kHybrid) {
            if (type != SEIS2D_VERTICAL_FORCE) atomicAdd(&f.vx[idx], force_x * g.dt / f.rhoOrig[idx]);
            if (type != SEIS2D_HORIZONTAL_FORCE) atomicAdd(&f.vz[idx], force_z * g.dt / f.rhoXZ[idx]);
        } else {
            if (type != SEIS2D_VERTICAL_FORCE) atomicAdd(&f.vx1[idx], force_x * g.dt / f.rho[idx]);
            if (type != SEIS2D_HORIZONTAL_FORCE) {
                const float rho_avg = 0.25f * (f.rho[idx] + f.rho[idx + 1] + f.rho[idx + g.NX] + f.rho[idx + g.NX + 1]);
                atomicAdd(&f.vz1[idx], force_z * g.dt / rho_avg);
            }
        }
    } else if (type == SEIS2D_EXPLOSIVE) {
        if (S == kHybrid) { atomicAdd(&f.sxx[idx], w); atomicAdd(&f.szz[idx], w); }
        else {
            atomicAdd(&f.sxx1[idx], w * 0.5f); atomicAdd(&f.sxx2[idx], w * 0.5f);
            atomicAdd(&f.szz1[idx], w * 0.5f); atomicAdd(&f.szz2[idx], w * 0.5f);
        }
    } else if (type == SEIS2D_SHEAR) {
        if (S == kHybrid) atomicAdd(&f.sxz[idx], w);
        else { atomicAdd(&f.sxz1[idx], w * 0.5f); atomicAdd(&f.sxz2[idx], w * 0.5f); }
    }
}

// Index written over an active source that has expired during an advancing run.
constexpr int kDroppedSource = INT32_MIN;

// One thread per active source.  With multiAdvance the source time moves by dt first and a
// source past 2.5 / f_peak is dropped, as the reference host loop does before each step
// (src/Seis2D/Workflow2D.inc:300-312); host arithmetic there, so the expiry test uses a
// correctly rounded division.
template <int S>
__global__ void injectSources(Grid2D g, Fields2D f, const Control2D* __restrict__ ctl) {
    const Control2D c = *ctl;
    const int r = threadIdx.x;
    if (r >= c.multiCount) return;
    seis2d_source src = c.sources[r];
    if (c.multiAdvance) {
        if (src.idx == kDroppedSource) return;  // expired earlier
        src.t = src.t + g.dt;
        c.sources[r].t = src.t;
        const float t_peak_host = __fdiv_rn(1.0f, src.f_peak);
        if (src.t > 2.5f * t_peak_host) { c.sources[r].idx = kDroppedSource; return; }
    }
    if (!isfinite(src.f_peak) || src.f_peak <= 0.0f || !isfinite(src.t)) return;
    const float t_peak = 1.0f / src.f_peak;
    const float x = 3.14159265358979323846 * src.f_peak * (src.t - t_peak);
    const float val = src.amp * (1.0f - 2.0f * x * x) * expf(-x * x);
    applySource<S>(g, f, c.srcType, c.srcAngle, val * SEIS2D_SOURCE_INJECTION_SCALE, src.idx);
}

// ---- batch boundaries ------------------------------------------------------------------

__global__ void configureRun(Control2D* ctl, Control2D value) { *ctl = value; }

// Completes the last step of a batch: its stress-type point source and its receivers, then
// advances the clock by the batch length.
template <int S>
__device__ void finishStep(const Grid2D& g, const Fields2D& f, const Control2D& c, int step, int tid, int nthreads) {
    recordStep<S>(g, f, c, step, tid, nthreads);
    if (tid == 0) {
        float w;
        if (stressSource(c, step, w)) {
            const int k = c.srcIdx;
            if (S == kHybrid) {
                if (c.srcType == SEIS2D_EXPLOSIVE) { f.sxx[k] += w; f.szz[k] += w; }
                else f.sxz[k] += w;
            } else if (c.srcType == SEIS2D_EXPLOSIVE) {
                f.sxx1[k] += w * 0.5f; f.sxx2[k] += w * 0.5f; f.szz1[k] += w * 0.5f; f.szz2[k] += w * 0.5f;
            } else {
                f.sxz1[k] += w * 0.5f; f.sxz2[k] += w * 0.5f;
            }
        }
    }
}

template <int S>
__global__ void finishBatch(Grid2D g, Fields2D f, Control2D* ctl, int slot, int batch) {
    const Control2D c = *ctl;
    finishStep<S>(g, f, c, c.base + slot, threadIdx.x, blockDim.x);
    __syncthreads();
    if (threadIdx.x == 0) ctl->base = c.base + batch;
}

// ---- persistent run (one cooperative launch for many steps) -----------------------------

// Grid barrier state of a persistent run, cleared before each launch.
struct GridSync {
    unsigned arrived;   // blocks that reached barriers so far (monotonic within a launch)
    unsigned failed;    // a barrier wait gave up; the run's results are invalid
    unsigned pad[2];
};

// Default bound of one barrier wait in SM clock cycles (about two seconds): the launch is
// cooperative, so every block is resident and a normal wait ends in microseconds.
constexpr long long kBarrierCycles = 4000000000LL;

// Bound of the barrier waits and the withheld-arrival test hook of one persistent run.
struct BarrierLimits {
    long long cycles;     // bound of every wait
    int withheldBlock;    // test hook: this block never arrives at the first barrier; -1 in use
};

// Grid-wide barrier number `epoch` (1, 2, ...): returns false when any wait timed out, in
// which case every block leaves the run.
__device__ __forceinline__ bool gridBarrier(GridSync* gs, unsigned epoch, const BarrierLimits& lim) {
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        __threadfence();
        if (epoch != 1 || int(blockIdx.x) != lim.withheldBlock) atomicAdd(&gs->arrived, 1u);
        const unsigned target = epoch * gridDim.x;
        const long long start = clock64();
        while (*reinterpret_cast<volatile unsigned*>(&gs->arrived) < target) {
            if (*reinterpret_cast<volatile unsigned*>(&gs->failed)) break;
            if (clock64() - start > lim.cycles) {
                atomicExch(&gs->failed, 1u);
                break;
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *reinterpret_cast<volatile unsigned*>(&gs->failed) == 0;
}

// `count` steps from ctl->base with every block resident: per step the stress phase over all
// tiles, a grid barrier, the velocity phase, a grid barrier.  The receivers of step-1 are
// sampled after the stress phase (velocities are final then) and the last step is completed
// as at a batch end.  Single-source runs only; multi-source runs use the per-step kernels.
template <int S>
__global__ void __launch_bounds__(kThreads, 3) runSteps(Grid2D g, Fields2D f, Control2D* ctl, GridSync* gs, int count,
                                                        BarrierLimits lim) {
    __shared__ float tiles[6 * kTile];
    const Control2D c = *ctl;
    const int tilesX = (g.NX + kBX - 1) / kBX, tilesY = (g.NZ + kBY - 1) / kBY, nTiles = tilesX * tilesY;
    const int gtid = blockIdx.x * kThreads + threadIdx.y * kBX + threadIdx.x, gthreads = gridDim.x * kThreads;
    unsigned epoch = 0;
    for (int q = 0; q < count; ++q) {
        const int step = c.base + q;
        for (int t = blockIdx.x; t < nTiles; t += gridDim.x) {
            stressTile<S>(g, f, c, step, q > 0, t % tilesX, t / tilesX, tiles);
            __syncthreads();
        }
        if (q > 0) recordStep<S>(g, f, c, step - 1, gtid, gthreads);
        if (!gridBarrier(gs, ++epoch, lim)) return;
        for (int t = blockIdx.x; t < nTiles; t += gridDim.x) {
            velocityTile<S>(g, f, c, step, t % tilesX, t / tilesX, tiles);
            __syncthreads();
        }
        if (!gridBarrier(gs, ++epoch, lim)) return;
    }
    finishStep<S>(g, f, c, c.base + count - 1, gtid, gthreads);
    if (gtid == 0) ctl->base = c.base + count;
}

// recordReceiverStepOnGpu / copyReceiverRecordsFromGpu sample (Cuda_Check.cu:793-818).
template <int S>
__global__ void extractReceivers(Grid2D g, Fields2D f, const int* __restrict__ idx, int count, float* outVx, float* outVz) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= count) return;
    float vx, vz;
    sampleReceiver<S>(g, f, idx[r], vx, vz);
    outVx[r] = vx;
    outVz[r] = vz;
}

// generateColorMapKernel (Cuda_Check.cu:700-790) behind generateWavefieldTextureOnGpu
// (:1136-1141): one RGBA pixel per grid cell, red for positive and blue for negative values of
// the selected component times scale and the component's balance factor.  `split` selects the
// split-field halves (flag_type 1 and 3) or the total fields (flag_type 2); any other scheme id
// reads the totals and shows no stress, as the reference's branches do.  The expressions keep
// the reference's operand order and its float-to-byte truncations.
struct ColorFields {
    const float *vx1, *vx2, *vz1, *vz2, *sxx1, *sxx2, *szz1, *szz2, *sxz1, *sxz2;
    const float *vx, *vz, *sxx, *szz, *sxz;
    const float *mu, *l2m;
};

__device__ __forceinline__ float colorVx(const ColorFields& f, int NX, int NZ, bool split, int i, int j) {
    const int r = i < 0 ? 0 : (i > NZ - 1 ? NZ - 1 : i);
    const int c = j < 0 ? 0 : (j > NX - 1 ? NX - 1 : j);
    const int k = r * NX + c;
    return split ? f.vx1[k] + f.vx2[k] : f.vx[k];
}

__device__ __forceinline__ float colorVz(const ColorFields& f, int NX, int NZ, bool split, int i, int j) {
    const int r = i < 0 ? 0 : (i > NZ - 1 ? NZ - 1 : i);
    const int c = j < 0 ? 0 : (j > NX - 1 ? NX - 1 : j);
    const int k = r * NX + c;
    return split ? f.vz1[k] + f.vz2[k] : f.vz[k];
}

__global__ void __launch_bounds__(256) colorMap(ColorFields f, int NX, int NZ, int flag, uchar4* out, float scale,
                                                int component) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= NZ || j >= NX) return;
    const int k = i * NX + j;
    const bool split = flag == 1 || flag == 3;
    float val = 0.0f, balance = 1.0f;
    if (component == 0) {
        const float vx = colorVx(f, NX, NZ, split, i, j), vz = colorVz(f, NX, NZ, split, i, j);
        val = sqrtf(vx * vx + vz * vz);
    } else if (component == 1) {
        val = colorVx(f, NX, NZ, split, i, j);
    } else if (component == 2) {
        val = colorVz(f, NX, NZ, split, i, j);
    } else if (component == 3) {
        // Normal stress scaled to a strain by lambda + 2 mu.
        float stress = 0.0f;
        if (split) stress = f.sxx1[k] + f.sxx2[k] + f.szz1[k] + f.szz2[k];
        else if (flag == 2) stress = f.sxx[k] + f.szz[k];
        const float l2m = f.l2m[k];
        val = l2m > 1000.0f ? stress / l2m : stress;
        val *= 1000;
        balance = 2.0f;
    } else if (component == 4) {
        // Shear stress scaled by mu.
        float shear = 0.0f;
        if (split) shear = f.sxz1[k] + f.sxz2[k];
        else if (flag == 2) shear = f.sxz[k];
        const float mu = f.mu[k];
        val = mu > 1000.0f ? shear / mu : shear;
        val *= 1000;
        balance = 3.0f;
    } else if (component == 5) {
        // Divergence (P waves).
        const float dvxdx = colorVx(f, NX, NZ, split, i, j) - colorVx(f, NX, NZ, split, i, j - 1);
        const float dvzdz = colorVz(f, NX, NZ, split, i, j) - colorVz(f, NX, NZ, split, i - 1, j);
        val = dvxdx + dvzdz;
        balance = 8.0f;
    } else if (component == 6) {
        // Curl (S waves).
        const float dvzdx = colorVz(f, NX, NZ, split, i, j) - colorVz(f, NX, NZ, split, i, j - 1);
        const float dvxdz = colorVx(f, NX, NZ, split, i, j) - colorVx(f, NX, NZ, split, i - 1, j);
        val = dvzdx - dvxdz;
        balance = 8.0f;
    }
    float norm = val * scale * balance;
    if (norm > 1.0f) norm = 1.0f;
    if (norm < -1.0f) norm = -1.0f;
    unsigned char r = 255, g = 255, b = 255;
    if (norm > 0.0f) {
        g = static_cast<unsigned char>(255.0f * (1.0f - norm));
        b = static_cast<unsigned char>(255.0f * (1.0f - norm));
    } else {
        r = static_cast<unsigned char>(255.0f * (1.0f + norm));
        g = static_cast<unsigned char>(255.0f * (1.0f + norm));
    }
    out[k] = make_uchar4(r, g, b, 255);
}

}  // namespace seis2d
