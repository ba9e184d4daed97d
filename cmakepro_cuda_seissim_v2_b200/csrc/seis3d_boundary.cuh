// seis3d_boundary.cuh - the learned thin boundary: a per-face MLP that corrects the interior
// cells next to a thin CPML so that the interior evolves as it would beside a wide one.
//
// Formulation.  A session with a thin CPML (4-7 cells) reflects part of every outgoing wave.
// After each step, every boundary column of each CPML face (a line of 8 cells along the face
// normal: 4 interior cells next to the interface and the first 4 CPML cells) is mapped by the
// face's network to a correction of the 9 wavefields on its 4 interior cells.  The training
// target is the difference between a run of the same model beside a 40-cell CPML and the thin
// run, both stepped in lock step with the thin run's interior reset to the wide run's after
// every step, so the network learns the one-step difference the thin layer introduces.
//
// Network (one per face, no reference counterpart): 256 inputs -> 64 -> 64 -> 36, ReLU,
// BF16 weights and activations into the tensor cores (mma.sync m16n8k16, FP32 accumulate),
// FP32 biases and master weights.  Inputs, per column: the 8-cell stencil of the 9 fields
// (velocities as they are, stresses divided by the column's P impedance), its central
// differences along the two directions within the face, the six CPML memories (psi) of the
// face's axis on the 4 CPML cells (times h; stress-derivative memories also divided by the
// impedance) -- the history the layer has absorbed, which one time slice of the fields does
// not show -- all divided by the column's RMS amplitude s; and five scheme numbers (local P
// and S Courant numbers, the maximum Courant number, frequency x dt, 1).  Outputs are the 36 corrections divided by s and by a per-face
// output scale, so the network works on unit-size numbers whatever the wave amplitude.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace seis3d {
namespace bnet {

constexpr int kDepth = 8;          // stencil cells per column: 4 interior, 4 CPML
constexpr int kBand = 4;           // corrected interior cells per column
constexpr int kColumnValues = 9 * kDepth;     // 72
constexpr int kFeatures = 3 * kColumnValues;  // 216: column, two lateral differences
constexpr int kMemoryValues = 6 * 4;          // 24: psi slots 0-5 on the 4 CPML cells
constexpr int kScheme = kFeatures + kMemoryValues;   // 240: 5 scheme inputs, then zero padding
constexpr int kIn = 256;
constexpr int kHidden = 64;
constexpr int kOut = 9 * kBand;    // 36
constexpr int kOutPad = 48;        // rows of W3 (36 used; the rest stay zero)
constexpr int kFaces = 6;          // 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+

// Parameter block of one face (FP32 master copy; the matrices also exist in BF16).
constexpr int kW1 = 0;                              // [64][256]
constexpr int kW2 = kW1 + kHidden * kIn;            // [64][64]
constexpr int kW3 = kW2 + kHidden * kHidden;        // [48][64]
constexpr int kMatrixCount = kW3 + kOutPad * kHidden;   // 23552
constexpr int kB1 = kMatrixCount;                   // [64]
constexpr int kB2 = kB1 + kHidden;                  // [64]
constexpr int kB3 = kB2 + kHidden;                  // [48]
constexpr int kParamCount = kB3 + kOutPad;          // 23728

// Shared-memory row strides (bf16 elements) chosen so that the 8 rows of an mma fragment
// fall on distinct banks.
constexpr int kLdIn = 264;
constexpr int kLdHid = 72;

// One CPML face as the kernels see it.
struct Face {
    int present;       // the face has a CPML (not the free surface, not reflecting)
    int nu, nw;        // lateral extents (physical cells)
    int64_t du, dw;    // element strides along the two lateral directions
    int64_t dn;        // element stride one cell outward along the normal
    int64_t base;      // element index of the interior cell next to the interface at (0, 0)
    int64_t wideBase;  // the same cell in the wide session (training only)
    int64_t wideDu, wideDw, wideDn;
    int columnBegin;   // first global column index of this face
    int loU, hiU, loW, hiW;   // face index owning the lateral ends' bands (-1 = none)
    const float* psi;  // CPML memories of the face's axis (slot 0)
    int64_t psiSlot;   // elements per slot
    int64_t psiBase;   // element of the first CPML cell (d = 4) of column (0, 0)
    int64_t psiDu, psiDw, psiDn;
};

struct Faces {
    Face f[kFaces];
    int columns;       // total columns over the present faces
    float cmax;        // maximum P Courant number maxVp dt / h
    float fdt;         // frequency x dt
    float dtOverH;
    float h;           // grid spacing
};

__device__ __forceinline__ uint32_t packBf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// D += A(16x16, row) * B(16x8, col), BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t lds32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ uint32_t pair16(const __nv_bfloat16* lo, const __nv_bfloat16* hi) {
    const uint32_t a = *reinterpret_cast<const unsigned short*>(lo);
    const uint32_t b = *reinterpret_cast<const unsigned short*>(hi);
    return a | (b << 16);
}

// Weights of one face staged in shared memory (padded rows) plus the FP32 biases.
struct SharedNet {
    __nv_bfloat16 w1[kHidden * kLdIn];
    __nv_bfloat16 w2[kHidden * kLdHid];
    __nv_bfloat16 w3[kOutPad * kLdHid];
    float b1[kHidden], b2[kHidden], b3[kOutPad];
};

__device__ __forceinline__ void loadNet(SharedNet& S, const __nv_bfloat16* w, const float* p, int tid, int threads) {
    for (int e = tid; e < kHidden * kIn / 2; e += threads) {
        const int r = (2 * e) / kIn, c = (2 * e) % kIn;
        *reinterpret_cast<uint32_t*>(&S.w1[r * kLdIn + c]) = lds32(w + kW1 + 2 * e);
    }
    for (int e = tid; e < kHidden * kHidden / 2; e += threads) {
        const int r = (2 * e) / kHidden, c = (2 * e) % kHidden;
        *reinterpret_cast<uint32_t*>(&S.w2[r * kLdHid + c]) = lds32(w + kW2 + 2 * e);
    }
    for (int e = tid; e < kOutPad * kHidden / 2; e += threads) {
        const int r = (2 * e) / kHidden, c = (2 * e) % kHidden;
        *reinterpret_cast<uint32_t*>(&S.w3[r * kLdHid + c]) = lds32(w + kW3 + 2 * e);
    }
    for (int e = tid; e < kHidden; e += threads) { S.b1[e] = p[kB1 + e]; S.b2[e] = p[kB2 + e]; }
    for (int e = tid; e < kOutPad; e += threads) S.b3[e] = p[kB3 + e];
}

// Forward pass of 16 rows (one warp) whose inputs sit in `a` (bf16, row stride kLdIn).
// Returns the layer-3 accumulators y[5][4] (C fragments: rows g, g+8; outputs 8n+2t, +1) and
// leaves the hidden activations as A fragments h1[4][4], h2[4][4] (for the backward pass).
struct Hidden { uint32_t h1[4][4], h2[4][4]; };

__device__ __forceinline__ void forward16(const SharedNet& S, const __nv_bfloat16* a, float (&y)[5][4], Hidden& H) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float acc[8][4];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const float b0 = S.b1[8 * n + 2 * t], b1 = S.b1[8 * n + 2 * t + 1];
        acc[n][0] = b0; acc[n][1] = b1; acc[n][2] = b0; acc[n][3] = b1;
    }
#pragma unroll 2
    for (int k = 0; k < kIn / 16; ++k) {
        uint32_t f[4];
        f[0] = lds32(a + g * kLdIn + 16 * k + 2 * t);
        f[1] = lds32(a + (g + 8) * kLdIn + 16 * k + 2 * t);
        f[2] = lds32(a + g * kLdIn + 16 * k + 8 + 2 * t);
        f[3] = lds32(a + (g + 8) * kLdIn + 16 * k + 8 + 2 * t);
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const __nv_bfloat16* w = S.w1 + (8 * n + g) * kLdIn + 16 * k + 2 * t;
            mma16816(acc[n], f, lds32(w), lds32(w + 8));
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        H.h1[j][0] = packBf16(fmaxf(acc[2 * j][0], 0.f), fmaxf(acc[2 * j][1], 0.f));
        H.h1[j][1] = packBf16(fmaxf(acc[2 * j][2], 0.f), fmaxf(acc[2 * j][3], 0.f));
        H.h1[j][2] = packBf16(fmaxf(acc[2 * j + 1][0], 0.f), fmaxf(acc[2 * j + 1][1], 0.f));
        H.h1[j][3] = packBf16(fmaxf(acc[2 * j + 1][2], 0.f), fmaxf(acc[2 * j + 1][3], 0.f));
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const float b0 = S.b2[8 * n + 2 * t], b1 = S.b2[8 * n + 2 * t + 1];
        acc[n][0] = b0; acc[n][1] = b1; acc[n][2] = b0; acc[n][3] = b1;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const __nv_bfloat16* w = S.w2 + (8 * n + g) * kLdHid + 16 * k + 2 * t;
            mma16816(acc[n], H.h1[k], lds32(w), lds32(w + 8));
        }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        H.h2[j][0] = packBf16(fmaxf(acc[2 * j][0], 0.f), fmaxf(acc[2 * j][1], 0.f));
        H.h2[j][1] = packBf16(fmaxf(acc[2 * j][2], 0.f), fmaxf(acc[2 * j][3], 0.f));
        H.h2[j][2] = packBf16(fmaxf(acc[2 * j + 1][0], 0.f), fmaxf(acc[2 * j + 1][1], 0.f));
        H.h2[j][3] = packBf16(fmaxf(acc[2 * j + 1][2], 0.f), fmaxf(acc[2 * j + 1][3], 0.f));
    }
#pragma unroll
    for (int n = 0; n < 5; ++n) {
        const float b0 = S.b3[8 * n + 2 * t], b1 = S.b3[8 * n + 2 * t + 1];
        y[n][0] = b0; y[n][1] = b1; y[n][2] = b0; y[n][3] = b1;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int n = 0; n < 5; ++n) {
            const __nv_bfloat16* w = S.w3 + (8 * n + g) * kLdHid + 16 * k + 2 * t;
            mma16816(y[n], H.h2[k], lds32(w), lds32(w + 8));
        }
}

// ---------------------------------------------------------------------------------------
// Column geometry and features.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int faceOf(const Faces& F, int column) {
    int f = 0;
#pragma unroll
    for (int k = 1; k < kFaces; ++k)
        if (F.f[k].present && column >= F.f[k].columnBegin) f = k;
    return f;
}

// Element index of stencil cell `d` (0..3 interior, deepest first; 4..7 CPML, nearest first).
__device__ __forceinline__ int64_t cellIndex(const Face& f, int u, int w, int d) {
    return f.base + int64_t(u) * f.du + int64_t(w) * f.dw + int64_t(d - 3) * f.dn;
}

// True when interior cell `d` (0..3) of column (u, w) of face `self` gets this face's
// correction: a cell within 4 cells of two faces belongs to the face it is nearer to (ties to
// the lower face index).
__device__ __forceinline__ bool owns(const Face& f, int self, int u, int w, int d) {
    const int depth = 3 - d;   // cells from the interface
    const int ends[4] = {f.loU, f.hiU, f.loW, f.hiW};
    const int dist[4] = {u, f.nu - 1 - u, w, f.nw - 1 - w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        if (ends[e] < 0 || dist[e] >= kBand) continue;
        if (dist[e] < depth || (dist[e] == depth && ends[e] < self)) return false;
    }
    return true;
}

struct Materials { const float* invRho; const float* lambda; const float* mu; };

// Inputs of one column written as bf16 into `row` (kIn values) and returned: s (0 when the
// column is at rest) and the impedance used for the stresses.  One thread per column half:
// `half` 0 writes the fields 0-4 part, 1 the rest, both compute s.
__device__ __forceinline__ void columnScale(const Face& f, const float* const* field, const Materials& M, int u, int w,
                                            float& s, float& z, float& cp, float& cs, float dtOverH) {
    const int64_t c = cellIndex(f, u, w, 3);
    const float invRho = M.invRho[c], modulus = M.lambda[c] + 2.0f * M.mu[c];
    z = sqrtf(modulus / invRho);
    cp = sqrtf(modulus * invRho) * dtOverH;
    cs = sqrtf(M.mu[c] * invRho) * dtOverH;
    const float iz = 1.0f / z;
    float sum = 0.0f;
    for (int k = 0; k < 9; ++k) {
        const float scale = k < 3 ? 1.0f : iz;
        for (int d = 0; d < kDepth; ++d) {
            const float v = field[k][cellIndex(f, u, w, d)] * scale;
            sum += v * v;
        }
    }
    s = sqrtf(sum / float(kColumnValues));
}

__device__ __forceinline__ void columnFeatures(const Face& f, const float* const* field, int u, int w, float s, float z,
                                               float cp, float cs, const Faces& F, int half, __nv_bfloat16* row) {
    const float inv = s > 0.0f ? 1.0f / s : 0.0f;
    const float iz = 1.0f / z;
    for (int i = half; i < kColumnValues; i += 2) {
        const int k = i / kDepth, d = i % kDepth;
        const float scale = (k < 3 ? 1.0f : iz) * inv;
        const float* p = field[k] + cellIndex(f, u, w, d);
        const float centre = p[0];
        const float du = p[f.du] - p[-f.du];
        const float dw = p[f.dw] - p[-f.dw];
        row[i] = __float2bfloat16_rn(centre * scale);
        row[kColumnValues + i] = __float2bfloat16_rn(du * scale);
        row[2 * kColumnValues + i] = __float2bfloat16_rn(dw * scale);
    }
    // CPML memories: half 0 the velocity pass's slots 0-2 (stress derivatives), half 1 the
    // stress pass's slots 3-5 (velocity derivatives).
    for (int slot = 3 * half; slot < 3 * half + 3; ++slot) {
        const float scale = (slot < 3 ? F.h * iz : F.h) * inv;
        const float* q = f.psi + slot * f.psiSlot + f.psiBase + int64_t(u) * f.psiDu + int64_t(w) * f.psiDw;
        for (int d = 0; d < 4; ++d) row[kFeatures + 4 * slot + d] = __float2bfloat16_rn(q[int64_t(d) * f.psiDn] * scale);
    }
    if (half == 0) {
        // Scheme numbers, then zeros up to the padded input width.
        const float extra[5] = {cp, cs, F.cmax, F.fdt, 1.0f};
        for (int e = 0; e < kIn - kScheme; ++e) row[kScheme + e] = __float2bfloat16_rn(e < 5 ? extra[e] : 0.0f);
    }
}

// ---------------------------------------------------------------------------------------
// Inference: corrections of every boundary column into `out` ([column][36], FP32), then
// added to the fields by applyCorrections (two launches, so that no column reads a cell
// another column has already corrected).
// ---------------------------------------------------------------------------------------
constexpr int kInferWarps = 4;
constexpr int kInferRows = 16 * kInferWarps;

struct InferArgs {
    Faces faces;
    const float* field[9];
    Materials mat;
    const __nv_bfloat16* weights;   // kFaces x kMatrixCount
    const float* params;            // kFaces x kParamCount (biases)
    const float* outScale;          // kFaces
    float* out;                     // columns x 36
};

__global__ void __launch_bounds__(32 * kInferWarps) correctionForward(InferArgs A, int face) {
    extern __shared__ __align__(16) unsigned char smemRaw[];
    SharedNet& S = *reinterpret_cast<SharedNet*>(smemRaw);
    __nv_bfloat16* tiles = reinterpret_cast<__nv_bfloat16*>(smemRaw + sizeof(SharedNet));
    __shared__ float rowScale[kInferRows], rowImpedance[kInferRows];
    const Face& f = A.faces.f[face];
    const int columns = f.nu * f.nw;
    loadNet(S, A.weights + size_t(face) * kMatrixCount, A.params + size_t(face) * kParamCount, threadIdx.x, blockDim.x);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    __nv_bfloat16* a = tiles + warp * 16 * kLdIn;
    const float outScale = A.outScale[face];
    for (int first = blockIdx.x * kInferRows + warp * 16; first < columns; first += gridDim.x * kInferRows) {
        const int r = lane & 15, half = lane >> 4;
        const int col = first + r;
        float s = 0.0f, z = 1.0f, cp = 0.0f, cs = 0.0f;
        int u = 0, w = 0;
        if (col < columns) {
            u = col % f.nu; w = col / f.nu;
            columnScale(f, A.field, A.mat, u, w, s, z, cp, cs, A.faces.dtOverH);
            columnFeatures(f, A.field, u, w, s, z, cp, cs, A.faces, half, a + r * kLdIn);
        } else {
            for (int i = half; i < kIn; i += 2) a[r * kLdIn + i] = __float2bfloat16_rn(0.0f);
        }
        if (half == 0) { rowScale[warp * 16 + r] = s; rowImpedance[warp * 16 + r] = z; }
        __syncwarp();
        float y[5][4];
        Hidden H;
        forward16(S, a, y, H);
        // Rows g and g+8, outputs 8n + 2t (+1): value x outScale x s (x z for stresses).
#pragma unroll
        for (int half8 = 0; half8 < 2; ++half8) {
            const int rr = g + 8 * half8, cc = first + rr;
            if (cc >= columns) continue;
            const float sr = rowScale[warp * 16 + rr] * outScale, zr = rowImpedance[warp * 16 + rr];
            float* o = A.out + size_t(f.columnBegin + cc) * kOut;
#pragma unroll
            for (int n = 0; n < 5; ++n)
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int out = 8 * n + 2 * t + q;
                    if (out >= kOut) continue;
                    const float v = y[n][2 * half8 + q] * sr * (out / kBand < 3 ? 1.0f : zr);
                    o[out] = v;
                }
        }
        __syncwarp();
    }
}

struct FieldPtrs { float* f[9]; };

// Adds gain x correction to every owned interior cell (one thread per column and output).
__global__ void applyCorrections(Faces F, FieldPtrs P, const float* corr, float gain) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(F.columns) * kOut) return;
    const int column = int(i / kOut), out = int(i % kOut);
    const int face = faceOf(F, column);
    const Face& f = F.f[face];
    const int local = column - f.columnBegin;
    const int u = local % f.nu, w = local / f.nu;
    const int k = out / kBand, d = out % kBand;
    if (!owns(f, face, u, w, d)) return;
    P.f[k][cellIndex(f, u, w, d)] += gain * corr[i];
}

// ---------------------------------------------------------------------------------------
// Training data: rows of the thin session's columns with the targets from the wide session.
// ---------------------------------------------------------------------------------------
struct CollectArgs {
    Faces faces;
    const float* thin[9];
    const float* wide[9];
    Materials mat;
    float fraction;                 // share of the columns recorded
    unsigned long long seed;
    int model;                      // index of the training model (for the per-model weight)
    // dataset of this face
    __nv_bfloat16* x;               // capacity x kIn
    float* y;                       // capacity x kOut
    float* s;                       // capacity
    int* modelOf;                   // capacity
    unsigned long long* count;      // rows written so far (may exceed capacity: excess dropped)
    unsigned long long capacity;
    unsigned* modelMax;             // per model: max s (float bits)
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void collectRows(CollectArgs A, int face) {
    const Face& f = A.faces.f[face];
    const int columns = f.nu * f.nw;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= columns) return;
    const unsigned long long h = mix64(A.seed ^ (unsigned long long)(f.columnBegin + col) * 0x2545F4914F6CDD1Dull);
    if (double(h >> 11) * (1.0 / 9007199254740992.0) >= double(A.fraction)) return;
    const int u = col % f.nu, w = col / f.nu;
    float s, z, cp, cs;
    columnScale(f, A.thin, A.mat, u, w, s, z, cp, cs, A.faces.dtOverH);
    if (!(s > 0.0f)) return;
    atomicMax(A.modelMax + A.model, __float_as_uint(s));
    const unsigned long long row = atomicAdd(A.count, 1ull);
    if (row >= A.capacity) return;
    __nv_bfloat16* x = A.x + row * kIn;
    columnFeatures(f, A.thin, u, w, s, z, cp, cs, A.faces, 0, x);
    columnFeatures(f, A.thin, u, w, s, z, cp, cs, A.faces, 1, x);
    float* y = A.y + row * kOut;
    const float inv = 1.0f / s, iz = 1.0f / z;
    for (int k = 0; k < 9; ++k)
        for (int d = 0; d < kBand; ++d) {
            const int64_t ct = cellIndex(f, u, w, d);
            const int64_t cw = f.wideBase + int64_t(u) * f.wideDu + int64_t(w) * f.wideDw + int64_t(d - 3) * f.wideDn;
            y[k * kBand + d] = (A.wide[k][cw] - A.thin[k][ct]) * (k < 3 ? 1.0f : iz) * inv;
        }
    A.s[row] = s;
    A.modelOf[row] = A.model;
}

// Teacher forcing: the thin session's interior (every physical cell) takes the wide
// session's values.  One thread per physical cell and field.
struct InteriorCopy {
    float* thin[9];
    const float* wide[9];
    int nx, ny, nz;
    int64_t thinBase, thinPitch, thinPlane;   // element index of physical (0, 0, 0)
    int64_t wideBase, widePitch, widePlane;
};

__global__ void copyInterior(InteriorCopy C) {
    const int64_t n = int64_t(C.nx) * C.ny * C.nz;
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = int(i % C.nx), y = int((i / C.nx) % C.ny), z = int(i / (int64_t(C.nx) * C.ny));
    const int64_t t = C.thinBase + z * C.thinPlane + y * C.thinPitch + x;
    const int64_t w = C.wideBase + z * C.widePlane + y * C.widePitch + x;
#pragma unroll
    for (int k = 0; k < 9; ++k) C.thin[k][t] = C.wide[k][w];
}

// ---------------------------------------------------------------------------------------
// Training: forward + backward of 64 rows per CTA on the tensor cores, gradients summed into
// FP32 global buffers; Adam on the FP32 master weights, BF16 copies refreshed.
// ---------------------------------------------------------------------------------------
constexpr int kTrainWarps = 4;
constexpr int kTrainRows = 16 * kTrainWarps;
constexpr int kLdOut = 56;   // bf16 row stride of the dY tile (48 used)

struct TrainTiles {
    __nv_bfloat16 x[kTrainRows * kLdIn];
    __nv_bfloat16 h1[kTrainRows * kLdHid], h2[kTrainRows * kLdHid];
    __nv_bfloat16 dz1[kTrainRows * kLdHid], dz2[kTrainRows * kLdHid];
    __nv_bfloat16 dy[kTrainRows * kLdOut];
    float target[kTrainRows * kOutPad];
    float weight[kTrainRows];
    float gb[kHidden + kHidden + kOutPad];
    float loss;
};

struct TrainArgs {
    const __nv_bfloat16* x;   // rows x kIn
    const float* y;           // rows x kOut (normalised by s)
    const float* rowWeight;   // rows (already including the 1 / (B * 36 * mean weight) factor), or null = 1
    const int* rowIndex;      // batch -> dataset row, or null = identity
    int rows;                 // batch size
    const __nv_bfloat16* weights;   // kMatrixCount
    const float* params;            // kParamCount
    float invOutScale;
    float* grad;                    // kParamCount (accumulated)
    float* loss;                    // accumulated sum of w (y - t)^2
};

// Stores the fp32 C fragments of an m16 x (8 x count) tile into a bf16 shared tile.
template <int N>
__device__ __forceinline__ void storeFragments(__nv_bfloat16* tile, int ld, int row0, const float (&c)[N][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int n = 0; n < N; ++n) {
        *reinterpret_cast<uint32_t*>(&tile[(row0 + g) * ld + 8 * n + 2 * t]) = packBf16(c[n][0], c[n][1]);
        *reinterpret_cast<uint32_t*>(&tile[(row0 + g + 8) * ld + 8 * n + 2 * t]) = packBf16(c[n][2], c[n][3]);
    }
}

__device__ __forceinline__ void storeHidden(__nv_bfloat16* tile, int row0, const uint32_t (&h)[4][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        *reinterpret_cast<uint32_t*>(&tile[(row0 + g) * kLdHid + 16 * j + 2 * t]) = h[j][0];
        *reinterpret_cast<uint32_t*>(&tile[(row0 + g + 8) * kLdHid + 16 * j + 2 * t]) = h[j][1];
        *reinterpret_cast<uint32_t*>(&tile[(row0 + g) * kLdHid + 16 * j + 8 + 2 * t]) = h[j][2];
        *reinterpret_cast<uint32_t*>(&tile[(row0 + g + 8) * kLdHid + 16 * j + 8 + 2 * t]) = h[j][3];
    }
}

__device__ __forceinline__ bool positive(uint32_t packed, int hi) {
    const unsigned short v = hi ? (packed >> 16) : (packed & 0xffff);
    return (v & 0x8000u) == 0 && v != 0;
}

// Column sums over the 16 rows of C fragments (8 x N outputs) into shared accumulators.
template <int N>
__device__ __forceinline__ void sumColumns(float* acc, const float (&c)[N][4], int limit) {
    const int lane = threadIdx.x & 31, t = lane & 3;
#pragma unroll
    for (int n = 0; n < N; ++n)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            float v = c[n][q] + c[n][2 + q];
            v += __shfl_xor_sync(0xffffffffu, v, 4);
            v += __shfl_xor_sync(0xffffffffu, v, 8);
            v += __shfl_xor_sync(0xffffffffu, v, 16);
            const int col = 8 * n + 2 * t + q;
            if (lane < 4 && col < limit) atomicAdd(&acc[col], v);
        }
}

// grad[m][n] += sum_rows A[row][m] * B[row][n] over the CTA's 64 rows (A, B bf16 shared tiles,
// row strides lda, ldb), tiles of 16 x 8 assigned round-robin to the warps.
__device__ __forceinline__ void weightGradient(float* grad, int ldg, const __nv_bfloat16* A, int lda, int mTiles,
                                               const __nv_bfloat16* B, int ldb, int nTiles, int mLimit) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int tile = warp; tile < mTiles * nTiles; tile += kTrainWarps) {
        const int m0 = 16 * (tile / nTiles), n0 = 8 * (tile % nTiles);
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < kTrainRows / 16; ++k) {
            const int r = 16 * k;
            uint32_t a[4];
            a[0] = pair16(&A[(r + 2 * t) * lda + m0 + g], &A[(r + 2 * t + 1) * lda + m0 + g]);
            a[1] = pair16(&A[(r + 2 * t) * lda + m0 + g + 8], &A[(r + 2 * t + 1) * lda + m0 + g + 8]);
            a[2] = pair16(&A[(r + 2 * t + 8) * lda + m0 + g], &A[(r + 2 * t + 9) * lda + m0 + g]);
            a[3] = pair16(&A[(r + 2 * t + 8) * lda + m0 + g + 8], &A[(r + 2 * t + 9) * lda + m0 + g + 8]);
            const uint32_t b0 = pair16(&B[(r + 2 * t) * ldb + n0 + g], &B[(r + 2 * t + 1) * ldb + n0 + g]);
            const uint32_t b1 = pair16(&B[(r + 2 * t + 8) * ldb + n0 + g], &B[(r + 2 * t + 9) * ldb + n0 + g]);
            mma16816(acc, a, b0, b1);
        }
        const int ma = m0 + g, mb = m0 + g + 8, n = n0 + 2 * t;
        if (ma < mLimit) { atomicAdd(&grad[ma * ldg + n], acc[0]); atomicAdd(&grad[ma * ldg + n + 1], acc[1]); }
        if (mb < mLimit) { atomicAdd(&grad[mb * ldg + n], acc[2]); atomicAdd(&grad[mb * ldg + n + 1], acc[3]); }
    }
}

__global__ void __launch_bounds__(32 * kTrainWarps) trainStep(TrainArgs A) {
    extern __shared__ __align__(16) unsigned char smemRaw[];
    SharedNet& S = *reinterpret_cast<SharedNet*>(smemRaw);
    TrainTiles& T = *reinterpret_cast<TrainTiles*>(smemRaw + sizeof(SharedNet));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    loadNet(S, A.weights, A.params, tid, blockDim.x);
    const int row0 = blockIdx.x * kTrainRows;
    for (int e = tid; e < kTrainRows * (kIn / 2); e += blockDim.x) {
        const int r = e / (kIn / 2), c = 2 * (e % (kIn / 2));
        const int b = row0 + r;
        uint32_t v = 0;
        if (b < A.rows) {
            const int src = A.rowIndex ? A.rowIndex[b] : b;
            v = lds32(A.x + size_t(src) * kIn + c);
        }
        *reinterpret_cast<uint32_t*>(&T.x[r * kLdIn + c]) = v;
    }
    for (int e = tid; e < kTrainRows * kOutPad; e += blockDim.x) {
        const int r = e / kOutPad, c = e % kOutPad, b = row0 + r;
        float v = 0.0f;
        if (b < A.rows && c < kOut) v = A.y[size_t(A.rowIndex ? A.rowIndex[b] : b) * kOut + c] * A.invOutScale;
        T.target[e] = v;
    }
    for (int e = tid; e < kTrainRows; e += blockDim.x) {
        const int b = row0 + e;
        T.weight[e] = b < A.rows ? (A.rowWeight ? A.rowWeight[b] : 1.0f) : 0.0f;
    }
    for (int e = tid; e < kHidden + kHidden + kOutPad; e += blockDim.x) T.gb[e] = 0.0f;
    if (tid == 0) T.loss = 0.0f;
    __syncthreads();

    const int r0 = 16 * warp;
    float y[5][4];
    Hidden H;
    forward16(S, T.x + r0 * kLdIn, y, H);
    storeHidden(T.h1, r0, H.h1);
    storeHidden(T.h2, r0, H.h2);
    // dL/dy = 2 w (y - t) (the row weight carries the batch normalisation).
    float dy[6][4];
    float lossPart = 0.0f;
#pragma unroll
    for (int n = 0; n < 5; ++n)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int rr = r0 + g + 8 * (q >> 1), cc = 8 * n + 2 * t + (q & 1);
            const float w = T.weight[rr];
            const float diff = cc < kOut ? y[n][q] - T.target[rr * kOutPad + cc] : 0.0f;
            lossPart += w * diff * diff;
            dy[n][q] = 2.0f * w * diff;
        }
    dy[5][0] = dy[5][1] = dy[5][2] = dy[5][3] = 0.0f;
    storeFragments<6>(T.dy, kLdOut, r0, dy);
    sumColumns<5>(T.gb + 2 * kHidden, *reinterpret_cast<float(*)[5][4]>(&dy), kOut);
    // dH2 = dY W3 (K = 48 outputs), masked by h2 > 0.
    float acc[8][4];
#pragma unroll
    for (int n = 0; n < 8; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        uint32_t a[4] = {packBf16(dy[2 * k][0], dy[2 * k][1]), packBf16(dy[2 * k][2], dy[2 * k][3]),
                         packBf16(dy[2 * k + 1][0], dy[2 * k + 1][1]), packBf16(dy[2 * k + 1][2], dy[2 * k + 1][3])};
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const int o = 16 * k + 2 * t, h = 8 * n + g;
            const uint32_t b0 = pair16(&S.w3[o * kLdHid + h], &S.w3[(o + 1) * kLdHid + h]);
            const uint32_t b1 = pair16(&S.w3[(o + 8) * kLdHid + h], &S.w3[(o + 9) * kLdHid + h]);
            mma16816(acc[n], a, b0, b1);
        }
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const uint32_t lo = H.h2[n >> 1][(n & 1) ? 2 : 0], hi = H.h2[n >> 1][(n & 1) ? 3 : 1];
        if (!positive(lo, 0)) acc[n][0] = 0.0f;
        if (!positive(lo, 1)) acc[n][1] = 0.0f;
        if (!positive(hi, 0)) acc[n][2] = 0.0f;
        if (!positive(hi, 1)) acc[n][3] = 0.0f;
    }
    storeFragments<8>(T.dz2, kLdHid, r0, acc);
    sumColumns<8>(T.gb + kHidden, acc, kHidden);
    // dH1 = dZ2 W2, masked by h1 > 0.
    float acc1[8][4];
#pragma unroll
    for (int n = 0; n < 8; ++n) acc1[n][0] = acc1[n][1] = acc1[n][2] = acc1[n][3] = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint32_t a[4] = {packBf16(acc[2 * k][0], acc[2 * k][1]), packBf16(acc[2 * k][2], acc[2 * k][3]),
                         packBf16(acc[2 * k + 1][0], acc[2 * k + 1][1]), packBf16(acc[2 * k + 1][2], acc[2 * k + 1][3])};
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const int o = 16 * k + 2 * t, h = 8 * n + g;
            const uint32_t b0 = pair16(&S.w2[o * kLdHid + h], &S.w2[(o + 1) * kLdHid + h]);
            const uint32_t b1 = pair16(&S.w2[(o + 8) * kLdHid + h], &S.w2[(o + 9) * kLdHid + h]);
            mma16816(acc1[n], a, b0, b1);
        }
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const uint32_t lo = H.h1[n >> 1][(n & 1) ? 2 : 0], hi = H.h1[n >> 1][(n & 1) ? 3 : 1];
        if (!positive(lo, 0)) acc1[n][0] = 0.0f;
        if (!positive(lo, 1)) acc1[n][1] = 0.0f;
        if (!positive(hi, 0)) acc1[n][2] = 0.0f;
        if (!positive(hi, 1)) acc1[n][3] = 0.0f;
    }
    storeFragments<8>(T.dz1, kLdHid, r0, acc1);
    sumColumns<8>(T.gb, acc1, kHidden);
    lossPart += __shfl_xor_sync(0xffffffffu, lossPart, 1);
    lossPart += __shfl_xor_sync(0xffffffffu, lossPart, 2);
    lossPart += __shfl_xor_sync(0xffffffffu, lossPart, 4);
    lossPart += __shfl_xor_sync(0xffffffffu, lossPart, 8);
    lossPart += __shfl_xor_sync(0xffffffffu, lossPart, 16);
    if (lane == 0) atomicAdd(&T.loss, lossPart);
    __syncthreads();

    // Weight gradients over the CTA's rows: dW3 = dY^T H2, dW2 = dZ2^T H1, dW1 = dZ1^T X.
    weightGradient(A.grad + kW3, kHidden, T.dy, kLdOut, 3, T.h2, kLdHid, 8, kOut);
    weightGradient(A.grad + kW2, kHidden, T.dz2, kLdHid, 4, T.h1, kLdHid, 8, kHidden);
    weightGradient(A.grad + kW1, kIn, T.dz1, kLdHid, 4, T.x, kLdIn, kIn / 8, kHidden);
    for (int e = tid; e < kHidden; e += blockDim.x) {
        atomicAdd(&A.grad[kB1 + e], T.gb[e]);
        atomicAdd(&A.grad[kB2 + e], T.gb[kHidden + e]);
    }
    for (int e = tid; e < kOut; e += blockDim.x) atomicAdd(&A.grad[kB3 + e], T.gb[2 * kHidden + e]);
    if (tid == 0) atomicAdd(A.loss, T.loss);
}

// Adam on the FP32 master parameters; refreshes the BF16 matrices.  Rows 36..47 of W3 and
// b3 never move (their gradients are zero).  Gradients are cleared for the next step.
__global__ void adamStep(float* p, float* grad, float* m, float* v, __nv_bfloat16* w, float lr, float beta1, float beta2,
                         float eps, float bias1, float bias2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParamCount) return;
    const float gr = grad[i];
    grad[i] = 0.0f;
    const float mi = beta1 * m[i] + (1.0f - beta1) * gr;
    const float vi = beta2 * v[i] + (1.0f - beta2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    const float value = p[i] - lr * (mi / bias1) / (sqrtf(vi / bias2) + eps);
    p[i] = value;
    if (i < kMatrixCount) w[i] = __float2bfloat16_rn(value);
}

// Batch rows drawn with replacement from the dataset, with their loss weights:
// weight = (s / max s of the row's model)^2 x norm.
__global__ void sampleBatch(int* index, float* weight, int batch, unsigned long long rows, unsigned long long seed,
                            const float* s, const int* modelOf, const unsigned* modelMax, float norm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    const unsigned long long h = mix64(seed * 0x9E3779B97F4A7C15ull + (unsigned long long)i);
    const unsigned long long r = h % rows;
    index[i] = int(r);
    const float mx = __uint_as_float(modelMax[modelOf[r]]);
    const float rel = mx > 0.0f ? s[r] / mx : 0.0f;
    weight[i] = rel * rel * norm;
}

// Sums over one face's dataset: sum of row weights (s / max s of the model)^2 and of weight x
// squared target (FP64 accumulation).
__global__ void datasetMoments(const float* y, const float* s, const int* modelOf, const unsigned* modelMax,
                               unsigned long long rows, double* out) {
    double w = 0.0, wy = 0.0;
    for (unsigned long long r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        const float mx = __uint_as_float(modelMax[modelOf[r]]);
        const double rel = mx > 0.0f ? double(s[r]) / mx : 0.0;
        double sq = 0.0;
        for (int k = 0; k < kOut; ++k) sq += double(y[r * kOut + k]) * y[r * kOut + k];
        w += rel * rel;
        wy += rel * rel * sq;
    }
    atomicAdd(out, w);
    atomicAdd(out + 1, wy);
}

}  // namespace bnet
}  // namespace seis3d
