// seis3d_views.cuh - display extraction of the 3-D solver (extractViews3D, reference
// cuda/Cuda_Seis3D.cu:334-418,627-646) without a graphics stack: three packed physical
// slices (XZ at y = sy, YZ at x = sx, XY at z = sz, each including the visible CPML) and an
// optional bounded volume resampled trilinearly at cell centres, written as interleaved
// (wave value, material value) pairs into a caller-owned device buffer, with the reference's
// colour statistics (largest |value|, material range, largest velocity magnitude).
//
// The per-sample arithmetic is the reference's (collocated face velocities, material
// transforms, trilinear weights), read from this solver's pitched volumes.  One thread per
// output sample; a warp reduces its statistics before one atomic per word, as the reference
// does.  Output samples are independent, so the kernel is a plain grid over the samples.
#pragma once

#include "../../include/seis3d_capi.h"

#include <cstdint>

namespace seis3d {

struct ViewArgs {
    const float* v[3];      // vx, vy, vz
    const float* s[3];      // sxx, syy, szz
    const float* invRho;
    const float* lambda;
    const float* mu;
    int64_t pitch, plane;
    int ox, oy, oz;         // physical origin inside the padded volume
    int nx, ny, nz;         // physical size
    seis3d_view_layout layout;
    int sx, sy, sz;
    int component, materialComponent;
    int includeBoundary;
    float* out;
    unsigned* stats;        // [0] |value| max, [2] material min, [3] material max, [4] |v| max
    unsigned* nonFinite;    // the session's non-finite flag
};

// sampleScalar3D (cuda/Cuda_Seis3D.cu:335-352) at physical cell (x, y, z).
__device__ __forceinline__ float viewScalar(const ViewArgs& a, int x, int y, int z, int component, float* magnitudeOut) {
    const int64_t i = int64_t(z + a.oz) * a.plane + int64_t(y + a.oy) * a.pitch + (x + a.ox);
    if (component == 5) return sqrtf((a.lambda[i] + 2 * a.mu[i]) * a.invRho[i]);
    if (component == 6) return sqrtf(a.mu[i] * a.invRho[i]);
    if (component == 7) return 1 / a.invRho[i];
    const float vx = 0.5f * (a.v[0][i] + a.v[0][i - 1]);
    const float vy = 0.5f * (a.v[1][i] + a.v[1][i - a.pitch]);
    const float vz = 0.5f * (a.v[2][i] + a.v[2][i - a.plane]);
    const float magnitude = sqrtf(vx * vx + vy * vy + vz * vz);
    if (magnitudeOut) *magnitudeOut = magnitude;
    if (component == 0) return vz;
    if (component == 1) return vx;
    if (component == 2) return vy;
    if (component == 3) return magnitude;
    if (component == 4) return -(a.s[0][i] + a.s[1][i] + a.s[2][i]) / 3;
    return 0;
}

// resampleScalar3D (:355-367): trilinear over the 8 cells around (x, y, z).
__device__ __forceinline__ float viewResample(const ViewArgs& a, float x, float y, float z, int component,
                                              float* magnitudeOut) {
    const int ix = int(floorf(x)), iy = int(floorf(y)), iz = int(floorf(z));
    const float fraction[3] = {x - ix, y - iy, z - iz};
    float result = 0;
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                const float weight = (dx ? fraction[0] : 1 - fraction[0]) * (dy ? fraction[1] : 1 - fraction[1]) *
                                     (dz ? fraction[2] : 1 - fraction[2]);
                if (weight > 0) {
                    float magnitude = 0;
                    result += weight * viewScalar(a, ix + dx, iy + dy, iz + dz, component,
                                                  magnitudeOut ? &magnitude : nullptr);
                    if (magnitudeOut) *magnitudeOut += weight * magnitude;
                }
            }
    return result;
}

__global__ void __launch_bounds__(256) extractViews(ViewArgs a, uint64_t limit) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= limit) return;
    const seis3d_view_layout& L = a.layout;
    const int nx = L.domainSize3D[0], ny = L.domainSize3D[1], nz = L.domainSize3D[2];
    const int ox = L.domainOrigin3D[0], oy = L.domainOrigin3D[1], oz = L.domainOrigin3D[2];
    int x, y, z;
    float fx = 0, fy = 0, fz = 0;
    if (i < L.sliceOffset3D[1]) {
        x = int(i % nx) + ox; y = a.sy; z = int(i / nx) + oz;
    } else if (i < L.sliceOffset3D[2]) {
        const uint64_t j = i - L.sliceOffset3D[1];
        x = a.sx; y = int(j % ny) + oy; z = int(j / ny) + oz;
    } else if (i < L.volumeOffset3D) {
        const uint64_t j = i - L.sliceOffset3D[2];
        x = int(j % nx) + ox; y = int(j / nx) + oy; z = a.sz;
    } else {
        const uint64_t j = i - L.volumeOffset3D;
        fx = (float(j % L.volumeX3D) + .5f) * float(nx) / L.volumeX3D - .5f + ox;
        fy = (float((j / L.volumeX3D) % L.volumeY3D) + .5f) * float(ny) / L.volumeY3D - .5f + oy;
        fz = (float(j / (uint64_t(L.volumeX3D) * L.volumeY3D)) + .5f) * float(nz) / L.volumeZ3D - .5f + oz;
        x = int(floorf(fx)); y = int(floorf(fy)); z = int(floorf(fz));
    }
    const bool volumeSample = i >= L.volumeOffset3D;
    float magnitude = 0;
    const float value = volumeSample ? viewResample(a, fx, fy, fz, a.component, &magnitude)
                                     : viewScalar(a, x, y, z, a.component, &magnitude);
    const float material = volumeSample ? viewResample(a, fx, fy, fz, a.materialComponent, nullptr)
                                        : viewScalar(a, x, y, z, a.materialComponent, nullptr);
    a.out[2 * i] = isfinite(value) ? value : 0;
    a.out[2 * i + 1] = isfinite(material) ? material : 0;
    if (!isfinite(value) || !isfinite(material) || !isfinite(magnitude) || material < 0) atomicExch(a.nonFinite, 1u);
    const bool physical = x >= 0 && x < a.nx && y >= 0 && y < a.ny && z >= 0 && z < a.nz;
    float waveMax = (physical || a.includeBoundary) && isfinite(value) ? fabsf(value) : 0;
    float velocityMax = (physical || a.includeBoundary) && isfinite(magnitude) ? magnitude : 0;
    float materialMin = physical && isfinite(material) ? material : 3.402823466e38f;
    float materialMax = physical && isfinite(material) ? material : 0;
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31, active = __popc(mask);
    for (int offset = 16; offset > 0; offset /= 2) {
        const float w = __shfl_down_sync(mask, waveMax, offset);
        const float v = __shfl_down_sync(mask, velocityMax, offset);
        const float lo = __shfl_down_sync(mask, materialMin, offset);
        const float hi = __shfl_down_sync(mask, materialMax, offset);
        if (lane + offset < active) {
            waveMax = fmaxf(waveMax, w);
            velocityMax = fmaxf(velocityMax, v);
            materialMin = fminf(materialMin, lo);
            materialMax = fmaxf(materialMax, hi);
        }
    }
    if (lane == 0) {
        // Non-negative floats order like their bit patterns.
        atomicMax(a.stats, __float_as_uint(waveMax));
        atomicMin(a.stats + 2, __float_as_uint(materialMin));
        atomicMax(a.stats + 3, __float_as_uint(materialMax));
        atomicMax(a.stats + 4, __float_as_uint(velocityMax));
    }
}

}  // namespace seis3d
