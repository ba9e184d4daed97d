// seis3d_shade.cuh - the workspace's display shaders as CUDA kernels, writing a device RGBA
// buffer instead of a GL framebuffer:
//
//   * shadeSlices  = shaders/seis3d_slice.frag:9-20 over the three extracted slices;
//   * renderVolume = shaders/seis3d_volume.frag:15-83, one ray per pixel through the bounded
//                    volume of the extracted views;
//   * both share the transfer function of shaders/seis3d_transfer.glsl:6-28.
//
// GLSL semantics kept: mix(a, b, t) = a(1 - t) + bt, clamp = min(max()), smoothstep with the
// cubic 3t^2 - 2t^3, normalize = v / |v|.  The slice pass of the reference draws a full-screen
// triangle into a target of the slice's own size, so every pixel samples its texel centre
// and the linear filter returns that texel: the shading is per view sample.  The volume
// texture is sampled here with an FP32 trilinear filter under clamp-to-edge addressing (the
// GL_LINEAR / GL_CLAMP_TO_EDGE state of src/Seis3D/Renderer3D.cpp:137-140).
#pragma once

#include "../../include/seis3d_capi.h"

#include <cstdint>

namespace seis3d {
namespace shade {

struct Rgb { float r, g, b; };

__host__ __device__ __forceinline__ Rgb rgb(float r, float g, float b) { return Rgb{r, g, b}; }
__host__ __device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__host__ __device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__host__ __device__ __forceinline__ Rgb mix3(Rgb a, Rgb b, float t) {
    return Rgb{mixf(a.r, b.r, t), mixf(a.g, b.g, t), mixf(a.b, b.b, t)};
}
__host__ __device__ __forceinline__ Rgb scale3(Rgb a, float s) { return Rgb{a.r * s, a.g * s, a.b * s}; }
__host__ __device__ __forceinline__ float smoothstepf(float e0, float e1, float x) {
    const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

// waveVisibility3D (seis3d_transfer.glsl:7-10).
__device__ __forceinline__ float waveVisibility(const seis3d_transfer& t, float magnitude) {
    const float visible = clampf((magnitude - t.waveThreshold3D) / fmaxf(1.0f - t.waveThreshold3D, 1e-6f), 0.0f, 1.0f);
    return powf(visible, fmaxf(t.waveGamma3D, 0.1f));
}

// waveColor3D (:12-16): the five-stop palette, signed or |value|.
__device__ __forceinline__ Rgb waveColor(const seis3d_transfer& t, float value) {
    const float q = clampf(t.unsignedWave3D != 0 ? fabsf(value) : value * 0.5f + 0.5f, 0.0f, 1.0f) * 4.0f;
    const int i = min(int(q), 3);
    const float* a = t.palette3D[i];
    const float* b = t.palette3D[i + 1];
    return mix3(rgb(a[0], a[1], a[2]), rgb(b[0], b[1], b[2]), q - float(i));
}

// materialColor3D (:18-28): material value in the shared range, five model styles.
__device__ __forceinline__ Rgb materialColor(const seis3d_transfer& t, float value) {
    const float lo = t.materialRange3D[0], hi = t.materialRange3D[1];
    const float span = hi - lo;
    const float q = span > fmaxf(1e-6f, fabsf(hi) * 1e-6f) ? clampf((value - lo) / span, 0.0f, 1.0f) : 0.5f;
    switch (t.modelStyle3D) {
        case 0: return mix3(rgb(.09f, .13f, .17f), rgb(.43f, .53f, .6f), q);
        case 1:
            return q < .5f ? mix3(rgb(.13f, .28f, .33f), rgb(.48f, .65f, .46f), q * 2.0f)
                           : mix3(rgb(.48f, .65f, .46f), rgb(.78f, .52f, .31f), (q - .5f) * 2.0f);
        case 2: { const float g = mixf(.12f, .85f, q); return rgb(g, g, g); }
        case 3: return waveColor(t, t.unsignedWave3D != 0 ? q : q * 2.0f - 1.0f);
        default: return mix3(rgb(.97f, .96f, .93f), rgb(.79f, .84f, .85f), q);
    }
}

// One pixel into the output in the requested format.
__device__ __forceinline__ void storePixel(void* out, uint64_t k, int format, Rgb c) {
    if (format == SEIS3D_PIXELS_RGBA32F) {
        reinterpret_cast<float4*>(out)[k] = make_float4(c.r, c.g, c.b, 1.0f);
    } else {
        const unsigned r = __float2uint_rn(clampf(c.r, 0.0f, 1.0f) * 255.0f);
        const unsigned g = __float2uint_rn(clampf(c.g, 0.0f, 1.0f) * 255.0f);
        const unsigned b = __float2uint_rn(clampf(c.b, 0.0f, 1.0f) * 255.0f);
        reinterpret_cast<uint32_t*>(out)[k] = r | (g << 8) | (b << 16) | (255u << 24);
    }
}

// seis3d_slice.frag main (:9-20) for view sample k of the slices.
__global__ void __launch_bounds__(256) shadeSlices(const float2* __restrict__ views, uint64_t count,
                                                   const __grid_constant__ seis3d_transfer t, float scale,
                                                   float gain, int format, void* out) {
    const uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const float2 sample = views[k];
    const float q = clampf(sample.x * gain / fmaxf(scale, 1e-20f), -1.0f, 1.0f);
    const Rgb background = t.modelStyle3D == 4 ? rgb(.97f, .96f, .93f) : rgb(0.028f, 0.045f, 0.052f);
    const Rgb material = materialColor(t, sample.y);
    const float alpha = waveVisibility(t, fabsf(q)) * t.waveOpacity3D;
    const Rgb base = t.displayMode3D == 1 ? background : scale3(material, t.materialBrightness3D);
    const Rgb mapped = t.displayMode3D == 2 ? material : mix3(base, waveColor(t, q), alpha);
    storePixel(out, k, format, mapped);
}

struct Vec3 { float x, y, z; };
__device__ __forceinline__ Vec3 v3(float x, float y, float z) { return Vec3{x, y, z}; }
__device__ __forceinline__ Vec3 operator+(Vec3 a, Vec3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ Vec3 operator-(Vec3 a, Vec3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ Vec3 operator*(Vec3 a, Vec3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ Vec3 operator/(Vec3 a, Vec3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ Vec3 operator*(float s, Vec3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot3(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Vec3 normalize3(Vec3 a) {
    const float n = sqrtf(dot3(a, a));
    return v3(a.x / n, a.y / n, a.z / n);
}
__device__ __forceinline__ Vec3 cross3(Vec3 a, Vec3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ Vec3 min3v(Vec3 a, Vec3 b) { return v3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__device__ __forceinline__ Vec3 max3v(Vec3 a, Vec3 b) { return v3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
__device__ __forceinline__ Vec3 abs3(Vec3 a) { return v3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
__device__ __forceinline__ Vec3 load3(const float* p) { return v3(p[0], p[1], p[2]); }
// Distance of a box-normalised point to the nearest edge (the second-smallest face distance).
__device__ __forceinline__ float edgeDistance(Vec3 p) {
    const Vec3 d = v3(fabsf(fabsf(p.x) - 0.5f), fabsf(fabsf(p.y) - 0.5f), fabsf(fabsf(p.z) - 0.5f));
    return fmaxf(fminf(d.x, d.y), fminf(fmaxf(d.x, d.y), d.z));
}

// Bounded volume of the views: volumeX3D x volumeY3D x volumeZ3D float2 texels, x fastest.
struct VolumeTexture {
    const float2* texels;
    int nx, ny, nz;
};

// texture(volumeTexture3D, uvw).rg with GL_LINEAR filtering and clamp-to-edge addressing:
// texel coordinate u * n - 1/2, the two neighbours per axis clamped to [0, n - 1].  The
// coordinate is first bounded to [-1, n], which changes no in-range result and keeps the
// indices finite for any input.
__device__ __forceinline__ float2 sampleVolume(const VolumeTexture& v, Vec3 uvw) {
    const float fx = clampf(uvw.x * float(v.nx) - 0.5f, -1.0f, float(v.nx));
    const float fy = clampf(uvw.y * float(v.ny) - 0.5f, -1.0f, float(v.ny));
    const float fz = clampf(uvw.z * float(v.nz) - 0.5f, -1.0f, float(v.nz));
    const float bx = floorf(fx), by = floorf(fy), bz = floorf(fz);
    const float ax = fx - bx, ay = fy - by, az = fz - bz;
    const int x0 = min(max(int(bx), 0), v.nx - 1), x1 = min(max(int(bx) + 1, 0), v.nx - 1);
    const int y0 = min(max(int(by), 0), v.ny - 1), y1 = min(max(int(by) + 1, 0), v.ny - 1);
    const int z0 = min(max(int(bz), 0), v.nz - 1), z1 = min(max(int(bz) + 1, 0), v.nz - 1);
    const uint64_t sx = 1, sy = uint64_t(v.nx), sz = uint64_t(v.nx) * v.ny;
    const float2* p = v.texels;
    const float2 c000 = __ldg(p + z0 * sz + y0 * sy + x0 * sx), c100 = __ldg(p + z0 * sz + y0 * sy + x1 * sx);
    const float2 c010 = __ldg(p + z0 * sz + y1 * sy + x0 * sx), c110 = __ldg(p + z0 * sz + y1 * sy + x1 * sx);
    const float2 c001 = __ldg(p + z1 * sz + y0 * sy + x0 * sx), c101 = __ldg(p + z1 * sz + y0 * sy + x1 * sx);
    const float2 c011 = __ldg(p + z1 * sz + y1 * sy + x0 * sx), c111 = __ldg(p + z1 * sz + y1 * sy + x1 * sx);
    float2 r;
    r.x = mixf(mixf(mixf(c000.x, c100.x, ax), mixf(c010.x, c110.x, ax), ay),
               mixf(mixf(c001.x, c101.x, ax), mixf(c011.x, c111.x, ax), ay), az);
    r.y = mixf(mixf(mixf(c000.y, c100.y, ax), mixf(c010.y, c110.y, ax), ay),
               mixf(mixf(c001.y, c101.y, ax), mixf(c011.y, c111.y, ax), ay), az);
    return r;
}

// seis3d_volume.frag main (:15-83) for pixel (px, py) of a width x height target.
__global__ void __launch_bounds__(128) renderVolume(VolumeTexture vol, const __grid_constant__ seis3d_transfer t,
                                                    const __grid_constant__ seis3d_volume_view u, int width,
                                                    int height, int format, void* out) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= width || py >= height) return;
    const float tcx = (float(px) + 0.5f) / float(width), tcy = (float(py) + 0.5f) / float(height);
    const Vec3 extent = load3(u.extent3D);
    const Vec3 forward = normalize3(v3(cosf(u.pitch3D) * sinf(u.yaw3D), sinf(u.pitch3D), cosf(u.pitch3D) * cosf(u.yaw3D)));
    const Vec3 right = normalize3(cross3(v3(0, 1, 0), forward));
    const Vec3 up = cross3(forward, right);
    const Vec3 target = u.pan3D[0] * right + u.pan3D[1] * up;
    const Vec3 origin = target + u.distance3D * forward;
    const float sx = (tcx - 0.5f) * 1.3f * u.aspect3D, sy = (tcy - 0.5f) * 1.3f;
    const Vec3 direction = normalize3(v3(-forward.x, -forward.y, -forward.z) + sx * right + sy * up);
    const Vec3 safe = v3(fabsf(direction.x) < 1e-7f ? 1e-7f : direction.x, fabsf(direction.y) < 1e-7f ? 1e-7f : direction.y,
                         fabsf(direction.z) < 1e-7f ? 1e-7f : direction.z);
    const Vec3 inverse = v3(1.0f / safe.x, 1.0f / safe.y, 1.0f / safe.z);
    const Vec3 first = (-0.5f * extent - origin) * inverse, second = (0.5f * extent - origin) * inverse;
    const Vec3 nearT = min3v(first, second), farT = max3v(first, second);
    float enter = fmaxf(fmaxf(nearT.x, nearT.y), nearT.z);
    const float exitT = fminf(fminf(farT.x, farT.y), farT.z);
    const uint64_t k = uint64_t(py) * width + px;
    const Rgb background = t.modelStyle3D == 4 ? rgb(.97f, .96f, .93f) : rgb(0.025f, 0.041f, 0.05f);
    if (exitT <= fmaxf(enter, 0.0f)) {
        storePixel(out, k, format, background);
        return;
    }
    enter = fmaxf(enter, 0.0f);
    float ar = 0, ag = 0, ab = 0, aa = 0;
    const Vec3 lo = load3(u.domainLow3D), hi = load3(u.domainHigh3D);
    const Vec3 plo = load3(u.physicalLow3D), phi = load3(u.physicalHigh3D);
    const Vec3 path = abs3(((exitT - enter) * direction) / extent);
    const Vec3 texturePath = v3(path.x, path.z, path.y) * (hi - lo);
    const Vec3 scaled = texturePath * v3(float(vol.nx), float(vol.ny), float(vol.nz));
    const int steps = int(clampf(ceilf(sqrtf(dot3(scaled, scaled)) * u.sampling3D), 192.0f, 1024.0f));
    const float delta = (exitT - enter) / float(steps);
    const float scaleFloor = fmaxf(u.scale3D, 1e-20f);
    for (int i = 0; i < steps; ++i) {
        const Vec3 q = (origin + (enter + (float(i) + 0.5f) * delta) * direction) / extent + v3(0.5f, 0.5f, 0.5f);
        const Vec3 w = v3(q.x, q.z, 1.0f - q.y);
        const Vec3 uvw = v3(mixf(lo.x, hi.x, w.x), mixf(lo.y, hi.y, w.y), mixf(lo.z, hi.z, w.z));
        const bool boundary = u.showBoundary3D != 0 &&
                              (uvw.x < plo.x || uvw.y < plo.y || uvw.z < plo.z || uvw.x > phi.x || uvw.y > phi.y || uvw.z > phi.z);
        const float2 sample = sampleVolume(vol, uvw);
        const float scalar = sample.x * u.gain3D * u.volumeGain3D / scaleFloor;
        const float magnitude = fabsf(scalar);
        const float waveDensity = t.displayMode3D == 2 || magnitude <= u.threshold3D
                                      ? 0.0f
                                      : powf(waveVisibility(t, magnitude), u.sharpness3D) * u.opacity3D * t.waveOpacity3D *
                                            28.0f * u.opticalScale3D;
        const float materialDensity = boundary ? u.boundaryOpacity3D * 1.8f : t.displayMode3D == 1 ? 0.0f : t.modelOpacity3D * 3.0f;
        const float density = waveDensity + materialDensity;
        const float alpha = 1.0f - expf(-density * delta);
        const Rgb tint = boundary ? rgb(.78f, .53f, .20f) : materialColor(t, sample.y);
        const Rgb wave = waveColor(t, scalar);
        const float norm = fmaxf(density, 1e-10f);
        const Rgb mapped = rgb((wave.r * waveDensity + tint.r * materialDensity) / norm,
                               (wave.g * waveDensity + tint.g * materialDensity) / norm,
                               (wave.b * waveDensity + tint.b * materialDensity) / norm);
        const float weight = (1.0f - aa) * alpha;
        ar += weight * mapped.r;
        ag += weight * mapped.g;
        ab += weight * mapped.b;
        aa += (1.0f - aa) * alpha;
        if (aa > 0.98f) break;
    }
    const float secondEdge = edgeDistance((origin + enter * direction) / extent);
    Rgb result = rgb(ar + (1.0f - aa) * background.r, ag + (1.0f - aa) * background.g, ab + (1.0f - aa) * background.b);
    const Rgb outline = t.modelStyle3D == 4 ? rgb(.22f, .43f, .46f) : rgb(0.35f, 0.76f, 0.38f);
    const bool hasLayer = u.showBoundary3D != 0 && (phi.x - plo.x < .999f || phi.y - plo.y < .999f || phi.z - plo.z < .999f);
    result = mix3(result, hasLayer ? rgb(.78f, .53f, .20f) : outline, 1.0f - smoothstepf(0.002f, 0.006f, secondEdge));
    if (hasLayer) {
        // The physical box inside the CPML shell, in the same depth-axis convention.
        const Vec3 pmin = (v3(plo.x, 1.0f - phi.z, plo.y) - v3(.5f, .5f, .5f)) * extent;
        const Vec3 pmax = (v3(phi.x, 1.0f - plo.z, phi.y) - v3(.5f, .5f, .5f)) * extent;
        const Vec3 a = (pmin - origin) * inverse, b = (pmax - origin) * inverse;
        const Vec3 nb = min3v(a, b), fb = max3v(a, b);
        const float boxEnter = fmaxf(fmaxf(nb.x, nb.y), nb.z);
        const float boxExit = fminf(fminf(fb.x, fb.y), fb.z);
        if (boxExit > fmaxf(boxEnter, 0.0f)) {
            const Vec3 p = (origin + boxEnter * direction - 0.5f * (pmin + pmax)) / (pmax - pmin);
            result = mix3(result, outline, 1.0f - smoothstepf(.002f, .006f, edgeDistance(p)));
        }
    }
    storePixel(out, k, format, result);
}

}  // namespace shade
}  // namespace seis3d
