// seis3d_shade_oracle.cpp - TEST INFRASTRUCTURE ONLY: a CPU restatement of the reference's
// display shaders, used by the tests to check the CUDA shading kernels of the B200 library.
//
//   shaders/seis3d_transfer.glsl:6-28  waveVisibility3D, waveColor3D, materialColor3D
//   shaders/seis3d_slice.frag:9-20     the slice composite (one pixel per texel centre)
//   shaders/seis3d_volume.frag:15-83   the raymarched volume with box / CPML outlines
//
// GLSL built-ins are written out from the GLSL specification: mix(x, y, a) = x(1 - a) + ya,
// clamp(x, lo, hi) = min(max(x, lo), hi), smoothstep(e0, e1, x) = t^2(3 - 2t) with
// t = clamp((x - e0)/(e1 - e0), 0, 1), normalize(v) = v/length(v).  The volume texture is
// sampled with the GL_LINEAR / GL_CLAMP_TO_EDGE rule (texel coordinate u*n - 1/2, neighbours
// clamped to the edge texels).  The GL shaders themselves cannot run here (no graphics stack),
// so parity of this restatement with the reference's drawn pixels is unpinned; the tests pin
// its pieces with hand-computed values instead.
//
// Built with -ffp-contract=off; FP32 throughout, like the shaders.
#include "../include/seis3d_capi.h"

#include <algorithm>
#include <cmath>
#include <cstdint>

namespace {

struct V3 {
    float x, y, z;
};
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 mul(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
V3 div(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
V3 muls(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 normalize(V3 a) {
    const float n = std::sqrt(dot(a, a));
    return {a.x / n, a.y / n, a.z / n};
}
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V3 vmin(V3 a, V3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
V3 vmax(V3 a, V3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
V3 of(const float* p) { return {p[0], p[1], p[2]}; }

float clampf(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }
float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
V3 mix(V3 x, V3 y, float a) { return {mix(x.x, y.x, a), mix(x.y, y.y, a), mix(x.z, y.z, a)}; }
float smoothstep(float e0, float e1, float x) {
    const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

float visibility(const seis3d_transfer& t, float magnitude) {
    const float v = clampf((magnitude - t.waveThreshold3D) / std::fmax(1.0f - t.waveThreshold3D, 1e-6f), 0.0f, 1.0f);
    return std::pow(v, std::fmax(t.waveGamma3D, 0.1f));
}

V3 waveColor(const seis3d_transfer& t, float value) {
    const float q = clampf(t.unsignedWave3D != 0 ? std::fabs(value) : value * 0.5f + 0.5f, 0.0f, 1.0f) * 4.0f;
    const int index = std::min(int(q), 3);
    return mix(of(t.palette3D[index]), of(t.palette3D[index + 1]), q - float(index));
}

V3 materialColor(const seis3d_transfer& t, float value) {
    const float span = t.materialRange3D[1] - t.materialRange3D[0];
    const float q = span > std::fmax(1e-6f, std::fabs(t.materialRange3D[1]) * 1e-6f)
                        ? clampf((value - t.materialRange3D[0]) / span, 0.0f, 1.0f)
                        : 0.5f;
    if (t.modelStyle3D == 0) return mix(V3{.09f, .13f, .17f}, V3{.43f, .53f, .6f}, q);
    if (t.modelStyle3D == 1)
        return q < .5f ? mix(V3{.13f, .28f, .33f}, V3{.48f, .65f, .46f}, q * 2.0f)
                       : mix(V3{.48f, .65f, .46f}, V3{.78f, .52f, .31f}, (q - .5f) * 2.0f);
    if (t.modelStyle3D == 2) {
        const float g = mix(.12f, .85f, q);
        return {g, g, g};
    }
    if (t.modelStyle3D == 3) return waveColor(t, t.unsignedWave3D != 0 ? q : q * 2.0f - 1.0f);
    return mix(V3{.97f, .96f, .93f}, V3{.79f, .84f, .85f}, q);
}

// texture() of the RG volume: trilinear, clamp to edge.
void sample(const float* texels, int nx, int ny, int nz, V3 uvw, float out[2]) {
    const float c[3] = {clampf(uvw.x * float(nx) - 0.5f, -1.0f, float(nx)),
                        clampf(uvw.y * float(ny) - 0.5f, -1.0f, float(ny)),
                        clampf(uvw.z * float(nz) - 0.5f, -1.0f, float(nz))};
    const int n[3] = {nx, ny, nz};
    int lo[3], hi[3];
    float f[3];
    for (int a = 0; a < 3; ++a) {
        const float b = std::floor(c[a]);
        f[a] = c[a] - b;
        lo[a] = std::clamp(int(b), 0, n[a] - 1);
        hi[a] = std::clamp(int(b) + 1, 0, n[a] - 1);
    }
    for (int ch = 0; ch < 2; ++ch) {
        auto at = [&](int x, int y, int z) { return texels[2 * ((int64_t(z) * ny + y) * nx + x) + ch]; };
        const float y0 = mix(mix(at(lo[0], lo[1], lo[2]), at(hi[0], lo[1], lo[2]), f[0]),
                             mix(at(lo[0], hi[1], lo[2]), at(hi[0], hi[1], lo[2]), f[0]), f[1]);
        const float y1 = mix(mix(at(lo[0], lo[1], hi[2]), at(hi[0], lo[1], hi[2]), f[0]),
                             mix(at(lo[0], hi[1], hi[2]), at(hi[0], hi[1], hi[2]), f[0]), f[1]);
        out[ch] = mix(y0, y1, f[2]);
    }
}

float edgeDistance(V3 p) {
    const float e[3] = {std::fabs(std::fabs(p.x) - 0.5f), std::fabs(std::fabs(p.y) - 0.5f), std::fabs(std::fabs(p.z) - 0.5f)};
    return std::fmax(std::fmin(e[0], e[1]), std::fmin(std::fmax(e[0], e[1]), e[2]));
}

V3 volumePixel(const float* texels, int nx, int ny, int nz, const seis3d_transfer& t, const seis3d_volume_view& u,
               float tx, float ty) {
    const V3 extent = of(u.extent3D);
    const V3 forward = normalize({std::cos(u.pitch3D) * std::sin(u.yaw3D), std::sin(u.pitch3D),
                                  std::cos(u.pitch3D) * std::cos(u.yaw3D)});
    const V3 right = normalize(cross({0, 1, 0}, forward));
    const V3 up = cross(forward, right);
    const V3 target = add(muls(u.pan3D[0], right), muls(u.pan3D[1], up));
    const V3 origin = add(target, muls(u.distance3D, forward));
    const float sx = (tx - 0.5f) * 1.3f * u.aspect3D, sy = (ty - 0.5f) * 1.3f;
    const V3 direction = normalize(add(add(V3{-forward.x, -forward.y, -forward.z}, muls(sx, right)), muls(sy, up)));
    const V3 safe = {std::fabs(direction.x) < 1e-7f ? 1e-7f : direction.x,
                     std::fabs(direction.y) < 1e-7f ? 1e-7f : direction.y,
                     std::fabs(direction.z) < 1e-7f ? 1e-7f : direction.z};
    const V3 inverse = {1.0f / safe.x, 1.0f / safe.y, 1.0f / safe.z};
    const V3 first = mul(sub(muls(-0.5f, extent), origin), inverse);
    const V3 second = mul(sub(muls(0.5f, extent), origin), inverse);
    const V3 nearT = vmin(first, second), farT = vmax(first, second);
    float enter = std::fmax(std::fmax(nearT.x, nearT.y), nearT.z);
    const float exitT = std::fmin(std::fmin(farT.x, farT.y), farT.z);
    const V3 background = t.modelStyle3D == 4 ? V3{.97f, .96f, .93f} : V3{0.025f, 0.041f, 0.05f};
    if (exitT <= std::fmax(enter, 0.0f)) return background;
    enter = std::fmax(enter, 0.0f);
    const V3 lo = of(u.domainLow3D), hi = of(u.domainHigh3D), plo = of(u.physicalLow3D), phi = of(u.physicalHigh3D);
    V3 path = div(muls(exitT - enter, direction), extent);
    path = {std::fabs(path.x), std::fabs(path.y), std::fabs(path.z)};
    const V3 texPath = mul(V3{path.x, path.z, path.y}, sub(hi, lo));
    const V3 scaled = mul(texPath, V3{float(nx), float(ny), float(nz)});
    const int steps = int(clampf(std::ceil(std::sqrt(dot(scaled, scaled)) * u.sampling3D), 192.0f, 1024.0f));
    const float delta = (exitT - enter) / float(steps);
    const float scaleFloor = std::fmax(u.scale3D, 1e-20f);
    float acc[4] = {0, 0, 0, 0};
    for (int i = 0; i < steps; ++i) {
        const V3 q = add(div(add(origin, muls(enter + (float(i) + 0.5f) * delta, direction)), extent), V3{0.5f, 0.5f, 0.5f});
        const V3 w = {q.x, q.z, 1.0f - q.y};
        const V3 uvw = {mix(lo.x, hi.x, w.x), mix(lo.y, hi.y, w.y), mix(lo.z, hi.z, w.z)};
        const bool boundary = u.showBoundary3D != 0 && (uvw.x < plo.x || uvw.y < plo.y || uvw.z < plo.z ||
                                                        uvw.x > phi.x || uvw.y > phi.y || uvw.z > phi.z);
        float s[2];
        sample(texels, nx, ny, nz, uvw, s);
        const float scalar = s[0] * u.gain3D * u.volumeGain3D / scaleFloor;
        const float magnitude = std::fabs(scalar);
        const float waveDensity = t.displayMode3D == 2 || magnitude <= u.threshold3D
                                      ? 0.0f
                                      : std::pow(visibility(t, magnitude), u.sharpness3D) * u.opacity3D *
                                            t.waveOpacity3D * 28.0f * u.opticalScale3D;
        const float materialDensity =
            boundary ? u.boundaryOpacity3D * 1.8f : t.displayMode3D == 1 ? 0.0f : t.modelOpacity3D * 3.0f;
        const float density = waveDensity + materialDensity;
        const float alpha = 1.0f - std::exp(-density * delta);
        const V3 tint = boundary ? V3{.78f, .53f, .20f} : materialColor(t, s[1]);
        const V3 wave = waveColor(t, scalar);
        const float norm = std::fmax(density, 1e-10f);
        const V3 mapped = {(wave.x * waveDensity + tint.x * materialDensity) / norm,
                           (wave.y * waveDensity + tint.y * materialDensity) / norm,
                           (wave.z * waveDensity + tint.z * materialDensity) / norm};
        const float weight = (1.0f - acc[3]) * alpha;
        acc[0] += weight * mapped.x;
        acc[1] += weight * mapped.y;
        acc[2] += weight * mapped.z;
        acc[3] += (1.0f - acc[3]) * alpha;
        if (acc[3] > 0.98f) break;
    }
    const float secondEdge = edgeDistance(div(add(origin, muls(enter, direction)), extent));
    V3 result = {acc[0] + (1.0f - acc[3]) * background.x, acc[1] + (1.0f - acc[3]) * background.y,
                 acc[2] + (1.0f - acc[3]) * background.z};
    const V3 outline = t.modelStyle3D == 4 ? V3{.22f, .43f, .46f} : V3{0.35f, 0.76f, 0.38f};
    const bool hasLayer = u.showBoundary3D != 0 && (phi.x - plo.x < .999f || phi.y - plo.y < .999f || phi.z - plo.z < .999f);
    result = mix(result, hasLayer ? V3{.78f, .53f, .20f} : outline, 1.0f - smoothstep(0.002f, 0.006f, secondEdge));
    if (hasLayer) {
        const V3 pmin = mul(sub(V3{plo.x, 1.0f - phi.z, plo.y}, V3{.5f, .5f, .5f}), extent);
        const V3 pmax = mul(sub(V3{phi.x, 1.0f - plo.z, phi.y}, V3{.5f, .5f, .5f}), extent);
        const V3 a = mul(sub(pmin, origin), inverse), b = mul(sub(pmax, origin), inverse);
        const V3 nb = vmin(a, b), fb = vmax(a, b);
        const float boxEnter = std::fmax(std::fmax(nb.x, nb.y), nb.z);
        const float boxExit = std::fmin(std::fmin(fb.x, fb.y), fb.z);
        if (boxExit > std::fmax(boxEnter, 0.0f)) {
            const V3 p = div(sub(add(origin, muls(boxEnter, direction)), muls(0.5f, add(pmin, pmax))), sub(pmax, pmin));
            result = mix(result, outline, 1.0f - smoothstep(.002f, .006f, edgeDistance(p)));
        }
    }
    return result;
}

}  // namespace

extern "C" {

// Slice composite of `count` view samples {wave, material} into RGBA floats.
void oracle_shade_slices(const float* views, uint64_t count, const seis3d_transfer* t, float scale, float gain,
                         float* rgba) {
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < int64_t(count); ++k) {
        const float value = views[2 * k], material = views[2 * k + 1];
        const float q = clampf(value * gain / std::fmax(scale, 1e-20f), -1.0f, 1.0f);
        const V3 background = t->modelStyle3D == 4 ? V3{.97f, .96f, .93f} : V3{0.028f, 0.045f, 0.052f};
        const V3 mat = materialColor(*t, material);
        const float alpha = visibility(*t, std::fabs(q)) * t->waveOpacity3D;
        const V3 base = t->displayMode3D == 1 ? background : muls(t->materialBrightness3D, mat);
        const V3 mapped = t->displayMode3D == 2 ? mat : mix(base, waveColor(*t, q), alpha);
        rgba[4 * k] = mapped.x;
        rgba[4 * k + 1] = mapped.y;
        rgba[4 * k + 2] = mapped.z;
        rgba[4 * k + 3] = 1.0f;
    }
}

// Volume composite of a width x height target (row 0 at the bottom) into RGBA floats.
void oracle_render_volume(const float* texels, int nx, int ny, int nz, const seis3d_transfer* t,
                          const seis3d_volume_view* u, int width, int height, float* rgba) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            const V3 c = volumePixel(texels, nx, ny, nz, *t, *u, (float(x) + 0.5f) / float(width),
                                     (float(y) + 0.5f) / float(height));
            float* o = rgba + 4 * (int64_t(y) * width + x);
            o[0] = c.x;
            o[1] = c.y;
            o[2] = c.z;
            o[3] = 1.0f;
        }
}

}  // extern "C"
