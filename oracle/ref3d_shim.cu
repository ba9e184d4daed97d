// ref3d_shim.cu - C ABI around the reference's own 3-D CUDA solver.
//
// TEST INFRASTRUCTURE ONLY.  This translation unit includes the reference's unmodified
// cuda/Cuda_Seis3D.cu from the reference tree (the include path is set by
// oracle/Makefile) and exposes its Seis3D:: functions as extern "C" so that the parity
// tests and bench.py's reference arm can drive the reference solver exactly as its own
// host code does (src/Seis3D_Sim.cpp:120-153).  Nothing of the reference is copied here;
// the build output goes to oracle/_ref/ only.
#include "Cuda_Seis3D.cu"

#include "../include/seis3d_capi.h"

#include <cstring>
#include <stdexcept>
#include <string>

namespace {

thread_local std::string refMessage;

Seis3D::SimulationContext3D toReference(const seis3d_context& in) {
    Seis3D::SimulationContext3D c;
    c.nx3D = in.nx3D; c.ny3D = in.ny3D; c.nz3D = in.nz3D; c.pml3D = in.pml3D;
    c.freeSurface3D = in.freeSurface3D != 0; c.reflecting3D = in.reflecting3D != 0;
    c.spacing3D = in.spacing3D; c.cfl3D = in.cfl3D; c.dt3D = in.dt3D;
    c.manualTimeStep3D = in.manualTimeStep3D != 0; c.requestedDtMs3D = in.requestedDtMs3D; c.safeDt3D = in.safeDt3D;
    c.vp3D = in.vp3D; c.vs3D = in.vs3D; c.density3D = in.density3D;
    c.layerVp3D = in.layerVp3D; c.layerVs3D = in.layerVs3D; c.layerDensity3D = in.layerDensity3D;
    c.maxVp3D = in.maxVp3D; c.frequency3D = in.frequency3D;
    c.modelKind3D = Seis3D::ModelKind3D(in.modelKind3D);
    c.interfaceDepth3D = in.interfaceDepth3D; c.layerDip3D = in.layerDip3D; c.layerThickness3D = in.layerThickness3D;
    c.faultThrow3D = in.faultThrow3D; c.anomalyRadius3D = in.anomalyRadius3D;
    c.gx3D = in.gx3D; c.gy3D = in.gy3D; c.gz3D = in.gz3D; c.ox3D = in.ox3D; c.oy3D = in.oy3D; c.oz3D = in.oz3D;
    c.cells3D = std::size_t(in.cells3D);
    return c;
}

void fromReference(const Seis3D::SimulationContext3D& c, seis3d_context& out) {
    out.nx3D = c.nx3D; out.ny3D = c.ny3D; out.nz3D = c.nz3D; out.pml3D = c.pml3D;
    out.freeSurface3D = c.freeSurface3D; out.reflecting3D = c.reflecting3D;
    out.spacing3D = c.spacing3D; out.cfl3D = c.cfl3D; out.dt3D = c.dt3D;
    out.manualTimeStep3D = c.manualTimeStep3D; out.requestedDtMs3D = c.requestedDtMs3D; out.safeDt3D = c.safeDt3D;
    out.vp3D = c.vp3D; out.vs3D = c.vs3D; out.density3D = c.density3D;
    out.layerVp3D = c.layerVp3D; out.layerVs3D = c.layerVs3D; out.layerDensity3D = c.layerDensity3D;
    out.maxVp3D = c.maxVp3D; out.frequency3D = c.frequency3D; out.modelKind3D = int(c.modelKind3D);
    out.interfaceDepth3D = c.interfaceDepth3D; out.layerDip3D = c.layerDip3D; out.layerThickness3D = c.layerThickness3D;
    out.faultThrow3D = c.faultThrow3D; out.anomalyRadius3D = c.anomalyRadius3D;
    out.gx3D = c.gx3D; out.gy3D = c.gy3D; out.gz3D = c.gz3D; out.ox3D = c.ox3D; out.oy3D = c.oy3D; out.oz3D = c.oz3D;
    out.cells3D = c.cells3D;
}

Seis3D::Source3D toReference(const seis3d_source& s) {
    Seis3D::Source3D r;
    r.x3D = s.x3D; r.y3D = s.y3D; r.z3D = s.z3D;
    r.kind3D = Seis3D::SourceKind3D(s.kind3D);
    r.amplitude3D = s.amplitude3D;
    for (int a = 0; a < 3; ++a) r.direction3D[a] = s.direction3D[a];
    return r;
}

struct RefSession {
    Seis3D::SimulationContext3D context;
    Seis3D::GPUSimData3D gpu;
};

// Map exceptions onto the status codes of include/seis3d_capi.h.
template <class F> int guarded(F&& body) {
    try {
        body();
        refMessage.clear();
        return SEIS3D_OK;
    } catch (const std::invalid_argument& e) {
        refMessage = e.what(); return SEIS3D_INVALID_ARGUMENT;
    } catch (const std::logic_error& e) {
        refMessage = e.what(); return SEIS3D_LOGIC_ERROR;
    } catch (const std::exception& e) {
        refMessage = e.what(); return SEIS3D_RUNTIME_ERROR;
    }
}

}  // namespace

extern "C" {

const char* ref3d_last_error(void) { return refMessage.c_str(); }

// The reference's own default member initialisers (include/Common3D.h:24-49).
void ref3d_default_context(seis3d_context* c) { fromReference(Seis3D::SimulationContext3D{}, *c); }

void ref3d_default_source(seis3d_source* s) {
    const Seis3D::Source3D r{};
    s->x3D = r.x3D; s->y3D = r.y3D; s->z3D = r.z3D;
    s->kind3D = int(r.kind3D);
    s->amplitude3D = r.amplitude3D;
    for (int a = 0; a < 3; ++a) s->direction3D[a] = r.direction3D[a];
}

int ref3d_validate(seis3d_context* c) {
    return guarded([&] {
        auto r = toReference(*c);
        Seis3D::validateContext3D(r);
        fromReference(r, *c);
    });
}

int ref3d_estimate_memory(const seis3d_context* c, seis3d_memory_budget* out) {
    return guarded([&] {
        const auto b = Seis3D::estimateMemory3D(toReference(*c));
        out->fieldBytes3D = b.fieldBytes3D; out->cpmlBytes3D = b.cpmlBytes3D;
        out->viewBytes3D = b.viewBytes3D; out->totalBytes3D = b.totalBytes3D;
    });
}

// The reference's FP64->FP32 CPML profile (cuda/Cuda_Seis3D.cu:45-64); host only.
int ref3d_make_coefficients(const seis3d_context* c, int axis, float* out) {
    const auto v = Seis3D::makeCoefficients3D(toReference(*c), axis);
    std::memcpy(out, v.data(), v.size() * sizeof(float));
    return int(v.size());
}

void* ref3d_create(const seis3d_context* c) {
    auto* s = new RefSession;
    s->context = toReference(*c);
    const int status = guarded([&] { Seis3D::initializeGpu3D(s->gpu, s->context); });
    if (status != SEIS3D_OK) { delete s; return nullptr; }
    return s;
}

void ref3d_destroy(void* handle) {
    auto* s = static_cast<RefSession*>(handle);
    if (!s) return;
    Seis3D::releaseGpu3D(s->gpu);
    delete s;
}

int ref3d_upload_plane(void* h, int z, const float* values) {
    auto* s = static_cast<RefSession*>(h);
    return guarded([&] { Seis3D::uploadModelPlane3D(s->gpu, s->context, z, values); });
}

int ref3d_finish_upload(void* h) {
    auto* s = static_cast<RefSession*>(h);
    return guarded([&] { Seis3D::finishModelUpload3D(s->gpu, s->context); });
}

int ref3d_reset(void* h) {
    auto* s = static_cast<RefSession*>(h);
    return guarded([&] { Seis3D::resetGpu3D(s->gpu, s->context); });
}

int ref3d_set_receivers(void* h, const seis3d_receiver* r, int count) {
    auto* s = static_cast<RefSession*>(h);
    static_assert(sizeof(seis3d_receiver) == sizeof(Seis3D::Receiver3D), "receiver layout");
    return guarded([&] {
        Seis3D::setReceivers3D(s->gpu, s->context, reinterpret_cast<const Seis3D::Receiver3D*>(r), count);
    });
}

// Enqueue `count` steps exactly as the reference loop does (runStep3D per step).
int ref3d_run_steps(void* h, const seis3d_source* src, uint64_t first, int count) {
    auto* s = static_cast<RefSession*>(h);
    const auto source = toReference(*src);
    return guarded([&] {
        for (int k = 0; k < count; ++k) Seis3D::runStep3D(s->gpu, s->context, source, first + uint64_t(k));
    });
}

// The recording loop of advanceSimulation3D (src/Seis3D_Sim.cpp:125-132): step, then
// sampleReceivers3D (D2H + stream sync) whenever (step+1) % stride == 0.
int ref3d_run_gather(void* h, const seis3d_source* src, uint64_t first, int count, int stride,
                     float* out, int capacity, int* taken) {
    auto* s = static_cast<RefSession*>(h);
    const auto source = toReference(*src);
    *taken = 0;
    return guarded([&] {
        const std::size_t perSample = std::size_t(s->gpu.receiverCount3D) * 3;
        for (int k = 0; k < count; ++k) {
            const uint64_t n = first + uint64_t(k);
            Seis3D::runStep3D(s->gpu, s->context, source, n);
            if (stride > 0 && (n + 1) % uint64_t(stride) == 0 && *taken < capacity) {
                const float* values = Seis3D::sampleReceivers3D(s->gpu, s->context);
                if (values) std::memcpy(out + std::size_t(*taken) * perSample, values, perSample * sizeof(float));
                ++*taken;
            }
        }
    });
}

// Device time of `count` reference steps with CUDA events on the session stream.
int ref3d_time_steps(void* h, const seis3d_source* src, uint64_t first, int count, float* ms) {
    auto* s = static_cast<RefSession*>(h);
    const auto source = toReference(*src);
    return guarded([&] {
        cudaEvent_t a, b;
        cudaEventCreate(&a); cudaEventCreate(&b);
        cudaEventRecord(a, s->gpu.stream3D);
        for (int k = 0; k < count; ++k) Seis3D::runStep3D(s->gpu, s->context, source, first + uint64_t(k));
        cudaEventRecord(b, s->gpu.stream3D);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(ms, a, b);
        cudaEventDestroy(a); cudaEventDestroy(b);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    });
}

int ref3d_sample(void* h, float* out) {
    auto* s = static_cast<RefSession*>(h);
    return guarded([&] {
        const float* values = Seis3D::sampleReceivers3D(s->gpu, s->context);
        if (values) std::memcpy(out, values, std::size_t(s->gpu.receiverCount3D) * 3 * sizeof(float));
    });
}

// Copy one field (0-8 wavefields, 9 = 1/rho, 10 = lambda, 11 = mu) to the host.
int ref3d_get_field(void* h, int f, float* out) {
    auto* s = static_cast<RefSession*>(h);
    return guarded([&] {
        const float* src = f < 9 ? s->gpu.field3D[f] : f == 9 ? s->gpu.inverseDensity3D : f == 10 ? s->gpu.lambda3D : s->gpu.mu3D;
        if (cudaStreamSynchronize(s->gpu.stream3D) != cudaSuccess) throw std::runtime_error("stream");
        if (cudaMemcpy(out, src, s->context.cells3D * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("copy field");
    });
}

int ref3d_set_field(void* h, int f, const float* in) {
    auto* s = static_cast<RefSession*>(h);
    return guarded([&] {
        float* dst = f < 9 ? s->gpu.field3D[f] : f == 9 ? s->gpu.inverseDensity3D : f == 10 ? s->gpu.lambda3D : s->gpu.mu3D;
        if (cudaStreamSynchronize(s->gpu.stream3D) != cudaSuccess) throw std::runtime_error("stream");
        if (cudaMemcpy(dst, in, s->context.cells3D * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("copy field");
    });
}

int ref3d_synchronize(void* h) {
    auto* s = static_cast<RefSession*>(h);
    return guarded([&] {
        const cudaError_t e = cudaStreamSynchronize(s->gpu.stream3D);
        if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    });
}


// extractViews3D of the reference into a device buffer it allocates, copied back to `out`
// (2 floats per sample).
int ref3d_extract_views(void* h, const seis3d_view_layout* l, const int slices[3], int component, int material,
                        int volume, int includeBoundary, float* out, float* maximum, float range[2], float* vmax) {
    auto* s = static_cast<RefSession*>(h);
    return guarded([&] {
        Seis3D::ViewLayout3D layout = Seis3D::makeViewLayout3D(s->context);
        (void)l;
        const std::size_t count = volume ? layout.totalSamples3D : layout.volumeOffset3D;
        float* device = nullptr;
        if (cudaMalloc(&device, std::max<std::size_t>(count, 1) * 2 * sizeof(float)) != cudaSuccess)
            throw std::runtime_error("view buffer");
        try {
            Seis3D::extractViews3D(s->gpu, s->context, device, layout, slices, component, material, volume != 0,
                                   *maximum, range, includeBoundary != 0, vmax);
            if (cudaMemcpy(out, device, count * 2 * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
                throw std::runtime_error("view copy");
        } catch (...) {
            cudaFree(device);
            throw;
        }
        cudaFree(device);
    });
}
}  // extern "C"
