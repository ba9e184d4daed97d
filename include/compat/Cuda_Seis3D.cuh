// Cuda_Seis3D.cuh - the namespace Seis3D solver functions of the SeisWave Lab 3-D API as a
// header-only C++ layer over the B200 solver's C ABI (include/seis3d_capi.h).
//
// Each function has the signature of its reference declaration (cuda/Cuda_Seis3D.cuh:7-42)
// and rethrows the library's status codes as the exception types the reference throws
// (std::invalid_argument, std::logic_error, std::runtime_error), so callers and tests written
// against the reference compile and behave unchanged.
#pragma once

#include "Common3D.h"

#include <stdexcept>
#include <string>

namespace Seis3D {

namespace compat3D {

inline void check(int status) {
    if (status == SEIS3D_OK) return;
    const std::string message = seis3d_last_error();
    if (status == SEIS3D_INVALID_ARGUMENT) throw std::invalid_argument(message);
    if (status == SEIS3D_LOGIC_ERROR) throw std::logic_error(message);
    throw std::runtime_error(message);
}

inline seis3d_session* session(const GPUSimData3D& g) {
    if (!g.session3D) throw std::logic_error("Seis3D: GPU resources are not initialized.");
    return g.session3D;
}

// Refreshes the GPUSimData3D members from the session after a call that may reallocate.
inline void refresh(GPUSimData3D& g) {
    seis3d_device_views v{};
    check(seis3d_get_views(session(g), &v));
    for (int k = 0; k < 9; ++k) g.field3D[k] = static_cast<float*>(v.field3D[k]);
    g.inverseDensity3D = static_cast<float*>(v.inverseDensity3D);
    g.lambda3D = static_cast<float*>(v.lambda3D);
    g.mu3D = static_cast<float*>(v.mu3D);
    for (int a = 0; a < 3; ++a) {
        g.cpml3D[a] = v.cpml3D[a];
        g.slabCells3D[a] = std::size_t(v.slabCells3D[a]);
        g.coefficients3D[a] = v.coefficients3D[a];
    }
    g.stream3D = static_cast<cudaStream_t>(v.stream3D);
    g.receiverCount3D = v.receiverCount3D;
    g.allocatedBytes3D = std::size_t(v.allocatedBytes3D);
    g.pitch3D = v.pitch;
}

}  // namespace compat3D

inline void validateContext3D(SimulationContext3D& context3D) {
    seis3d_context c = context3D.toC();
    compat3D::check(seis3d_validate_context(&c));
    context3D.assign(c);
}

inline MemoryBudget3D estimateMemory3D(const SimulationContext3D& context3D) {
    const seis3d_context c = context3D.toC();
    seis3d_memory_budget b{};
    compat3D::check(seis3d_estimate_memory(&c, &b));
    MemoryBudget3D out;
    out.fieldBytes3D = std::size_t(b.fieldBytes3D);
    out.cpmlBytes3D = std::size_t(b.cpmlBytes3D);
    out.viewBytes3D = std::size_t(b.viewBytes3D);
    out.totalBytes3D = std::size_t(b.totalBytes3D);
    return out;
}

inline ViewLayout3D makeViewLayout3D(const SimulationContext3D& context3D) {
    const seis3d_context c = context3D.toC();
    seis3d_view_layout l{};
    compat3D::check(seis3d_make_view_layout(&c, &l));
    ViewLayout3D out;
    for (int a = 0; a < 3; ++a) {
        out.sliceOffset3D[a] = std::size_t(l.sliceOffset3D[a]);
        out.sliceWidth3D[a] = l.sliceWidth3D[a];
        out.sliceHeight3D[a] = l.sliceHeight3D[a];
        out.domainSize3D[a] = l.domainSize3D[a];
        out.domainOrigin3D[a] = l.domainOrigin3D[a];
    }
    out.volumeOffset3D = std::size_t(l.volumeOffset3D);
    out.totalSamples3D = std::size_t(l.totalSamples3D);
    out.volumeX3D = l.volumeX3D; out.volumeY3D = l.volumeY3D; out.volumeZ3D = l.volumeZ3D;
    return out;
}

inline void releaseGpu3D(GPUSimData3D& gpu3D) noexcept {
    if (gpu3D.startEvent3D) cudaEventDestroy(gpu3D.startEvent3D);
    if (gpu3D.stopEvent3D) cudaEventDestroy(gpu3D.stopEvent3D);
    seis3d_release(gpu3D.session3D);
    gpu3D = GPUSimData3D{};
}

// The session uses the reference's unpitched rows when the tensor-map stride rule allows it.
inline void initializeGpu3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D) {
    seis3d_context c = context3D.toC();
    compat3D::check(seis3d_validate_context(&c));
    releaseGpu3D(gpu3D);
    seis3d_options options{};
    options.compact_rows = c.gx3D % 4 == 0;
    compat3D::check(seis3d_initialize(&gpu3D.session3D, &c, &options));
    try {
        compat3D::refresh(gpu3D);
        if (cudaEventCreate(&gpu3D.startEvent3D) != cudaSuccess || cudaEventCreate(&gpu3D.stopEvent3D) != cudaSuccess)
            throw std::runtime_error("Seis3D: cannot create timing events.");
    } catch (...) {
        releaseGpu3D(gpu3D);
        throw;
    }
}

inline void resetGpu3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D) {
    const seis3d_context c = context3D.toC();
    compat3D::check(seis3d_reset(compat3D::session(gpu3D), &c));
}

inline void refreshCpmlCoefficients3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D) {
    const seis3d_context c = context3D.toC();
    compat3D::check(seis3d_refresh_cpml(compat3D::session(gpu3D), &c));
    compat3D::refresh(gpu3D);
}

inline void runStep3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D, const Source3D& source3D,
                      std::uint64_t step3D) {
    const seis3d_context c = context3D.toC();
    const seis3d_source s = source3D.toC();
    compat3D::check(seis3d_run_step(compat3D::session(gpu3D), &c, &s, step3D));
}

inline void setReceivers3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D, const Receiver3D* receivers3D,
                           int count3D) {
    const seis3d_context c = context3D.toC();
    compat3D::check(seis3d_set_receivers(compat3D::session(gpu3D), &c,
                                         reinterpret_cast<const seis3d_receiver*>(receivers3D), count3D));
    compat3D::refresh(gpu3D);
}

inline const float* sampleReceivers3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D) {
    const seis3d_context c = context3D.toC();
    const float* values = nullptr;
    compat3D::check(seis3d_sample_receivers(compat3D::session(gpu3D), &c, &values));
    gpu3D.hostReceiverValues3D = const_cast<float*>(values);
    return values;
}

inline void probeMaterial3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D, const Receiver3D& point3D,
                            float values3D[3]) {
    const seis3d_context c = context3D.toC();
    compat3D::check(seis3d_probe_material(compat3D::session(gpu3D), &c,
                                          reinterpret_cast<const seis3d_receiver*>(&point3D), values3D));
}

inline void uploadModelPlane3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D, int plane3D,
                               const float* values3D) {
    const seis3d_context c = context3D.toC();
    compat3D::check(seis3d_upload_model_plane(compat3D::session(gpu3D), &c, plane3D, values3D));
}

inline void finishModelUpload3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D) {
    const seis3d_context c = context3D.toC();
    compat3D::check(seis3d_finish_model_upload(compat3D::session(gpu3D), &c));
}

// extractViews3D (cuda/Cuda_Seis3D.cu:627-646): the three slices and the bounded volume of
// one wavefield component and one material component into `output3D`, a device buffer of
// 2 * totalSamples3D floats (volumeOffset3D samples without the volume).  The layout passed
// in must be the one makeViewLayout3D gives for this context.
inline void extractViews3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D, float* output3D,
                           const ViewLayout3D& layout3D, const int slice3D[3], int component3D,
                           int materialComponent3D, bool volumeEnabled3D, float& maximum3D,
                           float materialRange3D[2], bool includeBoundary3D = false,
                           float* velocityMaximum3D = nullptr) {
    const seis3d_context c = context3D.toC();
    seis3d_view_layout l{};
    compat3D::check(seis3d_make_view_layout(&c, &l));
    for (int a = 0; a < 3; ++a)
        if (std::size_t(l.sliceOffset3D[a]) != layout3D.sliceOffset3D[a] || l.sliceWidth3D[a] != layout3D.sliceWidth3D[a] ||
            l.sliceHeight3D[a] != layout3D.sliceHeight3D[a])
            throw std::invalid_argument("Seis3D: view layout does not match the context.");
    if (std::size_t(l.volumeOffset3D) != layout3D.volumeOffset3D || std::size_t(l.totalSamples3D) != layout3D.totalSamples3D)
        throw std::invalid_argument("Seis3D: view layout does not match the context.");
    compat3D::check(seis3d_extract_views(compat3D::session(gpu3D), &c, output3D, &l, slice3D, component3D,
                                         materialComponent3D, volumeEnabled3D ? 1 : 0, includeBoundary3D ? 1 : 0,
                                         &maximum3D, materialRange3D, velocityMaximum3D));
}

inline void downloadModelPlane3D(GPUSimData3D& gpu3D, const SimulationContext3D& context3D, int plane3D,
                                 float* values3D) {
    const seis3d_context c = context3D.toC();
    compat3D::check(seis3d_download_model_plane(compat3D::session(gpu3D), &c, plane3D, values3D));
}

}  // namespace Seis3D
