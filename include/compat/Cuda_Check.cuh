// Cuda_Check.cuh - the 2-D GPU solver interface of the SeisWave Lab API
// (CUDA_Kernels/Cuda_Check.cuh:56-149) as a header-only C++ layer over the B200 solver's
// C ABI (include/seis2d_capi.h).
//
// GPUSimData keeps the reference member names; its device pointers are refreshed from the
// session after every call that may reallocate, so code that copies into d_szz_1,
// d_active_sources or d_rcv_grid_idx with cudaMemcpy keeps working.  Sessions run on the
// legacy default stream, as the reference's 2-D solver does, so such copies are ordered
// after the steps.  The extra member `session` is the library handle.  Every function
// rethrows the library status as the exception type the reference throws.  The GPU demo
// functions of the reference header (vector add, Game of Life) are not part of this library.
#pragma once

#include "Common.h"
#include "SolverNumerics.h"

#include <cuda_runtime.h>

#include <vector>

inline void checkCudaResult(cudaError_t result, const char* operation, const char* file, int line) {
    if (result != cudaSuccess)
        throw std::runtime_error(std::string("CUDA failure: ") + operation + " at " + file + ":" +
                                 std::to_string(line) + " | " + cudaGetErrorString(result));
}
#define CUDA_CHECK(call) checkCudaResult((call), #call, __FILE__, __LINE__)

struct GPUSimData {
    int NX = 0;
    int NZ = 0;
    int total_grid = 0;
    float dt = 0.0f;
    float inv_dt = 0.0f;
    int flag_type = 1;
    int npml = 0;
    int fs_idx = 0;
    bool upFlag = false;
    float c1_h = 0.0f, c2_h = 0.0f, c3_h = 0.0f, c4_h = 0.0f;

    float* d_vx_1 = nullptr; float* d_vx_2 = nullptr;
    float* d_vz_1 = nullptr; float* d_vz_2 = nullptr;
    float* d_sxx_1 = nullptr; float* d_sxx_2 = nullptr;
    float* d_szz_1 = nullptr; float* d_szz_2 = nullptr;
    float* d_sxz_1 = nullptr; float* d_sxz_2 = nullptr;

    float* d_vx = nullptr; float* d_vz = nullptr;
    float* d_sigmaxx = nullptr; float* d_sigmazz = nullptr; float* d_sigmaxz = nullptr;
    float* d_mu_x_flat = nullptr; float* d_lambda_x_flat = nullptr;
    float* d_lambda2mu_x_flat = nullptr; float* d_mu_z_flat = nullptr;
    float* d_rho_x_z_flat = nullptr; float* d_rho_orig_flat = nullptr;

    float* d_rho = nullptr;
    float* d_mu = nullptr;
    float* d_lambda = nullptr;
    float* d_lambda2mu = nullptr;

    float* d_dx = nullptr; float* d_dx_half = nullptr;
    float* d_dz = nullptr; float* d_dz_half = nullptr;
    float* d_dp_flat = nullptr;

    float* d_wavelet = nullptr;
    int* d_rcv_grid_idx = nullptr;
    float* d_record_vx_step = nullptr;
    float* d_record_vz_step = nullptr;

    GPUSource* d_active_sources = nullptr;
    float src_angle = 0.0f;
    int src_type = 0;
    int receiverCapacity = 0;

    seis2d_session* session = nullptr;  // B200 solver session (not in the reference struct)
};

namespace seis2d_compat {

struct ContextView {
    seis2d_context c{};
    explicit ContextView(const SimulationContext& s) {
        c.NX = s.NX; c.NZ = s.NZ; c.total_grid = s.total_grid; c.h = s.h; c.dt = s.dt; c.nt = s.nt;
        c.npml = s.npml; c.snap_spacenum = s.snap_spacenum; c.flag_type = s.flag_type;
        c.rho = view(s.rho); c.mu = view(s.mu); c.lambda = view(s.lambda); c.lambda2mu = view(s.lambda2mu);
        c.dp_flat = view(s.dp_flat);
        c.dx = view(s.dx); c.dx_half = view(s.dx_half); c.dz = view(s.dz); c.dz_half = view(s.dz_half);
        c.c1_h = s.c1_h; c.c2_h = s.c2_h; c.c3_h = s.c3_h; c.c4_h = s.c4_h;
        c.src_idx = s.src_idx; c.src_z_idx = s.src_z_idx;
        c.wavelet = view(s.wavelet);
        c.src_angle = s.src_angle; c.src_type = s.src_type; c.src_amp = s.src_amp;
        c.num_rcv = s.num_rcv;
        c.rcv_grid_idx = seis2d_int_view{s.rcv_grid_idx.data(), int64_t(s.rcv_grid_idx.size())};
        c.upFlag = s.upFlag ? 1 : 0;
    }
    static seis2d_float_view view(const std::vector<float>& v) { return seis2d_float_view{v.data(), int64_t(v.size())}; }
};

inline seis2d_session* session(const GPUSimData& g) {
    if (!g.session) throw std::logic_error("The GPU simulation is not initialized");
    return g.session;
}

inline void refresh(GPUSimData& g) {
    seis2d_device_views v{};
    check(seis2d_get_views(session(g), &v));
    g.NX = v.NX; g.NZ = v.NZ; g.total_grid = v.total_grid; g.dt = v.dt; g.inv_dt = v.inv_dt;
    g.flag_type = v.flag_type; g.npml = v.npml; g.fs_idx = v.fs_idx; g.upFlag = v.upFlag != 0;
    g.c1_h = v.c1_h; g.c2_h = v.c2_h; g.c3_h = v.c3_h; g.c4_h = v.c4_h;
    float** fields[SEIS2D_FIELD_COUNT] = {
        &g.d_vx_1, &g.d_vx_2, &g.d_vz_1, &g.d_vz_2, &g.d_sxx_1, &g.d_sxx_2, &g.d_szz_1, &g.d_szz_2, &g.d_sxz_1,
        &g.d_sxz_2, &g.d_vx, &g.d_vz, &g.d_sigmaxx, &g.d_sigmazz, &g.d_sigmaxz, &g.d_rho, &g.d_mu, &g.d_lambda,
        &g.d_lambda2mu, &g.d_mu_x_flat, &g.d_lambda_x_flat, &g.d_lambda2mu_x_flat, &g.d_mu_z_flat,
        &g.d_rho_x_z_flat, &g.d_rho_orig_flat};
    for (int q = 0; q < SEIS2D_FIELD_COUNT; ++q) *fields[q] = v.field[q];
    g.d_dx = v.d_dx; g.d_dx_half = v.d_dx_half; g.d_dz = v.d_dz; g.d_dz_half = v.d_dz_half;
    g.d_dp_flat = v.d_dp_flat;
    g.d_wavelet = v.d_wavelet;
    g.d_rcv_grid_idx = v.d_rcv_grid_idx;
    g.d_record_vx_step = v.d_record_vx_step;
    g.d_record_vz_step = v.d_record_vz_step;
    g.d_active_sources = reinterpret_cast<GPUSource*>(v.d_active_sources);
    g.receiverCapacity = v.receiverCapacity;
}

}  // namespace seis2d_compat

inline void releaseGpuSimulation(GPUSimData& gpu) {
    seis2d_release(gpu.session);
    gpu = GPUSimData{};
}

inline void validateSimulationContext(const SimulationContext& ctx) {
    const seis2d_compat::ContextView v(ctx);
    seis2d_compat::check(seis2d_validate_context(&v.c));
}

inline void initializeGpuSimulation(GPUSimData& gpu, const SimulationContext& ctx) {
    const seis2d_compat::ContextView v(ctx);
    seis2d_compat::check(seis2d_validate_context(&v.c));
    releaseGpuSimulation(gpu);
    seis2d_compat::check(seis2d_initialize(&gpu.session, &v.c));
    try {
        // The reference enqueues its 2-D solver on the legacy default stream.
        seis2d_compat::check(seis2d_set_stream(gpu.session, nullptr));
        seis2d_compat::refresh(gpu);
    } catch (...) {
        releaseGpuSimulation(gpu);
        throw;
    }
}

inline void updateGpuReceivers(GPUSimData& gpu, const std::vector<int>& receiverIndices) {
    if (receiverIndices.size() > size_t((std::numeric_limits<int>::max)()))
        throw std::invalid_argument("Too many receivers");
    seis2d_compat::check(seis2d_update_receivers(seis2d_compat::session(gpu), receiverIndices.data(),
                                                 int(receiverIndices.size())));
    seis2d_compat::refresh(gpu);
}

inline void runGpuSimulationStep(GPUSimData& gpu, int currentIteration, const SimulationContext& ctx,
                                 int activeSourceCount) {
    if (!gpu.session || gpu.total_grid <= 0)
        throw std::invalid_argument("Invalid GPU simulation state, iteration, or source count");
    gpu.src_type = ctx.src_type;
    gpu.src_angle = ctx.src_angle;
    const seis2d_compat::ContextView v(ctx);
    seis2d_compat::check(seis2d_run_step(gpu.session, currentIteration, &v.c, activeSourceCount));
}

inline void copyWavefieldToHost(GPUSimData& gpu, float* hostVzOutput) {
    if (!hostVzOutput || gpu.total_grid <= 0) throw std::invalid_argument("Invalid wavefield output buffer");
    seis2d_compat::check(seis2d_copy_wavefield(seis2d_compat::session(gpu), hostVzOutput));
}

inline void copyReceiverRecordsFromGpu(GPUSimData& gpu, int receiverCount, int timeSampleCount, int currentIteration,
                                       float* hostReceiverVx, float* hostReceiverVz) {
    if (receiverCount <= 0) return;
    seis2d_compat::check(seis2d_copy_receiver_records(seis2d_compat::session(gpu), receiverCount, timeSampleCount,
                                                      currentIteration, hostReceiverVx, hostReceiverVz));
}

inline void recordReceiverStepOnGpu(GPUSimData& gpu, int receiverCount, float* hostVxOutput, float* hostVzOutput) {
    if (receiverCount <= 0) return;
    seis2d_compat::check(seis2d_record_receiver_step(seis2d_compat::session(gpu), receiverCount, hostVxOutput,
                                                     hostVzOutput));
}

inline void generateWavefieldTextureOnGpu(GPUSimData& gpu, uchar4* deviceRgbaOutput, float colorScale,
                                          int componentIndex) {
    seis2d_compat::check(seis2d_wavefield_texture(seis2d_compat::session(gpu), deviceRgbaOutput, colorScale,
                                                  componentIndex));
}

inline void ReplayManager::uploadFrameToGpu(int frameIdx, GPUSimData& gpu) {
    if (frameIdx < 0 || frameIdx >= static_cast<int>(frames.size())) return;
    if (frames[frameIdx].size() != static_cast<size_t>(gpu.total_grid))
        throw std::invalid_argument("Replay frame dimensions do not match the active model");
    seis2d_session* s = seis2d_compat::session(gpu);
    if (gpu.flag_type == 1 || gpu.flag_type == 3) {
        const std::vector<float> zeros(frames[frameIdx].size(), 0.0f);
        seis2d_compat::check(seis2d_set_field(s, SEIS2D_VZ_1, frames[frameIdx].data()));
        seis2d_compat::check(seis2d_set_field(s, SEIS2D_VZ_2, zeros.data()));
    } else {
        seis2d_compat::check(seis2d_set_field(s, SEIS2D_VZ, frames[frameIdx].data()));
    }
}
