// ref2d_shim.cu - C ABI around the reference's own 2-D CUDA solver.
//
// TEST INFRASTRUCTURE ONLY.  This translation unit includes the reference's unmodified
// CUDA_Kernels/Cuda_Check.cu from the reference tree (include paths and the reference's
// --use_fast_math are set by oracle/Makefile; Common.h resolves to the headless stand-in in
// oracle/ref2d_include/) and exposes its 2-D solver functions as extern "C", so that the
// parity tests and the benchmark's reference arm drive the reference solver through its own
// entry points (Cuda_Check.cuh:126-149).  The build output goes to oracle/_ref/ only.
#include "Cuda_Check.cu"

#include "../include/seis2d_capi.h"

#include <cstring>
#include <exception>
#include <string>

namespace {

thread_local std::string refMessage;

template <class F> int call(F&& body) {
    try {
        body();
        return 0;
    } catch (const std::invalid_argument& e) {
        refMessage = e.what(); return SEIS2D_INVALID_ARGUMENT;
    } catch (const std::overflow_error& e) {
        refMessage = e.what(); return SEIS2D_OVERFLOW_ERROR;
    } catch (const std::logic_error& e) {
        refMessage = e.what(); return SEIS2D_LOGIC_ERROR;
    } catch (const std::exception& e) {
        refMessage = e.what(); return SEIS2D_RUNTIME_ERROR;
    }
}

template <class T> std::vector<T> vec(const T* p, int64_t n) {
    return (p && n > 0) ? std::vector<T>(p, p + n) : std::vector<T>(std::size_t(std::max<int64_t>(n, 0)));
}

SimulationContext toReference(const seis2d_context& in) {
    SimulationContext c{};
    c.NX = in.NX; c.NZ = in.NZ; c.total_grid = in.total_grid; c.h = in.h; c.dt = in.dt; c.nt = in.nt;
    c.npml = in.npml; c.snap_spacenum = in.snap_spacenum; c.flag_type = in.flag_type;
    c.rho = vec(in.rho.data, in.rho.size); c.mu = vec(in.mu.data, in.mu.size);
    c.lambda = vec(in.lambda.data, in.lambda.size); c.lambda2mu = vec(in.lambda2mu.data, in.lambda2mu.size);
    c.dp_flat = vec(in.dp_flat.data, in.dp_flat.size);
    c.dx = vec(in.dx.data, in.dx.size); c.dx_half = vec(in.dx_half.data, in.dx_half.size);
    c.dz = vec(in.dz.data, in.dz.size); c.dz_half = vec(in.dz_half.data, in.dz_half.size);
    c.c1_h = in.c1_h; c.c2_h = in.c2_h; c.c3_h = in.c3_h; c.c4_h = in.c4_h;
    c.src_idx = in.src_idx; c.src_z_idx = in.src_z_idx;
    c.wavelet = vec(in.wavelet.data, in.wavelet.size);
    c.src_angle = in.src_angle; c.src_type = in.src_type; c.src_amp = in.src_amp;
    c.num_rcv = in.num_rcv; c.rcv_grid_idx = vec(in.rcv_grid_idx.data, in.rcv_grid_idx.size);
    c.upFlag = in.upFlag != 0;
    return c;
}

struct RefSession {
    GPUSimData gpu;
    SimulationContext ctx;
};

}  // namespace

extern "C" {

const char* ref2d_last_error(void) { return refMessage.c_str(); }

int ref2d_validate(const seis2d_context* c) {
    return call([&] { validateSimulationContext(toReference(*c)); });
}

int ref2d_create(void** out, const seis2d_context* c) {
    return call([&] {
        *out = nullptr;
        auto* s = new RefSession;
        try {
            s->ctx = toReference(*c);
            initializeGpuSimulation(s->gpu, s->ctx);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

void ref2d_destroy(void* h) {
    auto* s = static_cast<RefSession*>(h);
    if (!s) return;
    releaseGpuSimulation(s->gpu);
    delete s;
}

// Replaces the per-step source parameters the reference reads from the context each step.
int ref2d_set_context(void* h, const seis2d_context* c) {
    return call([&] { static_cast<RefSession*>(h)->ctx = toReference(*c); });
}

int ref2d_update_receivers(void* h, const int* idx, int count) {
    return call([&] { updateGpuReceivers(static_cast<RefSession*>(h)->gpu, vec(idx, count)); });
}

int ref2d_set_sources(void* h, const seis2d_source* sources, int count) {
    return call([&] {
        auto* s = static_cast<RefSession*>(h);
        CUDA_CHECK(cudaMemcpy(s->gpu.d_active_sources, sources, std::size_t(count) * sizeof(GPUSource),
                              cudaMemcpyHostToDevice));
    });
}

int ref2d_step(void* h, int it, int numActive) {
    return call([&] {
        auto* s = static_cast<RefSession*>(h);
        runGpuSimulationStep(s->gpu, it, s->ctx, numActive);
    });
}

// The reference time loop without a display: one runGpuSimulationStep per step and, when
// rec_vx is given, recordReceiverStepOnGpu after each (src/Seis2D/Workflow2D.inc:297-345),
// writing [r][count].
int ref2d_run(void* h, int first, int count, int numActive, int nrcv, float* rec_vx, float* rec_vz) {
    return call([&] {
        auto* s = static_cast<RefSession*>(h);
        std::vector<float> vx(std::max(nrcv, 0)), vz(std::max(nrcv, 0));
        for (int q = 0; q < count; ++q) {
            runGpuSimulationStep(s->gpu, first + q, s->ctx, numActive);
            if (rec_vx && nrcv > 0) {
                recordReceiverStepOnGpu(s->gpu, nrcv, vx.data(), vz.data());
                for (int r = 0; r < nrcv; ++r) {
                    rec_vx[std::size_t(r) * count + q] = vx[r];
                    rec_vz[std::size_t(r) * count + q] = vz[r];
                }
            }
        }
        CUDA_CHECK(cudaDeviceSynchronize());
    });
}

// Device time of `count` steps of the reference loop (no recording), CUDA events on the
// legacy stream the reference launches on.
int ref2d_time_steps(void* h, int first, int count, float* ms) {
    return call([&] {
        auto* s = static_cast<RefSession*>(h);
        cudaEvent_t a, b;
        CUDA_CHECK(cudaEventCreate(&a));
        CUDA_CHECK(cudaEventCreate(&b));
        CUDA_CHECK(cudaEventRecord(a));
        for (int q = 0; q < count; ++q) runGpuSimulationStep(s->gpu, first + q, s->ctx, -1);
        CUDA_CHECK(cudaEventRecord(b));
        CUDA_CHECK(cudaEventSynchronize(b));
        CUDA_CHECK(cudaEventElapsedTime(ms, a, b));
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    });
}

int ref2d_record(void* h, int nrcv, float* vx, float* vz) {
    return call([&] { recordReceiverStepOnGpu(static_cast<RefSession*>(h)->gpu, nrcv, vx, vz); });
}

int ref2d_wavefield(void* h, float* vz) {
    return call([&] { copyWavefieldToHost(static_cast<RefSession*>(h)->gpu, vz); });
}

// Reads one device array of the reference's GPUSimData in the seis2d_field numbering.
int ref2d_field(void* h, int which, float* out) {
    return call([&] {
        auto& g = static_cast<RefSession*>(h)->gpu;
        float* table[SEIS2D_FIELD_COUNT] = {g.d_vx_1, g.d_vx_2, g.d_vz_1, g.d_vz_2, g.d_sxx_1, g.d_sxx_2, g.d_szz_1,
                                            g.d_szz_2, g.d_sxz_1, g.d_sxz_2, g.d_vx, g.d_vz, g.d_sigmaxx,
                                            g.d_sigmazz, g.d_sigmaxz, g.d_rho, g.d_mu, g.d_lambda, g.d_lambda2mu,
                                            g.d_mu_x_flat, g.d_lambda_x_flat, g.d_lambda2mu_x_flat, g.d_mu_z_flat,
                                            g.d_rho_x_z_flat, g.d_rho_orig_flat};
        if (which < 0 || which >= SEIS2D_FIELD_COUNT || !table[which]) throw std::invalid_argument("no such field");
        CUDA_CHECK(cudaMemcpy(out, table[which], std::size_t(g.total_grid) * 4, cudaMemcpyDeviceToHost));
    });
}

int ref2d_set_field(void* h, int which, const float* in) {
    return call([&] {
        auto& g = static_cast<RefSession*>(h)->gpu;
        float* table[SEIS2D_FIELD_COUNT] = {g.d_vx_1, g.d_vx_2, g.d_vz_1, g.d_vz_2, g.d_sxx_1, g.d_sxx_2, g.d_szz_1,
                                            g.d_szz_2, g.d_sxz_1, g.d_sxz_2, g.d_vx, g.d_vz, g.d_sigmaxx,
                                            g.d_sigmazz, g.d_sigmaxz, g.d_rho, g.d_mu, g.d_lambda, g.d_lambda2mu,
                                            g.d_mu_x_flat, g.d_lambda_x_flat, g.d_lambda2mu_x_flat, g.d_mu_z_flat,
                                            g.d_rho_x_z_flat, g.d_rho_orig_flat};
        if (which < 0 || which >= SEIS2D_FIELD_COUNT || !table[which]) throw std::invalid_argument("no such field");
        CUDA_CHECK(cudaMemcpy(table[which], in, std::size_t(g.total_grid) * 4, cudaMemcpyHostToDevice));
    });
}

// generateWavefieldTextureOnGpu of the reference into a device buffer of NX * NZ uchar4.
int ref2d_wavefield_texture(void* h, void* rgba, float scale, int component) {
    return call([&] {
        generateWavefieldTextureOnGpu(static_cast<RefSession*>(h)->gpu, static_cast<uchar4*>(rgba), scale, component);
        CUDA_CHECK(cudaDeviceSynchronize());
    });
}

}  // extern "C"
