/*
 * seis2d_capi.h - C ABI of the B200 2-D P-SV velocity-stress solver.
 *
 * Each entry point replaces one function of the reference's 2-D GPU solver interface
 * (CUDA_Kernels/Cuda_Check.cuh:126-149) or of the host set-up numerics it depends on
 * (Main_header/SolverNumerics.h, src/Seis2D/Numerics2D.inc), with the same meaning, the
 * same validation and the same error classes, expressed as plain C.
 *
 * The reference passes a host struct of std::vector (SimulationContext,
 * Main_header/Common.h:259-287); here every vector is a pointer + element count view so
 * the length checks of validateSimulationContext (Cuda_Check.cu:841-884) still apply.
 *
 * Status codes map one-to-one onto the exception types the reference throws:
 *   SEIS2D_INVALID_ARGUMENT <-> std::invalid_argument
 *   SEIS2D_LOGIC_ERROR      <-> std::logic_error
 *   SEIS2D_RUNTIME_ERROR    <-> std::runtime_error (CUDA failure, CUDA_CHECK)
 *   SEIS2D_OVERFLOW_ERROR   <-> std::overflow_error (index capacity, SolverNumerics.h:27-29)
 * seis2d_last_error() returns the thread-local message of the last failure.
 *
 * Threading: a session is not thread-safe.  All device work of a session runs on the
 * session's own non-blocking stream (the reference uses the legacy default stream,
 * Cuda_Check.cu:1039-1083); every function that returns host data synchronises that stream.
 */
#ifndef SEIS2D_CAPI_H
#define SEIS2D_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SEIS2D_ABI_VERSION 1

enum seis2d_status {
    SEIS2D_OK = 0,
    SEIS2D_INVALID_ARGUMENT = 1,
    SEIS2D_LOGIC_ERROR = 2,
    SEIS2D_RUNTIME_ERROR = 3,
    SEIS2D_OVERFLOW_ERROR = 4
};

/* Limits and constants of Main_header/SolverNumerics.h:9-12. */
#define SEIS2D_STENCIL_RADIUS 4
#define SEIS2D_MAX_ACTIVE_SOURCES 200
#define SEIS2D_SOURCE_INJECTION_SCALE 1e7f

/* Solver schemes (SimulationContext::flag_type, Common.h:265). */
enum seis2d_scheme { SEIS2D_SPLIT_PML = 1, SEIS2D_HYBRID_PML = 2, SEIS2D_FREE_SURFACE = 3 };
/* Source types (GPUSimData::src_type, Cuda_Check.cuh:119; applyPointSource, Cuda_Check.cu:567-634). */
enum seis2d_source_type { SEIS2D_VERTICAL_FORCE = 0, SEIS2D_HORIZONTAL_FORCE = 1, SEIS2D_EXPLOSIVE = 2,
                          SEIS2D_SHEAR = 3, SEIS2D_ROTATED_FORCE = 4 };

/* Device fields addressable through seis2d_copy_field / seis2d_set_field, named after the
 * GPUSimData members (Cuda_Check.cuh:86-109).  Fields 10-14 and 19-24 exist only for the
 * hybrid scheme; dp_flat only for the free-surface scheme. */
enum seis2d_field {
    SEIS2D_VX_1 = 0, SEIS2D_VX_2, SEIS2D_VZ_1, SEIS2D_VZ_2, SEIS2D_SXX_1, SEIS2D_SXX_2,
    SEIS2D_SZZ_1, SEIS2D_SZZ_2, SEIS2D_SXZ_1, SEIS2D_SXZ_2,
    SEIS2D_VX = 10, SEIS2D_VZ, SEIS2D_SIGMAXX, SEIS2D_SIGMAZZ, SEIS2D_SIGMAXZ,
    SEIS2D_RHO = 15, SEIS2D_MU, SEIS2D_LAMBDA, SEIS2D_LAMBDA2MU,
    SEIS2D_MU_X_FLAT = 19, SEIS2D_LAMBDA_X_FLAT, SEIS2D_LAMBDA2MU_X_FLAT, SEIS2D_MU_Z_FLAT,
    SEIS2D_RHO_X_Z_FLAT, SEIS2D_RHO_ORIG_FLAT,
    SEIS2D_FIELD_COUNT = 25
};

typedef struct seis2d_float_view { const float* data; int64_t size; } seis2d_float_view;
typedef struct seis2d_int_view { const int* data; int64_t size; } seis2d_int_view;

/* SimulationContext (Main_header/Common.h:259-287) with vectors as views; upFlag is an int.
 * record_vx / record_vz are host outputs of the reference loop and are not part of the
 * solver input, so they are left out. */
typedef struct seis2d_context {
    int NX, NZ;
    int total_grid;
    float h, dt;
    int nt, npml;
    int snap_spacenum;
    int flag_type;
    seis2d_float_view rho, mu, lambda, lambda2mu;
    seis2d_float_view dp_flat;
    seis2d_float_view dx, dx_half, dz, dz_half;
    float c1_h, c2_h, c3_h, c4_h;
    int src_idx;
    int src_z_idx;
    seis2d_float_view wavelet;
    float src_angle;
    int src_type;
    float src_amp;
    int num_rcv;
    seis2d_int_view rcv_grid_idx;
    int upFlag;
} seis2d_context;

/* GPUSource (Main_header/Common.h:251-256): one entry of the multi-source array. */
typedef struct seis2d_source {
    int idx;
    float t;
    float f_peak;
    float amp;
} seis2d_source;

typedef struct seis2d_session seis2d_session;

/* Raw device pointers of a session, named as the GPUSimData members
 * (Cuda_Check.cuh:68-121).  Absent buffers are NULL.  Layout: row-major
 * [NZ][NX] float, row stride NX (the reference layout). */
typedef struct seis2d_device_views {
    int NX, NZ, total_grid;
    float dt, inv_dt;
    int flag_type, npml, fs_idx, upFlag;
    float c1_h, c2_h, c3_h, c4_h;
    float* field[SEIS2D_FIELD_COUNT];     /* indexed by enum seis2d_field */
    float* d_dx; float* d_dx_half; float* d_dz; float* d_dz_half; float* d_dp_flat;
    float* d_wavelet;                     /* wavelet * src_amp * 1e7 of the last run, per step */
    int* d_rcv_grid_idx;
    float* d_record_vx_step; float* d_record_vz_step;
    seis2d_source* d_active_sources;      /* capacity SEIS2D_MAX_ACTIVE_SOURCES */
    int receiverCapacity;
    int reserved;
    void* stream;                         /* cudaStream_t of the session */
    uint64_t kernelLaunches;              /* kernels this session has enqueued so far */
} seis2d_device_views;

const char* seis2d_last_error(void);
int seis2d_abi_version(void);

/* ---- Shared numerics (Main_header/SolverNumerics.h) ------------------------------- */
/* kStaggeredDerivativeWeights (:15-17). */
void seis2d_stencil_weights(double weights[4]);
/* kCourantLimit2d, kSafeCourant2d (:21-22). */
float seis2d_courant_limit(void);
float seis2d_safe_courant(void);
/* checkedGridElementCount (:25-34): INVALID_ARGUMENT / OVERFLOW_ERROR. */
int seis2d_checked_grid_element_count(int nx, int nz, int64_t* count);
/* validateBoundaryGeometry (:37-47). */
int seis2d_validate_boundary_geometry(int nx, int nz, int pml_width, int free_surface);
/* getReceiverSamplingStride (:50-59). */
int seis2d_receiver_sampling_stride(double time_step, double sampling_rate_hz, int* stride);

/* ---- Host set-up (src/Seis2D/Numerics2D.inc) ---------------------------------------- */
/* generateRickerWavelet (:3-14): wavelet[i] for i < nt; FP32 host arithmetic. */
int seis2d_generate_ricker(float* wavelet, int nt, float dt, float f0, float t0);
/* updatePmlDampingArrays (:36-83): fills dx, dx_half (NX) and dz, dz_half (NZ) from the
 * context's grid, npml, h and materials (max Vp), after validateBoundaryGeometry. */
int seis2d_update_pml_damping(const seis2d_context* context, float* dx, float* dx_half, float* dz,
                              float* dz_half);
/* dp_flat of setupTestContext (:124-135): traction-free modulus (l2m^2 - lambda^2)/l2m on
 * the free-surface row npml, zero where l2m <= 0. */
int seis2d_free_surface_modulus(const seis2d_context* context, float* dp_flat);

/* ---- Solver (CUDA_Kernels/Cuda_Check.cuh:126-149) ----------------------------------- */
/* validateSimulationContext (Cuda_Check.cu:841-884). */
int seis2d_validate_context(const seis2d_context* context);
/* initializeGpuSimulation (Cuda_Check.cu:887-967): validates, releases *session (like the
 * reference releases the GPUSimData it is given), then allocates; on failure *session is
 * NULL and nothing stays allocated. */
int seis2d_initialize(seis2d_session** session, const seis2d_context* context);
/* releaseGpuSimulation (Cuda_Check.cu:970-989); NULL is a no-op. */
void seis2d_release(seis2d_session* session);
/* updateGpuReceivers (Cuda_Check.cu:992-1024): all-or-nothing replacement; count 0 clears. */
int seis2d_update_receivers(seis2d_session* session, const int* indices, int count);
/* Writes the device multi-source array (the reference caller copies into
 * GPUSimData::d_active_sources directly, src/Seis2D/Workflow2D.inc:314). */
int seis2d_set_active_sources(seis2d_session* session, const seis2d_source* sources, int count);
/* runGpuSimulationStep (Cuda_Check.cu:1027-1085): one step; num_active_sources < 0 injects
 * the context's single wavelet source, >= 0 the first num_active_sources active sources as
 * stored on the device (their time is not advanced). */
int seis2d_run_step(seis2d_session* session, int current_it, const seis2d_context* context,
                    int num_active_sources);
/* count consecutive steps first_it .. first_it+count-1, equal to count calls of
 * seis2d_run_step, replayed from captured CUDA graphs of the per-step kernels (or, with
 * SEIS2D_RUN_PERSISTENT and a single source, one cooperative launch with two grid barriers
 * per step).  With num_active_sources >= 0 the active sources
 * advance by dt before each step and expire after 2.5 / f_peak, as the reference time loop
 * does on the host (src/Seis2D/Workflow2D.inc:300-318).  An open gather records the steps
 * it selects. */
int seis2d_run_steps(seis2d_session* session, int first_it, int count, const seis2d_context* context,
                     int num_active_sources);
/* copyWavefieldToHost (Cuda_Check.cu:1088-1103): host_vz[total_grid] = vz_1 + vz_2 (or vz). */
int seis2d_copy_wavefield(seis2d_session* session, float* host_vz);
/* copyReceiverRecordsFromGpu (Cuda_Check.cu:1106-1135): writes [r * nt + current_it]. */
int seis2d_copy_receiver_records(seis2d_session* session, int num_rcv, int nt, int current_it, float* host_vx,
                                 float* host_vz);
/* recordReceiverStepOnGpu (Cuda_Check.cu:1147-1169): host_vx[r], host_vz[r] of the current state. */
int seis2d_record_receiver_step(seis2d_session* session, int num_rcv, float* host_vx, float* host_vz);

/* generateWavefieldTextureOnGpu (Cuda_Check.cu:1136-1141, kernel :700-790): NX * NZ RGBA8
 * pixels of `component` (0 |v|, 1 vx, 2 vz, 3 normal stress / (lambda + 2 mu), 4 shear stress
 * / mu, 5 divergence, 6 curl) times color_scale and the component's balance factor, red for
 * positive, blue for negative, into `device_rgba` (a device buffer of the caller, 4-byte
 * aligned).  Enqueued on the session stream without waiting, like the reference's launch. */
int seis2d_wavefield_texture(seis2d_session* session, void* device_rgba, float color_scale, int component);

/* ---- Device-resident recording of seis2d_run_steps ---------------------------------- */
/* Records step `it` when (it - capture_start_step) % stride == 0 and the sample index is
 * below `samples`, after the step, exactly as the reference recording loop
 * (src/Seis2D/Workflow2D.inc:320-345) but without a host round trip per sample. */
int seis2d_gather_begin(seis2d_session* session, int capture_start_step, int stride, int samples);
/* Copies the gather as [receiver][sample] (recorded_vx / recorded_vz layout); *taken = the
 * number of samples recorded so far. */
int seis2d_gather_fetch(seis2d_session* session, float* host_vx, float* host_vz, int samples, int* taken);
int seis2d_gather_end(seis2d_session* session);

/* ---- Inspection --------------------------------------------------------------------- */
int seis2d_get_views(seis2d_session* session, seis2d_device_views* views);
int seis2d_copy_field(seis2d_session* session, int field, float* host);
int seis2d_set_field(seis2d_session* session, int field, const float* host);
/* Copies bytes between host memory and a device range that lies inside one of the
 * session's own buffers (what the reference tests do with cudaMemcpy on GPUSimData
 * pointers); other device addresses are rejected. */
int seis2d_write_device(seis2d_session* session, void* device_dst, const void* host_src, size_t bytes);
int seis2d_read_device(seis2d_session* session, void* host_dst, const void* device_src, size_t bytes);
int seis2d_synchronize(seis2d_session* session);
/* Test hook (host-side fault injection): with nth > 0 the nth device allocation made by the
 * library from now on fails as out of memory, with the call's rollback; 0 disarms it. */
void seis2d_debug_fail_allocation(int nth);
/* Test hook of the bounded grid barriers of the persistent run mode (no reference
 * counterpart).  Every barrier wait gives up after `cycles` SM cycles (0 restores the default,
 * about two seconds), and with withheld_block >= 0 that block of the cooperative launch never
 * arrives at the first barrier, so every wait runs out: the blocks leave the run and the next
 * synchronising call fails with SEIS2D_RUNTIME_ERROR.  -1 withholds nothing.  Meant for tests
 * of the failure path only. */
int seis2d_debug_barrier_wait(seis2d_session* session, long long cycles, int withheld_block);
/* Runs the session's later work on `stream` (a cudaStream_t; NULL = the legacy default
 * stream, where the reference enqueues its 2-D kernels, so plain cudaMemcpy calls of the
 * caller are ordered after the steps as they are with the reference).  The session's own
 * non-blocking stream is the default; the previous stream is synchronised first. */
int seis2d_set_stream(seis2d_session* session, void* stream);
/* How seis2d_run_steps executes single-source runs (no reference counterpart); graph replay is
 * the default (on a B200 a grid barrier costs about as much as a kernel boundary). */
enum seis2d_run_mode { SEIS2D_RUN_PERSISTENT = 0, SEIS2D_RUN_GRAPH = 1 };
int seis2d_set_run_mode(seis2d_session* session, int mode);
/* Device time of count steps replayed as in seis2d_run_steps, split into the stress and
 * velocity kernels: ms[0] = whole replay, ms[1] = stress kernels, ms[2] = velocity kernels. */
int seis2d_profile_steps(seis2d_session* session, int first_it, int count, const seis2d_context* context,
                         float ms[3]);

#ifdef __cplusplus
}
#endif

#endif
