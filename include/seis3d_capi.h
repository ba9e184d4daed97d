/*
 * seis3d_capi.h - C ABI of the B200 3-D elastic velocity-stress solver.
 *
 * Every entry point replaces one free function of the SeisWave Lab solver API
 * (namespace Seis3D, cuda/Cuda_Seis3D.cuh:7-42) with the same meaning, the same
 * validation and the same error classes, expressed as plain C: POD structs,
 * pointers and sizes, an opaque session handle and an int status.
 *
 * Status codes map one-to-one onto the exception types the reference throws:
 *   SEIS3D_INVALID_ARGUMENT  <-> std::invalid_argument (rejected before any allocation)
 *   SEIS3D_LOGIC_ERROR       <-> std::logic_error      (lifecycle misuse)
 *   SEIS3D_RUNTIME_ERROR     <-> std::runtime_error    (VRAM budget, CUDA failure,
 *                                                       non-finite wavefield)
 * seis3d_last_error() returns the thread-local message of the last failure.
 *
 * Threading: a session is not thread-safe; one host thread drives it.  All work of a
 * session is enqueued on the session's own non-blocking stream and functions
 * synchronise only that stream (reference cuda/Cuda_Seis3D.cu:534,547,641,678).
 */
#ifndef SEIS3D_CAPI_H
#define SEIS3D_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SEIS3D_ABI_VERSION 1

enum seis3d_status {
    SEIS3D_OK = 0,
    SEIS3D_INVALID_ARGUMENT = 1,
    SEIS3D_LOGIC_ERROR = 2,
    SEIS3D_RUNTIME_ERROR = 3
};

/* Limits of the reference (include/Common3D.h:9-16). */
#define SEIS3D_STENCIL_RADIUS 4
#define SEIS3D_MAX_PHYSICAL_NODES 36000000ULL
#define SEIS3D_MAX_VOLUME_AXIS 256
#define SEIS3D_MAX_VOLUME_OUTPUT 1536
#define SEIS3D_MEMORY_LIMIT 4294967296ULL
#define SEIS3D_MAX_RECEIVERS 300
#define SEIS3D_MAX_SEGY_SAMPLES 32767
#define SEIS3D_MAX_SEGY_INTERVAL_US 32767

/* Field order of the nine wavefields (include/Common3D.h:18). */
enum seis3d_field { SEIS3D_VX, SEIS3D_VY, SEIS3D_VZ, SEIS3D_SXX, SEIS3D_SYY, SEIS3D_SZZ,
                    SEIS3D_SXY, SEIS3D_SYZ, SEIS3D_SXZ };
/* Procedural model ids (include/Common3D.h:20-21). */
enum seis3d_model_kind { SEIS3D_MODEL_UNIFORM, SEIS3D_MODEL_TWO_LAYER, SEIS3D_MODEL_SPHERE,
                         SEIS3D_MODEL_IMPORTED, SEIS3D_MODEL_THREE_LAYER, SEIS3D_MODEL_DIPPING_LAYER,
                         SEIS3D_MODEL_LOW_VELOCITY_LAYER, SEIS3D_MODEL_FAULT, SEIS3D_MODEL_GRADIENT,
                         SEIS3D_MODEL_SALT_DOME };
/* Source kinds (include/Common3D.h:22). */
enum seis3d_source_kind { SEIS3D_SOURCE_EXPLOSION = 0, SEIS3D_SOURCE_FORCE = 1 };

/* SimulationContext3D (include/Common3D.h:24-42); bools are ints, names keep the
 * reference's 3D suffix so host code maps field by field. */
typedef struct seis3d_context {
    int nx3D, ny3D, nz3D;
    int pml3D;
    int freeSurface3D;
    int reflecting3D;
    float spacing3D, cfl3D, dt3D;
    int manualTimeStep3D;
    float requestedDtMs3D;
    float safeDt3D;
    float vp3D, vs3D, density3D;
    float layerVp3D, layerVs3D, layerDensity3D;
    float maxVp3D, frequency3D;
    int modelKind3D;
    float interfaceDepth3D, layerDip3D, layerThickness3D;
    float faultThrow3D, anomalyRadius3D;
    int gx3D, gy3D, gz3D, ox3D, oy3D, oz3D;
    uint64_t cells3D;
} seis3d_context;

/* Source3D (include/Common3D.h:44-49). */
typedef struct seis3d_source {
    int x3D, y3D, z3D;
    int kind3D;
    float amplitude3D;
    float direction3D[3];
} seis3d_source;

/* Receiver3D (include/Common3D.h:51). */
typedef struct seis3d_receiver { int x3D, y3D, z3D; } seis3d_receiver;

/* MemoryBudget3D (include/Common3D.h:72-74). */
typedef struct seis3d_memory_budget {
    uint64_t fieldBytes3D, cpmlBytes3D, viewBytes3D, totalBytes3D;
} seis3d_memory_budget;

/* ViewLayout3D (include/Common3D.h:53-60). */
typedef struct seis3d_view_layout {
    uint64_t sliceOffset3D[3];
    int sliceWidth3D[3], sliceHeight3D[3];
    uint64_t volumeOffset3D, totalSamples3D;
    int volumeX3D, volumeY3D, volumeZ3D;
    int domainSize3D[3], domainOrigin3D[3];
} seis3d_view_layout;

/* Storage precision.  Arithmetic is FP32 in every mode.
 *   SEIS3D_STORAGE_FP32       everything in FP32 (the parity mode).
 *   SEIS3D_STORAGE_FP16/BF16  16-bit wavefields and materials: not provided (rejected by
 *                             seis3d_initialize); their receiver traces move by more than
 *                             1e-3 relative L2 against an FP64 run of the scheme.
 *   SEIS3D_STORAGE_BF16_CPML  wavefields and materials FP32, CPML memories stored in BF16
 *                             (each FP32 update is used in full; only the kept memory is
 *                             rounded, to nearest even).  Halves the memory traffic of the
 *                             CPML slabs; traces stay within 1e-3 of FP64, not within the
 *                             1e-5 parity bar.  The learned boundary needs FP32 memories. */
enum seis3d_storage {
    SEIS3D_STORAGE_FP32 = 0,
    SEIS3D_STORAGE_FP16 = 1,
    SEIS3D_STORAGE_BF16 = 2,
    SEIS3D_STORAGE_BF16_CPML = 3
};

/* Session options (no reference counterpart: the reference has one fixed kernel shape).
 * Zero-initialised options select FP32 storage and the tuned default tile. */
typedef struct seis3d_options {
    int storage;        /* enum seis3d_storage */
    int tile_y;         /* rows of the xy tile of the z-marching kernels (0 = default) */
    int z_chunk;        /* planes per CTA along z (0 = default) */
    int compact_rows;   /* 1: row pitch = gx3D, the reference's unpitched device layout
                           (cells3D contiguous floats per field); needs gx3D % 4 == 0 */
    int tune;           /* 1 (with z_chunk 0): at initialisation, time both passes on the zeroed
                           fields for z chunks 16..40 and the default choice, and keep the
                           fastest (a few tens of ms; results do not depend on the chunk) */
    int thin_cpml;      /* 1: accept a CPML of 4..7 cells (the learned-boundary mode; the
                           reference and seis3d_validate_context require 8..40) */
    int reserved[2];
} seis3d_options;

/* Device views of a session (the GPUSimData3D members of include/Common3D.h:76-93).
 * Fields and materials use the padded X-contiguous layout of the reference with a row
 * pitch rounded up to 32 elements:  index(x,y,z) = (z*gy + y)*pitch + x.  In FP16/BF16
 * storage the pointers address 2-byte elements and field_scale[] holds the per-field
 * scale (stored = physical / scale). */
typedef struct seis3d_device_views {
    void* field3D[9];
    void* inverseDensity3D;
    void* lambda3D;
    void* mu3D;
    float* cpml3D[3];               /* 2-byte BF16 elements in SEIS3D_STORAGE_BF16_CPML */
    uint64_t slabCells3D[3];
    float* coefficients3D[3];
    void* stream3D;                 /* cudaStream_t */
    int receiverCount3D;
    int storage;
    int64_t pitch;                  /* elements per row */
    int64_t plane;                  /* elements per z plane */
    float field_scale[12];          /* 9 fields, 1/rho, lambda, mu */
    uint64_t allocatedBytes3D;
    uint64_t kernelLaunches;        /* kernels enqueued by this session so far (graph nodes counted) */
} seis3d_device_views;

typedef struct seis3d_session seis3d_session;

/* ---- host-only functions (no GPU needed) ------------------------------------ */

/* Message of the last failing call on this thread ("" when none). */
const char* seis3d_last_error(void);
/* ABI version of the loaded library. */
int seis3d_abi_version(void);
/* Reference defaults of SimulationContext3D / Source3D (include/Common3D.h:24-49). */
void seis3d_default_context(seis3d_context* context);
void seis3d_default_source(seis3d_source* source);
/* validateContext3D (cuda/Cuda_Seis3D.cu:433-483): derive padding, offsets, CFL-limited
 * integer-microsecond dt; SEIS3D_INVALID_ARGUMENT on any rejected input. */
int seis3d_validate_context(seis3d_context* context);
/* estimateMemory3D (cuda/Cuda_Seis3D.cu:504-516). */
int seis3d_estimate_memory(const seis3d_context* context, seis3d_memory_budget* budget);
/* makeViewLayout3D (cuda/Cuda_Seis3D.cu:486-501). */
int seis3d_make_view_layout(const seis3d_context* context, seis3d_view_layout* layout);
/* makeCoefficients3D (cuda/Cuda_Seis3D.cu:45-64): FP64 CPML profile of one axis as FP32
 * {a, b, 1/kappa} triples, centre nodes then half-grid nodes; writes n*6 floats where
 * n = gx, gy or gz.  `capacity` is in floats. */
int seis3d_make_cpml_coefficients(const seis3d_context* context, int axis, float* values, size_t capacity);

/* ---- session lifecycle ---------------------------------------------------------- */

/* initializeGpu3D (cuda/Cuda_Seis3D.cu:519-555): validate, check the VRAM budget, allocate
 * the session on the current device, build the CPML profiles and the procedural model.
 * `options` may be NULL.  Rolls back every allocation on failure. */
int seis3d_initialize(seis3d_session** session, const seis3d_context* context,
                      const seis3d_options* options);
/* releaseGpu3D (cuda/Cuda_Seis3D.cu:558-569): idempotent, accepts NULL. */
void seis3d_release(seis3d_session* session);
/* resetGpu3D (cuda/Cuda_Seis3D.cu:572-577): clear fields, CPML memories and the
 * non-finite flag; keep model and receivers. */
int seis3d_reset(seis3d_session* session, const seis3d_context* context);
/* refreshCpmlCoefficients3D (cuda/Cuda_Seis3D.cu:580-599): transactional coefficient swap. */
int seis3d_refresh_cpml(seis3d_session* session, const seis3d_context* context);
/* runStep3D (cuda/Cuda_Seis3D.cu:602-624): enqueue one leapfrog step at time index `step`. */
int seis3d_run_step(seis3d_session* session, const seis3d_context* context,
                    const seis3d_source* source, uint64_t step);
/* Enqueue `count` consecutive steps starting at `first_step`, replayed from a CUDA graph
 * that is captured once per (source, count) and reused.  With an active gather
 * (seis3d_gather_begin) receivers are sampled on the device, in the reference's cadence
 * (src/Seis3D_Sim.cpp:127-132), with no host synchronisation.  Equivalent to `count`
 * calls of seis3d_run_step plus the sampling calls. */
int seis3d_run_steps(seis3d_session* session, const seis3d_context* context,
                     const seis3d_source* source, uint64_t first_step, int count);
/* Capture (or re-capture) the step graph that seis3d_run_steps replays for `source`, so
 * that the next seis3d_run_steps of at least one batch replays without capturing.  No
 * step is executed. */
int seis3d_prepare_steps(seis3d_session* session, const seis3d_context* context,
                         const seis3d_source* source);
/* setReceivers3D (cuda/Cuda_Seis3D.cu:649-668): validate and atomically replace. */
int seis3d_set_receivers(seis3d_session* session, const seis3d_context* context,
                         const seis3d_receiver* receivers, int count);
/* sampleReceivers3D (cuda/Cuda_Seis3D.cu:671-681): collocated [r][vx,vy,vz] into the
 * session's pinned buffer, valid until the next set_receivers/release.  *values is NULL
 * when no receivers are set.  SEIS3D_RUNTIME_ERROR when the wavefield went non-finite. */
int seis3d_sample_receivers(seis3d_session* session, const seis3d_context* context,
                            const float** values);
/* probeMaterial3D (cuda/Cuda_Seis3D.cu:684-693): {vp, vs, rho}; no-op outside the model. */
int seis3d_probe_material(seis3d_session* session, const seis3d_context* context,
                          const seis3d_receiver* point, float values[3]);
/* uploadModelPlane3D (cuda/Cuda_Seis3D.cu:696-711): one physical z plane of interleaved
 * SI vp,vs,rho ([y][x][3] floats). */
int seis3d_upload_model_plane(seis3d_session* session, const seis3d_context* context,
                              int plane, const float* values);
/* The whole model in one call from three host volumes [nz][ny][nx] of SI vp, vs, rho: the
 * same validation, materials (bit for bit) and edge extension as nz calls of
 * seis3d_upload_model_plane plus seis3d_finish_model_upload, with the conversion done on the
 * device (no reference counterpart; the reference streams planes through host staging). */
int seis3d_upload_model(seis3d_session* session, const seis3d_context* context, const float* vp,
                        const float* vs, const float* rho);
/* finishModelUpload3D (cuda/Cuda_Seis3D.cu:714-717): extend edge materials into padding. */
int seis3d_finish_model_upload(seis3d_session* session, const seis3d_context* context);
/* downloadModelPlane3D (cuda/Cuda_Seis3D.cu:720-733). */
int seis3d_download_model_plane(seis3d_session* session, const seis3d_context* context,
                                int plane, float* values);

/* ---- device-resident gather (replaces the per-sample host sync of
 *      src/Seis3D_Sim.cpp:128-132 / cuda/Cuda_Seis3D.cu:671-681) ------------------ */

/* Start recording: a sample is taken after every step whose (step+1) % stride == 0,
 * into a device buffer [sample][receiver][vx,vy,vz] of `target_samples` samples. */
int seis3d_gather_begin(seis3d_session* session, int stride, int target_samples);
/* Copy the recorded samples to `host` (capacity in floats) and report how many samples
 * were taken; SEIS3D_RUNTIME_ERROR when the wavefield went non-finite. */
int seis3d_gather_fetch(seis3d_session* session, float* host, size_t capacity, int* sample_count);
/* Stop recording (the buffer is kept until the next gather_begin or release). */
int seis3d_gather_end(seis3d_session* session);

/* ---- display views ------------------------------------------------------------------ */

/* extractViews3D (cuda/Cuda_Seis3D.cu:627-646) without a graphics stack: the three slices and
 * (volume != 0) the bounded volume of `layout` (from seis3d_make_view_layout for this context)
 * as interleaved {wave, material} floats into `output`, a device buffer of the caller holding
 * 2 floats per sample (volumeOffset3D or totalSamples3D samples).  component 0..7 = vz, vx,
 * vy, |v|, pressure, vp, vs, rho; material_component 5..7.  Returns the largest |value| (and
 * |v|) over the physical cells, or over the visible CPML too with include_boundary, and the
 * physical material range.  SEIS3D_INVALID_ARGUMENT for bad parameters or an output range that
 * is not inside one device allocation; SEIS3D_RUNTIME_ERROR when the wavefield is non-finite. */
int seis3d_extract_views(seis3d_session* session, const seis3d_context* context, float* output,
                         const seis3d_view_layout* layout, const int slices[3], int component,
                         int material_component, int volume, int include_boundary, float* maximum,
                         float material_range[2], float* velocity_maximum);

/* ---- display shading: the workspace's slice and volume shaders as CUDA kernels -------- */
/* Both shading calls are enqueued on the session stream and return without waiting: the
 * output is ready after seis3d_synchronize (or any later call that synchronises the
 * session), and buffers written on other streams must be complete before the call. */

/* Uniforms of the shared transfer function (shaders/seis3d_transfer.glsl:1-5, set by
 * src/Seis3D/Renderer3D.cpp:148-160).  palette3D = the five stops of the wave style. */
typedef struct seis3d_transfer {
    float palette3D[5][3];
    int displayMode3D, modelStyle3D, unsignedWave3D;
    float materialRange3D[2];
    float waveOpacity3D, waveThreshold3D, modelOpacity3D;
    float waveGamma3D, materialBrightness3D;
} seis3d_transfer;

/* Uniforms of the raymarched volume (shaders/seis3d_volume.frag:4-12, set by
 * src/Seis3D/Renderer3D.cpp:236-267).  Axes of extent3D are display x, up (model z) and
 * depth (model y); domain and physical bounds are normalised texture coordinates. */
typedef struct seis3d_volume_view {
    float extent3D[3];
    float pan3D[2];
    float domainLow3D[3], domainHigh3D[3], physicalLow3D[3], physicalHigh3D[3];
    int showBoundary3D;
    float boundaryOpacity3D;
    float yaw3D, pitch3D, distance3D, scale3D, gain3D, opacity3D, threshold3D;
    float aspect3D, sampling3D, sharpness3D;
    float volumeGain3D, opticalScale3D;
} seis3d_volume_view;

/* The display settings of the workspace (Seis3D_State, include/Seis3D_Sim.h:110-160, with
 * its defaults from seis3d_default_display) from which the renderer derives the uniforms.
 * scale3D is displayScale3D() of that state (include/Seis3D_Sim.h:189-192): the auto-scaled
 * or held-peak maximum, or the manual scale. */
typedef struct seis3d_display {
    int displayMode3D, waveStyle3D, modelStyle3D, component3D;
    int materialRangeAuto3D;
    float materialRange3D[2], manualMaterialRange3D[2];
    float waveOpacity3D, waveThreshold3D, modelOpacity3D, waveGamma3D, materialBrightness3D;
    float gain3D, scale3D;
    int showBoundary3D;
    float boundaryOpacity3D;
    float yaw3D, pitch3D, distance3D, pan3D[2];
    float volumeOpacity3D, volumeThreshold3D, volumeSampling3D, volumeSharpness3D, volumeGain3D;
    int volumeSizeCompensation3D;
    int volumeRequestedWidth3D, volumeRequestedHeight3D;
} seis3d_display;

/* Pixel formats of the shaded outputs: RGBA8 is the GL_RGBA8 render target (each channel
 * clamped to [0, 1] and rounded to the nearest of 255 steps); RGBA32F keeps the FP32 colour. */
enum seis3d_pixel_format { SEIS3D_PIXELS_RGBA8 = 0, SEIS3D_PIXELS_RGBA32F = 1 };

/* The workspace defaults of the display settings (include/Seis3D_Sim.h:110-160, camera
 * :25-28). */
void seis3d_default_display(seis3d_display* display);
/* wavePalette (Main_header/WavePalettes.h:9-29): the five stops of wave style 0..13 (clamped). */
void seis3d_wave_palette(int style, float stops[5][3]);
/* The uniforms that Renderer3D derives from the display settings for this context and layout
 * (src/Seis3D/Renderer3D.cpp:148-160, 211, 224-267), and the volume target size (requested
 * size clamped to 1..SEIS3D_MAX_VOLUME_OUTPUT).  Host arithmetic only. */
int seis3d_make_display_uniforms(const seis3d_context* context, const seis3d_view_layout* layout,
                                 const seis3d_display* display, seis3d_transfer* transfer,
                                 seis3d_volume_view* volume, int* width, int* height);
/* The slice shader (shaders/seis3d_slice.frag:9-20) over the three slices of `views` (the
 * device buffer filled by seis3d_extract_views for `layout`).  The full-screen pass samples
 * each slice texture at its texel centres, so pixel k of slice p is the shading of view
 * sample sliceOffset3D[p] + k: `output` (device) receives volumeOffset3D pixels in the view
 * order, 4 bytes (RGBA8) or 16 bytes (RGBA32F) each.  scale and gain are the shader's
 * scale3D and gain3D. */
int seis3d_shade_slices(seis3d_session* session, const seis3d_view_layout* layout, const float* views,
                        const seis3d_transfer* transfer, float scale, float gain, int format, void* output);
/* The volume shader (shaders/seis3d_volume.frag:15-83): one ray per pixel of a width x height
 * target through the bounded volume of `views` (trilinear, clamp-to-edge texture sampling in
 * FP32), front-to-back compositing with the shader's early exit, and the box and CPML-layer
 * outlines.  `output` (device) receives width * height pixels, row 0 at the bottom as in the
 * GL framebuffer.  1 <= width, height <= SEIS3D_MAX_VOLUME_OUTPUT. */
int seis3d_render_volume(seis3d_session* session, const seis3d_view_layout* layout, const float* views,
                         const seis3d_transfer* transfer, const seis3d_volume_view* volume, int width,
                         int height, int format, void* output);

/* ---- batched shots (no reference counterpart) ----------------------------------------- */

/* Many shots, each a session on its own grid (e.g. a cropped window of a large model), stepped
 * together on one device: one CUDA graph replay per 64 steps holds every shot's step chain as an
 * independent branch, so CTAs of several shots share the SMs.  Each shot runs exactly the
 * launches of seis3d_run_steps: its fields, receivers and device gather are bit-identical to a
 * solo run.  The sessions stay owned by the caller and must outlive the batch; calls on a
 * session after seis3d_batch_run_steps are ordered after the batch's work. */
#define SEIS3D_MAX_BATCH_SHOTS 64

typedef struct seis3d_batch seis3d_batch;

typedef struct seis3d_batch_options {
    int shots_per_launch;   /* shots whose branches run concurrently (0 = all of them) */
    int z_chunk;            /* planes per CTA for every shot (0 = each session's choice) */
    int tune;               /* 1: on the first run long enough, time the candidates of the
                               z chunk (session choice, 16, 24, 32, 48) and of the shots per
                               launch (all, 1, half) that are not fixed above, two steps each
                               after one warm-up replay, and keep the fastest */
    int reserved[5];
} seis3d_batch_options;

typedef struct seis3d_batch_info {
    int shots, shots_per_launch, z_chunk, tuned, candidates;
    float tuned_ms_per_step;    /* device time of one step of all shots with the chosen pair */
    uint64_t kernel_launches;   /* kernels the batch has enqueued (graph nodes counted) */
    void* stream;               /* cudaStream_t the batch graph is replayed on */
} seis3d_batch_info;

/* `sessions[0..count)` (1 <= count <= SEIS3D_MAX_BATCH_SHOTS, distinct, one device). */
int seis3d_batch_create(seis3d_batch** batch, seis3d_session* const* sessions, int count,
                        const seis3d_batch_options* options);
/* `count` steps first .. first+count-1 of every shot, shot i firing sources[i] (validated like
 * seis3d_run_step).  Asynchronous: returns once the work is enqueued. */
int seis3d_batch_run_steps(seis3d_batch* batch, const seis3d_source* sources, uint64_t first, int count);
/* Waits for the batch and its sessions; SEIS3D_RUNTIME_ERROR when a wavefield went non-finite. */
int seis3d_batch_synchronize(seis3d_batch* batch);
int seis3d_batch_get_info(seis3d_batch* batch, seis3d_batch_info* info);
/* Waits for the batch's work and frees it (not the sessions); NULL is a no-op. */
void seis3d_batch_release(seis3d_batch* batch);

/* ---- checkpoints (no reference counterpart) ------------------------------------------- */

/* The state a run continues from: the nine wavefields (ghosts and CPML cells included), the
 * CPML memories and the step clock, in an unpitched little-endian layout behind a 72-byte
 * header that names the grid.  Materials (part of the model) and the device gather (fetch it
 * first) are not included.  A checkpoint restores into any session of the same grid,
 * boundary and storage mode (the memories are BF16 in SEIS3D_STORAGE_BF16_CPML), with either
 * row layout; the restored session continues bit-identically. */
int seis3d_checkpoint_bytes(seis3d_session* session, uint64_t* bytes);
/* Writes the checkpoint to a host buffer of at least seis3d_checkpoint_bytes bytes.
 * SEIS3D_RUNTIME_ERROR if the wavefield is non-finite. */
int seis3d_save_checkpoint(seis3d_session* session, void* host, uint64_t capacity);
/* Restores a checkpoint (SEIS3D_INVALID_ARGUMENT: another grid or storage mode, bad magic, truncated;
 * SEIS3D_LOGIC_ERROR: a gather is active). */
int seis3d_load_checkpoint(seis3d_session* session, const void* host, uint64_t bytes);
/* The same through a file: written to `path`.part and renamed, read completely before the
 * session is touched. */
int seis3d_write_checkpoint(seis3d_session* session, const char* path);
int seis3d_read_checkpoint(seis3d_session* session, const char* path);

/* ---- files: .s3dm models and SEG-Y rev1 gathers ---------------------------------------- */

/* Survey3D (include/Seis3D_Sim.h:36-45): receiver mesh and shot spread in physical cells. */
typedef struct seis3d_survey {
    int receiverCountX3D, receiverCountY3D;
    int receiverOrigin3D[3];
    int receiverSpacing3D[2];
    int shotCountX3D, shotCountY3D;
    int shotOrigin3D[3];
    int shotSpacing3D[2];
    double worldOrigin3D[2];
    float cmpBinSize3D[2];
} seis3d_survey;

/* Gather3D (include/Seis3D_Sim.h:47-57) with its receiver and sample vectors as views;
 * samples3D is [sample][receiver][vx, vy, vz] (the device gather's layout). */
typedef struct seis3d_gather_record {
    seis3d_context context3D;
    seis3d_source source3D;
    seis3d_survey survey3D;
    const seis3d_receiver* receivers3D;
    int receiverCount3D;
    const float* samples3D;
    int sampleCount3D, targetSamples3D, stride3D, shotId3D;
    int sampleIntervalUs3D;
    int coordinateScalar3D;
    double firstSampleTime3D;
} seis3d_gather_record;

void seis3d_default_survey(seis3d_survey* survey);
/* The metadata and checks of startGather3D (src/Seis3D/Acquisition3D.cpp:188-230): fills
 * sampleIntervalUs3D, firstSampleTime3D = (stride - 1/2) dt and coordinateScalar3D. */
int seis3d_freeze_gather(seis3d_gather_record* gather);
/* cmpBin3D (src/Seis3D/Acquisition3D.cpp:64-73): one-based inline (y) / crossline (x) bins. */
int seis3d_cmp_bin(const seis3d_gather_record* gather, const seis3d_receiver* receiver, int* inline_bin,
                   int* crossline_bin);
/* writeSegyComponent3D (src/Seis3D/Acquisition3D.cpp:76-153): component 0 vx, 1 vy, 2 vz. */
int seis3d_write_segy_component(const seis3d_gather_record* gather, const char* path, int component);
/* exportGather3D (src/Seis3D/Acquisition3D.cpp:156-185): three SEG-Y files and the geometry CSV. */
int seis3d_export_gather(const seis3d_gather_record* gather, const char* directory, const char* prefix);
/* inspectModel3D (src/Seis3D/ModelIo3D.cpp:35-65): validates a .s3dm file and returns the
 * imported context (dimensions, CPML, boundary, spacing and maxVp3D from the file; the other
 * settings from *context). */
int seis3d_inspect_model(const char* path, seis3d_context* context);
/* One [y][x][vp, vs, rho] plane of an inspected .s3dm file. */
int seis3d_read_model_plane(const char* path, const seis3d_context* context, int plane, float* values);
/* importModel3D (src/Seis3D/ModelIo3D.cpp:68-77): plane-by-plane upload + edge extension. */
int seis3d_import_model(seis3d_session* session, const seis3d_context* context, const char* path);
/* exportModel3D (src/Seis3D/ModelIo3D.cpp:80-102): the session's model into a new file. */
int seis3d_export_model(seis3d_session* session, const seis3d_context* context, const char* path);
/* A new .s3dm file from host planes (nz x ny x nx x 3 floats); no reference counterpart
 * (the reference writes only from its GPU session), used to produce model inputs. */
int seis3d_write_model(const char* path, const seis3d_context* context, const float* values);

/* ---- inspection -------------------------------------------------------------------- */

/* Device pointers and layout of the session (GPUSimData3D members). */
int seis3d_get_views(seis3d_session* session, seis3d_device_views* views);
/* The session's z chunk setting (0: the default choice; the tuned value after options.tune)
 * and the planes per CTA its step kernels run with. */
int seis3d_get_z_chunk(seis3d_session* session, int* setting, int* planes);
/* Copy one whole padded field (0-8 wavefields, 9 = 1/rho, 10 = lambda, 11 = mu) between
 * the device and a host array in the reference's unpitched layout (z*gy + y)*gx + x,
 * converting from/to FP32.  direction 0 = device->host, 1 = host->device. */
int seis3d_copy_field(seis3d_session* session, int field, int direction, float* host);
/* Device time of each launch class over `count` steps run without a graph, measured with
 * CUDA events on the session stream (the reference's computeMs3D event pair,
 * src/Seis3D_Sim.cpp:122,150-152, split per pass):  ms[0] velocity pass, ms[1] stress
 * pass, ms[2] boundary images + step tail, ms[3] whole steps. */
int seis3d_profile_steps(seis3d_session* session, const seis3d_context* context,
                         const seis3d_source* source, uint64_t first_step, int count, float ms[4]);
/* Wait for the session stream. */
int seis3d_synchronize(seis3d_session* session);
/* Test hook (host-side fault injection): with nth > 0 the nth device or pinned allocation made
 * by the library from now on fails as out of memory (SEIS3D_RUNTIME_ERROR, with the call's
 * rollback); 0 disarms it.  Process-wide; meant for tests of the rollback paths. */
void seis3d_debug_fail_allocation(int nth);
/* ---- learned thin boundary (no reference counterpart) ---------------------------------
 * A session with a thin CPML (seis3d_options.thin_cpml, 4..7 cells) plus one small network per
 * CPML face that corrects, after every step, the four interior cells next to the layer on every
 * boundary column, so that the interior evolves as it would beside a wide layer.  Each network
 * is an MLP 256 -> 64 -> 64 -> 36 (ReLU) with BF16 weights on the tensor cores and FP32
 * accumulation; its inputs are the 8-cell stencil of the nine fields along the face normal (4
 * interior, 4 CPML cells), its two lateral central differences and the six CPML memories of the
 * face's axis on the 4 CPML cells (times the spacing), divided by the column's RMS amplitude,
 * plus five scheme numbers (local P and S Courant numbers, maximum Courant number,
 * frequency x dt, 1); its outputs are the 36 corrections (9 fields x 4 cells) divided by the
 * same amplitude and a per-face output scale.  Stresses (and stress-derivative memories) enter
 * and leave divided by the column's P impedance.  Faces: 0 x-, 1 x+, 2 y-, 3 y+, 4 z- (absent with a free surface), 5 z+.
 *
 * Training data come from the solver itself: a thin session and a session of the same model
 * with a 40-cell CPML are stepped in lock step; after each step seis3d_boundary_collect records
 * rows (inputs from the thin session, targets = wide minus thin on the corrected cells) and
 * resets the thin session's interior to the wide one's.  seis3d_boundary_train runs Adam on
 * the device (hand-written forward and backward kernels).  A cell within 4 cells of two faces
 * is corrected by the nearer face only (ties: the lower face index). */
#define SEIS3D_BOUNDARY_PARAMETERS 23728   /* FP32 parameters per face: W1[64][256], W2[64][64],
                                              W3[48][64] (rows 36..47 zero), b1[64], b2[64], b3[48] */
typedef struct seis3d_boundary_net seis3d_boundary_net;
typedef struct seis3d_boundary_dataset seis3d_boundary_dataset;
/* validateContext3D with the thin layers of this mode allowed (CPML 4..40 cells). */
int seis3d_validate_thin_context(seis3d_context* context);
/* Networks for a CPML of `pml` cells, He-initialised from `seed` (last layer zero, so an
 * untrained network corrects nothing), on the current device. */
int seis3d_boundary_net_create(seis3d_boundary_net** out, int pml, uint64_t seed);
void seis3d_boundary_net_release(seis3d_boundary_net* net);
/* FP32 parameters of one face (SEIS3D_BOUNDARY_PARAMETERS floats) and its output scale. */
int seis3d_boundary_net_get(seis3d_boundary_net* net, int face, float* params, float* out_scale);
int seis3d_boundary_net_set(seis3d_boundary_net* net, int face, const float* params, float out_scale);
/* Device dataset of up to rows_per_face rows per face (664 bytes a row). */
int seis3d_boundary_dataset_create(seis3d_boundary_dataset** out, uint64_t rows_per_face);
void seis3d_boundary_dataset_release(seis3d_boundary_dataset* dataset);
/* Rows per face recorded so far (capped at the capacity). */
int seis3d_boundary_dataset_rows(seis3d_boundary_dataset* dataset, uint64_t rows[6]);
/* Rows first..first+count-1 of one face: inputs (count x 256, the stored BF16 values as FP32),
 * targets (count x 36, normalised by the row's amplitude) and amplitudes s (count).  Rows are
 * in no particular order (columns are appended by concurrent threads). */
int seis3d_boundary_dataset_read(seis3d_boundary_dataset* dataset, int face, uint64_t first, uint64_t count,
                                 float* inputs, float* targets, float* amplitudes);
/* Starts a new training model: later rows are weighted by (s / max s of their model)^2. */
int seis3d_boundary_begin_model(seis3d_boundary_dataset* dataset);
/* After both sessions took the same step: records a `fraction` of the thin session's boundary
 * columns (chosen by a hash of `seed` and the column), then copies the wide session's interior
 * into the thin one.  Both sessions must hold the same physical model, spacing, dt, frequency
 * and free-surface setting; the wide one may have any CPML. */
int seis3d_boundary_collect(seis3d_session* thin, seis3d_session* wide, seis3d_boundary_dataset* dataset,
                            float fraction, uint64_t seed);
/* `iterations` Adam steps (learning rate lr) on batches of `batch` rows of one face drawn with
 * replacement; the first call on a face sets its output scale from the dataset.  loss receives
 * the weighted mean squared error of the last batch (normalised units). */
int seis3d_boundary_train(seis3d_boundary_net* net, seis3d_boundary_dataset* dataset, int face, int iterations,
                          int batch, float lr, uint64_t seed, float* loss);
/* One forward and backward pass of face `face` on `rows` given rows (inputs rows x 256 FP32,
 * rounded to BF16 as the dataset stores them; targets rows x 36 in normalised units; weights
 * rows): the parameter gradient (SEIS3D_BOUNDARY_PARAMETERS floats) of
 * sum_rows w (y - t / out_scale)^2 and that sum.  For checks against a CPU restatement. */
int seis3d_boundary_gradients(seis3d_boundary_net* net, int face, const float* inputs, const float* targets,
                              const float* weights, int rows, float* gradient, float* loss);
/* Applies `net` after every step of `session` with the corrections scaled by `gain`
 * (NULL detaches).  The session's CPML must have the network's thickness. */
int seis3d_boundary_attach(seis3d_session* session, seis3d_boundary_net* net, float gain);

/* Test hook of the bounded stage waits (no reference counterpart).  Every wait of the
 * z-marching passes on a TMA stage gives up after `cycles` SM cycles (0 restores the default,
 * about two seconds), and with withheld_stage >= 0 each CTA never issues the copies of that
 * plane of its z chunk, so the wait for it runs out: the CTA records a staging stall, waits
 * (bounded) for the copies it did issue and exits, and the next synchronising call fails with
 * SEIS3D_RUNTIME_ERROR.  -1 withholds nothing.  Meant for tests of the failure path only: the
 * session's results are invalid once a stall has been recorded. */
int seis3d_debug_stage_wait(seis3d_session* session, long long cycles, int withheld_stage);
/* Read and clear nothing: 1 when a non-finite value was seen since the last reset. */
int seis3d_non_finite(seis3d_session* session, int* flag);

/* ---- sampling without allocation --------------------------------------------------- */

/* No counterpart in the reference.  For callers that cannot allocate device memory while
 * they run (a host whose device memory all belongs to its own pool allocator, a loop in
 * which an allocation or the synchronisation it may imply is not allowed, a plugin that
 * is only lent another owner's wavefield buffers): collocated [vx, vy, vz] of up to
 * SEIS3D_NOALLOC_MAX_RECEIVERS receivers read from caller-owned velocity fields
 * (device pointers, padded layout index = (z*gy + y)*pitch + x of the validated
 * `context`) into the host array `values` ([count][3] floats), on `stream`
 * (a cudaStream_t, NULL = legacy default stream), which the call synchronises.
 * The only device scratch is a fixed 8,400-byte static array that every GPU loading the
 * library holds until exit; the call makes no cudaMalloc, cudaFree or other allocating
 * call.  The first call on a device looks up that array's device address (issue it before
 * any stream capture).  All calls share the array, so calls that overlap on the GPU
 * (different streams or threads) race; serialise them.  More receivers than the maximum,
 * a receiver outside the physical model, or a context whose offsets (each at least 1) and
 * physical sizes do not fit its padded grid is SEIS3D_INVALID_ARGUMENT; the message is in
 * seis3d_noalloc_last_error(). */
#define SEIS3D_NOALLOC_MAX_RECEIVERS 300
int seis3d_sample_receivers_noalloc(const seis3d_context* context, const float* vx, const float* vy,
                                    const float* vz, int64_t pitch, const seis3d_receiver* receivers,
                                    int count, float* values, void* stream);
const char* seis3d_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SEIS3D_CAPI_H */
