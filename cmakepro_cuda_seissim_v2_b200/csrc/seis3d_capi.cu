// seis3d_capi.cu - host side of the B200 solver behind the C ABI of include/seis3d_capi.h.
//
// Each exported function keeps the contract of the reference free function it replaces
// (cited per function): the same validation order, the same error class, the same
// transactional rollback.  Device work is enqueued on the session's own non-blocking
// stream; step batches are captured once into a CUDA graph and replayed.
#include "../../include/seis3d_capi.h"
#include "seis3d_kernels.cuh"
#include "seis3d_views.cuh"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

using namespace seis3d;

namespace {

thread_local std::string lastError;

struct InvalidArgument : std::runtime_error { using std::runtime_error::runtime_error; };
struct LogicError : std::runtime_error { using std::runtime_error::runtime_error; };
struct RuntimeError : std::runtime_error { using std::runtime_error::runtime_error; };

void cudaCheck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw RuntimeError(std::string("Seis3D / ") + what + ": " + cudaGetErrorString(e));
}

// NVTX range around an API call (a no-op unless a profiler is attached), so that traces and
// ncu's --nvtx filters see the solver's calls by name.
struct ApiRange {
    explicit ApiRange(const char* name) { nvtxRangePushA(name); }
    ~ApiRange() { nvtxRangePop(); }
    ApiRange(const ApiRange&) = delete;
    ApiRange& operator=(const ApiRange&) = delete;
};

// Allocation seam for host-side fault injection (seis3d_debug_fail_allocation): when armed
// with n > 0, the n-th device or pinned allocation from then on reports out of memory, so
// the tests can drive every rollback path without touching the GPU's real limits.
std::atomic<int> failAllocation{0};

bool injectFailure() {
    int n = failAllocation.load();
    while (n > 0 && !failAllocation.compare_exchange_weak(n, n - 1)) {
    }
    return n == 1;
}

template <class T> cudaError_t deviceMalloc(T** p, std::size_t bytes) {
    if (injectFailure()) return cudaErrorMemoryAllocation;
    return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}

template <class T> cudaError_t hostMalloc(T** p, std::size_t bytes) {
    if (injectFailure()) return cudaErrorMemoryAllocation;
    return cudaMallocHost(reinterpret_cast<void**>(p), bytes);
}

template <class F> int guarded(F&& body) {
    try {
        body();
        return SEIS3D_OK;
    } catch (const InvalidArgument& e) {
        lastError = e.what(); return SEIS3D_INVALID_ARGUMENT;
    } catch (const LogicError& e) {
        lastError = e.what(); return SEIS3D_LOGIC_ERROR;
    } catch (const std::bad_alloc&) {
        lastError = "Seis3D: host allocation failed"; return SEIS3D_RUNTIME_ERROR;
    } catch (const std::exception& e) {
        lastError = e.what(); return SEIS3D_RUNTIME_ERROR;
    }
}

// Material admissibility (cuda/Cuda_Seis3D.cu:30-34).
bool admissible(float vp, float vs, float rho) {
    return std::isfinite(vp) && std::isfinite(vs) && std::isfinite(rho) && vp > 0 && vp <= 30000 && vs >= 0 &&
           vs < vp && vp * vp > (4.0f / 3.0f) * vs * vs && rho > 0 && rho <= 50000;
}

int activePml(const seis3d_context& c) { return c.reflecting3D ? 0 : c.pml3D; }

// Context derivation (cuda/Cuda_Seis3D.cu:433-483); throws InvalidArgument.  `minPml` is the
// reference's 8 everywhere except for the thin layers of the learned boundary (4).
void validate(seis3d_context& c, int minPml = 8) {
    if (c.reflecting3D) c.freeSurface3D = 0;
    if (c.modelKind3D < 0 || c.modelKind3D > SEIS3D_MODEL_SALT_DOME || !std::isfinite(c.interfaceDepth3D) ||
        c.interfaceDepth3D < .1f || c.interfaceDepth3D > .9f || !std::isfinite(c.layerDip3D) ||
        std::abs(c.layerDip3D) > .6f || !std::isfinite(c.layerThickness3D) || c.layerThickness3D < .03f ||
        c.layerThickness3D > .5f || !std::isfinite(c.faultThrow3D) || std::abs(c.faultThrow3D) > .4f ||
        !std::isfinite(c.anomalyRadius3D) || c.anomalyRadius3D < .05f || c.anomalyRadius3D > .4f)
        throw InvalidArgument("Seis3D: invalid procedural model geometry.");
    if (c.nx3D < 16 || c.ny3D < 16 || c.nz3D < 16)
        throw InvalidArgument("Seis3D: every physical dimension must be at least 16.");
    const std::size_t cap = SEIS3D_MAX_PHYSICAL_NODES;
    if (std::size_t(c.nx3D) > cap / std::size_t(c.ny3D) ||
        std::size_t(c.nx3D) * std::size_t(c.ny3D) > cap / std::size_t(c.nz3D))
        throw InvalidArgument("Seis3D: physical node count exceeds 300 x 300 x 400 (36,000,000).");
    if (c.pml3D < minPml || c.pml3D > 40 || !std::isfinite(c.spacing3D) || c.spacing3D <= 0 ||
        !std::isfinite(c.frequency3D) || c.frequency3D <= 0 || c.frequency3D > 10000 || !std::isfinite(c.cfl3D) ||
        c.cfl3D <= 0 || c.cfl3D > 0.9f)
        throw InvalidArgument("Seis3D: invalid CPML, spacing, frequency or CFL safety factor.");
    if (!admissible(c.vp3D, c.vs3D, c.density3D) || !admissible(c.layerVp3D, c.layerVs3D, c.layerDensity3D))
        throw InvalidArgument("Seis3D: Vp/Vs/rho must be finite with positive bulk modulus.");
    if (c.modelKind3D != SEIS3D_MODEL_IMPORTED)
        c.maxVp3D = c.modelKind3D == SEIS3D_MODEL_UNIFORM ? c.vp3D : std::max(c.vp3D, c.layerVp3D);
    if (!std::isfinite(c.maxVp3D) || c.maxVp3D <= 0 || c.maxVp3D > 30000)
        throw InvalidArgument("Seis3D: invalid model maximum Vp.");
    const int p = activePml(c);
    c.ox3D = c.oy3D = p + 4;
    c.oz3D = c.freeSurface3D ? 4 : p + 4;
    c.gx3D = c.nx3D + 2 * p + 8;
    c.gy3D = c.ny3D + 2 * p + 8;
    c.gz3D = c.nz3D + (c.freeSurface3D ? 1 : 2) * p + 8;
    c.cells3D = uint64_t(c.gx3D) * c.gy3D * c.gz3D;
    const double sumWeights = 1225.0 / 1024 + 245.0 / 3072 + 49.0 / 5120 + 5.0 / 7168;
    const double safeDt = c.cfl3D * c.spacing3D / (std::sqrt(3.0) * c.maxVp3D * sumWeights);
    const double microseconds = std::floor(safeDt * 1.0e6);
    if (microseconds < 1 || microseconds > 65535)
        throw InvalidArgument("Seis3D: safe dt is outside the implemented 1..65535 microsecond range.");
    c.safeDt3D = float(microseconds * 1.0e-6);
    c.dt3D = c.safeDt3D;
    if (c.manualTimeStep3D) {
        const double requested = double(c.requestedDtMs3D) * 1000;
        const double rounded = std::round(requested);
        if (!std::isfinite(requested) || rounded < 1 || rounded > 65535)
            throw InvalidArgument("Seis3D: manual dt must be between 0.001 and 65.535 ms.");
        if (std::abs(requested - rounded) > 0.05)
            throw InvalidArgument("Seis3D: manual dt must use whole microseconds (0.001 ms increments).");
        if (rounded > microseconds)
            throw InvalidArgument("Seis3D: manual dt exceeds the model CFL ceiling; reduce dt or select Automatic CFL.");
        c.dt3D = float(rounded * 1.0e-6);
    }
}

// Display layout (cuda/Cuda_Seis3D.cu:486-501); part of the memory budget.
seis3d_view_layout viewLayout(const seis3d_context& c) {
    seis3d_view_layout l{};
    const int p = activePml(c);
    const int nx = c.nx3D + 2 * p, ny = c.ny3D + 2 * p, nz = c.nz3D + (c.freeSurface3D ? 1 : 2) * p;
    l.domainSize3D[0] = nx; l.domainSize3D[1] = ny; l.domainSize3D[2] = nz;
    l.domainOrigin3D[0] = -p; l.domainOrigin3D[1] = -p; l.domainOrigin3D[2] = c.freeSurface3D ? 0 : -p;
    l.sliceWidth3D[0] = nx; l.sliceHeight3D[0] = nz;
    l.sliceWidth3D[1] = ny; l.sliceHeight3D[1] = nz;
    l.sliceWidth3D[2] = nx; l.sliceHeight3D[2] = ny;
    l.sliceOffset3D[1] = uint64_t(nx) * nz;
    l.sliceOffset3D[2] = l.sliceOffset3D[1] + uint64_t(ny) * nz;
    l.volumeOffset3D = l.sliceOffset3D[2] + uint64_t(nx) * ny;
    l.volumeX3D = std::min(SEIS3D_MAX_VOLUME_AXIS, nx);
    l.volumeY3D = std::min(SEIS3D_MAX_VOLUME_AXIS, ny);
    l.volumeZ3D = std::min(SEIS3D_MAX_VOLUME_AXIS, nz);
    l.totalSamples3D = l.volumeOffset3D + uint64_t(l.volumeX3D) * l.volumeY3D * l.volumeZ3D;
    return l;
}

// Reference slab cell count per axis (cuda/Cuda_Seis3D.cu:37-42); used for the budget.
uint64_t referenceSlabCells(const seis3d_context& c, int axis) {
    if (c.reflecting3D) return 0;
    if (axis == 0) return uint64_t(2 * c.pml3D) * c.gy3D * c.gz3D;
    if (axis == 1) return uint64_t(2 * c.pml3D) * c.gx3D * c.gz3D;
    return uint64_t((c.freeSurface3D ? 1 : 2) * c.pml3D) * c.gx3D * c.gy3D;
}

// Memory budget (cuda/Cuda_Seis3D.cu:504-516).
seis3d_memory_budget budget(const seis3d_context& context, int minPml = 8) {
    seis3d_context c = context;
    validate(c, minPml);
    seis3d_memory_budget b{};
    b.fieldBytes3D = c.cells3D * 12 * sizeof(float);
    for (int a = 0; a < 3; ++a) b.cpmlBytes3D += referenceSlabCells(c, a) * 6 * sizeof(float);
    const auto l = viewLayout(c);
    b.viewBytes3D = l.totalSamples3D * 4 * sizeof(float) + l.volumeOffset3D * 4 +
                    uint64_t(SEIS3D_MAX_VOLUME_OUTPUT) * SEIS3D_MAX_VOLUME_OUTPUT * 4;
    b.totalBytes3D = b.fieldBytes3D + b.cpmlBytes3D + b.viewBytes3D + uint64_t(c.gx3D + c.gy3D + c.gz3D) * 6 * sizeof(float) +
                     uint64_t(SEIS3D_MAX_RECEIVERS) * (sizeof(seis3d_receiver) + 3 * sizeof(float)) + 2 * 1024 * 1024;
    return b;
}

// CPML profile of one axis in FP64, rounded to FP32 {a, b, 1/kappa} (cuda/Cuda_Seis3D.cu:45-64).
std::vector<float> coefficients(const seis3d_context& c, int axis) {
    const int n = axis == 0 ? c.gx3D : axis == 1 ? c.gy3D : c.gz3D;
    std::vector<float> v(std::size_t(n) * 6);
    const double sigmaMax = -4.0 * c.maxVp3D * std::log(1.0e-6) / (2.0 * c.pml3D * c.spacing3D);
    const bool topFree = axis == 2 && c.freeSurface3D;
    for (int half = 0; half < 2; ++half)
        for (int i = 0; i < n; ++i) {
            const double at = i + 0.5 * half;
            double d = (at - (n - kRadius - c.pml3D - 0.5)) / c.pml3D;
            if (!topFree) d = std::max(d, (kRadius + c.pml3D - 0.5 - at) / c.pml3D);
            d = std::clamp(d, 0.0, 1.0);
            const double cube = d * d * d;
            const double sigma = sigmaMax * cube, kappa = 1.0 + 2.0 * cube;
            const double alpha = d > 0 ? 3.141592653589793 * c.frequency3D * (1.0 - d) : 0.0;
            const double b = std::exp(-(sigma / kappa + alpha) * c.dt3D);
            const double a = sigma > 0 ? sigma * (b - 1.0) / (kappa * (sigma + kappa * alpha)) : 0.0;
            float* slot = v.data() + (std::size_t(half) * n + i) * 3;
            slot[0] = float(a); slot[1] = float(b); slot[2] = float(1.0 / kappa);
        }
    return v;
}

int64_t roundUp(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

}  // namespace

// --------------------------------------------------------------------------------------
// Session.
// --------------------------------------------------------------------------------------
struct seis3d_session {
    seis3d_context ctx{};
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t pitch = 0, plane = 0;
    float* pool = nullptr;          // 12 padded volumes: 9 fields, 3 materials
    std::size_t poolBytes = 0;
    float* field[9]{};
    float* invRho = nullptr;
    float* lambda = nullptr;
    float* mu = nullptr;
    float* psi[3]{};                // CPML memories (FP32, or BF16 elements in SEIS3D_STORAGE_BF16_CPML)
    std::size_t psiCount[3]{};
    int storage = SEIS3D_STORAGE_FP32;
    std::size_t psiBytes(int a) const { return psiCount[a] * (storage == SEIS3D_STORAGE_BF16_CPML ? 2 : 4); }
    float* coef[3]{};
    unsigned* status = nullptr;     // [0] non-finite flag, [1] staging stall
    unsigned* viewStats = nullptr;  // colour statistics of the view extraction (5 words)
    CUtensorMap* maps = nullptr;    // device copy of the TMA descriptor table
    Clock* clock = nullptr;
    uint64_t hostClock = std::numeric_limits<uint64_t>::max();
    // receivers
    int4* recv = nullptr;
    float* recvValues = nullptr;
    float* hostRecv = nullptr;      // pinned
    int recvCount = 0;
    // device gather
    float* gather = nullptr;
    std::size_t gatherFloats = 0;
    int gatherStride = 0, gatherTarget = 0;
    bool gatherActive = false;
    // model staging (pinned, 3 planes of nx*ny)
    float* stage = nullptr;
    // graph cache of a batch of steps
    cudaGraphExec_t graph = nullptr;
    int graphSteps = 0;
    seis3d_source graphSource{};
    bool graphGather = false;
    // launch shape
    int tileY = 8;
    int zChunk = 0;
    int smCount = 148;
    int residentCtas = 296;         // CTAs of one pass resident on the whole device
    uint64_t launches = 0;          // kernels enqueued (graph replays add their node count)
    float* uploadHost[2] = {nullptr, nullptr};   // pinned chunks of seis3d_upload_model
    cudaEvent_t uploadDone[2] = {nullptr, nullptr};
    std::size_t uploadCapacity = 0;              // cells per pinned chunk
    float* uploadRaw = nullptr;                  // device staging of seis3d_upload_model (3 volumes)
    std::size_t uploadRawCells = 0;
    uint64_t graphNodes = 0;
    std::size_t allocated = 0;
    // stage-wait bound and the withheld-stage test hook (seis3d_debug_stage_wait)
    long long waitCycles = tma::kWaitCycles;
    int withheldStage = -1;
    // learned thin boundary (seis3d_boundary_attach): network, gain, corrections scratch
    seis3d_boundary_net* net = nullptr;
    float netGain = 1.0f;
    float* netCorr = nullptr;
    std::size_t netCorrFloats = 0;

    Geometry geometry() const {
        Geometry G{};
        G.gx = ctx.gx3D; G.gy = ctx.gy3D; G.gz = ctx.gz3D;
        G.pml = ctx.pml3D; G.freeSurface = ctx.freeSurface3D; G.reflecting = ctx.reflecting3D;
        G.thick[0] = G.thick[1] = 2 * ctx.pml3D;
        G.thick[2] = (ctx.freeSurface3D ? 1 : 2) * ctx.pml3D;
        G.pitch = pitch; G.plane = plane;
        G.invH = 1.0f / ctx.spacing3D;
        const float weights[4] = {SEIS3D_W0, SEIS3D_W1, SEIS3D_W2, SEIS3D_W3};
        for (int r = 0; r < 4; ++r) G.w[r] = weights[r];
        G.w[4] = G.invH;
        G.h = ctx.spacing3D;
        G.dt = ctx.dt3D;
        G.frequency = ctx.frequency3D;
        G.ox = ctx.ox3D; G.oy = ctx.oy3D; G.oz = ctx.oz3D;
        G.nx = ctx.nx3D; G.ny = ctx.ny3D; G.nz = ctx.nz3D;
        G.waitCycles = waitCycles;
        G.withheldStage = withheldStage;
        return G;
    }
    Fields fields() const {
        Fields F{};
        for (int k = 0; k < 9; ++k) F.f[k] = field[k];
        F.invRho = invRho; F.lambda = lambda; F.mu = mu;
        for (int a = 0; a < 3; ++a) { F.psi[a] = psi[a]; F.coef[a] = coef[a]; }
        F.status = status;
        F.clock = clock;
        F.maps = maps;
        return F;
    }
    void dropGraph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        graphSteps = 0;
    }
};

namespace {

void releaseSession(seis3d_session* s) noexcept {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    s->dropGraph();
    cudaFree(s->pool);
    for (int a = 0; a < 3; ++a) { cudaFree(s->psi[a]); cudaFree(s->coef[a]); }
    cudaFree(s->status);
    cudaFree(s->viewStats);
    cudaFree(s->clock);
    cudaFree(s->maps);
    cudaFree(s->recv);
    cudaFree(s->recvValues);
    cudaFree(s->gather);
    cudaFree(s->netCorr);
    if (s->hostRecv) cudaFreeHost(s->hostRecv);
    if (s->stage) cudaFreeHost(s->stage);
    for (float* h : s->uploadHost)
        if (h) cudaFreeHost(h);
    cudaFree(s->uploadRaw);
    for (cudaEvent_t e : s->uploadDone)
        if (e) cudaEventDestroy(e);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

void requireSession(seis3d_session* s) {
    if (!s || !s->stream) throw LogicError("Seis3D: simulation not initialized.");
}

// Read the device status words; a staging stall is a runtime error.
unsigned readStatus(seis3d_session* s) {
    unsigned st[2] = {0, 0};
    cudaCheck(cudaMemcpyAsync(st, s->status, sizeof(st), cudaMemcpyDeviceToHost, s->stream), "read status");
    cudaCheck(cudaStreamSynchronize(s->stream), "read status");
    if (st[1]) throw RuntimeError("Seis3D: TMA staging pipeline stalled; results of the affected steps are invalid.");
    return st[0];
}

// The caller's context must describe the session's grid (the reference passes both).
void requireSameGrid(const seis3d_session* s, const seis3d_context* c) {
    if (!c) throw InvalidArgument("Seis3D: null context.");
    if (c->gx3D != s->ctx.gx3D || c->gy3D != s->ctx.gy3D || c->gz3D != s->ctx.gz3D || c->ox3D != s->ctx.ox3D ||
        c->oy3D != s->ctx.oy3D || c->oz3D != s->ctx.oz3D || c->freeSurface3D != s->ctx.freeSurface3D ||
        c->reflecting3D != s->ctx.reflecting3D || c->pml3D != s->ctx.pml3D)
        throw LogicError("Seis3D: context does not describe this session's grid.");
}

// Pick up time-dependent scalars of the caller's context (dt, spacing, frequency).
void adoptScalars(seis3d_session* s, const seis3d_context* c) {
    if (s->ctx.dt3D != c->dt3D || s->ctx.frequency3D != c->frequency3D || s->ctx.spacing3D != c->spacing3D) {
        s->ctx.dt3D = c->dt3D; s->ctx.frequency3D = c->frequency3D; s->ctx.spacing3D = c->spacing3D;
        s->dropGraph();
    }
}

void checkSource(const seis3d_context& c, const seis3d_source& src) {
    if (src.x3D < 1 || src.x3D >= c.nx3D - 1 || src.y3D < 1 || src.y3D >= c.ny3D - 1 || src.z3D < 2 ||
        src.z3D >= c.nz3D - 1 || !std::isfinite(src.amplitude3D))
        throw InvalidArgument("Seis3D: source must be inside the physical volume, at depth >=2.");
    for (float d : src.direction3D)
        if (!std::isfinite(d)) throw InvalidArgument("Seis3D: invalid force direction.");
}

SourceParams sourceParams(const seis3d_context& c, const seis3d_source& src) {
    SourceParams S{};
    S.gxs = src.x3D + c.ox3D; S.gys = src.y3D + c.oy3D; S.gzs = src.z3D + c.oz3D;
    S.kind = src.kind3D;
    S.amplitude = src.amplitude3D;
    for (int a = 0; a < 3; ++a) S.direction[a] = src.direction3D[a];
    return S;
}

void launchCheck(const char* what) { cudaCheck(cudaGetLastError(), what); }

constexpr std::size_t kVelocitySmem = std::size_t(tma::kStages) * VelocityStage::SIZE * sizeof(float);
constexpr std::size_t kStressSmem = std::size_t(tma::kStages) * StressStage::SIZE * sizeof(float);

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

using AddressRange = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);

// cuMemGetAddressRange through the runtime's driver entry point (no -lcuda needed).
AddressRange addressRange() {
    static AddressRange fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        cudaCheck(cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q), "driver entry point");
        if (!p || q != cudaDriverEntryPointSuccess) throw RuntimeError("Seis3D: cuMemGetAddressRange is unavailable.");
        fn = reinterpret_cast<AddressRange>(p);
    }
    return fn;
}

// True when [p, p + bytes) lies inside one device allocation of the session's device.
bool deviceRange(const seis3d_session* s, const void* p, std::size_t bytes) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if ((attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) || attr.device != s->device) return false;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (addressRange()(&base, &size, CUdeviceptr(reinterpret_cast<uintptr_t>(p))) != CUDA_SUCCESS) return false;
    const uintptr_t a = reinterpret_cast<uintptr_t>(p), b = uintptr_t(base);
    return a >= b && bytes <= size && a - b <= size - bytes;
}

EncodeTiled encoder() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        cudaCheck(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q), "driver entry point");
        if (!p || q != cudaDriverEntryPointSuccess) throw RuntimeError("Seis3D: cuTensorMapEncodeTiled is unavailable.");
        fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

// TMA descriptor table of a session (tma::MapIndex): FP32 volumes gx * gy * gz with the
// pitched row and plane strides, zero fill outside the volume.
void buildTensorMaps(seis3d_session* s);

void configureKernels() {
    static bool done = false;
    if (done) return;
    for (auto k : {velocityPass, velocityPassBf16Cpml})
        cudaCheck(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kVelocitySmem)),
                  "velocity pass shared memory");
    for (auto k : {stressPass, stressPassBf16Cpml})
        cudaCheck(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kStressSmem)),
                  "stress pass shared memory");
    done = true;
}

// The pass kernels of a session's storage mode.
using PassKernel = void (*)(Geometry, Fields, SourceParams, int);
PassKernel velocityKernel(const seis3d_session* s) {
    return s->storage == SEIS3D_STORAGE_BF16_CPML ? velocityPassBf16Cpml : velocityPass;
}
PassKernel stressKernel(const seis3d_session* s) {
    return s->storage == SEIS3D_STORAGE_BF16_CPML ? stressPassBf16Cpml : stressPass;
}

// Launch shapes of the two passes.
struct Shape { dim3 grid, block; int zChunk; };

Shape passShape(const seis3d_session* s) {
    const int nxA = s->ctx.gx3D - 8, nyA = s->ctx.gy3D - 8, nzA = s->ctx.gz3D - 8;
    const int tilesX = (nxA + kTX - 1) / kTX, tilesY = (nyA + kTY - 1) / kTY;
    const int tiles = tilesX * tilesY;
    int chunks = 1;
    if (s->zChunk > 0) {
        chunks = (nzA + s->zChunk - 1) / s->zChunk;
    } else {
        // Chunks of 18-32 planes (measured best on B200: many CTAs per SM over the run
        // keep the HBM streams spread), picking the split that fills whole waves of the
        // resident CTA slots best, with each chunk's 7-plane ring warm-up as overhead.
        const double slots = double(std::max(1, s->residentCtas));
        double best = -1.0;
        const int lo = std::max(1, nzA / 32), hi = std::max(lo, nzA / 18);
        for (int n = lo; n <= hi; ++n) {
            const double waves = tiles * double(n) / slots;
            const double fill = waves / std::ceil(waves);
            const double chunk = std::ceil(double(nzA) / n);
            const double score = fill * chunk / (chunk + 7.0);
            if (score > best + 1e-9) { best = score; chunks = n; }
        }
    }
    Shape sh;
    sh.zChunk = (nzA + chunks - 1) / chunks;
    sh.block = dim3(kTX, kWarps);
    sh.grid = dim3(tilesX, tilesY, (nzA + sh.zChunk - 1) / sh.zChunk);
    return sh;
}

// True when the passes write the free-surface images themselves: the first z chunk of each
// pass writes those of its columns before its z rings read them, which needs chunks of at
// least 4 planes (a shorter first chunk leaves ghost planes to the next chunk's rings).
bool foldedImages(const Shape& sh) { return sh.zChunk >= kRadius; }

// Slip-wall images of the velocities or the stresses, and with `surface` the free-surface
// images (in a step only when the passes do not write them, foldedImages).
void launchImages(seis3d_session* s, bool velocities, cudaStream_t stream = nullptr, bool surface = true) {
    const Geometry G = s->geometry();
    const Fields F = s->fields();
    if (!stream) stream = s->stream;
    if (s->ctx.freeSurface3D && surface) {
        const dim3 b(32, 8), g((s->ctx.gx3D - 8 + 31) / 32, (s->ctx.gy3D - 8 + 7) / 8);
        if (velocities) velocityImages<<<g, b, 0, stream>>>(G, F);
        else stressImages<<<g, b, 0, stream>>>(G, F);
        launchCheck("free-surface images");
        ++s->launches;
    }
    if (s->ctx.reflecting3D) {
        const int len[3] = {s->ctx.gx3D, s->ctx.gy3D, s->ctx.gz3D};
        for (int axis = 0; axis < 3; ++axis) {
            const dim3 b(16, 16), g((len[(axis + 1) % 3] + 15) / 16, (len[(axis + 2) % 3] + 15) / 16);
            reflectingImages<<<g, b, 0, stream>>>(G, F, axis, velocities ? 1 : 0);
            launchCheck("reflecting images");
            ++s->launches;
        }
    }
}

// One leapfrog step in the reference order (cuda/Cuda_Seis3D.cu:602-624), reading the
// step index from the device clock; `leadingImages` re-applies the start-of-step slip-wall
// stress images (idempotent after a previous step, needed after a reset or a field upload).
// The free-surface stress images are written at the start of every velocity pass, where the
// reference's step starts with stressGhostKernel3D; its step also ends with them (:621), which
// closingImages does once per API call (between the steps of a call nothing reads them).
// Optional events bracket the passes for seis3d_profile_steps.
struct PassEvents { cudaEvent_t start, afterVelocity, afterImages, afterStress, end; };

void enqueueBoundaryCorrection(seis3d_session* s, cudaStream_t stream);   // seis3d_boundary.inc

void enqueueStep(seis3d_session* s, const SourceParams& S, bool leadingImages, const PassEvents* ev = nullptr,
                 cudaStream_t stream = nullptr) {
    const Geometry G = s->geometry();
    const Fields F = s->fields();
    const Shape sh = passShape(s);
    if (!stream) stream = s->stream;
    const bool folded = foldedImages(sh);
    if (leadingImages) launchImages(s, false, stream);
    if (ev) cudaEventRecord(ev->start, stream);
    velocityKernel(s)<<<sh.grid, sh.block, kVelocitySmem, stream>>>(G, F, S, sh.zChunk);
    launchCheck("velocity pass");
    ++s->launches;
    if (ev) cudaEventRecord(ev->afterVelocity, stream);
    launchImages(s, true, stream, !folded);
    if (ev) cudaEventRecord(ev->afterImages, stream);
    stressKernel(s)<<<sh.grid, sh.block, kStressSmem, stream>>>(G, F, S, sh.zChunk);
    launchCheck("stress pass");
    ++s->launches;
    if (ev) cudaEventRecord(ev->afterStress, stream);
    launchImages(s, false, stream, !folded || s->net != nullptr);
    if (s->net) {
        // Learned thin boundary: corrections of the boundary columns after the full step (on
        // the imaged state), then the stress images again for the corrected cells.
        enqueueBoundaryCorrection(s, stream);
        launchImages(s, false, stream);
    }
    stepTail<<<1, 256, 0, stream>>>(G, F, s->recv, s->recvCount, s->gatherActive ? s->gather : nullptr);
    launchCheck("step tail");
    ++s->launches;
    if (ev) cudaEventRecord(ev->end, stream);
}

// The free-surface stress images after the last step of an API call, so that the state
// between calls is the reference's (its step ends with stressGhostKernel3D).  With the
// learned boundary every step already ends with them.
void closingImages(seis3d_session* s, cudaStream_t stream = nullptr) {
    if (!s->ctx.freeSurface3D || s->net) return;
    const dim3 b(32, 8), g((s->ctx.gx3D - 8 + 31) / 32, (s->ctx.gy3D - 8 + 7) / 8);
    stressImages<<<g, b, 0, stream ? stream : s->stream>>>(s->geometry(), s->fields());
    launchCheck("free-surface images");
    ++s->launches;
}

// Picks the z chunk of a new session by timing both passes on its zeroed fields (zero fields
// and zero-amplitude source stay zero, so nothing the session later computes is touched; the
// kernels' work does not depend on the values).  One warm-up and three timed pass pairs per
// candidate; the session keeps the fastest.
void tuneZChunk(seis3d_session* s) {
    const int candidates[] = {0, 16, 20, 24, 28, 32, 40};
    SourceParams S{};
    S.gxs = s->ctx.gx3D / 2; S.gys = s->ctx.gy3D / 2; S.gzs = s->ctx.gz3D / 2;
    S.kind = 0; S.amplitude = 0.0f;
    const Geometry G = s->geometry();
    const Fields F = s->fields();
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaCheck(cudaEventCreate(&t0), "tuner event");
    cudaCheck(cudaEventCreate(&t1), "tuner event");
    float best = std::numeric_limits<float>::max();
    int chosen = 0;
    try {
        for (int z : candidates) {
            s->zChunk = z;
            const Shape sh = passShape(s);
            auto pair = [&] {
                velocityKernel(s)<<<sh.grid, sh.block, kVelocitySmem, s->stream>>>(G, F, S, sh.zChunk);
                stressKernel(s)<<<sh.grid, sh.block, kStressSmem, s->stream>>>(G, F, S, sh.zChunk);
                launchCheck("z chunk tuning");
                s->launches += 2;
            };
            pair();
            cudaCheck(cudaEventRecord(t0, s->stream), "tuner event");
            for (int k = 0; k < 3; ++k) pair();
            cudaCheck(cudaEventRecord(t1, s->stream), "tuner event");
            cudaCheck(cudaEventSynchronize(t1), "tuner wait");
            float ms = 0.0f;
            cudaCheck(cudaEventElapsedTime(&ms, t0, t1), "tuner time");
            if (ms < best) { best = ms; chosen = z; }
        }
    } catch (...) {
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        throw;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    s->zChunk = chosen;
    if (readStatus(s)) throw RuntimeError("Seis3D: z chunk tuning produced non-finite values.");
}

void syncClock(seis3d_session* s, uint64_t step) {
    if (s->hostClock != step) {
        setClock<<<1, 1, 0, s->stream>>>(s->clock, step);
        launchCheck("set clock");
        ++s->launches;
    }
}

}  // namespace

namespace {

void buildTensorMaps(seis3d_session* s) {
    const EncodeTiled encode = encoder();
    std::vector<CUtensorMap> table(tma::kMapCount);
    const cuuint64_t dims[3] = {cuuint64_t(s->ctx.gx3D), cuuint64_t(s->ctx.gy3D), cuuint64_t(s->ctx.gz3D)};
    const cuuint64_t strides[2] = {cuuint64_t(s->pitch) * 4, cuuint64_t(s->plane) * 4};
    const cuuint32_t unit[3] = {1, 1, 1};
    auto make = [&](int index, float* base, cuuint32_t w, cuuint32_t h) {
        const cuuint32_t box[3] = {w, h, 1};
        const CUresult r = encode(&table[index], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, unit,
                                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) throw RuntimeError("Seis3D: cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ").");
    };
    for (int k = 0; k < 9; ++k) make(tma::kCenter0 + k, s->field[k], kTX, kTY);
    make(tma::kCenter0 + 9, s->invRho, kTX, kTY);
    make(tma::kCenter0 + 10, s->lambda, kTX, kTY);
    make(tma::kCenter0 + 11, s->mu, kTX, kTY);
    make(tma::kSxxX, s->field[3], kTX + 8, kTY);
    make(tma::kSxzX, s->field[8], kTX + 8, kTY);
    make(tma::kSxyXY, s->field[6], kTX + 8, kTY + 8);
    make(tma::kSyyY, s->field[4], kTX, kTY + 8);
    make(tma::kSyzY, s->field[7], kTX, kTY + 8);
    make(tma::kVxXY, s->field[0], kTX + 8, kTY + 8);
    make(tma::kVyXY, s->field[1], kTX + 8, kTY + 8);
    make(tma::kVzXY, s->field[2], kTX + 8, kTY + 8);
    make(tma::kRhoT, s->invRho, 36, kTY + 1);
    make(tma::kMuT, s->mu, 36, kTY + 1);
    cudaCheck(deviceMalloc(&s->maps, table.size() * sizeof(CUtensorMap)), "allocate tensor maps");
    cudaCheck(cudaMemcpyAsync(s->maps, table.data(), table.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, s->stream),
              "upload tensor maps");
    cudaCheck(cudaStreamSynchronize(s->stream), "upload tensor maps");
}

}  // namespace

// --------------------------------------------------------------------------------------
// C ABI.
// --------------------------------------------------------------------------------------
extern "C" {

const char* seis3d_last_error(void) { return lastError.c_str(); }

int seis3d_abi_version(void) { return SEIS3D_ABI_VERSION; }

// Defaults of include/Common3D.h:24-42.
void seis3d_default_context(seis3d_context* c) {
    if (!c) return;
    *c = seis3d_context{};
    c->nx3D = 300; c->ny3D = 50; c->nz3D = 300;
    c->pml3D = 12;
    c->freeSurface3D = 1; c->reflecting3D = 0;
    c->spacing3D = 10.0f; c->cfl3D = 0.85f; c->dt3D = 0.0f;
    c->manualTimeStep3D = 0; c->requestedDtMs3D = 0.5f; c->safeDt3D = 0.0f;
    c->vp3D = 3000.0f; c->vs3D = 1700.0f; c->density3D = 2200.0f;
    c->layerVp3D = 4200.0f; c->layerVs3D = 2400.0f; c->layerDensity3D = 2500.0f;
    c->maxVp3D = 4200.0f; c->frequency3D = 20.0f;
    c->modelKind3D = SEIS3D_MODEL_TWO_LAYER;
    c->interfaceDepth3D = 0.5f; c->layerDip3D = 0.25f; c->layerThickness3D = 0.15f;
    c->faultThrow3D = 0.18f; c->anomalyRadius3D = 0.187f;
}

// Defaults of include/Common3D.h:44-49.
void seis3d_default_source(seis3d_source* s) {
    if (!s) return;
    *s = seis3d_source{};
    s->x3D = 48; s->y3D = 48; s->z3D = 24;
    s->kind3D = SEIS3D_SOURCE_EXPLOSION;
    s->amplitude3D = 1.0e8f;
    s->direction3D[0] = 0.0f; s->direction3D[1] = 0.0f; s->direction3D[2] = 1.0f;
}

int seis3d_validate_context(seis3d_context* c) {
    return guarded([&] {
        if (!c) throw InvalidArgument("Seis3D: null context.");
        validate(*c);
    });
}

int seis3d_validate_thin_context(seis3d_context* c) {
    return guarded([&] {
        if (!c) throw InvalidArgument("Seis3D: null context.");
        validate(*c, 4);
    });
}

int seis3d_estimate_memory(const seis3d_context* c, seis3d_memory_budget* b) {
    return guarded([&] {
        if (!c || !b) throw InvalidArgument("Seis3D: null argument.");
        *b = budget(*c);
    });
}

int seis3d_make_view_layout(const seis3d_context* c, seis3d_view_layout* l) {
    return guarded([&] {
        if (!c || !l) throw InvalidArgument("Seis3D: null argument.");
        *l = viewLayout(*c);
    });
}

int seis3d_make_cpml_coefficients(const seis3d_context* c, int axis, float* values, size_t capacity) {
    return guarded([&] {
        if (!c || !values || axis < 0 || axis > 2) throw InvalidArgument("Seis3D: invalid coefficient request.");
        const auto v = coefficients(*c, axis);
        if (capacity < v.size()) throw InvalidArgument("Seis3D: coefficient buffer too small.");
        std::memcpy(values, v.data(), v.size() * sizeof(float));
    });
}

// initializeGpu3D (cuda/Cuda_Seis3D.cu:519-555).
int seis3d_initialize(seis3d_session** out, const seis3d_context* context, const seis3d_options* options) {
    const ApiRange range("seis3d_initialize");
    return guarded([&] {
        if (!out || !context) throw InvalidArgument("Seis3D: null argument.");
        if (*out) throw LogicError("Seis3D: release the previous session before initializing.");
        seis3d_context c = *context;
        const seis3d_options opt = options ? *options : seis3d_options{};
        const int minPml = opt.thin_cpml ? 4 : 8;
        const auto b = budget(c, minPml);   // validates
        validate(c, minPml);
        if (opt.storage == SEIS3D_STORAGE_FP16 || opt.storage == SEIS3D_STORAGE_BF16)
            throw InvalidArgument("Seis3D: 16-bit wavefield storage is not provided (its trace error against FP64 "
                                  "exceeds 1e-3); SEIS3D_STORAGE_BF16_CPML keeps only the CPML memories in 16 bits.");
        if (opt.storage != SEIS3D_STORAGE_FP32 && opt.storage != SEIS3D_STORAGE_BF16_CPML)
            throw InvalidArgument("Seis3D: unknown storage mode.");
        if (opt.tile_y != 0 && opt.tile_y != kTY) throw InvalidArgument("Seis3D: tile_y must be 0 or 16.");
        if (opt.z_chunk < 0) throw InvalidArgument("Seis3D: z_chunk must be >= 0.");
        // The tensor maps need 16-byte row strides, so unpitched rows need gx3D % 4 == 0.
        if (opt.compact_rows && c.gx3D % 4 != 0)
            throw InvalidArgument("Seis3D: the unpitched layout needs gx3D (nx3D + 2 pml3D + 8) to be a multiple of 4.");
        int device = 0;
        cudaCheck(cudaGetDevice(&device), "query current device");
        std::size_t freeBytes = 0, totalBytes = 0;
        cudaCheck(cudaMemGetInfo(&freeBytes, &totalBytes), "query VRAM");
        const std::size_t reserve = std::max(std::size_t(512) * 1024 * 1024, totalBytes / 5);
        if (b.totalBytes3D > SEIS3D_MEMORY_LIMIT || freeBytes < reserve || b.totalBytes3D > freeBytes - reserve)
            throw RuntimeError("Seis3D: VRAM budget exceeded; reduce grid size or CPML thickness.");

        auto* s = new seis3d_session;
        try {
            s->ctx = c;
            s->device = device;
            s->tileY = kTY;
            s->zChunk = opt.z_chunk;
            s->storage = opt.storage;
            cudaCheck(cudaDeviceGetAttribute(&s->smCount, cudaDevAttrMultiProcessorCount, device), "query SM count");
            configureKernels();
            {
                int perSmV = 0, perSmS = 0;
                cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSmV, velocityKernel(s), kThreads,
                                                                        kVelocitySmem), "velocity pass occupancy");
                cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSmS, stressKernel(s), kThreads, kStressSmem),
                          "stress pass occupancy");
                if (perSmV < 1 || perSmS < 1) throw RuntimeError("Seis3D: the step kernels do not fit on this device.");
                s->residentCtas = std::min(perSmV, perSmS) * s->smCount;
            }
            cudaCheck(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "create stream");
            s->pitch = opt.compact_rows ? c.gx3D : roundUp(c.gx3D, 32);
            s->plane = s->pitch * c.gy3D;
            const std::size_t volume = std::size_t(s->plane) * c.gz3D;
            s->poolBytes = volume * 12 * sizeof(float);
            cudaCheck(deviceMalloc(&s->pool, s->poolBytes), "allocate fields");
            cudaCheck(cudaMemsetAsync(s->pool, 0, s->poolBytes, s->stream), "clear fields");
            for (int k = 0; k < 9; ++k) s->field[k] = s->pool + k * volume;
            s->invRho = s->pool + 9 * volume;
            s->lambda = s->pool + 10 * volume;
            s->mu = s->pool + 11 * volume;
            s->allocated = s->poolBytes;
            if (!c.reflecting3D) {
                const int thick[3] = {2 * c.pml3D, 2 * c.pml3D, (c.freeSurface3D ? 1 : 2) * c.pml3D};
                s->psiCount[0] = std::size_t(6) * c.gz3D * c.gy3D * thick[0];
                s->psiCount[1] = std::size_t(6) * c.gz3D * thick[1] * s->pitch;
                s->psiCount[2] = std::size_t(6) * thick[2] * c.gy3D * s->pitch;
                for (int a = 0; a < 3; ++a) {
                    cudaCheck(deviceMalloc(&s->psi[a], s->psiBytes(a)), "allocate CPML memories");
                    cudaCheck(cudaMemsetAsync(s->psi[a], 0, s->psiBytes(a), s->stream), "clear CPML");
                    s->allocated += s->psiBytes(a);
                    const auto k = coefficients(c, a);
                    cudaCheck(deviceMalloc(&s->coef[a], k.size() * sizeof(float)), "allocate CPML coefficients");
                    cudaCheck(cudaMemcpyAsync(s->coef[a], k.data(), k.size() * sizeof(float), cudaMemcpyHostToDevice,
                                              s->stream), "upload CPML coefficients");
                    cudaCheck(cudaStreamSynchronize(s->stream), "finish coefficient upload");
                }
            }
            cudaCheck(deviceMalloc(&s->status, 4 * sizeof(unsigned)), "allocate status");
            cudaCheck(cudaMemsetAsync(s->status, 0, 4 * sizeof(unsigned), s->stream), "clear status");
            configureKernels();
            buildTensorMaps(s);
            cudaCheck(deviceMalloc(&s->clock, sizeof(Clock)), "allocate clock");
            cudaCheck(cudaMemsetAsync(s->clock, 0, sizeof(Clock), s->stream), "clear clock");
            s->hostClock = 0;
            cudaCheck(hostMalloc(&s->stage, std::size_t(c.nx3D) * c.ny3D * 3 * sizeof(float)), "allocate staging");
            ModelParams M{};
            M.kind = c.modelKind3D;
            M.vp = c.vp3D; M.vs = c.vs3D; M.rho = c.density3D;
            M.layerVp = c.layerVp3D; M.layerVs = c.layerVs3D; M.layerRho = c.layerDensity3D;
            M.interfaceDepth = c.interfaceDepth3D; M.layerDip = c.layerDip3D; M.layerThickness = c.layerThickness3D;
            M.faultThrow = c.faultThrow3D; M.anomalyRadius = c.anomalyRadius3D;
            const int64_t cells = int64_t(c.cells3D);
            generateMaterials<<<unsigned((cells + 255) / 256), 256, 0, s->stream>>>(s->geometry(), s->fields(), M);
            launchCheck("generate materials");
            cudaCheck(cudaStreamSynchronize(s->stream), "initialize model");
            if (opt.tune && opt.z_chunk == 0) tuneZChunk(s);
        } catch (...) {
            releaseSession(s);
            throw;
        }
        *out = s;
    });
}

void seis3d_release(seis3d_session* s) { releaseSession(s); }

// resetGpu3D (cuda/Cuda_Seis3D.cu:572-577).
int seis3d_reset(seis3d_session* s, const seis3d_context* c) {
    return guarded([&] {
        requireSession(s);
        requireSameGrid(s, c);
        const std::size_t volume = std::size_t(s->plane) * s->ctx.gz3D;
        cudaCheck(cudaMemsetAsync(s->pool, 0, volume * 9 * sizeof(float), s->stream), "reset wavefield");
        for (int a = 0; a < 3; ++a)
            if (s->psi[a]) cudaCheck(cudaMemsetAsync(s->psi[a], 0, s->psiBytes(a), s->stream), "reset CPML");
        cudaCheck(cudaMemsetAsync(s->status, 0, 4 * sizeof(unsigned), s->stream), "reset diagnostics");
    });
}

// refreshCpmlCoefficients3D (cuda/Cuda_Seis3D.cu:580-599): build all profiles first, then
// swap on success only.
int seis3d_refresh_cpml(seis3d_session* s, const seis3d_context* c) {
    return guarded([&] {
        requireSession(s);
        requireSameGrid(s, c);
        if (c->reflecting3D) return;
        std::vector<float> profiles[3];
        for (int a = 0; a < 3; ++a) profiles[a] = coefficients(*c, a);
        float* replacement[3]{};
        try {
            for (int a = 0; a < 3; ++a) {
                cudaCheck(deviceMalloc(&replacement[a], profiles[a].size() * sizeof(float)), "allocate CPML coefficients");
                cudaCheck(cudaMemcpyAsync(replacement[a], profiles[a].data(), profiles[a].size() * sizeof(float),
                                          cudaMemcpyHostToDevice, s->stream), "refresh CPML coefficients");
            }
            cudaCheck(cudaStreamSynchronize(s->stream), "finish CPML refresh");
        } catch (...) {
            cudaStreamSynchronize(s->stream);
            for (auto p : replacement) cudaFree(p);
            throw;
        }
        for (int a = 0; a < 3; ++a) {
            std::swap(s->coef[a], replacement[a]);
            cudaFree(replacement[a]);
        }
        adoptScalars(s, c);
        s->dropGraph();
    });
}

// runStep3D (cuda/Cuda_Seis3D.cu:602-624).
int seis3d_run_step(seis3d_session* s, const seis3d_context* c, const seis3d_source* src, uint64_t step) {
    const ApiRange range("seis3d_run_step");
    return guarded([&] {
        requireSession(s);
        if (!src) throw InvalidArgument("Seis3D: null source.");
        checkSource(*c, *src);
        requireSameGrid(s, c);
        adoptScalars(s, c);
        syncClock(s, step);
        enqueueStep(s, sourceParams(s->ctx, *src), true);
        closingImages(s);
        s->hostClock = step + 1;
    });
}

// Steps are replayed from a captured graph of kGraphBatch steps; the graph reads the step
// index from the device clock, so one capture serves every start step.
constexpr int kGraphBatch = 64;

static void ensureGraph(seis3d_session* s, const seis3d_source& src, const SourceParams& S) {
    if (s->graph && std::memcmp(&s->graphSource, &src, sizeof(seis3d_source)) == 0 &&
        s->graphGather == s->gatherActive)
        return;
    s->dropGraph();
    cudaGraph_t g = nullptr;
    const uint64_t before = s->launches;
    cudaCheck(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        for (int k = 0; k < kGraphBatch; ++k) enqueueStep(s, S, false);
    } catch (...) {
        cudaStreamEndCapture(s->stream, &g);
        if (g) cudaGraphDestroy(g);
        s->launches = before;
        throw;
    }
    cudaCheck(cudaStreamEndCapture(s->stream, &g), "end capture");
    s->graphNodes = s->launches - before;
    s->launches = before;  // captured, not launched
    const cudaError_t e = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    cudaCheck(e, "instantiate step graph");
    s->graphSteps = kGraphBatch;
    s->graphSource = src;
    s->graphGather = s->gatherActive;
}

int seis3d_run_steps(seis3d_session* s, const seis3d_context* c, const seis3d_source* src, uint64_t first, int count) {
    const ApiRange range("seis3d_run_steps");
    return guarded([&] {
        requireSession(s);
        if (!src) throw InvalidArgument("Seis3D: null source.");
        if (count < 0) throw InvalidArgument("Seis3D: negative step count.");
        checkSource(*c, *src);
        requireSameGrid(s, c);
        adoptScalars(s, c);
        if (count == 0) return;
        syncClock(s, first);
        const SourceParams S = sourceParams(s->ctx, *src);
        // Start-of-step stress images once; later steps inherit them from the step before.
        launchImages(s, false);
        int done = 0;
        if (count >= kGraphBatch) {
            ensureGraph(s, *src, S);
            for (; count - done >= kGraphBatch; done += kGraphBatch) {
                cudaCheck(cudaGraphLaunch(s->graph, s->stream), "launch step graph");
                s->launches += s->graphNodes;
            }
        }
        for (; done < count; ++done) enqueueStep(s, S, false);
        closingImages(s);
        s->hostClock = first + uint64_t(count);
    });
}

int seis3d_prepare_steps(seis3d_session* s, const seis3d_context* c, const seis3d_source* src) {
    const ApiRange range("seis3d_prepare_steps");
    return guarded([&] {
        requireSession(s);
        if (!src) throw InvalidArgument("Seis3D: null source.");
        checkSource(*c, *src);
        requireSameGrid(s, c);
        adoptScalars(s, c);
        ensureGraph(s, *src, sourceParams(s->ctx, *src));
    });
}

// setReceivers3D (cuda/Cuda_Seis3D.cu:649-668).
int seis3d_set_receivers(seis3d_session* s, const seis3d_context* c, const seis3d_receiver* r, int count) {
    return guarded([&] {
        if (count < 0 || count > SEIS3D_MAX_RECEIVERS || (count && !r))
            throw InvalidArgument("Seis3D: invalid receiver count.");
        requireSession(s);
        requireSameGrid(s, c);
        for (int a = 0; a < count; ++a)
            if (r[a].x3D < 0 || r[a].x3D >= c->nx3D || r[a].y3D < 0 || r[a].y3D >= c->ny3D || r[a].z3D < 0 ||
                r[a].z3D >= c->nz3D)
                throw InvalidArgument("Seis3D: receiver outside the physical domain.");
        if (s->gatherActive) throw LogicError("Seis3D: stop the active gather before replacing receivers.");
        int4* positions = nullptr;
        float* values = nullptr;
        float* host = nullptr;
        std::vector<int4> grid(static_cast<std::size_t>(count));
        for (int a = 0; a < count; ++a) grid[a] = make_int4(r[a].x3D + c->ox3D, r[a].y3D + c->oy3D, r[a].z3D + c->oz3D, 0);
        try {
            if (count) {
                cudaCheck(deviceMalloc(&positions, std::size_t(count) * sizeof(int4)), "allocate receivers");
                cudaCheck(deviceMalloc(&values, std::size_t(count) * 3 * sizeof(float)), "allocate receiver values");
                cudaCheck(hostMalloc(&host, std::size_t(count) * 3 * sizeof(float)), "allocate pinned receivers");
                cudaCheck(cudaMemcpyAsync(positions, grid.data(), std::size_t(count) * sizeof(int4), cudaMemcpyHostToDevice,
                                          s->stream), "upload receivers");
            }
            cudaCheck(cudaStreamSynchronize(s->stream), "finish receiver update");
        } catch (...) {
            cudaFree(positions); cudaFree(values);
            if (host) cudaFreeHost(host);
            throw;
        }
        cudaFree(s->recv); cudaFree(s->recvValues);
        if (s->hostRecv) cudaFreeHost(s->hostRecv);
        s->recv = positions; s->recvValues = values; s->hostRecv = host; s->recvCount = count;
        s->dropGraph();
    });
}

// sampleReceivers3D (cuda/Cuda_Seis3D.cu:671-681).
int seis3d_sample_receivers(seis3d_session* s, const seis3d_context* c, const float** values) {
    const ApiRange range("seis3d_sample_receivers");
    return guarded([&] {
        if (!values) throw InvalidArgument("Seis3D: null output.");
        *values = nullptr;
        requireSession(s);
        requireSameGrid(s, c);
        if (!s->recvCount) return;
        sampleReceivers<<<(s->recvCount + 255) / 256, 256, 0, s->stream>>>(s->geometry(), s->fields(), s->recv,
                                                                            s->recvCount, s->recvValues);
        launchCheck("sample receivers");
        cudaCheck(cudaMemcpyAsync(s->hostRecv, s->recvValues, std::size_t(s->recvCount) * 3 * sizeof(float),
                                  cudaMemcpyDeviceToHost, s->stream), "gather receivers");
        cudaCheck(cudaStreamSynchronize(s->stream), "finish receiver gather");
        if (readStatus(s)) throw RuntimeError("Seis3D: non-finite wavefield detected; capture stopped before export.");
        *values = s->hostRecv;
    });
}

// probeMaterial3D (cuda/Cuda_Seis3D.cu:684-693).
int seis3d_probe_material(seis3d_session* s, const seis3d_context* c, const seis3d_receiver* p, float values[3]) {
    return guarded([&] {
        requireSession(s);
        requireSameGrid(s, c);
        if (!p || !values) throw InvalidArgument("Seis3D: null argument.");
        if (p->x3D < 0 || p->x3D >= c->nx3D || p->y3D < 0 || p->y3D >= c->ny3D || p->z3D < 0 || p->z3D >= c->nz3D) return;
        const int64_t i = int64_t(p->z3D + c->oz3D) * s->plane + int64_t(p->y3D + c->oy3D) * s->pitch + p->x3D + c->ox3D;
        float inverse = 0, m = 0, l = 0;
        cudaCheck(cudaMemcpyAsync(&inverse, s->invRho + i, 4, cudaMemcpyDeviceToHost, s->stream), "probe density");
        cudaCheck(cudaMemcpyAsync(&m, s->mu + i, 4, cudaMemcpyDeviceToHost, s->stream), "probe mu");
        cudaCheck(cudaMemcpyAsync(&l, s->lambda + i, 4, cudaMemcpyDeviceToHost, s->stream), "probe lambda");
        cudaCheck(cudaStreamSynchronize(s->stream), "finish material probe");
        values[0] = std::sqrt((l + 2 * m) * inverse);
        values[1] = std::sqrt(m * inverse);
        values[2] = 1 / inverse;
    });
}

// uploadModelPlane3D (cuda/Cuda_Seis3D.cu:696-711): validate the whole plane, convert to
// 1/rho, lambda, mu in FP32 on the host as the reference does, pitched copies.
int seis3d_upload_model_plane(seis3d_session* s, const seis3d_context* c, int z, const float* values) {
    const ApiRange range("seis3d_upload_model_plane");
    return guarded([&] {
        requireSession(s);
        requireSameGrid(s, c);
        if (z < 0 || z >= c->nz3D || !values) throw InvalidArgument("Seis3D: invalid model plane.");
        const std::size_t n = std::size_t(c->nx3D) * c->ny3D;
        cudaCheck(cudaStreamSynchronize(s->stream), "reuse staging");
        float* m = s->stage;
        for (std::size_t i = 0; i < n; ++i) {
            const float vp = values[3 * i], vs = values[3 * i + 1], rho = values[3 * i + 2];
            if (!admissible(vp, vs, rho) || vp > s->ctx.maxVp3D * (1 + 1.0e-6f))
                throw InvalidArgument("Seis3D: invalid or changed imported material.");
            m[i] = 1 / rho;
            m[n + i] = rho * (vp * vp - 2 * vs * vs);
            m[2 * n + i] = rho * vs * vs;
        }
        const int64_t offset = int64_t(z + c->oz3D) * s->plane + int64_t(c->oy3D) * s->pitch + c->ox3D;
        float* dst[3] = {s->invRho, s->lambda, s->mu};
        for (int a = 0; a < 3; ++a)
            cudaCheck(cudaMemcpy2DAsync(dst[a] + offset, std::size_t(s->pitch) * 4, m + a * n, std::size_t(c->nx3D) * 4,
                                        std::size_t(c->nx3D) * 4, c->ny3D, cudaMemcpyHostToDevice, s->stream),
                      "upload material plane");
        cudaCheck(cudaStreamSynchronize(s->stream), "finish material plane");
    });
}

// The whole model from three host volumes in one call: every cell is validated first (on
// host threads, before anything on the device changes, with the rejection of
// uploadModelPlane3D), then chunks of raw planes are copied and converted on the device, then
// the materials are extended as finishModelUpload3D does.
int seis3d_upload_model(seis3d_session* s, const seis3d_context* c, const float* vp, const float* vs,
                        const float* rho) {
    const ApiRange range("seis3d_upload_model");
    return guarded([&] {
        requireSession(s);
        requireSameGrid(s, c);
        if (!vp || !vs || !rho) throw InvalidArgument("Seis3D: invalid model volume.");
        const std::size_t n = std::size_t(c->nx3D) * c->ny3D, total = n * std::size_t(c->nz3D);
        const float limit = s->ctx.maxVp3D * (1 + 1.0e-6f);
        const unsigned workers = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        // The raw volumes go to a device staging area and are converted only after every cell
        // passed validation, so a rejected model leaves the session untouched.  Host work is
        // one pass per chunk of whole planes: worker threads validate the cells and pack them
        // into one of two pinned buffers while the DMA engine copies the previous chunk.
        // The staging area stays with the session (like the pinned chunks), so repeated uploads
        // neither allocate nor free device memory (a free synchronises the device).
        if (s->uploadRawCells < total) {
            cudaFree(s->uploadRaw);
            s->allocated -= s->uploadRawCells * 3 * sizeof(float);
            s->uploadRaw = nullptr;
            s->uploadRawCells = 0;
            cudaCheck(deviceMalloc(&s->uploadRaw, total * 3 * sizeof(float)), "model staging");
            s->uploadRawCells = total;
            s->allocated += total * 3 * sizeof(float);
        }
        float* raw = s->uploadRaw;
        struct Staging {
            cudaStream_t stream;
            ~Staging() { cudaStreamSynchronize(stream); }   // no copy outlives a rejected call
        } staging{s->stream};
        const std::size_t planes = std::max<std::size_t>(1, std::min<std::size_t>(c->nz3D, (std::size_t(32) << 20) / (n * 12)));
        const std::size_t chunk = planes * n;
        if (s->uploadCapacity < chunk) {
            for (auto& h : s->uploadHost) {
                if (h) cudaFreeHost(h);
                h = nullptr;
            }
            s->uploadCapacity = 0;
            for (auto& h : s->uploadHost) cudaCheck(hostMalloc(&h, chunk * 3 * sizeof(float)), "pinned model staging");
            s->uploadCapacity = chunk;
        }
        for (auto& e : s->uploadDone)
            if (!e) cudaCheck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "model staging event");
        std::size_t at = 0;
        for (int k = 0; at < total; ++k, at += chunk) {
            const std::size_t count = std::min(chunk, total - at);
            const int b = k & 1;
            float* host = s->uploadHost[b];
            if (k >= 2) cudaCheck(cudaEventSynchronize(s->uploadDone[b]), "model staging reuse");
            std::vector<char> bad(workers, 0);
            std::vector<std::thread> pool;
            for (unsigned w = 0; w < workers; ++w)
                pool.emplace_back([&, w] {
                    const std::size_t begin = count * w / workers, end = count * (w + 1) / workers;
                    for (std::size_t i = begin; i < end; ++i) {
                        const float p = vp[at + i], q = vs[at + i], r = rho[at + i];
                        if (!admissible(p, q, r) || p > limit) { bad[w] = 1; return; }
                        host[i] = p;
                        host[count + i] = q;
                        host[2 * count + i] = r;
                    }
                });
            for (auto& t : pool) t.join();
            for (char x : bad)
                if (x) throw InvalidArgument("Seis3D: invalid or changed imported material.");
            for (int a = 0; a < 3; ++a)
                cudaCheck(cudaMemcpyAsync(raw + a * total + at, host + a * count, count * sizeof(float),
                                          cudaMemcpyHostToDevice, s->stream), "upload model chunk");
            cudaCheck(cudaEventRecord(s->uploadDone[b], s->stream), "model staging event");
        }
        convertMaterials<<<unsigned((total + 255) / 256), 256, 0, s->stream>>>(s->geometry(), s->fields(), raw,
                                                                                raw + total, raw + 2 * total, 0,
                                                                                c->nz3D);
        launchCheck("convert materials");
        ++s->launches;
        cudaCheck(cudaStreamSynchronize(s->stream), "upload model");
        const int status = seis3d_finish_model_upload(s, c);
        if (status != SEIS3D_OK) throw RuntimeError(lastError);
    });
}

// finishModelUpload3D (cuda/Cuda_Seis3D.cu:714-717).
int seis3d_finish_model_upload(seis3d_session* s, const seis3d_context* c) {
    return guarded([&] {
        requireSession(s);
        requireSameGrid(s, c);
        const int64_t cells = int64_t(s->ctx.cells3D);
        extendMaterials<<<unsigned((cells + 255) / 256), 256, 0, s->stream>>>(s->geometry(), s->fields());
        launchCheck("extend materials");
        cudaCheck(cudaStreamSynchronize(s->stream), "finish model import");
    });
}

// downloadModelPlane3D (cuda/Cuda_Seis3D.cu:720-733).
int seis3d_download_model_plane(seis3d_session* s, const seis3d_context* c, int z, float* values) {
    return guarded([&] {
        requireSession(s);
        requireSameGrid(s, c);
        if (z < 0 || z >= c->nz3D || !values) throw InvalidArgument("Seis3D: invalid export plane.");
        const std::size_t n = std::size_t(c->nx3D) * c->ny3D;
        std::vector<float> m(n * 3);
        const int64_t offset = int64_t(z + c->oz3D) * s->plane + int64_t(c->oy3D) * s->pitch + c->ox3D;
        const float* src[3] = {s->invRho, s->lambda, s->mu};
        for (int a = 0; a < 3; ++a)
            cudaCheck(cudaMemcpy2DAsync(m.data() + a * n, std::size_t(c->nx3D) * 4, src[a] + offset,
                                        std::size_t(s->pitch) * 4, std::size_t(c->nx3D) * 4, c->ny3D,
                                        cudaMemcpyDeviceToHost, s->stream), "download material plane");
        cudaCheck(cudaStreamSynchronize(s->stream), "finish model plane export");
        for (std::size_t i = 0; i < n; ++i) {
            values[3 * i] = std::sqrt((m[n + i] + 2 * m[2 * n + i]) * m[i]);
            values[3 * i + 1] = std::sqrt(m[2 * n + i] * m[i]);
            values[3 * i + 2] = 1 / m[i];
        }
    });
}

int seis3d_gather_begin(seis3d_session* s, int stride, int target) {
    return guarded([&] {
        requireSession(s);
        if (stride < 1 || stride > 10000 || target < 1 || target > SEIS3D_MAX_SEGY_SAMPLES)
            throw InvalidArgument("Seis3D: gather sample count must be 1..32767 with stride 1..10000.");
        if (!s->recvCount) throw LogicError("Seis3D: set receivers before starting a gather.");
        const std::size_t need = std::size_t(target) * s->recvCount * 3;
        if (need * sizeof(float) > std::size_t(512) * 1024 * 1024)
            throw InvalidArgument("Seis3D: shot gather exceeds the 512 MiB budget.");
        if (need > s->gatherFloats) {
            float* g = nullptr;
            cudaCheck(deviceMalloc(&g, need * sizeof(float)), "allocate gather");
            cudaFree(s->gather);
            s->gather = g;
            s->gatherFloats = need;
            s->dropGraph();
        }
        cudaCheck(cudaMemsetAsync(s->gather, 0, need * sizeof(float), s->stream), "clear gather");
        Clock host{};
        cudaCheck(cudaMemcpyAsync(&host, s->clock, sizeof(Clock), cudaMemcpyDeviceToHost, s->stream), "read clock");
        cudaCheck(cudaStreamSynchronize(s->stream), "read clock");
        host.sample = 0; host.stride = stride; host.target = target;
        cudaCheck(cudaMemcpyAsync(s->clock, &host, sizeof(Clock), cudaMemcpyHostToDevice, s->stream), "write clock");
        cudaCheck(cudaStreamSynchronize(s->stream), "write clock");
        s->gatherStride = stride; s->gatherTarget = target;
        if (!s->gatherActive) s->dropGraph();
        s->gatherActive = true;
    });
}

int seis3d_gather_fetch(seis3d_session* s, float* host, size_t capacity, int* sampleCount) {
    const ApiRange range("seis3d_gather_fetch");
    return guarded([&] {
        requireSession(s);
        if (!sampleCount) throw InvalidArgument("Seis3D: null sample count.");
        Clock clk{};
        cudaCheck(cudaMemcpyAsync(&clk, s->clock, sizeof(Clock), cudaMemcpyDeviceToHost, s->stream), "read clock");
        cudaCheck(cudaStreamSynchronize(s->stream), "finish gather");
        const unsigned flag = readStatus(s);
        *sampleCount = s->gather ? clk.sample : 0;
        if (host && s->gather && clk.sample > 0) {
            const std::size_t n = std::size_t(clk.sample) * s->recvCount * 3;
            if (capacity < n) throw InvalidArgument("Seis3D: gather buffer too small.");
            cudaCheck(cudaMemcpyAsync(host, s->gather, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream), "fetch gather");
            cudaCheck(cudaStreamSynchronize(s->stream), "fetch gather");
        }
        if (flag) throw RuntimeError("Seis3D: non-finite wavefield detected; capture stopped before export.");
    });
}

int seis3d_gather_end(seis3d_session* s) {
    return guarded([&] {
        requireSession(s);
        if (!s->gatherActive) return;
        Clock host{};
        cudaCheck(cudaMemcpyAsync(&host, s->clock, sizeof(Clock), cudaMemcpyDeviceToHost, s->stream), "read clock");
        cudaCheck(cudaStreamSynchronize(s->stream), "read clock");
        host.stride = 0;
        cudaCheck(cudaMemcpyAsync(s->clock, &host, sizeof(Clock), cudaMemcpyHostToDevice, s->stream), "write clock");
        cudaCheck(cudaStreamSynchronize(s->stream), "write clock");
        s->gatherActive = false;
        s->dropGraph();
    });
}

int seis3d_get_views(seis3d_session* s, seis3d_device_views* v) {
    return guarded([&] {
        requireSession(s);
        if (!v) throw InvalidArgument("Seis3D: null views.");
        *v = seis3d_device_views{};
        for (int k = 0; k < 9; ++k) v->field3D[k] = s->field[k];
        v->inverseDensity3D = s->invRho; v->lambda3D = s->lambda; v->mu3D = s->mu;
        for (int a = 0; a < 3; ++a) {
            v->cpml3D[a] = s->psi[a];
            v->slabCells3D[a] = s->psiCount[a] / 6;
            v->coefficients3D[a] = s->coef[a];
        }
        v->stream3D = s->stream;
        v->receiverCount3D = s->recvCount;
        v->storage = s->storage;
        v->pitch = s->pitch; v->plane = s->plane;
        for (int k = 0; k < 12; ++k) v->field_scale[k] = 1.0f;
        v->allocatedBytes3D = s->allocated;
        v->kernelLaunches = s->launches;
    });
}

int seis3d_profile_steps(seis3d_session* s, const seis3d_context* c, const seis3d_source* src, uint64_t first,
                         int count, float ms[4]) {
    const ApiRange range("seis3d_profile_steps");
    return guarded([&] {
        requireSession(s);
        if (!src || !ms || count < 1) throw InvalidArgument("Seis3D: invalid profiling request.");
        checkSource(*c, *src);
        requireSameGrid(s, c);
        adoptScalars(s, c);
        syncClock(s, first);
        const SourceParams S = sourceParams(s->ctx, *src);
        launchImages(s, false);
        std::vector<PassEvents> ev(static_cast<std::size_t>(count));
        for (auto& e : ev)
            for (cudaEvent_t* p : {&e.start, &e.afterVelocity, &e.afterImages, &e.afterStress, &e.end})
                cudaCheck(cudaEventCreate(p), "create event");
        for (int k = 0; k < count; ++k) enqueueStep(s, S, false, &ev[std::size_t(k)]);
        closingImages(s);
        s->hostClock = first + uint64_t(count);
        cudaCheck(cudaStreamSynchronize(s->stream), "profile steps");
        for (int j = 0; j < 4; ++j) ms[j] = 0;
        for (auto& e : ev) {
            float a = 0, b = 0, d = 0, t = 0;
            cudaEventElapsedTime(&a, e.start, e.afterVelocity);
            cudaEventElapsedTime(&b, e.afterImages, e.afterStress);
            cudaEventElapsedTime(&t, e.start, e.end);
            float i1 = 0, i2 = 0;
            cudaEventElapsedTime(&i1, e.afterVelocity, e.afterImages);
            cudaEventElapsedTime(&i2, e.afterStress, e.end);
            d = i1 + i2;
            ms[0] += a; ms[1] += b; ms[2] += d; ms[3] += t;
            for (cudaEvent_t p : {e.start, e.afterVelocity, e.afterImages, e.afterStress, e.end}) cudaEventDestroy(p);
        }
    });
}


int seis3d_copy_field(seis3d_session* s, int f, int direction, float* host) {
    return guarded([&] {
        requireSession(s);
        if (f < 0 || f > 11 || !host || (direction != 0 && direction != 1)) throw InvalidArgument("Seis3D: invalid field copy.");
        float* dev = f < 9 ? s->field[f] : f == 9 ? s->invRho : f == 10 ? s->lambda : s->mu;
        const std::size_t rowBytes = std::size_t(s->ctx.gx3D) * 4;
        const std::size_t rows = std::size_t(s->ctx.gy3D) * s->ctx.gz3D;
        if (direction == 0)
            cudaCheck(cudaMemcpy2DAsync(host, rowBytes, dev, std::size_t(s->pitch) * 4, rowBytes, rows,
                                        cudaMemcpyDeviceToHost, s->stream), "copy field");
        else {
            cudaCheck(cudaMemcpy2DAsync(dev, std::size_t(s->pitch) * 4, host, rowBytes, rowBytes, rows,
                                        cudaMemcpyHostToDevice, s->stream), "copy field");
        }
        cudaCheck(cudaStreamSynchronize(s->stream), "copy field");
    });
}

// extractViews3D (cuda/Cuda_Seis3D.cu:627-646).
int seis3d_extract_views(seis3d_session* s, const seis3d_context* c, float* output, const seis3d_view_layout* layout,
                         const int slices[3], int component, int material_component, int volume,
                         int include_boundary, float* maximum, float material_range[2], float* velocity_maximum) {
    const ApiRange range("seis3d_extract_views");
    return guarded([&] {
        requireSession(s);
        requireSameGrid(s, c);
        if (!output || !layout || !slices || !maximum || !material_range || material_component < 5 ||
            material_component > 7 || component < 0 || component > 7 || slices[0] < 0 || slices[0] >= c->nx3D ||
            slices[1] < 0 || slices[1] >= c->ny3D || slices[2] < 0 || slices[2] >= c->nz3D)
            throw InvalidArgument("Seis3D: invalid view parameters.");
        const seis3d_view_layout expected = viewLayout(s->ctx);
        if (std::memcmp(&expected, layout, sizeof(expected)) != 0)
            throw InvalidArgument("Seis3D: the view layout does not describe this session (use seis3d_make_view_layout).");
        const uint64_t count = volume ? layout->totalSamples3D : layout->volumeOffset3D;
        if (!deviceRange(s, output, std::size_t(count) * 2 * sizeof(float)))
            throw InvalidArgument("Seis3D: the view output must be a device buffer of 2 floats per sample.");
        if (!s->viewStats) cudaCheck(deviceMalloc(&s->viewStats, 8 * sizeof(unsigned)), "allocate view statistics");
        const unsigned initial[5] = {0u, 0u, 0x7f7fffffu, 0u, 0u};
        cudaCheck(cudaMemcpyAsync(s->viewStats, initial, sizeof(initial), cudaMemcpyHostToDevice, s->stream),
                  "reset view statistics");
        ViewArgs a{};
        for (int k = 0; k < 3; ++k) { a.v[k] = s->field[k]; a.s[k] = s->field[3 + k]; }
        a.invRho = s->invRho; a.lambda = s->lambda; a.mu = s->mu;
        a.pitch = s->pitch; a.plane = s->plane;
        a.ox = s->ctx.ox3D; a.oy = s->ctx.oy3D; a.oz = s->ctx.oz3D;
        a.nx = s->ctx.nx3D; a.ny = s->ctx.ny3D; a.nz = s->ctx.nz3D;
        a.layout = *layout;
        a.sx = slices[0]; a.sy = slices[1]; a.sz = slices[2];
        a.component = component; a.materialComponent = material_component;
        a.includeBoundary = include_boundary != 0;
        a.out = output;
        a.stats = s->viewStats;
        a.nonFinite = s->status;
        if (count > 0) {
            extractViews<<<unsigned((count + 255) / 256), 256, 0, s->stream>>>(a, count);
            launchCheck("extract views");
            ++s->launches;
        }
        unsigned stats[5] = {};
        cudaCheck(cudaMemcpyAsync(stats, s->viewStats, sizeof(stats), cudaMemcpyDeviceToHost, s->stream),
                  "read view statistics");
        if (readStatus(s)) throw RuntimeError("Seis3D: non-finite wavefield detected; session stopped.");
        std::memcpy(maximum, stats, sizeof(float));
        std::memcpy(material_range, stats + 2, 2 * sizeof(float));
        if (velocity_maximum) std::memcpy(velocity_maximum, stats + 4, sizeof(float));
    });
}

int seis3d_get_z_chunk(seis3d_session* s, int* setting, int* planes) {
    return guarded([&] {
        requireSession(s);
        if (!setting || !planes) throw InvalidArgument("Seis3D: null output.");
        *setting = s->zChunk;
        *planes = passShape(s).zChunk;
    });
}

void seis3d_debug_fail_allocation(int nth) { failAllocation.store(nth > 0 ? nth : 0); }

int seis3d_debug_stage_wait(seis3d_session* s, long long cycles, int withheld_stage) {
    return guarded([&] {
        requireSession(s);
        if (cycles < 0 || withheld_stage < -1) throw InvalidArgument("Seis3D: invalid stage-wait test settings.");
        s->waitCycles = cycles ? cycles : tma::kWaitCycles;
        s->withheldStage = withheld_stage;
        s->dropGraph();   // captured launches carry the old settings
    });
}

int seis3d_synchronize(seis3d_session* s) {
    return guarded([&] {
        requireSession(s);
        cudaCheck(cudaStreamSynchronize(s->stream), "synchronize");
        readStatus(s);
    });
}

int seis3d_non_finite(seis3d_session* s, int* flag) {
    return guarded([&] {
        requireSession(s);
        if (!flag) throw InvalidArgument("Seis3D: null flag.");
        *flag = readStatus(s) ? 1 : 0;
    });
}

}  // extern "C"

#include "seis3d_io.inc"
#include "seis3d_shade.inc"
#include "seis3d_batch.inc"
#include "seis3d_checkpoint.inc"
#include "seis3d_boundary.inc"
