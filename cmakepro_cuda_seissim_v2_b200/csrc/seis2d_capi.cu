// seis2d_capi.cu - host side of the B200 2-D P-SV solver behind include/seis2d_capi.h.
//
// Each exported function keeps the contract of the reference function it replaces (cited
// per function): the same validation order and messages, the same error class, the same
// all-or-nothing buffer replacement.  Device work runs on the session's own stream; runs of
// many steps are captured once per batch length into a CUDA graph and replayed.
#include "../../include/seis2d_capi.h"
#include "seis2d_kernels.cuh"

#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

using namespace seis2d;

namespace {

thread_local std::string lastError;

struct InvalidArgument : std::runtime_error { using std::runtime_error::runtime_error; };
struct LogicError : std::runtime_error { using std::runtime_error::runtime_error; };
struct RuntimeError : std::runtime_error { using std::runtime_error::runtime_error; };
struct OverflowError : std::runtime_error { using std::runtime_error::runtime_error; };

void cudaCheck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw RuntimeError(std::string("CUDA failure: ") + what + " | " + cudaGetErrorString(e));
}

// Allocation seam for host-side fault injection (seis2d_debug_fail_allocation): when armed
// with n > 0, the n-th device allocation from then on reports out of memory.
std::atomic<int> failAllocation{0};

bool injectFailure() {
    int n = failAllocation.load();
    while (n > 0 && !failAllocation.compare_exchange_weak(n, n - 1)) {
    }
    return n == 1;
}

template <class F> int guarded(F&& body) {
    try {
        body();
        return SEIS2D_OK;
    } catch (const InvalidArgument& e) {
        lastError = e.what(); return SEIS2D_INVALID_ARGUMENT;
    } catch (const LogicError& e) {
        lastError = e.what(); return SEIS2D_LOGIC_ERROR;
    } catch (const OverflowError& e) {
        lastError = e.what(); return SEIS2D_OVERFLOW_ERROR;
    } catch (const std::bad_alloc&) {
        lastError = "host allocation failed"; return SEIS2D_RUNTIME_ERROR;
    } catch (const std::exception& e) {
        lastError = e.what(); return SEIS2D_RUNTIME_ERROR;
    }
}

// ---- SolverNumerics.h ------------------------------------------------------------------

constexpr double kWeights[4] = {1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0};
constexpr double kWeightMagnitude = kWeights[0] - kWeights[1] + kWeights[2] - kWeights[3];
constexpr float kCourantLimit = static_cast<float>(1.0 / (1.4142135623730951 * kWeightMagnitude));
constexpr float kSafeCourant = 0.480f;
constexpr double kPi = 3.14159265358979323846;  // M_PI of the C math headers (a double)

// checkedGridElementCount (SolverNumerics.h:25-34).
std::size_t checkedCount(int nx, int nz) {
    if (nx <= 2 * SEIS2D_STENCIL_RADIUS || nz <= 2 * SEIS2D_STENCIL_RADIUS)
        throw InvalidArgument("Grid dimensions must exceed the 8-cell stencil guard region");
    const std::size_t n = std::size_t(nx) * std::size_t(nz);
    if (n > std::size_t((std::numeric_limits<int>::max)()))
        throw OverflowError("The 2D solver index capacity was exceeded");
    return n;
}

// validateBoundaryGeometry (SolverNumerics.h:37-47).
void checkBoundary(int nx, int nz, int pml, bool freeSurface) {
    checkedCount(nx, nz);
    if (pml < 0 || pml > (nx - 2 * SEIS2D_STENCIL_RADIUS - 1) / 2 || pml > (nz - 2 * SEIS2D_STENCIL_RADIUS - 1) / 2)
        throw InvalidArgument("PML width leaves no physical interior grid");
    if (freeSurface && pml < SEIS2D_STENCIL_RADIUS)
        throw InvalidArgument("A free surface requires at least 4 top ghost rows");
}

void checkView(const seis2d_float_view& v) {
    if (v.size < 0 || (v.size > 0 && !v.data)) throw InvalidArgument("Simulation array view has no data");
}

// validateSimulationContext (Cuda_Check.cu:841-884), same checks in the same order.
void validate(const seis2d_context& c) {
    const std::size_t n = checkedCount(c.NX, c.NZ);
    checkBoundary(c.NX, c.NZ, c.npml, c.flag_type == 3 && c.upFlag);
    if (c.flag_type < 1 || c.flag_type > 3 || std::size_t(std::max(c.total_grid, 0)) != n || c.total_grid < 0 ||
        !std::isfinite(c.dt) || c.dt <= 0.0f || !std::isfinite(c.h) || c.h <= 0.0f || c.nt <= 0)
        throw InvalidArgument("Invalid solver, time grid, or spatial grid");
    for (const auto* v : {&c.rho, &c.mu, &c.lambda, &c.lambda2mu, &c.dp_flat, &c.dx, &c.dx_half, &c.dz, &c.dz_half,
                          &c.wavelet})
        checkView(*v);
    if (c.rcv_grid_idx.size < 0 || (c.rcv_grid_idx.size > 0 && !c.rcv_grid_idx.data))
        throw InvalidArgument("Simulation array view has no data");
    const int64_t count = int64_t(n);
    if (c.rho.size != count || c.mu.size != count || c.lambda.size != count || c.lambda2mu.size != count ||
        c.dx.size != c.NX || c.dx_half.size != c.NX || c.dz.size != c.NZ || c.dz_half.size != c.NZ ||
        (c.flag_type == 3 && c.dp_flat.size != c.NX) || c.wavelet.size < int64_t(c.nt) || c.num_rcv < 0 ||
        c.rcv_grid_idx.size != int64_t(c.num_rcv))
        throw InvalidArgument("Simulation array lengths do not match the grid or receiver count");
    float maximumVp = 0.0f;
    for (std::size_t k = 0; k < n; ++k) {
        const float rho = c.rho.data[k], mu = c.mu.data[k], lambda = c.lambda.data[k], l2m = c.lambda2mu.data[k];
        if (!std::isfinite(rho) || rho <= 0.0f || !std::isfinite(mu) || mu < 0.0f || !std::isfinite(lambda) ||
            !std::isfinite(l2m) || l2m <= 0.0f)
            throw InvalidArgument("Density/stiffness must be finite with rho > 0, mu >= 0, lambda2mu > 0");
        maximumVp = std::max(maximumVp, std::sqrt(l2m / rho));
        if (l2m - (4.0f / 3.0f) * mu <= 0.0f) throw InvalidArgument("Elastic bulk modulus must be positive");
    }
    if (!std::isfinite(maximumVp) || c.dt * maximumVp / c.h > kCourantLimit)
        throw InvalidArgument("The time step exceeds the 2D staggered-grid CFL limit");
    for (const auto* v : {&c.dx, &c.dx_half, &c.dz, &c.dz_half})
        for (int64_t q = 0; q < v->size; ++q)
            if (!std::isfinite(v->data[q]) || v->data[q] < 0.0f)
                throw InvalidArgument("PML damping must be finite and nonnegative");
    for (int r = 0; r < c.num_rcv; ++r)
        if (c.rcv_grid_idx.data[r] < 0 || c.rcv_grid_idx.data[r] >= c.total_grid)
            throw InvalidArgument("A receiver lies outside the simulation grid");
}

int kernelScheme(int flag, bool upFlag) {
    if (flag == 2) return kHybrid;
    return flag == 3 && upFlag ? kFree : kSplit;
}

}  // namespace

struct seis2d_session {
    Grid2D g{};
    int flag = 1;
    int upFlag = 0;
    int scheme = kSplit;
    Fields2D f{};
    float* field[SEIS2D_FIELD_COUNT] = {};
    cudaStream_t stream = nullptr;  // where work is enqueued (own stream, or the caller's)
    cudaStream_t own = nullptr;     // the session's non-blocking stream; graphs are captured on it
    std::vector<std::pair<void*, std::size_t>> allocations;
    Control2D* ctl = nullptr;
    float* series = nullptr;
    std::size_t seriesCapacity = 0;
    std::vector<float> seriesHost;
    bool seriesUploaded = false;
    int* rcvIdx = nullptr;
    float* stepVx = nullptr;
    float* stepVz = nullptr;
    int receiverCapacity = 0;
    seis2d_source* sources = nullptr;
    int* gatherIdx = nullptr;
    float* gatherVx = nullptr;
    float* gatherVz = nullptr;
    int gatherReceivers = 0, gatherStart = 0, gatherStride = 1, gatherSamples = 0, gatherTaken = 0;
    bool gatherOn = false;
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;  // (batch, with multi-source) -> graph
    GridSync* gridSync = nullptr;   // barrier state of the persistent runs
    int persistentBlocks = 0;       // co-resident blocks of the persistent kernel (0: not usable)
    int runMode = SEIS2D_RUN_GRAPH;
    bool persistentPending = false; // a persistent run has not been checked yet
    BarrierLimits barrier{kBarrierCycles, -1};   // seis2d_debug_barrier_wait
    uint64_t launches = 0;

    template <class T> T* alloc(std::size_t count) {
        void* p = nullptr;
        const std::size_t bytes = std::max<std::size_t>(count * sizeof(T), 16);
        cudaCheck(injectFailure() ? cudaErrorMemoryAllocation : cudaMalloc(&p, bytes), "cudaMalloc");
        allocations.emplace_back(p, bytes);
        cudaCheck(cudaMemsetAsync(p, 0, bytes, stream), "cudaMemset");
        return static_cast<T*>(p);
    }
    void free(void* p) {
        if (!p) return;
        for (auto it = allocations.begin(); it != allocations.end(); ++it)
            if (it->first == p) { allocations.erase(it); break; }
        cudaFree(p);
    }
    // The arrays of initialisation share one zeroed allocation (one cudaMalloc and one memset
    // instead of some thirty: the allocator's cost was most of a session's set-up time).
    // Each carved array keeps its own extent for the range checks of the device read/write
    // entry points, so a range that crosses from one array into the next is still refused.
    char* arena = nullptr;
    std::size_t arenaSize = 0, arenaUsed = 0;
    std::vector<std::pair<void*, std::size_t>> carved;
    template <class T> T* carve(std::size_t count) {
        const std::size_t bytes = std::max<std::size_t>(count * sizeof(T), 16);
        const std::size_t slot = (bytes + 255) & ~std::size_t(255);
        if (slot > arenaSize - arenaUsed) return alloc<T>(count);
        T* p = reinterpret_cast<T*>(arena + arenaUsed);
        arenaUsed += slot;
        carved.emplace_back(p, bytes);
        return p;
    }
    float* upload(const float* host, std::size_t count) {
        float* d = carve<float>(count);
        if (count) cudaCheck(cudaMemcpyAsync(d, host, count * sizeof(float), cudaMemcpyHostToDevice, stream), "upload");
        return d;
    }
    void sync() {
        cudaCheck(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        if (persistentPending) {
            persistentPending = false;
            GridSync state{};
            cudaCheck(cudaMemcpy(&state, gridSync, sizeof(state), cudaMemcpyDeviceToHost), "read run status");
            if (state.failed) throw RuntimeError("A persistent run gave up at a grid barrier; its results are invalid");
        }
    }
    ~seis2d_session() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        if (stream) cudaStreamSynchronize(stream);
        if (own && own != stream) cudaStreamSynchronize(own);
        for (auto& a : allocations) cudaFree(a.first);
        if (own) cudaStreamDestroy(own);
    }
};

namespace {

dim3 stressGrid(const Grid2D& g) { return dim3((g.NX + kBX - 1) / kBX, (g.NZ + kBY - 1) / kBY + 1); }
dim3 velocityGrid(const Grid2D& g) { return dim3((g.NX + kBX - 1) / kBX, (g.NZ + kBY - 1) / kBY); }
const dim3 kBlock(kBX, kBY);
constexpr int kSourceThreads = 256;
constexpr int kGraphBatch = 64;
static_assert(kSourceThreads >= SEIS2D_MAX_ACTIVE_SOURCES, "one thread per active source");

template <int S> void launchStress(seis2d_session* s, int slot) {
    stressStep<S><<<stressGrid(s->g), kBlock, 0, s->stream>>>(s->g, s->f, s->ctl, slot);
}
template <int S> void launchVelocity(seis2d_session* s, int slot) {
    velocityStep<S><<<velocityGrid(s->g), kBlock, 0, s->stream>>>(s->g, s->f, s->ctl, slot);
}
template <int S> void launchInject(seis2d_session* s) {
    injectSources<S><<<1, kSourceThreads, 0, s->stream>>>(s->g, s->f, s->ctl);
}
template <int S> void launchFinish(seis2d_session* s, int slot, int batch) {
    finishBatch<S><<<1, 256, 0, s->stream>>>(s->g, s->f, s->ctl, slot, batch);
}

template <class F> void dispatch(int scheme, F&& fn) {
    if (scheme == kHybrid) fn(std::integral_constant<int, kHybrid>{});
    else if (scheme == kFree) fn(std::integral_constant<int, kFree>{});
    else fn(std::integral_constant<int, kSplit>{});
}

// Enqueues `batch` steps (graph slots 0..batch-1) and the batch end.
void enqueueBatch(seis2d_session* s, int batch, bool multi) {
    dispatch(s->scheme, [&](auto tag) {
        constexpr int S = decltype(tag)::value;
        for (int slot = 0; slot < batch; ++slot) {
            launchStress<S>(s, slot);
            launchVelocity<S>(s, slot);
            if (multi) launchInject<S>(s);
        }
        launchFinish<S>(s, batch - 1, batch);
    });
    cudaCheck(cudaGetLastError(), "step kernel launch");
    s->launches += uint64_t(batch) * (multi ? 3 : 2) + 1;
}

// Blocks of the persistent kernel that fit on the device at once (cooperative launch bound).
template <int S> int residentBlocks() {
    int device = 0, sms = 0, perSm = 0;
    cudaCheck(cudaGetDevice(&device), "device");
    cudaCheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, runSteps<S>, kThreads, 0), "occupancy");
    return perSm * sms;
}

// One cooperative launch of `count` steps (after configure()).
void launchPersistent(seis2d_session* s, int count) {
    const int tiles = ((s->g.NX + kBX - 1) / kBX) * ((s->g.NZ + kBY - 1) / kBY);
    const int blocks = std::min(tiles, s->persistentBlocks);
    cudaCheck(cudaMemsetAsync(s->gridSync, 0, sizeof(GridSync), s->stream), "clear grid barrier");
    dispatch(s->scheme, [&](auto tag) {
        constexpr int S = decltype(tag)::value;
        void* args[] = {&s->g, &s->f, &s->ctl, &s->gridSync, &count, &s->barrier};
        cudaCheck(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(runSteps<S>), dim3(blocks), kBlock, args, 0,
                                              s->stream),
                  "persistent launch");
    });
    s->launches += 1;
    s->persistentPending = true;
}

cudaGraphExec_t batchGraph(seis2d_session* s, int batch, bool multi) {
    const auto key = std::make_pair(batch, int(multi));
    auto it = s->graphs.find(key);
    if (it != s->graphs.end()) return it->second;
    cudaGraph_t graph = nullptr;
    // Capture on the session's own stream (the work stream may be the legacy default
    // stream, which cannot be captured); the graph is launched on the work stream.
    const cudaStream_t work = s->stream;
    s->stream = s->own;
    cudaCheck(cudaStreamBeginCapture(s->own, cudaStreamCaptureModeThreadLocal), "begin capture");
    const uint64_t before = s->launches;
    try {
        enqueueBatch(s, batch, multi);
    } catch (...) {
        cudaStreamEndCapture(s->own, &graph);
        s->stream = work;
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    s->launches = before;
    s->stream = work;
    cudaCheck(cudaStreamEndCapture(s->own, &graph), "end capture");
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    cudaCheck(e, "graph instantiate");
    s->graphs.emplace(key, exec);
    return exec;
}

// Source series of the context: wavelet[it] * src_amp * kSourceInjectionScale2D, computed on
// the host in FP32 exactly as runGpuSimulationStep does (Cuda_Check.cu:1070-1071), for the
// steps that have a wavelet sample (it < nt and it < wavelet.size(), :1069).
int prepareSeries(seis2d_session* s, const seis2d_context& c) {
    if (c.wavelet.size < 0 || (c.wavelet.size > 0 && !c.wavelet.data))
        throw InvalidArgument("Simulation array view has no data");
    const int64_t length = std::max<int64_t>(0, std::min<int64_t>(c.nt, c.wavelet.size));
    std::vector<float> series(static_cast<std::size_t>(length));
    for (int64_t n = 0; n < length; ++n) series[n] = c.wavelet.data[n] * c.src_amp * SEIS2D_SOURCE_INJECTION_SCALE;
    const bool same = s->seriesUploaded && series.size() == s->seriesHost.size() &&
                      (series.empty() || std::memcmp(series.data(), s->seriesHost.data(), series.size() * 4) == 0);
    if (!same) {
        if (series.size() > s->seriesCapacity) {
            s->free(s->series);
            s->series = nullptr;
            s->seriesCapacity = 0;
            s->series = s->alloc<float>(series.size());
            s->seriesCapacity = series.size();
        }
        s->seriesHost = std::move(series);
        if (!s->seriesHost.empty())
            cudaCheck(cudaMemcpyAsync(s->series, s->seriesHost.data(), s->seriesHost.size() * 4, cudaMemcpyHostToDevice,
                                      s->stream),
                      "upload source series");
        // The pageable copy above is staged before it returns; the host vector stays as the cache.
        s->seriesUploaded = true;
    }
    return int(length);
}

// Control block of a run: the source index after the free-surface clamp of
// runGpuSimulationStep (Cuda_Check.cu:1073-1074) and the bounds checks of applyPointSource
// (:568-573), the receivers of the open gather and the multi-source mode.
Control2D runControl(seis2d_session* s, const seis2d_context& c, int first, int numActive, bool advance) {
    Control2D v{};
    v.base = first;
    v.srcSingle = numActive < 0;
    v.srcType = c.src_type;
    v.srcAngle = c.src_angle;
    v.series = s->series;
    if (numActive < 0) {
        v.srcLength = prepareSeries(s, c);
        v.series = s->series;
        const bool clamp = s->flag == 3 && s->upFlag;
        const int64_t z = clamp ? std::max<int64_t>(c.src_z_idx, s->g.fs + 1) : c.src_z_idx;
        const int64_t idx = z * s->g.NX + int64_t(c.src_idx % s->g.NX);
        bool valid = idx >= 0 && idx < s->g.total;
        if (valid) {
            const int x = int(idx % s->g.NX), zz = int(idx / s->g.NX);
            valid = x >= 4 && x < s->g.NX - 4 && zz >= 4 && zz < s->g.NZ - 4 && !(clamp && zz <= s->g.fs);
        }
        v.srcValid = valid;
        v.srcIdx = valid ? int(idx) : -1;
    } else {
        v.srcIdx = -1;
    }
    v.multiCount = std::max(numActive, 0);
    v.multiAdvance = advance;
    v.sources = s->sources;
    v.gatherOn = s->gatherOn;
    v.rcvCount = s->gatherOn ? s->gatherReceivers : 0;
    v.rcvIdx = s->gatherIdx;
    v.gatherVx = s->gatherVx;
    v.gatherVz = s->gatherVz;
    v.gatherStart = s->gatherStart;
    v.gatherStride = s->gatherStride;
    v.gatherSamples = s->gatherSamples;
    return v;
}

void noteGather(seis2d_session* s, int first, int count) {
    if (!s->gatherOn || count <= 0) return;
    const int64_t last = int64_t(first) + count - 1;
    if (last < s->gatherStart) return;
    int64_t sample = std::min<int64_t>((last - s->gatherStart) / s->gatherStride, s->gatherSamples - 1);
    if (int64_t(s->gatherStart) + sample * s->gatherStride < first) return;  // nothing recorded by this run
    s->gatherTaken = int(std::max<int64_t>(s->gatherTaken, sample + 1));
}

void configure(seis2d_session* s, const Control2D& v) {
    configureRun<<<1, 1, 0, s->stream>>>(s->ctl, v);
    cudaCheck(cudaGetLastError(), "configure run");
    s->launches += 1;
}

seis2d_session* checkedSession(seis2d_session* s) {
    if (!s) throw LogicError("The GPU simulation is not initialized");
    return s;
}

float* fieldPointer(seis2d_session* s, int field) {
    if (field < 0 || field >= SEIS2D_FIELD_COUNT) throw InvalidArgument("Unknown field index");
    float* p = s->field[field];
    if (!p) throw InvalidArgument("The field is not allocated for this solver scheme");
    return p;
}

// True when [p, p + bytes) lies inside one device allocation (any owner).
bool deviceRange(const void* p, std::size_t bytes) {
    using AddressRange = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
    static AddressRange range = nullptr;
    if (!range) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        cudaCheck(cudaGetDriverEntryPoint("cuMemGetAddressRange", &fn, cudaEnableDefault, &q), "driver entry point");
        if (!fn || q != cudaDriverEntryPointSuccess) throw RuntimeError("cuMemGetAddressRange is unavailable");
        range = reinterpret_cast<AddressRange>(fn);
    }
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) return false;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (range(&base, &size, CUdeviceptr(reinterpret_cast<uintptr_t>(p))) != CUDA_SUCCESS) return false;
    const uintptr_t a = reinterpret_cast<uintptr_t>(p), b = uintptr_t(base);
    return a >= b && bytes <= size && a - b <= size - bytes;
}

bool insideSession(const seis2d_session* s, const void* p, std::size_t bytes) {
    const auto a = reinterpret_cast<uintptr_t>(p);
    auto inside = [&](const std::pair<void*, std::size_t>& al) {
        const auto b = reinterpret_cast<uintptr_t>(al.first);
        return a >= b && bytes <= al.second && a - b <= al.second - bytes;
    };
    for (const auto& al : s->allocations)
        if (al.first != s->arena && inside(al)) return true;
    for (const auto& al : s->carved)
        if (inside(al)) return true;
    return false;
}

template <int S> void launchExtract(seis2d_session* s, int count) {
    extractReceivers<S><<<(count + 127) / 128, 128, 0, s->stream>>>(s->g, s->f, s->rcvIdx, count, s->stepVx, s->stepVz);
}

void extractStep(seis2d_session* s, int count, std::vector<float>& vx, std::vector<float>& vz) {
    dispatch(s->scheme, [&](auto tag) { launchExtract<decltype(tag)::value>(s, count); });
    cudaCheck(cudaGetLastError(), "receiver kernel launch");
    s->launches += 1;
    vx.resize(count);
    vz.resize(count);
    cudaCheck(cudaMemcpyAsync(vx.data(), s->stepVx, count * 4, cudaMemcpyDeviceToHost, s->stream), "receiver D2H");
    cudaCheck(cudaMemcpyAsync(vz.data(), s->stepVz, count * 4, cudaMemcpyDeviceToHost, s->stream), "receiver D2H");
    s->sync();
}

}  // namespace

extern "C" {

const char* seis2d_last_error(void) { return lastError.c_str(); }
int seis2d_abi_version(void) { return SEIS2D_ABI_VERSION; }

void seis2d_stencil_weights(double weights[4]) {
    if (weights) for (int q = 0; q < 4; ++q) weights[q] = kWeights[q];
}
float seis2d_courant_limit(void) { return kCourantLimit; }
float seis2d_safe_courant(void) { return kSafeCourant; }

int seis2d_checked_grid_element_count(int nx, int nz, int64_t* count) {
    return guarded([&] {
        const std::size_t n = checkedCount(nx, nz);
        if (count) *count = int64_t(n);
    });
}

int seis2d_validate_boundary_geometry(int nx, int nz, int pml_width, int free_surface) {
    return guarded([&] { checkBoundary(nx, nz, pml_width, free_surface != 0); });
}

// getReceiverSamplingStride (SolverNumerics.h:50-59).
int seis2d_receiver_sampling_stride(double time_step, double rate, int* stride) {
    return guarded([&] {
        if (!std::isfinite(time_step) || time_step <= 0.0 || !std::isfinite(rate) || rate <= 0.0)
            throw InvalidArgument("Sampling rate and simulation time step must be finite and positive");
        const double value = std::round(1.0 / (rate * time_step));
        if (!std::isfinite(value) || value > (std::numeric_limits<int>::max)())
            throw OverflowError("Receiver sampling stride is too large");
        if (stride) *stride = value < 1.0 ? 1 : static_cast<int>(value);
    });
}

// generateRickerWavelet (src/Seis2D/Numerics2D.inc:3-14).
int seis2d_generate_ricker(float* wavelet, int nt, float dt, float f0, float t0) {
    return guarded([&] {
        if (nt <= 0 || !std::isfinite(dt) || dt <= 0.0f || !std::isfinite(f0) || f0 <= 0.0f || !std::isfinite(t0))
            throw InvalidArgument("Invalid Ricker wavelet sampling or frequency");
        if (!wavelet) throw InvalidArgument("Invalid wavelet output buffer");
        for (int i = 0; i < nt; ++i) {
            const float t = i * dt - t0;
            const float pi2_f0 = kPi * kPi * f0 * f0;
            wavelet[i] = (1.0f - 2.0f * pi2_f0 * t * t) * std::exp(-pi2_f0 * t * t);
        }
    });
}

// updatePmlDampingArrays (src/Seis2D/Numerics2D.inc:36-83).
int seis2d_update_pml_damping(const seis2d_context* context, float* dx, float* dx_half, float* dz, float* dz_half) {
    return guarded([&] {
        if (!context || !dx || !dx_half || !dz || !dz_half) throw InvalidArgument("null argument");
        const seis2d_context& c = *context;
        checkBoundary(c.NX, c.NZ, c.npml, c.flag_type == 3 && c.upFlag);
        checkView(c.rho);
        checkView(c.lambda2mu);
        const int64_t n = int64_t(c.NX) * c.NZ;
        if (c.total_grid != n || c.rho.size != n || c.lambda2mu.size != n)
            throw InvalidArgument("Simulation array lengths do not match the grid or receiver count");
        float max_vp = 0.0f;
        for (int64_t k = 0; k < n; ++k) {
            const float vp = std::sqrt(c.lambda2mu.data[k] / c.rho.data[k]);
            if (vp > max_vp) max_vp = vp;
        }
        if (max_vp <= 350.0f) max_vp = 2000.0f;
        std::fill(dx, dx + c.NX, 0.0f);
        std::fill(dx_half, dx_half + c.NX, 0.0f);
        std::fill(dz, dz + c.NZ, 0.0f);
        std::fill(dz_half, dz_half + c.NZ, 0.0f);
        if (c.npml > 0) {
            const float L = c.npml * c.h;
            const float d_max = (3.0f * max_vp * 16.12f * 3.5f) / (2.0f * L);
            const float power = 2.5f;
            for (int i = 0; i < c.npml; ++i) {
                const float thick = (c.npml - i) / float(c.npml);
                float thick_half = (c.npml - (i + 0.5f)) / float(c.npml);
                if (thick_half < 0.0f) thick_half = 0.0f;
                const float val = d_max * std::pow(thick, power);
                const float val_half = d_max * std::pow(thick_half, power);
                dx[i] = val; dx[c.NX - 1 - i] = val;
                dx_half[i] = val_half; dx_half[c.NX - 1 - i] = val_half;
                dz[i] = val; dz[c.NZ - 1 - i] = val;
                dz_half[i] = val_half; dz_half[c.NZ - 1 - i] = val_half;
            }
        }
    });
}

// dp_flat of setupTestContext (src/Seis2D/Numerics2D.inc:124-135).
int seis2d_free_surface_modulus(const seis2d_context* context, float* dp_flat) {
    return guarded([&] {
        if (!context || !dp_flat) throw InvalidArgument("null argument");
        const seis2d_context& c = *context;
        checkView(c.lambda);
        checkView(c.lambda2mu);
        const int64_t n = int64_t(c.total_grid);
        if (c.NX <= 0 || c.lambda.size != n || c.lambda2mu.size != n)
            throw InvalidArgument("Simulation array lengths do not match the grid or receiver count");
        const int fs = c.npml;
        for (int j = 0; j < c.NX; ++j) {
            dp_flat[j] = 0.0f;
            const int64_t k = int64_t(fs) * c.NX + j;
            if (k >= 0 && k < n && c.lambda2mu.data[k] > 0.0f) {
                const float l2m = c.lambda2mu.data[k], lam = c.lambda.data[k];
                dp_flat[j] = (l2m * l2m - lam * lam) / l2m;
            }
        }
    });
}

int seis2d_validate_context(const seis2d_context* context) {
    return guarded([&] {
        if (!context) throw InvalidArgument("null context");
        validate(*context);
    });
}

void seis2d_release(seis2d_session* session) { delete session; }

// updateGpuReceivers (Cuda_Check.cu:992-1024): new buffers first, then the swap.
int seis2d_update_receivers(seis2d_session* session, const int* indices, int count) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (count < 0 || (count > 0 && !indices)) throw InvalidArgument("Too many receivers");
        for (int r = 0; r < count; ++r)
            if (indices[r] < 0 || indices[r] >= s->g.total)
                throw InvalidArgument("Receiver index is outside the active GPU grid");
        int* newIdx = nullptr;
        float* newVx = nullptr;
        float* newVz = nullptr;
        try {
            if (count > 0) {
                newIdx = s->alloc<int>(count);
                cudaCheck(cudaMemcpyAsync(newIdx, indices, std::size_t(count) * 4, cudaMemcpyHostToDevice, s->stream),
                          "receiver upload");
                newVx = s->alloc<float>(count);
                newVz = s->alloc<float>(count);
                s->sync();
            }
        } catch (...) {
            s->free(newIdx); s->free(newVx); s->free(newVz);
            throw;
        }
        s->sync();
        s->free(s->rcvIdx); s->free(s->stepVx); s->free(s->stepVz);
        s->rcvIdx = newIdx;
        s->stepVx = newVx;
        s->stepVz = newVz;
        s->receiverCapacity = count;
    });
}

// initializeGpuSimulation (Cuda_Check.cu:887-967).
int seis2d_initialize(seis2d_session** session, const seis2d_context* context) {
    return guarded([&] {
        if (!session || !context) throw InvalidArgument("null argument");
        const seis2d_context& c = *context;
        validate(c);
        seis2d_release(*session);
        *session = nullptr;
        auto* s = new seis2d_session;
        try {
            Grid2D& g = s->g;
            g.NX = c.NX; g.NZ = c.NZ; g.total = c.total_grid;
            g.npml = c.npml; g.fs = c.npml;
            g.dt = c.dt; g.inv_dt = 1.0f / c.dt;
            g.c1 = c.c1_h; g.c2 = c.c2_h; g.c3 = c.c3_h; g.c4 = c.c4_h;
            s->flag = c.flag_type;
            s->upFlag = c.upFlag != 0;
            s->scheme = kernelScheme(c.flag_type, s->upFlag);
            cudaCheck(cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking), "stream");
            s->stream = s->own;
            const std::size_t n = std::size_t(c.total_grid);
            {
                auto slot = [](std::size_t bytes) { return (std::max<std::size_t>(bytes, 16) + 255) & ~std::size_t(255); };
                const std::size_t volumes = 14 + (c.flag_type == 2 ? 11 : 0);
                const std::size_t lines = 4 + (c.flag_type == 3 ? 1 : 0);
                s->arenaSize = volumes * slot(n * sizeof(float)) +
                               lines * slot(std::size_t(std::max(c.NX, c.NZ)) * sizeof(float)) +
                               slot(SEIS2D_MAX_ACTIVE_SOURCES * sizeof(seis2d_source)) + slot(sizeof(Control2D)) +
                               slot(sizeof(GridSync));
                s->arena = s->alloc<char>(s->arenaSize);
            }
            Fields2D& f = s->f;
            float** splits[10] = {&f.vx1, &f.vx2, &f.vz1, &f.vz2, &f.sxx1, &f.sxx2, &f.szz1, &f.szz2, &f.sxz1, &f.sxz2};
            for (int q = 0; q < 10; ++q) s->field[q] = *splits[q] = s->carve<float>(n);
            f.rho = s->field[SEIS2D_RHO] = s->upload(c.rho.data, n);
            f.mu = s->field[SEIS2D_MU] = s->upload(c.mu.data, n);
            f.lambda = s->field[SEIS2D_LAMBDA] = s->upload(c.lambda.data, n);
            f.l2m = s->field[SEIS2D_LAMBDA2MU] = s->upload(c.lambda2mu.data, n);
            f.dx = s->upload(c.dx.data, c.NX);
            f.dxh = s->upload(c.dx_half.data, c.NX);
            f.dz = s->upload(c.dz.data, c.NZ);
            f.dzh = s->upload(c.dz_half.data, c.NZ);
            s->sources = s->carve<seis2d_source>(SEIS2D_MAX_ACTIVE_SOURCES);
            if (c.flag_type == 2) {
                float** totals[5] = {&f.vx, &f.vz, &f.sxx, &f.szz, &f.sxz};
                for (int q = 0; q < 5; ++q) s->field[SEIS2D_VX + q] = *totals[q] = s->carve<float>(n);
                // Staggered-point averages of the hybrid scheme (Cuda_Check.cu:922-939), FP32.
                std::vector<float> mu_x(n), lambda_x(n), l2m_x(n), mu_z(n), rho_xz(n), rho_orig(n);
                for (int i = 0; i < c.NZ; ++i)
                    for (int j = 0; j < c.NX; ++j) {
                        const std::size_t k = std::size_t(i) * c.NX + j;
                        rho_orig[k] = c.rho.data[k];
                        const std::size_t kx = j < c.NX - 1 ? k + 1 : k;
                        const std::size_t kz = i < c.NZ - 1 ? k + c.NX : k;
                        mu_x[k] = 0.5f * (c.mu.data[k] + c.mu.data[kx]);
                        lambda_x[k] = 0.5f * (c.lambda.data[k] + c.lambda.data[kx]);
                        l2m_x[k] = 0.5f * (c.lambda2mu.data[k] + c.lambda2mu.data[kx]);
                        mu_z[k] = 0.5f * (c.mu.data[k] + c.mu.data[kz]);
                        const std::size_t kd = (i < c.NZ - 1 && j < c.NX - 1) ? k + c.NX + 1 : k;
                        rho_xz[k] = 0.25f * (c.rho.data[k] + c.rho.data[kx] + c.rho.data[kz] + c.rho.data[kd]);
                    }
                f.muX = s->field[SEIS2D_MU_X_FLAT] = s->upload(mu_x.data(), n);
                f.lambdaX = s->field[SEIS2D_LAMBDA_X_FLAT] = s->upload(lambda_x.data(), n);
                f.l2mX = s->field[SEIS2D_LAMBDA2MU_X_FLAT] = s->upload(l2m_x.data(), n);
                f.muZ = s->field[SEIS2D_MU_Z_FLAT] = s->upload(mu_z.data(), n);
                f.rhoXZ = s->field[SEIS2D_RHO_X_Z_FLAT] = s->upload(rho_xz.data(), n);
                f.rhoOrig = s->field[SEIS2D_RHO_ORIG_FLAT] = s->upload(rho_orig.data(), n);
                s->sync();  // the host vectors die at the end of this scope
            }
            if (c.flag_type == 3) f.dp = s->upload(c.dp_flat.data, c.NX);
            s->ctl = s->carve<Control2D>(1);
            s->gridSync = s->carve<GridSync>(1);
            int cooperative = 0, device = 0;
            cudaCheck(cudaGetDevice(&device), "device");
            cudaCheck(cudaDeviceGetAttribute(&cooperative, cudaDevAttrCooperativeLaunch, device), "cooperative launch");
            if (cooperative) dispatch(s->scheme, [&](auto tag) { s->persistentBlocks = residentBlocks<decltype(tag)::value>(); });
            s->sync();
            *session = s;
            const int status = seis2d_update_receivers(s, c.rcv_grid_idx.data, c.num_rcv);
            if (status != SEIS2D_OK) throw RuntimeError(lastError);
        } catch (...) {
            *session = nullptr;
            delete s;
            throw;
        }
    });
}

int seis2d_set_active_sources(seis2d_session* session, const seis2d_source* sources, int count) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (count < 0 || count > SEIS2D_MAX_ACTIVE_SOURCES || (count > 0 && !sources))
            throw InvalidArgument("Active source capacity exceeded");
        if (count)
            cudaCheck(cudaMemcpyAsync(s->sources, sources, std::size_t(count) * sizeof(seis2d_source),
                                      cudaMemcpyHostToDevice, s->stream),
                      "active source upload");
        s->sync();
    });
}

// runGpuSimulationStep (Cuda_Check.cu:1027-1085).
int seis2d_run_step(seis2d_session* session, int current_it, const seis2d_context* context, int num_active_sources) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (!context) throw InvalidArgument("null context");
        if (s->g.total <= 0 || current_it < 0 || num_active_sources > SEIS2D_MAX_ACTIVE_SOURCES)
            throw InvalidArgument("Invalid GPU simulation state, iteration, or source count");
        configure(s, runControl(s, *context, current_it, num_active_sources, false));
        enqueueBatch(s, 1, num_active_sources > 0);
        noteGather(s, current_it, 1);
    });
}

int seis2d_run_steps(seis2d_session* session, int first_it, int count, const seis2d_context* context,
                     int num_active_sources) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (!context) throw InvalidArgument("null context");
        if (s->g.total <= 0 || first_it < 0 || count < 0 || num_active_sources > SEIS2D_MAX_ACTIVE_SOURCES ||
            int64_t(first_it) + count > (std::numeric_limits<int>::max)())
            throw InvalidArgument("Invalid GPU simulation state, iteration, or source count");
        if (count == 0) return;
        const bool multi = num_active_sources > 0;
        configure(s, runControl(s, *context, first_it, num_active_sources, num_active_sources >= 0));
        if (num_active_sources < 0 && s->runMode == SEIS2D_RUN_PERSISTENT && s->persistentBlocks > 0) {
            launchPersistent(s, count);
            noteGather(s, first_it, count);
            return;
        }
        int done = 0;
        while (done < count) {
            const int batch = std::min(kGraphBatch, count - done);
            cudaCheck(cudaGraphLaunch(batchGraph(s, batch, multi), s->stream), "graph launch");
            s->launches += uint64_t(batch) * (multi ? 3 : 2) + 1;
            done += batch;
        }
        noteGather(s, first_it, count);
    });
}

// copyWavefieldToHost (Cuda_Check.cu:1088-1103).
int seis2d_copy_wavefield(seis2d_session* session, float* host_vz) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (!host_vz || s->g.total <= 0) throw InvalidArgument("Invalid wavefield output buffer");
        const std::size_t n = std::size_t(s->g.total);
        if (s->flag == 1 || s->flag == 3) {
            std::vector<float> a(n), b(n);
            cudaCheck(cudaMemcpyAsync(a.data(), s->f.vz1, n * 4, cudaMemcpyDeviceToHost, s->stream), "wavefield D2H");
            cudaCheck(cudaMemcpyAsync(b.data(), s->f.vz2, n * 4, cudaMemcpyDeviceToHost, s->stream), "wavefield D2H");
            s->sync();
            for (std::size_t i = 0; i < n; ++i) host_vz[i] = a[i] + b[i];
        } else {
            cudaCheck(cudaMemcpyAsync(host_vz, s->f.vz, n * 4, cudaMemcpyDeviceToHost, s->stream), "wavefield D2H");
            s->sync();
        }
    });
}

// copyReceiverRecordsFromGpu (Cuda_Check.cu:1106-1135).
int seis2d_copy_receiver_records(seis2d_session* session, int num_rcv, int nt, int current_it, float* host_vx,
                                 float* host_vz) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (num_rcv <= 0) return;
        if (num_rcv > s->receiverCapacity || nt <= 0 || current_it < 0 || current_it >= nt || !host_vx || !host_vz)
            throw InvalidArgument("Invalid receiver trace count, time index, or host output buffer");
        std::vector<float> vx, vz;
        extractStep(s, num_rcv, vx, vz);
        for (int r = 0; r < num_rcv; ++r) {
            host_vx[std::size_t(r) * nt + current_it] = vx[r];
            host_vz[std::size_t(r) * nt + current_it] = vz[r];
        }
    });
}

// recordReceiverStepOnGpu (Cuda_Check.cu:1147-1169).
int seis2d_record_receiver_step(seis2d_session* session, int num_rcv, float* host_vx, float* host_vz) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (num_rcv <= 0) return;
        if (num_rcv > s->receiverCapacity || !host_vx || !host_vz)
            throw InvalidArgument("Invalid receiver count or host output buffer");
        std::vector<float> vx, vz;
        extractStep(s, num_rcv, vx, vz);
        std::copy(vx.begin(), vx.end(), host_vx);
        std::copy(vz.begin(), vz.end(), host_vz);
    });
}

int seis2d_gather_begin(seis2d_session* session, int capture_start_step, int stride, int samples) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (stride < 1 || samples < 1 || capture_start_step < 0)
            throw InvalidArgument("Recording stride, sample count and start step must be positive");
        if (s->receiverCapacity <= 0) throw InvalidArgument("Recording buffers do not match receiver channels");
        const std::size_t cells = std::size_t(s->receiverCapacity) * std::size_t(samples);
        s->free(s->gatherIdx); s->free(s->gatherVx); s->free(s->gatherVz);
        s->gatherIdx = nullptr; s->gatherVx = s->gatherVz = nullptr;
        s->gatherOn = false;
        s->gatherIdx = s->alloc<int>(s->receiverCapacity);
        s->gatherVx = s->alloc<float>(cells);
        s->gatherVz = s->alloc<float>(cells);
        cudaCheck(cudaMemcpyAsync(s->gatherIdx, s->rcvIdx, std::size_t(s->receiverCapacity) * 4,
                                  cudaMemcpyDeviceToDevice, s->stream),
                  "freeze receivers");
        s->sync();
        s->gatherReceivers = s->receiverCapacity;
        s->gatherStart = capture_start_step;
        s->gatherStride = stride;
        s->gatherSamples = samples;
        s->gatherTaken = 0;
        s->gatherOn = true;
    });
}

int seis2d_gather_fetch(seis2d_session* session, float* host_vx, float* host_vz, int samples, int* taken) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (!s->gatherOn) throw LogicError("No receiver gather is open");
        if (samples != s->gatherSamples || !host_vx || !host_vz)
            throw InvalidArgument("Recording buffers do not match receiver channels");
        const std::size_t bytes = std::size_t(s->gatherReceivers) * samples * 4;
        cudaCheck(cudaMemcpyAsync(host_vx, s->gatherVx, bytes, cudaMemcpyDeviceToHost, s->stream), "gather D2H");
        cudaCheck(cudaMemcpyAsync(host_vz, s->gatherVz, bytes, cudaMemcpyDeviceToHost, s->stream), "gather D2H");
        s->sync();
        if (taken) *taken = s->gatherTaken;
    });
}

int seis2d_gather_end(seis2d_session* session) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        s->sync();
        s->free(s->gatherIdx); s->free(s->gatherVx); s->free(s->gatherVz);
        s->gatherIdx = nullptr; s->gatherVx = s->gatherVz = nullptr;
        s->gatherOn = false;
        s->gatherReceivers = s->gatherSamples = s->gatherTaken = 0;
    });
}

int seis2d_get_views(seis2d_session* session, seis2d_device_views* views) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (!views) throw InvalidArgument("null views");
        seis2d_device_views v{};
        v.NX = s->g.NX; v.NZ = s->g.NZ; v.total_grid = s->g.total;
        v.dt = s->g.dt; v.inv_dt = s->g.inv_dt;
        v.flag_type = s->flag; v.npml = s->g.npml; v.fs_idx = s->g.fs; v.upFlag = s->upFlag;
        v.c1_h = s->g.c1; v.c2_h = s->g.c2; v.c3_h = s->g.c3; v.c4_h = s->g.c4;
        for (int q = 0; q < SEIS2D_FIELD_COUNT; ++q) v.field[q] = s->field[q];
        v.d_dx = const_cast<float*>(s->f.dx); v.d_dx_half = const_cast<float*>(s->f.dxh);
        v.d_dz = const_cast<float*>(s->f.dz); v.d_dz_half = const_cast<float*>(s->f.dzh);
        v.d_dp_flat = const_cast<float*>(s->f.dp);
        v.d_wavelet = s->series;
        v.d_rcv_grid_idx = s->rcvIdx;
        v.d_record_vx_step = s->stepVx; v.d_record_vz_step = s->stepVz;
        v.d_active_sources = s->sources;
        v.receiverCapacity = s->receiverCapacity;
        v.stream = s->stream;
        v.kernelLaunches = s->launches;
        *views = v;
    });
}

int seis2d_copy_field(seis2d_session* session, int field, float* host) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (!host) throw InvalidArgument("null output");
        float* p = fieldPointer(s, field);
        cudaCheck(cudaMemcpyAsync(host, p, std::size_t(s->g.total) * 4, cudaMemcpyDeviceToHost, s->stream), "field D2H");
        s->sync();
    });
}

int seis2d_set_field(seis2d_session* session, int field, const float* host) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (!host) throw InvalidArgument("null input");
        float* p = fieldPointer(s, field);
        cudaCheck(cudaMemcpyAsync(p, host, std::size_t(s->g.total) * 4, cudaMemcpyHostToDevice, s->stream), "field H2D");
        s->sync();
    });
}

int seis2d_write_device(seis2d_session* session, void* device_dst, const void* host_src, size_t bytes) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (!host_src || !insideSession(s, device_dst, bytes))
            throw InvalidArgument("The device range is not inside a buffer of this session");
        cudaCheck(cudaMemcpyAsync(device_dst, host_src, bytes, cudaMemcpyHostToDevice, s->stream), "device write");
        s->sync();
    });
}

int seis2d_read_device(seis2d_session* session, void* host_dst, const void* device_src, size_t bytes) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (!host_dst || !insideSession(s, device_src, bytes))
            throw InvalidArgument("The device range is not inside a buffer of this session");
        cudaCheck(cudaMemcpyAsync(host_dst, device_src, bytes, cudaMemcpyDeviceToHost, s->stream), "device read");
        s->sync();
    });
}

int seis2d_wavefield_texture(seis2d_session* session, void* device_rgba, float color_scale, int component) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        const std::size_t bytes = std::size_t(s->g.total) * 4;
        if (!device_rgba || reinterpret_cast<uintptr_t>(device_rgba) % 4 != 0 || !deviceRange(device_rgba, bytes))
            throw InvalidArgument("The texture must be a device buffer of NX * NZ RGBA8 pixels");
        const Fields2D& f = s->f;
        const ColorFields c{f.vx1, f.vx2, f.vz1, f.vz2, f.sxx1, f.sxx2, f.szz1, f.szz2, f.sxz1, f.sxz2,
                            f.vx,  f.vz,  f.sxx, f.szz, f.sxz, f.mu,   f.l2m};
        // Fields a scheme does not allocate are never read: the split halves exist for every
        // scheme and the totals only where flag_type 2 (or an unknown id) selects them.
        if (!(s->flag == 1 || s->flag == 3) && !f.vx) throw InvalidArgument("The total fields are not allocated");
        const dim3 block(32, 8), grid(unsigned((s->g.NX + 31) / 32), unsigned((s->g.NZ + 7) / 8));
        colorMap<<<grid, block, 0, s->stream>>>(c, s->g.NX, s->g.NZ, s->flag, static_cast<uchar4*>(device_rgba),
                                               color_scale, component);
        cudaCheck(cudaGetLastError(), "color map");
        ++s->launches;
    });
}

void seis2d_debug_fail_allocation(int nth) { failAllocation.store(nth > 0 ? nth : 0); }

int seis2d_debug_barrier_wait(seis2d_session* session, long long cycles, int withheld_block) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (cycles < 0 || withheld_block < -1) throw InvalidArgument("Invalid barrier-wait test settings");
        s->barrier.cycles = cycles ? cycles : kBarrierCycles;
        s->barrier.withheldBlock = withheld_block;
    });
}

int seis2d_synchronize(seis2d_session* session) {
    return guarded([&] { checkedSession(session)->sync(); });
}

int seis2d_set_run_mode(seis2d_session* session, int mode) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (mode != SEIS2D_RUN_PERSISTENT && mode != SEIS2D_RUN_GRAPH) throw InvalidArgument("Unknown run mode");
        s->runMode = mode;
    });
}

int seis2d_set_stream(seis2d_session* session, void* stream) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        s->sync();
        s->stream = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
    });
}

int seis2d_profile_steps(seis2d_session* session, int first_it, int count, const seis2d_context* context, float ms[3]) {
    return guarded([&] {
        seis2d_session* s = checkedSession(session);
        if (!context || !ms || count <= 0 || first_it < 0) throw InvalidArgument("invalid profile request");
        configure(s, runControl(s, *context, first_it, -1, false));
        std::vector<cudaEvent_t> ev(std::size_t(count) * 3 + 1);
        for (auto& e : ev) cudaCheck(cudaEventCreate(&e), "event");
        try {
            dispatch(s->scheme, [&](auto tag) {
                constexpr int S = decltype(tag)::value;
                for (int q = 0; q < count; ++q) {
                    // Each step is its own batch of one, so slot 0 and the batch end keep the
                    // field state of the reference after every step.
                    cudaEventRecord(ev[3 * q], s->stream);
                    launchStress<S>(s, 0);
                    cudaEventRecord(ev[3 * q + 1], s->stream);
                    launchVelocity<S>(s, 0);
                    cudaEventRecord(ev[3 * q + 2], s->stream);
                    launchFinish<S>(s, 0, 1);
                }
            });
            cudaEventRecord(ev.back(), s->stream);
            cudaCheck(cudaGetLastError(), "profile launch");
            s->launches += uint64_t(count) * 3;
            s->sync();
            float total = 0, stress = 0, velocity = 0, t = 0;
            cudaCheck(cudaEventElapsedTime(&total, ev[0], ev.back()), "elapsed");
            for (int q = 0; q < count; ++q) {
                cudaEventElapsedTime(&t, ev[3 * q], ev[3 * q + 1]); stress += t;
                cudaEventElapsedTime(&t, ev[3 * q + 1], ev[3 * q + 2]); velocity += t;
            }
            ms[0] = total; ms[1] = stress; ms[2] = velocity;
        } catch (...) {
            for (auto& e : ev) cudaEventDestroy(e);
            throw;
        }
        for (auto& e : ev) cudaEventDestroy(e);
    });
}

}  // extern "C"
