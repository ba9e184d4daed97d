// seis3d_noalloc.cu - receiver sampling that allocates no memory.
//
// Some callers cannot call cudaMalloc while they run the solver: a host that hands every
// byte of device memory to its own pool allocator up front, code that runs between the
// steps of a latency-critical loop where an allocation (and the device synchronisation
// it may imply) is not allowed, or a plugin that is only lent the wavefield buffers of
// another owner.  seis3d_sample_receivers_noalloc serves them: it reads the collocated
// receiver velocities straight from caller-owned velocity fields, using as its only
// device scratch the file-scope array below, and allocates nothing (no cudaMalloc,
// cudaFree, pinned host memory or allocating library call).
#include "../../include/seis3d_capi.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

namespace {

// Device scratch shared by every call on a device: receiver grid positions followed by
// the gathered [receiver][vx, vy, vz] values.  8,400 bytes; every GPU that loads this
// library holds it until the process exits.
constexpr int kMaxReceivers = SEIS3D_NOALLOC_MAX_RECEIVERS;
constexpr std::size_t kPositionBytes = std::size_t(kMaxReceivers) * sizeof(int4);
constexpr std::size_t kScratchBytes = kPositionBytes + std::size_t(kMaxReceivers) * 3 * sizeof(float);
static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

// Host-side device addresses of g_noallocScratch, looked up once per device.  In host
// code the symbol itself is only a stand-in, not a device address.
constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
unsigned char* g_scratchAddress[kMaxDevices] = {};

thread_local std::string g_error;

int fail(int status, const char* message) {
    g_error = message;
    return status;
}

// Collocated velocities at the receivers (the same arithmetic as sampleScalar3D,
// cuda/Cuda_Seis3D.cu:341-343): vx = (vx[i] + vx[i-1]) / 2, vy with i - pitch, vz with
// i - plane.
__global__ void gatherReceivers(const float* vx, const float* vy, const float* vz, int64_t pitch, int64_t plane,
                                const int4* positions, int count, float* out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= count) return;
    const int4 p = positions[r];
    const int64_t i = int64_t(p.z) * plane + int64_t(p.y) * pitch + p.x;
    out[3 * r + 0] = 0.5f * (vx[i] + vx[i - 1]);
    out[3 * r + 1] = 0.5f * (vy[i] + vy[i - pitch]);
    out[3 * r + 2] = 0.5f * (vz[i] + vz[i - plane]);
}

}  // namespace

extern "C" {

const char* seis3d_noalloc_last_error(void) { return g_error.c_str(); }

int seis3d_sample_receivers_noalloc(const seis3d_context* c, const float* vx, const float* vy, const float* vz,
                                    int64_t pitch, const seis3d_receiver* receivers, int count, float* values,
                                    void* stream) {
    if (!c || !vx || !vy || !vz || (count && (!receivers || !values)))
        return fail(SEIS3D_INVALID_ARGUMENT, "Seis3D no-alloc sampling: null argument.");
    if (count < 0 || count > kMaxReceivers)
        return fail(SEIS3D_INVALID_ARGUMENT,
                    "Seis3D no-alloc sampling: receiver count must be 0..300 (the size of its static scratch).");
    if (c->gx3D <= 8 || c->gy3D <= 8 || c->gz3D <= 8 || pitch < c->gx3D)
        return fail(SEIS3D_INVALID_ARGUMENT, "Seis3D no-alloc sampling: context not validated or pitch < gx.");
    // The collocation reads one node below each receiver along every axis, so each offset
    // must be at least 1 and the physical box must lie inside the padded grid.
    if (c->nx3D < 1 || c->ny3D < 1 || c->nz3D < 1 || c->ox3D < 1 || c->oy3D < 1 || c->oz3D < 1 ||
        int64_t(c->ox3D) + c->nx3D > c->gx3D || int64_t(c->oy3D) + c->ny3D > c->gy3D ||
        int64_t(c->oz3D) + c->nz3D > c->gz3D)
        return fail(SEIS3D_INVALID_ARGUMENT,
                    "Seis3D no-alloc sampling: context offsets and sizes do not fit the padded grid.");
    int4 positions[kMaxReceivers];
    for (int r = 0; r < count; ++r) {
        const seis3d_receiver p = receivers[r];
        if (p.x3D < 0 || p.x3D >= c->nx3D || p.y3D < 0 || p.y3D >= c->ny3D || p.z3D < 0 || p.z3D >= c->nz3D)
            return fail(SEIS3D_INVALID_ARGUMENT, "Seis3D no-alloc sampling: receiver outside the physical domain.");
        positions[r] = make_int4(p.x3D + c->ox3D, p.y3D + c->oy3D, p.z3D + c->oz3D, 0);
    }
    if (count == 0) return SEIS3D_OK;

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
        return fail(SEIS3D_RUNTIME_ERROR, "Seis3D no-alloc sampling: no usable current CUDA device.");
    unsigned char* scratch = nullptr;
    {
        // Set-up once per device, with that device current: resolve the device address
        // of the static scratch array.
        std::lock_guard<std::mutex> lock(g_setupMutex);
        if (!g_scratchAddress[device]) {
            void* address = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&address, g_noallocScratch);
            if (e != cudaSuccess || !address) {
                g_error = std::string("Seis3D no-alloc sampling: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
                return SEIS3D_RUNTIME_ERROR;
            }
            g_scratchAddress[device] = static_cast<unsigned char*>(address);
        }
        scratch = g_scratchAddress[device];
    }
    int4* devPositions = reinterpret_cast<int4*>(scratch);
    float* devValues = reinterpret_cast<float*>(scratch + kPositionBytes);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t plane = pitch * c->gy3D;

    // Every entry the kernel reads (positions) is written first and every value read back
    // is written by the kernel, so nothing in the scratch has to start at zero.
    cudaError_t e = cudaMemcpyAsync(devPositions, positions, std::size_t(count) * sizeof(int4), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        gatherReceivers<<<(count + 127) / 128, 128, 0, s>>>(vx, vy, vz, pitch, plane, devPositions, count, devValues);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(values, devValues, std::size_t(count) * 3 * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        g_error = std::string("Seis3D no-alloc sampling: ") + cudaGetErrorString(e);
        return SEIS3D_RUNTIME_ERROR;
    }
    return SEIS3D_OK;
}

}  // extern "C"
