// seis3d_tma.cuh - Tensor Memory Accelerator staging for the z-marching passes (sm_100a).
//
// Each CTA streams the planes of its column tile through a ring of kStages shared-memory
// stages.  One elected thread fills a stage with cp.async.bulk.tensor tile copies whose
// completion is tracked by the stage's mbarrier (expect-tx bytes); every thread waits on
// that mbarrier before reading the stage.  Waits are bounded: a stage that does not
// arrive within the session's wait limit (~2 s of SM clock by default) sets a stall flag
// that the host reports, and the CTA drains its in-flight copies (again bounded) and
// exits.  No cluster multicast is used.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace seis3d {
namespace tma {

constexpr int kStages = 3;

constexpr long long kWaitCycles = 4000000000LL;   // default wait limit, ~2 s at 1.9 GHz

// Tensor-map table (one CUtensorMap per array and box shape), kept in global memory.
enum MapIndex : int {
    kCenter0 = 0,        // 0..8: field k, 32 x TY box; 9 = 1/rho, 10 = lambda, 11 = mu
    kSxxX = 12,          // sigma_xx, (32+8) x TY (x halo)
    kSxzX = 13,          // sigma_xz, (32+8) x TY
    kSxyXY = 14,         // sigma_xy, (32+8) x (TY+8)
    kSyyY = 15,          // sigma_yy, 32 x (TY+8)
    kSyzY = 16,          // sigma_yz, 32 x (TY+8)
    kVxXY = 17,          // vx, vy, vz: (32+8) x (TY+8)
    kVyXY = 18,
    kVzXY = 19,
    kRhoT = 20,          // 1/rho, 36 x (TY+1)
    kMuT = 21,           // mu, 36 x (TY+1)
    kMapCount = 22
};

__device__ __forceinline__ uint32_t smemAddress(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void barrierInit(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddress(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void barrierInitFence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void arriveExpectTx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddress(bar)), "r"(bytes)
                 : "memory");
}

// Test the phase; if it is incomplete the thread may be suspended for a short,
// system-defined time before the instruction returns.  (A long explicit suspend-time hint
// measured 30 % slower on B200: suspended warps resume late after the phase completes.)
__device__ __forceinline__ bool tryWait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smemAddress(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait of at most `limit` SM cycles on one stage; returns false when it timed out.
__device__ __forceinline__ bool waitStage(uint64_t* bar, uint32_t parity, long long limit) {
    if (tryWait(bar, parity)) return true;
    const long long start = clock64();
    while (!tryWait(bar, parity))
        if (clock64() - start > limit) return false;
    return true;
}

// Order this thread's earlier generic-proxy shared-memory accesses before its later
// async-proxy (TMA) accesses.
__device__ __forceinline__ void fenceProxyAsync() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One 3-D tile copy global -> shared, completing on `bar`.
__device__ __forceinline__ void load3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smemAddress(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smemAddress(bar))
        : "memory");
}

}  // namespace tma
}  // namespace seis3d
