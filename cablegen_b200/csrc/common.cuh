// common.cuh -- shared host/device helpers of the engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>
#include <vector>

namespace cgb {

typedef uint64_t u64;
typedef unsigned int u32;

// Device error word bits.  Every kernel that can fail ORs a bit into a
// device-resident word that the host reads after each phase; nothing traps.
enum : u32 {
    ERR_LOOKBACK_TIMEOUT = 1u << 0,   // a decoupled look-back wait ran out
    ERR_CAPACITY = 1u << 1,           // an output would exceed its buffer
    ERR_UNSORTED = 1u << 2,           // an input that must be sorted was not
    ERR_TOO_LARGE = 1u << 3,          // a size beyond a kernel's 32-bit counters
    ERR_COPY_TIMEOUT = 1u << 4,       // a bulk copy into shared memory did not complete
};

// Bounded spin: a wait on another CTA gives up after this many polls.
constexpr u32 SPIN_LIMIT = 1u << 22;

constexpr int NUM_SMS_B200 = 148;

std::string err_string(u32 err);

// record the first CUDA error of an API call; returns false on failure
bool cuda_ok(cudaError_t e, const char *what, const char *file, int line);
#define CGB_CUDA(call) ::cgb::cuda_ok((call), #call, __FILE__, __LINE__)

void set_error(const std::string &msg);
const char *last_error();

// Per-kernel device time and algorithmic bytes, accumulated over launches.
// Launch time comes from CUDA events recorded around each launch on the
// launching stream and resolved at the next host synchronisation point.
struct KernelStats {
    u64 launches = 0;
    double hist_ms = 0, onesweep_ms = 0, unique_ms = 0, merge_ms = 0, expand_ms = 0, spawn_ms = 0,
           solve_ms = 0, index_ms = 0;
    u64 hist_bytes = 0, onesweep_bytes = 0, unique_bytes = 0, merge_bytes = 0, expand_bytes = 0,
        spawn_bytes = 0, solve_bytes = 0;
    u64 onesweep_launches = 0, solve_launches = 0, solve_boards = 0, lookups = 0;
    u64 index_builds = 0, compact_index_builds = 0;
    u64 moves_raw = 0, moves_kept = 0;  // move results before / after the per-block set
    u64 pool_trims = 0;  // failed allocations that returned the pool's cache to the device
};
KernelStats &kstats();

class KClock {
  public:
    void begin(cudaStream_t s, double *acc);
    void end(cudaStream_t s);
    void flush();  // call after the stream has been synchronised
  private:
    struct Pending {
        cudaEvent_t a, b;
        double *acc;
    };
    cudaEvent_t take();
    std::vector<cudaEvent_t> free_;
    std::vector<Pending> pend_;
    cudaEvent_t open_ = nullptr;
    double *open_acc_ = nullptr;
};
KClock &kclock();

#ifdef __CUDACC__
__device__ __forceinline__ u32 ld_acquire(const u32 *p)
{
    u32 v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(u32 *p, u32 v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// relaxed (non-caching) accesses: enough when the word carries its own flag
__device__ __forceinline__ u32 ld_relaxed(const u32 *p)
{
    u32 v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(u32 *p, u32 v)
{
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ u64 ld_acquire64(const u64 *p)
{
    u64 v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release64(u64 *p, u64 v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ u32 lanemask_lt()
{
    u32 m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// inclusive warp scan
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// exclusive block scan of one value per thread (blockDim.x a multiple of 32,
// at most 1024); `scratch` holds 33 T.  Returns the exclusive prefix and the
// block total in *total.  Contains __syncthreads().
template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *scratch, T *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    T inc = warp_inclusive_scan(v);
    if (lane == 31) scratch[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nwarps ? scratch[lane] : T(0);
        T wi = warp_inclusive_scan(w);
        scratch[lane] = wi - w;
        if (lane == 31) scratch[32] = wi;
    }
    __syncthreads();
    *total = scratch[32];
    T r = scratch[warp] + inc - v;
    __syncthreads();
    return r;
}
#endif


// ---- shared-memory barriers and bulk async copies (sm_90+) -----------------
// One-dimensional global -> shared bulk copies completed on an mbarrier: the
// copying thread announces the byte count (expect_tx), the copy engine
// decrements it, waiters poll the phase parity.  No multicast forms.
__device__ __forceinline__ u32 smem_addr(const void *p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, u32 count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// make barrier initialisation and earlier generic-proxy shared accesses
// visible to the async proxy before a bulk copy is issued
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, u32 bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}"
                 ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// bytes: multiple of 16; both addresses 16-byte aligned
__device__ __forceinline__ void bulk_load(void *dst_smem, const void *src_gmem, u32 bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_addr(dst_smem)), "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, u32 parity)
{
    u32 ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// bounded wait for the phase of the given parity; false (and ERR_COPY_TIMEOUT
// in *err) if it did not complete within SPIN_LIMIT polls
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, u32 parity, u32 *err)
{
    for (u32 spins = 0; !mbar_try_wait(bar, parity); spins++) {
        if (spins > SPIN_LIMIT) {
            atomicOr(err, ERR_COPY_TIMEOUT);
            return false;
        }
    }
    return true;
}

}  // namespace cgb
