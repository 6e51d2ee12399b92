// noalloc.cu -- sort + unique of a board set without any device allocation.
//
// Some callers cannot let a library allocate device memory: a host that owns
// the whole GPU through its own caching allocator with a hard budget (a
// framework process, a plugin inside a serving system), or latency-sensitive
// code that cannot afford cudaMalloc's implicit device-wide synchronisation.
// cgb_sort_unique_noalloc serves them: it runs the same histogram, onesweep
// digit-pass and unique kernels as cgb_sort/cgb_unique, but all of its
// scratch (the ping-pong key buffer, digit histograms, tile counters,
// look-back state, error word and count) lives in one file-scope
// __device__ array of fixed size (a little over 8 MiB).
//
// Limits and rules of use:
//  * at most CGB_NOALLOC_MAX_KEYS (2^20) keys per call; larger inputs are
//    rejected with an error, nothing is launched;
//  * set-up: the first call on a device resolves the array's device address
//    with cudaGetSymbolAddress (with that device current) and caches it.  The
//    CUDA runtime loads this file's device code lazily, so that first call is
//    also when the driver places the array on the GPU -- the one moment it
//    allocates device memory and may synchronise the device.  A call with
//    n = 0 does only this set-up: make it once per device outside any
//    budgeted or latency-sensitive region and before any stream capture.
//    From then on every GPU that was set up holds the array until the
//    process exits;
//  * every call on a device shares the one array and leaves its contents
//    behind; the call clears what must start at zero, but two calls whose
//    work overlaps on the GPU (other host threads, other streams) race on
//    it -- serialise them.
//  * the call returns when its work on `stream` is complete.
#include "common.cuh"
#include <cuda_runtime.h>
#include <mutex>

namespace cgb {

// kernels and tile shapes shared with sort.cu (SORT_THREADS=256 x 16 keys,
// UNQ_THREADS=256 x 16 keys)
__global__ void digit_histogram_kernel(const u64 *__restrict__ keys, u64 n, u32 *__restrict__ hist);
__global__ void onesweep_kernel(const u64 *__restrict__ src, u64 *__restrict__ dst, u32 n, int shift,
                                const u32 *__restrict__ digit_hist, u32 *lookback, u32 *tile_counter, u32 *err);
__global__ void unique_kernel(const u64 *__restrict__ in, u32 n, u64 *__restrict__ out, u32 *lookback,
                              u32 *tile_counter, u32 *out_count, u32 *err, unsigned long long *empties);
int sort_plan(const u32 *hist_host, u64 n, int *digits);

namespace noalloc {

constexpr u64 MAX_KEYS = 1ull << 20;
constexpr u64 TILE = 4096;                     // keys per onesweep / unique tile
constexpr u64 MAX_TILES = MAX_KEYS / TILE;     // 256
constexpr u64 HIST_WORDS = 8 * 256;            // u32: eight digit histograms
constexpr u64 CTR_WORDS = 16;                  // u32: per-pass tile counters
constexpr u64 LB_WORDS = MAX_TILES * 256;      // u32: look-back state of one pass
// layout in u32 words after the key buffer
constexpr u64 OFF_HIST = 0, OFF_CTR = OFF_HIST + HIST_WORDS, OFF_ERR = OFF_CTR + CTR_WORDS,
              OFF_COUNT = OFF_ERR + 1, OFF_LB = OFF_COUNT + 15, STATE_WORDS = OFF_LB + LB_WORDS;
constexpr u64 ARRAY_WORDS64 = MAX_KEYS + (STATE_WORDS + 1) / 2;

static __device__ __align__(256) u64 scratch[ARRAY_WORDS64];

static std::mutex g_mu;
static u64 *g_addr[64];  // device address of `scratch`, per device ordinal

static bool scratch_address(u64 **out)
{
    int dev = 0;
    if (!CGB_CUDA(cudaGetDevice(&dev))) return false;
    if (dev < 0 || dev >= 64) {
        set_error("cgb_sort_unique_noalloc: device ordinal out of range");
        return false;
    }
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        if (!CGB_CUDA(cudaGetSymbolAddress(&p, scratch))) return false;
        g_addr[dev] = (u64 *)p;
    }
    *out = g_addr[dev];
    return true;
}

}  // namespace noalloc
}  // namespace cgb

using namespace cgb;

extern "C" int cgb_sort_unique_noalloc(const uint64_t *d_in, uint64_t n, uint64_t *d_out, uint64_t *n_out,
                                       void *stream)
{
    using namespace cgb::noalloc;
    if (n_out) *n_out = 0;
    if (n > MAX_KEYS) {
        char buf[160];
        snprintf(buf, sizeof buf, "cgb_sort_unique_noalloc: %llu keys exceed the fixed scratch of %llu keys",
                 (unsigned long long)n, (unsigned long long)MAX_KEYS);
        set_error(buf);
        return -1;
    }
    u64 *base = nullptr;
    if (!scratch_address(&base)) return -1;  // the set-up; n = 0 stops after it
    if (n == 0) return 0;
    if (!d_in || !d_out || !n_out) {
        set_error("cgb_sort_unique_noalloc: null pointer");
        return -1;
    }
    cudaStream_t s = (cudaStream_t)stream;
    u64 *keys_tmp = base;                             // MAX_KEYS keys
    u32 *state = (u32 *)(base + MAX_KEYS);
    u32 *hist = state + OFF_HIST, *ctr = state + OFF_CTR, *err = state + OFF_ERR, *count = state + OFF_COUNT;
    u32 *lookback = state + OFF_LB;
    const u32 tiles = (u32)((n + TILE - 1) / TILE);

    // zero what accumulates: histograms, counters, error word, count
    if (!CGB_CUDA(cudaMemsetAsync(state, 0, OFF_LB * sizeof(u32), s))) return -1;
    const int hist_blocks = (int)std::min<u64>((n + 255) / 256, (u64)NUM_SMS_B200 * 8);
    digit_histogram_kernel<<<hist_blocks, 256, 0, s>>>(d_in, n, hist);
    if (!CGB_CUDA(cudaGetLastError())) return -1;
    u32 h[8 * 256];
    if (!CGB_CUDA(cudaMemcpyAsync(h, hist, sizeof h, cudaMemcpyDeviceToHost, s))) return -1;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return -1;
    int digits[8];
    const int np = sort_plan(h, n, digits);

    // ping-pong between d_out and the scratch buffer so that the last pass
    // lands in scratch; unique then writes d_out
    const u64 *src = d_in;
    for (int p = 0; p < np; p++) {
        u64 *dst = ((np - p) % 2 == 1) ? keys_tmp : d_out;
        if (!CGB_CUDA(cudaMemsetAsync(lookback, 0, (u64)tiles * 256 * sizeof(u32), s))) return -1;
        onesweep_kernel<<<tiles, 256, 0, s>>>(src, dst, (u32)n, 8 * digits[p], hist + digits[p] * 256, lookback,
                                              ctr + p, err);
        if (!CGB_CUDA(cudaGetLastError())) return -1;
        src = dst;
    }
    if (!CGB_CUDA(cudaMemsetAsync(lookback, 0, (u64)tiles * sizeof(u32), s))) return -1;
    unique_kernel<<<tiles, 256, 0, s>>>(src, (u32)n, d_out, lookback, ctr + 8, count, err, nullptr);
    if (!CGB_CUDA(cudaGetLastError())) return -1;
    u32 res[2];
    if (!CGB_CUDA(cudaMemcpyAsync(res, err, 2 * sizeof(u32), cudaMemcpyDeviceToHost, s))) return -1;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return -1;
    if (res[0]) {
        set_error("cgb_sort_unique_noalloc: device error " + err_string(res[0]));
        return -1;
    }
    *n_out = res[1];
    return 0;
}
