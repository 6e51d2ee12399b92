// solve.cu -- backward expectimax over one layer (src/solve.c:226-302).
//
// One thread per board of layer s:
//   * satisfied (src/solve.c:233-244): with nox the board wins (1.0) when it
//     holds tile nox; otherwise when it matches any winstate image.
//   * otherwise expectimax (src/solve.c:257-281): for every empty cell in
//     cell order 0..15, a 2 (weight 0.9) and a 4 (weight 0.1) are placed; the
//     value of each spawn is the best of the four moves (src/solve.c:246-256),
//     each successor looked up, canonicalised, in the s+2 / s+4 table; a miss
//     is 0.0 (src/solve.c:108-164).  res = 0.9*S2/k + 0.1*S4/k.
//
// The FP64 kernel evaluates exactly the reference's operation sequence with
// round-to-nearest intrinsics (no FMA contraction), so its values are
// bit-identical.  The FP32 kernel keeps tables in FP32, accumulates the two
// spawn sums with Kahan compensation, and forms the final weighted mean in
// FP64 before rounding once to FP32 (a 0.9f weight would bias every layer by
// 2.6e-8 relative).
#include "engine.h"

namespace cgb {

constexpr int SOLVE_THREADS = 512;
constexpr int TABLE_BYTES_S = 65536 * 2 + 2048 * 4;

// ---- lookup ---------------------------------------------------------------
template <typename V>
struct DevTable {
    const u64 *keys;
    const V *vals;
    u64 n;
    const u32 *bucket;  // optional bucket offsets over the bits after the prefix
    int prefix, bits;
    u64 prefix_value;
};

template <typename V>
__device__ __forceinline__ V table_lookup(const DevTable<V> &t, u64 key)
{
    if (t.n == 0) return V(0);
    u64 lo = 0, len = t.n;
    if (t.bucket) {
        if (t.prefix > 0 && (key >> (64 - t.prefix)) != t.prefix_value) return V(0);
        const u32 bk = (u32)((key << t.prefix) >> (64 - t.bits));
        const u32 b0 = __ldg(t.bucket + bk), b1 = __ldg(t.bucket + bk + 1);
        lo = b0;
        len = b1 - b0;
        if (len == 0) return V(0);
    }
    while (len > 1) {
        const u64 half = len >> 1;
        lo = (__ldg(t.keys + lo + half) <= key) ? lo + half : lo;
        len -= half;
    }
    return __ldg(t.keys + lo) == key ? __ldg(t.vals + lo) : V(0);
}

__device__ __forceinline__ double vmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }

// best of the four moves of b, successors looked up canonicalised
template <typename V>
__device__ __forceinline__ V best_move(const RowTable &rt, u64 b, const DevTable<V> &t, u32 &probes)
{
    u64 v[4];
    views(b, v);
    V p[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        u64 m;
        const bool legal = move_left(rt, v[k], &m) == 2;
        probes += legal;
        p[k] = legal ? table_lookup(t, canonical(m)) : V(0);
    }
    return vmax(vmax(p[0], p[1]), vmax(p[2], p[3]));
}

__device__ __forceinline__ void add_probes(u32 probes, u64 *counter)
{
    const u32 w = __reduce_add_sync(0xffffffffu, probes);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd((unsigned long long *)counter, (unsigned long long)w);
}

__device__ __forceinline__ bool satisfied(u64 b, const SolveRules &r)
{
    if (r.nox && !r.score) return has_tile(b, r.nox);
    if (r.score) return false;
    for (int i = 0; i < r.n_winstates; i++)
        if (matches(b, __ldg(r.winstates + i))) return true;
    return false;
}

__device__ __forceinline__ void stage_table_s(unsigned char *smem, const unsigned short *g_move)
{
    const uint4 *src = (const uint4 *)g_move;
    uint4 *dst = (uint4 *)smem;
    for (int i = threadIdx.x; i < TABLE_BYTES_S / 16; i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
}

__global__ void __launch_bounds__(SOLVE_THREADS, 1) solve_f64_kernel(const u64 *__restrict__ keys, u64 n,
                                                                     double *__restrict__ out, DevTable<double> t2,
                                                                     DevTable<double> t4, SolveRules r,
                                                                     const unsigned short *g_move, u64 *probes_out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    stage_table_s(smem, g_move);
    const RowTable rt{(const unsigned short *)smem, (const u32 *)(smem + 65536 * 2)};
    u32 probes = 0;
    for (u64 i = (u64)blockIdx.x * SOLVE_THREADS + threadIdx.x; i < n; i += (u64)gridDim.x * SOLVE_THREADS) {
        const u64 b = keys[i];
        double res;
        if (satisfied(b, r)) {
            res = 1.0;
        } else {
            u64 e = empty_mask(b);
            const int spaces = popc64(e);
            double s2 = 0.0, s4 = 0.0;
            while (e) {  // cells in order 0..15 = highest nibble first
                const int bit = 63 - __clzll(e);
                e &= ~(1ull << bit);
                s2 = __dadd_rn(s2, best_move(rt, b | (1ull << bit), t2, probes));
                s4 = __dadd_rn(s4, best_move(rt, b | (2ull << bit), t4, probes));
            }
            res = 0.0;
            if (spaces) {
                const double k = (double)spaces;
                res = __dadd_rn(__ddiv_rn(__dmul_rn(0.9, s2), k), __ddiv_rn(__dmul_rn(0.1, s4), k));
            }
            if (r.score && res == 0.0) res = (double)tile_sum(b);
        }
        out[i] = res;
    }
    add_probes(probes, probes_out);
}

__global__ void __launch_bounds__(SOLVE_THREADS, 1) solve_f32_kernel(const u64 *__restrict__ keys, u64 n,
                                                                     float *__restrict__ out, DevTable<float> t2,
                                                                     DevTable<float> t4, SolveRules r,
                                                                     const unsigned short *g_move, u64 *probes_out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    stage_table_s(smem, g_move);
    const RowTable rt{(const unsigned short *)smem, (const u32 *)(smem + 65536 * 2)};
    u32 probes = 0;
    for (u64 i = (u64)blockIdx.x * SOLVE_THREADS + threadIdx.x; i < n; i += (u64)gridDim.x * SOLVE_THREADS) {
        const u64 b = keys[i];
        float res;
        if (satisfied(b, r)) {
            res = 1.0f;
        } else {
            u64 e = empty_mask(b);
            const int spaces = popc64(e);
            float s2 = 0.f, c2 = 0.f, s4 = 0.f, c4 = 0.f;  // Kahan sums
            while (e) {
                const int bit = 63 - __clzll(e);
                e &= ~(1ull << bit);
                const float y2 = __fsub_rn(best_move(rt, b | (1ull << bit), t2, probes), c2);
                const float u2 = __fadd_rn(s2, y2);
                c2 = __fsub_rn(__fsub_rn(u2, s2), y2);
                s2 = u2;
                const float y4 = __fsub_rn(best_move(rt, b | (2ull << bit), t4, probes), c4);
                const float u4 = __fadd_rn(s4, y4);
                c4 = __fsub_rn(__fsub_rn(u4, s4), y4);
                s4 = u4;
            }
            double d = 0.0;
            if (spaces) {
                const double k = (double)spaces;
                const double S2 = (double)s2 - (double)c2, S4 = (double)s4 - (double)c4;
                d = __dadd_rn(__ddiv_rn(__dmul_rn(0.9, S2), k), __ddiv_rn(__dmul_rn(0.1, S4), k));
            }
            if (r.score && d == 0.0) d = (double)tile_sum(b);
            res = (float)d;
        }
        out[i] = res;
    }
    add_probes(probes, probes_out);
}

// ---- bucket offsets --------------------------------------------------------
__global__ void bucket_offsets_kernel(const u64 *__restrict__ keys, u64 n, u32 *__restrict__ off, int prefix,
                                      int bits)
{
    const u64 nb = 1ull << bits;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (u64)gridDim.x * blockDim.x) {
        const u64 bk = i < n ? (keys[i] << prefix) >> (64 - bits) : nb;
        const u64 bp = i ? (keys[i - 1] << prefix) >> (64 - bits) : 0;
        const u64 from = i ? bp + 1 : 0;
        for (u64 j = from; j <= bk && j <= nb; j++) off[j] = (u32)i;
    }
}

bool build_index(LayerIndex &ix, u32 **storage, u64 *capacity, int bits_hint, cudaStream_t s)
{
    ix.bucket = nullptr;
    ix.bits = 0;
    if (ix.n < 64 || bits_hint <= 0) return true;
    u64 first, last;
    if (!CGB_CUDA(cudaMemcpyAsync(&first, ix.keys, 8, cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaMemcpyAsync(&last, ix.keys + ix.n - 1, 8, cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    const u64 x = first ^ last;
    const int prefix = x ? __builtin_clzll(x) : 64;
    int bits = bits_hint;
    if (bits > 64 - prefix) bits = 64 - prefix;
    if (bits <= 0) return true;
    const u64 need = (1ull << bits) + 1;
    if (*capacity < need) {
        if (*storage) dev_free(*storage, s);
        *storage = nullptr;
        if (!dev_alloc((void **)storage, need * sizeof(u32), s)) return false;
        *capacity = need;
    }
    const int grid = (int)std::min<u64>((ix.n + 256) / 256, (u64)NUM_SMS_B200 * 16);
    bucket_offsets_kernel<<<grid, 256, 0, s>>>(ix.keys, ix.n, *storage, prefix, bits);
    if (!CGB_CUDA(cudaGetLastError())) return false;
    ix.bucket = *storage;
    ix.prefix = prefix;
    ix.bits = bits;
    ix.prefix_value = prefix ? first >> (64 - prefix) : 0;
    return true;
}

template <typename V>
static DevTable<V> dev_table(const LayerIndex &ix)
{
    DevTable<V> t;
    t.keys = ix.keys;
    t.vals = (const V *)ix.vals;
    t.n = ix.n;
    t.bucket = ix.bucket;
    t.prefix = ix.prefix;
    t.bits = ix.bits;
    t.prefix_value = ix.prefix_value;
    return t;
}

static int solve_grid(u64 n)
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = NUM_SMS_B200;
    const u64 need = (n + SOLVE_THREADS - 1) / SOLVE_THREADS;
    return (int)std::max<u64>(1, std::min<u64>(need, (u64)sms));
}

template <typename K, typename V>
static bool launch_solve(K kernel, const u64 *keys, u64 n, V *out, DevTable<V> t2, DevTable<V> t4,
                         const SolveRules &r, const DeviceRowTable &rt, Counters &c, cudaStream_t s, int vbytes)
{
    if (!CGB_CUDA(cudaMemsetAsync(c.d + 2, 0, sizeof(u64), s))) return false;
    kclock().begin(s, &kstats().solve_ms);
    kernel<<<solve_grid(n), SOLVE_THREADS, TABLE_BYTES_S, s>>>(keys, n, out, t2, t4, r, rt.move, c.d + 2);
    kclock().end(s);
    if (!CGB_CUDA(cudaGetLastError())) return false;
    u64 probes = 0;
    if (!CGB_CUDA(cudaMemcpyAsync(&probes, c.d + 2, sizeof(u64), cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    kclock().flush();
    KernelStats &k = kstats();
    k.solve_launches++;
    k.solve_boards += n;
    k.lookups += probes;
    // keys in, values out, one key sector and one value sector per probe
    k.solve_bytes += (8 + vbytes) * n + 64 * probes;
    return true;
}

bool solve_layer_f64(const u64 *keys, u64 n, double *out, const LayerIndex &t2, const LayerIndex &t4,
                     const SolveRules &r, const DeviceRowTable &rt, Counters &c, cudaStream_t s)
{
    if (n == 0) return true;
    static bool attr = false;
    if (!attr) {
        if (!CGB_CUDA(cudaFuncSetAttribute(solve_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           TABLE_BYTES_S)))
            return false;
        attr = true;
    }
    return launch_solve(solve_f64_kernel, keys, n, out, dev_table<double>(t2), dev_table<double>(t4), r, rt, c, s,
                        8);
}

bool solve_layer_f32(const u64 *keys, u64 n, float *out, const LayerIndex &t2, const LayerIndex &t4,
                     const SolveRules &r, const DeviceRowTable &rt, Counters &c, cudaStream_t s)
{
    if (n == 0) return true;
    static bool attr = false;
    if (!attr) {
        if (!CGB_CUDA(cudaFuncSetAttribute(solve_f32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           TABLE_BYTES_S)))
            return false;
        attr = true;
    }
    return launch_solve(solve_f32_kernel, keys, n, out, dev_table<float>(t2), dev_table<float>(t4), r, rt, c, s,
                        4);
}

}  // namespace cgb
