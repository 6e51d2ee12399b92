// sweep.cu -- generation + solve with every layer resident in HBM.
//
// The reference runs generate() (src/generate.c:551-615), writing every layer
// to disk, then solve() (src/solve.c:172-224), reading them back top-down with
// the s+2 and s+4 tables in memory.  Here the layers stay on the device
// (packed in a LayerStore), the solve walks them top-down, and each solved
// layer is turned into a lookup index for the two layers below it.  Host
// copies, when asked for, run on a second stream into double-buffered pinned
// memory and overlap the following layers' kernels.
//
// Precision 0 runs the FP64 and the FP32 chains side by side and reports,
// per layer, the largest and mean |fp32 - fp64|.
#include "async_out.h"
#include "cgb_engine.h"
#include <algorithm>
#include <functional>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

using namespace cgb;

namespace {

bool narrow_values(const double *a, float *b, u64 n, cudaStream_t s);

struct Layer {
    int sum;
    LayerStore::Handle h;
    bool live;
    const u64 *host = nullptr;  // host copy of the keys (host_layers), when kept
};

// device -> host copy on the I/O stream after the main stream's work so far;
// returns the event that marks its completion
cudaEvent_t copy_to_host(void *dst, const void *src, u64 bytes, cudaStream_t main, cudaStream_t io)
{
    cudaEvent_t before = nullptr, after = nullptr;
    if (!CGB_CUDA(cudaEventCreateWithFlags(&before, cudaEventDisableTiming)) ||
        !CGB_CUDA(cudaEventCreateWithFlags(&after, cudaEventDisableTiming)))
        return nullptr;
    const bool ok = CGB_CUDA(cudaEventRecord(before, main)) && CGB_CUDA(cudaStreamWaitEvent(io, before, 0)) &&
                    (bytes == 0 || CGB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, io))) &&
                    CGB_CUDA(cudaEventRecord(after, io));
    cudaEventDestroy(before);
    if (!ok) {
        cudaEventDestroy(after);
        return nullptr;
    }
    return after;
}

struct StoreSink : LayerSink {
    std::vector<Layer> layers;
    LayerStore store;
    cgb_layer_fn fn = nullptr;
    void *user = nullptr;
    AsyncOut *out = nullptr;
    u64 reserve_bytes = 0;
    size_t checked_at = 0;  // store chunks at the last free-memory check
    int device = 0;
    HostArena *host = nullptr;  // set when layers and tables both go to the host
    u64 host_cap = 0;
    u64 host_d2h = 0;
    // layer callbacks waiting for their copies, run in order
    std::deque<std::pair<cudaEvent_t, std::function<bool()>>> deferred;
    bool run_deferred(bool all)
    {
        while (!deferred.empty()) {
            auto &d = deferred.front();
            if (!all && cudaEventQuery(d.first) == cudaErrorNotReady) return true;
            if (!CGB_CUDA(cudaEventSynchronize(d.first))) return false;
            cudaEventDestroy(d.first);
            const bool ok = d.second();
            deferred.pop_front();
            if (!ok) {
                set_error("host callback failed");
                return false;
            }
        }
        return true;
    }
    bool layer(int sum, u64 *d, u64 n, cudaStream_t s, bool *kept) override
    {
        // the engine's layer buffer is reused by the next layer step: keep an
        // exact-size copy in the store (8 B/board)
        *kept = false;
        Layer L{sum, {}, true};
        if (!store.push(n, s, &L.h)) return false;
        u64 *keys = store.ptr(L.h, s);
        if (!keys) return false;
        if (n && !CGB_CUDA(cudaMemcpyAsync(keys, d, n * 8, cudaMemcpyDeviceToDevice, s))) return false;
        if (fn) {
            cgb_layer_fn f = fn;
            void *u = user;
            // with tables wanted too, the layer's host copy is kept for them, so
            // the keys cross the link once; else one of the two pinned slots
            u64 *hk = host && host->used + n * 8 + 16 <= host_cap ? (u64 *)host->take(n * 8 + 16) : nullptr;
            if (hk) {
                cudaEvent_t ev = copy_to_host(hk, keys, n * 8, s, out->io);
                if (!ev) return false;
                L.host = hk;
                host_d2h += n * 8;
                deferred.push_back({ev, [f, u, sum, n, hk] { return f(u, sum, hk, n) == 0; }});
                if (!run_deferred(false)) return false;
            } else if (!out->enqueue({{keys, n * 8}}, [f, u, sum, n](const char *h) {
                           return f(u, sum, (const uint64_t *)h, n) == 0;
                       })) {
                return false;
            }
        }
        layers.push_back(L);
        // keep room for the next layer steps: the working set grows with the
        // layer, so the reserve scales with it
        // (the device query is not free: ask only when the store took a new chunk)
        if (store.chunk_count() != checked_at) {
            const u64 want = reserve_bytes + 12 * n * 8;
            const u64 avail = device_available_bytes(device);
            // false when nothing is left to spill: carry on, an allocation may still fit
            if (avail < want) store.spill(want - avail, s, out->io);
            checked_at = store.chunk_count();
        }
        return true;
    }
};

// one precision's solve state: the current layer and the two above it.  An
// FP32 chain solves its `fp64_above` window -- the highest layers, solved
// first, whose values come straight from the winstates -- in FP64 and narrows
// those tables to FP32 when the first FP32 layer below needs them.
struct Chain {
    int vbytes = 8;
    int fp64_above = 1 << 30;  // FP32 chain: layers with sum > this are solved in FP64
    struct Solved {
        int sum = 0;
        int vb = 8;  // bytes per value of this layer's table
        const u64 *keys = nullptr;
        void *vals = nullptr;
        u64 n = 0;
        IndexStorage store;
        LayerIndex ix;
    };
    Solved t2, t4, cur;

    int layer_vbytes(int sum) const { return vbytes == 4 && sum > fp64_above ? 8 : vbytes; }

    // an FP64 table of the window turned into the FP32 table the chain below reads
    bool narrow(Engine &e, Solved &x, cudaStream_t s)
    {
        if (x.vb == 4 || !x.vals) return true;
        void *f = nullptr;
        if (!dev_alloc(&f, x.n * 4 + 8, s)) return false;
        if (x.n && !narrow_values((const double *)x.vals, (float *)f, x.n, s)) return false;
        dev_free(x.vals, s);
        x.vals = f;
        x.vb = 4;
        x.ix.keys = x.keys;
        x.ix.vals = x.vals;
        x.ix.n = x.n;
        return build_index(x.ix, e.index_kind, 4, x.store, e.bucket_bits, e.ctr, s);
    }
    bool solve(Engine &e, const SolveRules &r, cudaStream_t s)
    {
        cur.vb = layer_vbytes(cur.sum);
        if (cur.vb == 4 && !(narrow(e, t2, s) && narrow(e, t4, s))) return false;
        if (!dev_alloc(&cur.vals, cur.n * cur.vb + 8, s)) return false;
        if (cur.vb == 4)
            return solve_layer_f32(cur.keys, cur.n, (float *)cur.vals, t2.ix, t4.ix, r, e.rt, e.ctr, s, e.plan);
        return solve_layer_f64(cur.keys, cur.n, (double *)cur.vals, t2.ix, t4.ix, r, e.rt, e.ctr, s, e.plan);
    }
    bool index(Engine &e, cudaStream_t s)
    {
        cur.ix.keys = cur.keys;
        cur.ix.vals = cur.vals;
        cur.ix.n = cur.n;
        return build_index(cur.ix, e.index_kind, cur.vb, cur.store, e.bucket_bits, e.ctr, s);
    }
    void rotate(cudaStream_t s)
    {
        if (t4.vals) dev_free(t4.vals, s);
        if (t4.store.p) dev_free(t4.store.p, s);
        t4 = t2;
        t2 = cur;
        cur = Solved{};
    }
    void release(cudaStream_t s)
    {
        for (Solved *x : {&t2, &t4, &cur}) {
            if (x->vals) dev_free(x->vals, s);
            if (x->store.p) dev_free(x->store.p, s);
            *x = Solved{};
        }
    }
};

__global__ void narrow_kernel(const double *__restrict__ a, float *__restrict__ b, u64 n)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

bool narrow_values(const double *a, float *b, u64 n, cudaStream_t s)
{
    const int grid = (int)std::min<u64>((n + 255) / 256, (u64)NUM_SMS_B200 * 8);
    narrow_kernel<<<grid, 256, 0, s>>>(a, b, n);
    kstats().launches++;
    return CGB_CUDA(cudaGetLastError());
}

// max and sum of |a - b| over a layer (a: fp64, b: fp32)
__global__ void abs_diff_kernel(const double *__restrict__ a, const float *__restrict__ b, u64 n, u64 *max_bits,
                                double *sum)
{
    double m = 0, t = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const double d = fabs(a[i] - (double)b[i]);
        m = fmax(m, d);
        t += d;
    }
    for (int o = 16; o; o >>= 1) {
        m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
        t += __shfl_down_sync(0xffffffffu, t, o);
    }
    if ((threadIdx.x & 31) == 0) {
        // non-negative doubles order like their bit patterns
        atomicMax((unsigned long long *)max_bits, (unsigned long long)__double_as_longlong(m));
        atomicAdd(sum, t);
    }
}

}  // namespace

extern "C" int cgb_sweep_run(const cgb_sweep *w, cgb_stats *stats)
{
    if (!ensure_rules_for_api()) return -1;
    Engine &e = Engine::get();
    cudaStream_t s = e.stream;
    if (stats) *stats = cgb_stats{};
    if (w->precision != 0 && w->precision != 32 && w->precision != 64) {
        set_error("cgb_sweep_run: precision must be 64, 32 or 0");
        return -1;
    }
    AsyncOut out;
    if (!out.init(s, e.io_stream, e.out_stage)) return -1;
    StoreSink sink;
    sink.fn = w->layer_fn;
    sink.user = w->user;
    sink.out = &out;
    sink.reserve_bytes = e.spill_reserve;
    sink.store.chunk_bytes = e.store_chunk;
    sink.device = e.device;
    if (w->layer_fn && w->table_fn) {
        e.host_layers.reset();
        sink.host = &e.host_layers;
        sink.host_cap = e.host_layers_cap;
    }
    GenTimes tm;
    const KernelStats k0 = kstats();
    cudaEvent_t ev[3];
    for (auto &x : ev) cudaEventCreate(&x);
    cudaEventRecord(ev[0], s);
    bool ok = e.generate(w->initial, w->n_initial, w->start, w->end_gen, sink, &tm);
    // every layer callback has run (and every kept host copy is complete)
    if (!sink.run_deferred(true)) ok = false;
    cudaEventRecord(ev[1], s);

    // ---- solve, top-down (src/solve.c:203-219) ----
    std::map<int, size_t> by_sum;
    for (size_t i = 0; i < sink.layers.size(); i++) by_sum[sink.layers[i].sum] = i;
    std::vector<u64> ws = expand_winstates(w->winstates, w->n_winstates);
    u64 *d_ws = nullptr;
    std::vector<Chain> chains;
    if (w->precision == 0) {
        chains.resize(2);
        chains[0].vbytes = 8;
        chains[1].vbytes = 4;
    } else {
        chains.resize(1);
        chains[0].vbytes = w->precision == 32 ? 4 : 8;
    }
    for (auto &c : chains) c.fp64_above = w->end_gen - 2 * e.fp64_top_layers;
    u64 *d_err = nullptr;  // [max bits, sum]
    u64 solved = 0;
    double max_err = 0;
    if (ok) ok = dev_alloc((void **)&d_ws, ws.size() * 8 + 8, s);
    if (ok && !ws.empty()) ok = CGB_CUDA(cudaMemcpyAsync(d_ws, ws.data(), ws.size() * 8, cudaMemcpyHostToDevice, s));
    if (ok && w->precision == 0) ok = dev_alloc((void **)&d_err, 16, s);
    const SolveRules rules = make_solve_rules(e.rules, d_ws, (int)ws.size());
    const int lo = std::max(w->end_solve, 0);
    for (int sum = w->end_gen; ok && sum >= lo && sum > 0; sum -= 2) {
        auto it = by_sum.find(sum);
        const u64 *keys = nullptr;
        u64 n = 0;
        if (it != by_sum.end()) {
            n = sink.layers[it->second].h.n;
            keys = sink.store.ptr(sink.layers[it->second].h, s);
            if (!keys) {
                ok = false;
                break;
            }
        }
        for (auto &c : chains) {
            c.cur.sum = sum;
            c.cur.keys = keys;
            c.cur.n = n;
            ok = ok && c.solve(e, rules, s);
        }
        if (!ok) break;
        solved += n;
        if (w->precision == 0 && n && chains[1].cur.vb == 8) {
            // the FP32 chain's FP64 window: the same operations on the same tables as chain 0
            if (w->error_fn && w->error_fn(w->user, sum, n, 0.0, 0.0) != 0) {
                set_error("error callback failed");
                ok = false;
                break;
            }
        } else if (w->precision == 0 && n) {
            ok = CGB_CUDA(cudaMemsetAsync(d_err, 0, 16, s));
            const int grid = (int)std::min<u64>((n + 255) / 256, (u64)NUM_SMS_B200 * 8);
            kstats().launches++;
            abs_diff_kernel<<<grid, 256, 0, s>>>((const double *)chains[0].cur.vals, (const float *)chains[1].cur.vals,
                                                 n, d_err, (double *)(d_err + 1));
            u64 h[2];
            ok = ok && CGB_CUDA(cudaGetLastError()) &&
                 CGB_CUDA(cudaMemcpyAsync(h, d_err, 16, cudaMemcpyDeviceToHost, s)) &&
                 CGB_CUDA(cudaStreamSynchronize(s));
            if (!ok) break;
            double mx, sm;
            memcpy(&mx, &h[0], 8);
            memcpy(&sm, &h[1], 8);
            max_err = std::max(max_err, mx);
            if (w->error_fn && w->error_fn(w->user, sum, n, mx, sm / (double)n) != 0) {
                set_error("error callback failed");
                ok = false;
                break;
            }
        }
        bool enqueued = false;  // this layer's table copy (reads only this layer)
        if (w->table_fn) {
            enqueued = true;
            Chain &c = chains[0];
            const int prec = c.cur.vb == 8 ? 64 : 32;
            cgb_table_fn f = w->table_fn;
            void *u = w->user;
            static const uint64_t none = 0;
            const u64 *hk = it != by_sum.end() ? sink.layers[it->second].host : nullptr;
            if (hk || n == 0) {  // the keys are on the host already: copy the values only
                const uint64_t *k = hk ? hk : &none;
                ok = out.enqueue({{c.cur.vals, n * (u64)c.cur.vb}}, [f, u, sum, n, prec, k](const char *h) {
                    return f(u, sum, k, h, n, prec) == 0;
                });
            } else {
                ok = out.enqueue({{keys, n * 8}, {c.cur.vals, n * (u64)c.cur.vb}},
                                 [f, u, sum, n, prec](const char *h) {
                                     return f(u, sum, (const uint64_t *)h, h + n * 8, n, prec) == 0;
                                 });
            }
            if (!ok) break;
        }
        for (auto &c : chains) ok = ok && c.index(e, s);
        if (!ok) break;
        // the s+4 layer is no longer needed by anyone.  When this layer's table
        // was enqueued, the copies still in flight are this layer's and the
        // previous one's (an enqueue first completes the copy it replaces, two
        // layers back), so none reads s+4 and the main stream need not wait;
        // otherwise fence every pending copy (layer copies of the generation)
        if (!enqueued) ok = out.fence_main();
        const int gone = chains[0].t4.sum;
        for (auto &c : chains) c.rotate(s);
        auto it4 = by_sum.find(gone);
        if (gone && it4 != by_sum.end() && sink.layers[it4->second].live) {
            sink.store.release(sink.layers[it4->second].h, s);
            sink.layers[it4->second].live = false;
        }
    }
    if (ok) ok = out.drain();
    out.fence_main();
    for (auto &c : chains) c.release(s);
    sink.store.clear(s);
    dev_free(d_ws, s);
    dev_free(d_err, s);
    cudaEventRecord(ev[2], s);
    cudaEventSynchronize(ev[2]);
    float gen_ms = 0, solve_ms = 0;
    cudaEventElapsedTime(&gen_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&solve_ms, ev[1], ev[2]);
    for (auto &x : ev) cudaEventDestroy(x);
    if (stats) {
        fill_stats(stats, tm, k0, kstats());
        stats->layers = sink.layers.size();
        stats->boards_solved = solved;
        stats->gen_ms = gen_ms;
        stats->solve_ms = solve_ms;
        stats->total_ms = gen_ms + solve_ms;
        stats->h2d_bytes = w->n_initial * 8;
        stats->d2h_bytes = out.d2h + sink.host_d2h;
        stats->max_abs_err = max_err;
        stats->spilled_chunks = sink.store.spills;
        stats->restored_chunks = sink.store.restores;
    }
    return ok ? 0 : -1;
}
