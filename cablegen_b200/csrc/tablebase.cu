// tablebase.cu -- the C ABI of the engine (include/cablegen_b200.h).
#include "cgb_engine.h"
#include <algorithm>
#include <map>
#include <vector>

using namespace cgb;

namespace cgb {

// the 8 images of a winstate (get_all_rots, src/board.c:349-374)
std::vector<u64> expand_winstates(const u64 *w, int n)
{
    std::vector<u64> out;
    for (int i = 0; i < n; i++) {
        const u64 b = w[i], f = flip_v(b);
        const u64 imgs[8] = {b, rot_cw(b), rot_cw(rot_cw(b)), rot_ccw(b),
                             f, rot_cw(f), rot_cw(rot_cw(f)), rot_ccw(f)};
        for (u64 x : imgs) out.push_back(x);
    }
    return out;
}

SolveRules make_solve_rules(const cgb_rules &r, const u64 *d_ws, int nws)
{
    SolveRules s;
    s.nox = (int)(signed char)r.nox;  // the solver keeps nox in a char (src/solve.c:18)
    s.score = r.score ? 1 : 0;
    s.winstates = d_ws;
    s.n_winstates = nws;
    return s;
}

}  // namespace cgb

namespace cgb {
bool set_lookback_test(u32 spin_limit, int hold_first_tile);
extern u64 g_dev_mem_cap;
static u32 g_test_spin = 0;
static int g_test_hold = 0;
extern int g_solve_variant;
extern int g_sort_variant;
extern int g_hash_load_pct;
extern int g_hash_compact;
extern int g_region_build;
extern int g_move_window;
}

static Engine &E() { return Engine::get(); }

#define CGB_TRY(x)      \
    do {                \
        if (!(x)) return -1; \
    } while (0)

extern "C" {

const char *cgb_last_error(void) { return last_error(); }

int cgb_get_kernel_stats(cgb_kernel_stats *o)
{
    const KernelStats &k = kstats();
    o->launches = k.launches;
    o->hist_ms = k.hist_ms;
    o->onesweep_ms = k.onesweep_ms;
    o->unique_ms = k.unique_ms;
    o->merge_ms = k.merge_ms;
    o->expand_ms = k.expand_ms;
    o->spawn_ms = k.spawn_ms;
    o->solve_ms = k.solve_ms;
    o->index_ms = k.index_ms;
    o->hist_bytes = k.hist_bytes;
    o->onesweep_bytes = k.onesweep_bytes;
    o->unique_bytes = k.unique_bytes;
    o->merge_bytes = k.merge_bytes;
    o->expand_bytes = k.expand_bytes;
    o->spawn_bytes = k.spawn_bytes;
    o->solve_bytes = k.solve_bytes;
    o->onesweep_launches = k.onesweep_launches;
    o->solve_launches = k.solve_launches;
    o->solve_boards = k.solve_boards;
    o->lookups = k.lookups;
    o->index_builds = k.index_builds;
    o->compact_index_builds = k.compact_index_builds;
    o->moves_raw = k.moves_raw;
    o->moves_kept = k.moves_kept;
    o->pool_trims = k.pool_trims;
    return 0;
}

int cgb_reset_kernel_stats(void)
{
    kstats() = KernelStats{};
    return 0;
}

int cgb_set_option(const char *name, long long value)
{
    const std::string k = name ? name : "";
    if (k == "index") {
        if (value < INDEX_BISECT || value > INDEX_HASH) {
            set_error("cgb_set_option: index must be 0 (bisect), 1 (bucket) or 2 (hash)");
            return -1;
        }
        E().index_kind = (int)value;
    } else if (k == "solve_variant") {
        if (value < 0 || value > 1) {
            set_error("cgb_set_option: solve_variant must be 0 (one thread per board) or 1 (board-cell pairs)");
            return -1;
        }
        g_solve_variant = (int)value;
    } else if (k == "sort_variant") {
        if (value < 0 || value > 5) {
            set_error("cgb_set_option: sort_variant must be 0 (match ranking), 1 (ballot ranking), 2 (pipelined), "
                      "3 (byte-digit ballot ranking), 4 (byte-digit, 8192-key tiles) or 5 (4 with match ranking)");
            return -1;
        }
        g_sort_variant = (int)value;
    } else if (k == "hash_load_pct") {
        if (value != 0 && (value < 10 || value > 90)) {
            set_error("cgb_set_option: hash_load_pct must be 0 (by size) or in [10, 90]");
            return -1;
        }
        g_hash_load_pct = (int)value;
    } else if (k == "spill_reserve_mb") {
        if (value < 0) {
            set_error("cgb_set_option: spill_reserve_mb must be >= 0");
            return -1;
        }
        E().spill_reserve = (u64)value << 20;
    } else if (k == "host_layers_mb") {
        if (value < 0) {
            set_error("cgb_set_option: host_layers_mb must be >= 0");
            return -1;
        }
        E().host_layers_cap = (u64)value << 20;
    } else if (k == "store_chunk_mb") {
        if (value < 1) {
            set_error("cgb_set_option: store_chunk_mb must be >= 1");
            return -1;
        }
        E().store_chunk = (u64)value << 20;
    } else if (k == "max_sort_keys") {
        if (value < (1 << 16) || value > (1 << 30)) {
            set_error("cgb_set_option: max_sort_keys must be in [2^16, 2^30]");
            return -1;
        }
        E().max_sort_keys = (u64)value;
    } else if (k == "lookback_spin_limit" || k == "lookback_hold_first_tile") {
        // failure-path tests: a lower poll limit for look-back waits (0 = default), and a
        // digit pass whose tile 0 never publishes, so tile 1's wait must run out
        if (value < 0 || value > 0xFFFFFFFFll) {
            set_error("cgb_set_option: " + k + " must be in 0..2^32-1");
            return -1;
        }
        if (!E().ready && !E().init(0)) return -1;
        if (k == "lookback_spin_limit") g_test_spin = (u32)value;
        else g_test_hold = value ? 1 : 0;
        if (!set_lookback_test(g_test_spin, g_test_hold)) return -1;
    } else if (k == "device_mem_cap_mb") {
        // a capped device allocator: allocations through the engine fail once the
        // bytes it holds would exceed the cap (0 = no cap)
        if (value < 0) {
            set_error("cgb_set_option: device_mem_cap_mb must be >= 0");
            return -1;
        }
        g_dev_mem_cap = (u64)value << 20;
    } else if (k == "region_build") {
        if (value < 0 || value > 1) {
            set_error("cgb_set_option: region_build must be 0 or 1");
            return -1;
        }
        g_region_build = (int)value;
    } else if (k == "move_window") {
        if (value < 1 || value > 4) {
            set_error("cgb_set_option: move_window must be in [1, 4]");
            return -1;
        }
        g_move_window = (int)value;
    } else if (k == "hash_compact") {
        if (value < 0 || value > 1) {
            set_error("cgb_set_option: hash_compact must be 0 or 1");
            return -1;
        }
        g_hash_compact = (int)value;
    } else if (k == "fp64_top_layers") {
        if (value < 0 || value > 100000) {
            set_error("cgb_set_option: fp64_top_layers must be in 0..100000");
            return -1;
        }
        E().fp64_top_layers = (int)value;
    } else if (k == "bucket_bits") {
        if (value < 0 || value > 30) {
            set_error("cgb_set_option: bucket_bits must be in 0..30");
            return -1;
        }
        E().bucket_bits = (int)value;
    } else {
        set_error("cgb_set_option: unknown option " + k);
        return -1;
    }
    return 0;
}

long long cgb_get_option(const char *name)
{
    const std::string k = name ? name : "";
    if (k == "index") return E().index_kind;
    if (k == "bucket_bits") return E().bucket_bits;
    if (k == "solve_variant") return g_solve_variant;
    if (k == "sort_variant") return g_sort_variant;
    if (k == "hash_load_pct") return g_hash_load_pct;
    if (k == "spill_reserve_mb") return (long long)(E().spill_reserve >> 20);
    if (k == "max_sort_keys") return (long long)E().max_sort_keys;
    if (k == "store_chunk_mb") return (long long)(E().store_chunk >> 20);
    if (k == "host_layers_mb") return (long long)(E().host_layers_cap >> 20);
    if (k == "fp64_top_layers") return E().fp64_top_layers;
    if (k == "hash_compact") return g_hash_compact;
    if (k == "region_build") return g_region_build;
    if (k == "move_window") return g_move_window;
    if (k == "lookback_spin_limit") return g_test_spin;
    if (k == "lookback_hold_first_tile") return g_test_hold;
    if (k == "device_mem_cap_mb") return (long long)(g_dev_mem_cap >> 20);
    return -1;
}

int cgb_init(int device)
{
    CGB_TRY(E().init(device));
    return 0;
}

static bool ensure_init()
{
    if (E().ready) return true;
    return E().init(0);
}

int cgb_set_rules(const cgb_rules *r)
{
    CGB_TRY(ensure_init());
    CGB_TRY(E().set_rules(*r));
    return 0;
}

bool ensure_rules_for_api()
{
    if (!ensure_init()) return false;
    if (E().rt.move) return true;
    cgb_rules r{};
    r.stsl = 200;
    r.ltc = 5;
    r.smallest_large = 6;
    return E().set_rules(r);
}

int cgb_expand_moves(const uint64_t *d_in, uint64_t n, uint64_t *d_out, uint64_t cap, uint64_t *n_out)
{
    CGB_TRY(ensure_rules_for_api());
    if (cap < 4 * n) {
        set_error("cgb_expand_moves: the output needs 4n slots");
        return -1;
    }
    CGB_TRY(expand_moves(d_in, n, d_out, cap, n_out, E().rt, E().prune_params(), E().ctr, E().stream));
    return 0;
}

int cgb_count_spawns(const uint64_t *d_in, uint64_t n, uint64_t *total)
{
    CGB_TRY(ensure_init());
    CGB_TRY(count_spawns(d_in, n, total, E().ctr, E().stream));
    return 0;
}

int cgb_expand_spawns(const uint64_t *d_in, uint64_t n, uint64_t *d_out2, uint64_t *d_out4, uint64_t cap,
                      uint64_t *n_out)
{
    CGB_TRY(ensure_init());
    CGB_TRY(expand_spawns(d_in, n, d_out2, d_out4, cap, n_out, E().ctr, E().stream));
    return 0;
}

int cgb_sort(uint64_t *d_keys, uint64_t *d_tmp, uint64_t n, int *result_in_tmp, int *passes)
{
    CGB_TRY(ensure_init());
    u64 *sorted = nullptr;
    SortStats st;
    CGB_TRY(sort_keys(d_keys, d_tmp, n, &sorted, E().ws, E().stream, &st));
    CGB_TRY(sort_check(E().ws, E().stream));
    if (result_in_tmp) *result_in_tmp = (sorted == d_tmp) ? 1 : 0;
    if (passes) *passes = st.passes;
    return 0;
}

int cgb_unique(const uint64_t *d_in, uint64_t n, uint64_t *d_out, uint64_t *n_out)
{
    CGB_TRY(ensure_init());
    CGB_TRY(unique_keys(d_in, n, d_out, n_out, E().ws, E().stream));
    return 0;
}

int cgb_merge_unique(const uint64_t *d_a, uint64_t na, const uint64_t *d_b, uint64_t nb, uint64_t *d_out,
                     uint64_t *n_out)
{
    CGB_TRY(ensure_init());
    CGB_TRY(merge_unique(d_a, na, d_b, nb, d_out, n_out, E().ws, E().stream));
    return 0;
}

}  // extern "C"

__global__ void canonicalize_kernel(const u64 *__restrict__ in, u64 n, u64 *__restrict__ out)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        out[i] = canonical(in[i]);
}

extern "C" int cgb_canonicalize(const uint64_t *d_in, uint64_t n, uint64_t *d_out)
{
    CGB_TRY(ensure_init());
    if (n == 0) return 0;
    const int grid = (int)std::min<u64>((n + 255) / 256, (u64)NUM_SMS_B200 * 8);
    canonicalize_kernel<<<grid, 256, 0, E().stream>>>(d_in, n, d_out);
    CGB_TRY(CGB_CUDA(cudaGetLastError()));
    CGB_TRY(E().sync());
    return 0;
}

extern "C" int cgb_solve_layer(const uint64_t *d_keys, uint64_t n, void *d_out, int precision,
                               const uint64_t *d_k2, const void *d_v2, uint64_t n2, const uint64_t *d_k4,
                               const void *d_v4, uint64_t n4, const uint64_t *h_winstates, int n_winstates)
{
    CGB_TRY(ensure_rules_for_api());
    cudaStream_t s = E().stream;
    std::vector<u64> ws = expand_winstates(h_winstates, n_winstates);
    u64 *d_ws = nullptr;
    CGB_TRY(dev_alloc((void **)&d_ws, ws.size() * 8 + 8, s));
    if (!ws.empty())
        CGB_TRY(CGB_CUDA(cudaMemcpyAsync(d_ws, ws.data(), ws.size() * 8, cudaMemcpyHostToDevice, s)));
    LayerIndex t2, t4;
    t2.keys = d_k2;
    t2.vals = d_v2;
    t2.n = n2;
    t4.keys = d_k4;
    t4.vals = d_v4;
    t4.n = n4;
    const int vb = precision == 32 ? 4 : 8;
    IndexStorage st2, st4;
    bool ok = build_index(t2, E().index_kind, vb, st2, E().bucket_bits, E().ctr, s) &&
              build_index(t4, E().index_kind, vb, st4, E().bucket_bits, E().ctr, s);
    const SolveRules r = make_solve_rules(E().rules, d_ws, (int)ws.size());
    // the images that can be canonical follow the 0xf mask of the first board
    CanonPlan plan;
    if (ok && n) {
        u64 first = 0;
        ok = CGB_CUDA(cudaMemcpyAsync(&first, d_keys, 8, cudaMemcpyDeviceToHost, s)) &&
             CGB_CUDA(cudaStreamSynchronize(s));
        plan = make_canon_plan(first, E().rules.free_formation != 0);
    }
    if (ok) {
        if (precision == 32)
            ok = solve_layer_f32(d_keys, n, (float *)d_out, t2, t4, r, E().rt, E().ctr, s, plan);
        else
            ok = solve_layer_f64(d_keys, n, (double *)d_out, t2, t4, r, E().rt, E().ctr, s, plan);
    }
    dev_free(d_ws, s);
    dev_free(st2.p, s);
    dev_free(st4.p, s);
    CGB_TRY(ok);
    CGB_TRY(E().sync());
    return 0;
}

int cgb_lookup_batch(const uint64_t *d_keys, const void *d_vals, uint64_t n, int precision, const uint64_t *d_boards,
                     uint64_t m, int canonicalize, double *d_out)
{
    CGB_TRY(ensure_init());
    if (precision != 32 && precision != 64) {
        set_error("cgb_lookup_batch: precision must be 32 or 64");
        return -1;
    }
    cudaStream_t s = E().stream;
    LayerIndex ix;
    ix.keys = d_keys;
    ix.vals = d_vals;
    ix.n = n;
    const int vb = precision == 32 ? 4 : 8;
    IndexStorage st;
    const bool ok = build_index(ix, E().index_kind, vb, st, E().bucket_bits, E().ctr, s) &&
                    lookup_batch(ix, vb, d_boards, m, canonicalize != 0, d_out, s);
    dev_free(st.p, s);
    CGB_TRY(ok);
    CGB_TRY(E().sync());
    return 0;
}

// ---------------------------------------------------------------- sweeps
namespace {

struct CopyOutSink : LayerSink {
    cgb_layer_fn fn = nullptr;
    void *user = nullptr;
    HostStage stage;
    u64 d2h = 0;
    bool failed = false;
    bool layer(int sum, u64 *d, u64 n, cudaStream_t s, bool *kept) override
    {
        *kept = false;
        if (!fn) return true;
        if (!stage.reserve(n * 8 + 8)) return false;
        if (n && !CGB_CUDA(cudaMemcpyAsync(stage.p, d, n * 8, cudaMemcpyDeviceToHost, s))) return false;
        if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
        d2h += n * 8;
        if (fn(user, sum, (const u64 *)stage.p, n) != 0) {
            set_error("layer callback failed");
            return false;
        }
        return true;
    }
};

// per-phase device times as the difference of two kernel-clock snapshots
}  // namespace

namespace cgb {
void fill_stats(cgb_stats *st, const GenTimes &tm, const KernelStats &k0, const KernelStats &k1)
{
    if (!st) return;
    st->boards_generated += tm.boards;
    st->expand_ms += (k1.expand_ms - k0.expand_ms) + (k1.spawn_ms - k0.spawn_ms);
    st->sort_ms += (k1.onesweep_ms - k0.onesweep_ms) + (k1.hist_ms - k0.hist_ms);
    st->unique_ms += k1.unique_ms - k0.unique_ms;
    st->merge_ms += k1.merge_ms - k0.merge_ms;
    st->solve_kernel_ms += k1.solve_ms - k0.solve_ms;
    st->index_ms += k1.index_ms - k0.index_ms;
    st->sorted_keys += tm.sorted_keys;
    st->sort_key_passes += tm.sort_passes;
    st->layer_slices += tm.chunks;
    st->gpu_launches += k1.launches - k0.launches;
    st->lookups_bytes += k1.solve_bytes - k0.solve_bytes;
}

}  // namespace cgb

extern "C" int cgb_generate(const uint64_t *h_initial, uint64_t n, int start, int end, cgb_layer_fn fn, void *user,
                            cgb_stats *stats)
{
    CGB_TRY(ensure_rules_for_api());
    CopyOutSink sink;
    sink.fn = fn;
    sink.user = user;
    GenTimes tm;
    const KernelStats k0 = kstats();
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, E().stream);
    const bool ok = E().generate(h_initial, n, start, end, sink, &tm);
    cudaEventRecord(b, E().stream);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (stats) {
        *stats = cgb_stats{};
        fill_stats(stats, tm, k0, kstats());
        stats->gen_ms = ms;
        stats->total_ms = ms;
        stats->h2d_bytes = n * 8;
        stats->d2h_bytes = sink.d2h;
        stats->layers = (end >= start) ? (u64)((end - start) / 2 + 1) : 0;
    }
    CGB_TRY(ok);
    return 0;
}

extern "C" int cgb_tablebase(const uint64_t *h_initial, uint64_t n, int start, int end_gen, int end_solve,
                             const uint64_t *h_winstates, int n_winstates, int precision, cgb_layer_fn layer_fn,
                             cgb_table_fn table_fn, void *user, cgb_stats *stats)
{
    cgb_sweep w{};
    w.initial = h_initial;
    w.n_initial = n;
    w.start = start;
    w.end_gen = end_gen;
    w.end_solve = end_solve;
    w.winstates = h_winstates;
    w.n_winstates = n_winstates;
    w.precision = precision;
    w.layer_fn = layer_fn;
    w.table_fn = table_fn;
    w.user = user;
    return cgb_sweep_run(&w, stats);
}
