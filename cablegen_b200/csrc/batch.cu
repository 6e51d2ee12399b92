// batch.cu -- many formations in one generation + solve sweep.
//
// The reference generates and solves one formation per call (generate(),
// src/generate.c:551-615; solve(), src/solve.c:172-224).  A batch advances all
// its formations together: at step t formation f is at tile sum start_f + 2t,
// and the boards of every formation go through the same expansion, sort,
// unique and merge launches.  This works because a canonical board names its
// formation: fixed cells (0xf) never move, so the board's fixed-cell mask is
// one of the 8 images of its formation's mask, and formations whose mask
// orbits are disjoint never share a board.  A 65536-entry table maps a mask to
// the formation id; formations whose orbits meet are put in separate groups.
//
// Generation: the layer recurrence of the single sweep (engine.cu) runs on the
// union of the formations' boards; expand_moves drops the boards of
// formations past their last layer; each step's layer is partitioned by
// formation id (one stable digit pass) into the resident layer store, so a
// formation's layer is one contiguous range.
//
// Solve: step tau solves, for every formation still solving, its layer at
// end_f - 2 tau.  The ranges are gathered into one array, solved by one
// launch against hash indexes of the two previous steps' unions (a successor
// of a board of formation f only matches boards of formation f), and indexed
// in turn.  That launch sequence is captured as a CUDA graph per step (the
// graph of the previous step is updated in place when the topology allows).
// Winstates are per formation (SolveRules::fid / ws_begin).
#include "async_out.h"
#include "cgb_engine.h"
#include <algorithm>
#include <cstring>
#include <vector>

using namespace cgb;

namespace {

struct Plan {
    int index = 0;              // position in the caller's array
    int start = 0, end_gen = 0, lo_solve = 0;
    int steps = 0;              // layers start, start+2, ..., end_gen
    u32 mask = 0;               // fixed_pattern of the formation
    std::vector<u64> initial;   // sorted, unique
    std::vector<u64> winstates; // expanded x8
};

// the 8 fixed-cell masks a board of this formation can show after canonicalisation
void mask_orbit(u32 mask, u32 out[8])
{
    u64 b = 0;
    for (int i = 0; i < 16; i++)
        if (mask >> i & 1) b |= 0xFull << (4 * i);
    u64 img[8];
    images(b, img);
    for (int k = 0; k < 8; k++) out[k] = fixed_pattern(img[k]);
}

int tile_sum_host(u64 b)
{
    int s = 0;
    for (int c = 0; c < 16; c++) {
        const int e = tile_at(b, c);
        if (e != 0 && e != 0xE && e != 0xF) s += 1 << e;
    }
    return s;
}

// where formation f's layer of generation step t lives
struct Range {
    int block = -1;  // index into the sink's blocks
    u64 off = 0, n = 0;
};

struct BatchSink : LayerSink {
    Engine *e = nullptr;
    const std::vector<Plan> *plans = nullptr;
    const unsigned char *d_fid = nullptr;
    unsigned char *d_active = nullptr;
    std::vector<unsigned char> active;  // host copy of the active flags
    AsyncOut *out = nullptr;
    cgb_batch_layer_fn fn = nullptr;
    void *user = nullptr;
    LayerStore store;
    struct Block {
        LayerStore::Handle h;
        int refs = 0;  // ranges of this step not yet gathered by the solve
        bool live = true;
    };
    std::vector<Block> blocks;
    std::vector<std::vector<Range>> ranges;  // [formation][step]
    int step = 0;
    u64 reserve_bytes = 0;
    size_t checked_at = 0;  // store chunks at the last free-memory check

    bool set_active(cudaStream_t s)
    {
        bool changed = false;
        for (size_t f = 0; f < plans->size(); f++) {
            const unsigned char a = step < (*plans)[f].steps ? 1 : 0;
            changed |= active[f] != a;
            active[f] = a;
        }
        // pageable source: the copy is staged before the call returns
        return !changed || CGB_CUDA(cudaMemcpyAsync(d_active, active.data(), 256, cudaMemcpyHostToDevice, s));
    }

    bool layer(int, u64 *d, u64 n, cudaStream_t s, bool *kept) override
    {
        *kept = false;
        Block b;
        if (!store.push(n, s, &b.h)) return false;
        u64 *dst = store.ptr(b.h, s);
        if (!dst) return false;
        u32 counts[256];
        if (!partition_by_formation(d, n, dst, d_fid, counts, e->ws, s)) return false;
        if (counts[0xFF]) {
            set_error("cgb_batch_run: boards without a formation of the batch (do fixed cells move?)");
            return false;
        }
        const int bi = (int)blocks.size();
        std::vector<std::pair<int, Range>> mine;  // (formation, range) of this step
        u64 off = 0;
        for (size_t f = 0; f < plans->size(); f++) {
            const u64 c = counts[f];
            if (step < (*plans)[f].steps) {
                Range r{bi, off, c};
                ranges[f].push_back(r);
                mine.push_back({(int)f, r});
                b.refs++;
            } else if (c) {
                set_error("cgb_batch_run: a finished formation produced boards");
                return false;
            }
            off += c;
        }
        blocks.push_back(b);
        if (fn) {
            cgb_batch_layer_fn f = fn;
            void *u = user;
            const std::vector<Plan> *p = plans;
            const int t = step;
            if (!out->enqueue({{dst, n * 8}}, [f, u, p, t, mine](const char *h) {
                    for (auto &m : mine) {
                        const Plan &pl = (*p)[m.first];
                        if (f(u, pl.index, pl.start + 2 * t, (const uint64_t *)h + m.second.off, m.second.n) != 0)
                            return false;
                    }
                    return true;
                }))
                return false;
        }
        step++;
        if (!set_active(s)) return false;
        // keep room for the next steps (older steps move to pinned host memory)
        // (the device query is not free: ask only when the store took a new chunk)
        if (store.chunk_count() != checked_at) {
            const u64 want = reserve_bytes + 12 * n * 8;
            const u64 avail = device_available_bytes(e->device);
            // false when nothing is left to spill: carry on, an allocation may still fit
            if (avail < want) store.spill(want - avail, s, out->io);
            checked_at = store.chunk_count();
        }
        return true;
    }
};

// one solved union of layers, indexed by a hash table
struct Solved {
    u64 *keys = nullptr;
    void *vals = nullptr;
    void *slots = nullptr;
    u64 n = 0;
    LayerIndex ix;
    std::vector<std::pair<int, Range>> parts;  // (formation, range in this array)
    std::vector<int> sums;                      // sum of each part
};

void free_solved(Solved &x, cudaStream_t s)
{
    dev_free(x.keys, s);
    dev_free(x.vals, s);
    dev_free(x.slots, s);
    x = Solved{};
}

struct GraphRunner {
    cudaGraphExec_t exec = nullptr;
    u64 launches = 0;
    ~GraphRunner()
    {
        if (exec) cudaGraphExecDestroy(exec);
    }
    // ends the capture on s and launches it, reusing the previous executable
    // graph when the new one has the same topology
    bool finish(cudaStream_t s, bool captured_ok)
    {
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(s, &g);
        if (!captured_ok || !CGB_CUDA(ec)) {
            if (g) cudaGraphDestroy(g);
            return false;
        }
        bool ok = true;
        if (exec) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(exec, g, &info) != cudaSuccess) {
                cudaGetLastError();  // a topology change is not an error: instantiate anew
                cudaGraphExecDestroy(exec);
                exec = nullptr;
            }
        }
        if (!exec) ok = CGB_CUDA(cudaGraphInstantiate(&exec, g, 0));
        cudaGraphDestroy(g);
        if (ok) ok = CGB_CUDA(cudaGraphLaunch(exec, s));
        launches += ok;
        return ok;
    }
};

bool run_group(Engine &e, const cgb_batch *b, std::vector<Plan> &plans, cgb_batch_stats *st, AsyncOut &out)
{
    cudaStream_t s = e.stream;
    const int nf = (int)plans.size();
    // formation tables
    std::vector<unsigned char> fid(65536, 0xFF);
    for (int f = 0; f < nf; f++) {
        u32 orbit[8];
        mask_orbit(plans[f].mask, orbit);
        for (u32 m : orbit) fid[m] = (unsigned char)f;
    }
    std::vector<u32> ws_begin(nf + 1, 0);
    std::vector<u64> ws;
    for (int f = 0; f < nf; f++) {
        ws_begin[f] = (u32)ws.size();
        ws.insert(ws.end(), plans[f].winstates.begin(), plans[f].winstates.end());
    }
    ws_begin[nf] = (u32)ws.size();
    unsigned char *d_tab = nullptr;  // fid[65536] | active[256] | ws_begin | winstates | probes, err
    const u64 off_active = 65536, off_wsb = off_active + 256, off_ws = off_wsb + 8 * ((4 * (nf + 1) + 7) / 8);
    const u64 off_ctr = off_ws + 8 * (ws.size() + 1), tab_bytes = off_ctr + 16;
    if (!dev_alloc((void **)&d_tab, tab_bytes, s)) return false;
    u64 *d_probes = (u64 *)(d_tab + off_ctr);
    u32 *d_err = (u32 *)(d_tab + off_ctr + 8);
    bool ok = CGB_CUDA(cudaMemcpyAsync(d_tab, fid.data(), 65536, cudaMemcpyHostToDevice, s)) &&
              CGB_CUDA(cudaMemsetAsync(d_tab + off_active, 0, 256, s)) &&
              CGB_CUDA(cudaMemcpyAsync(d_tab + off_wsb, ws_begin.data(), 4 * (nf + 1), cudaMemcpyHostToDevice, s)) &&
              (ws.empty() ||
               CGB_CUDA(cudaMemcpyAsync(d_tab + off_ws, ws.data(), 8 * ws.size(), cudaMemcpyHostToDevice, s))) &&
              CGB_CUDA(cudaMemsetAsync(d_tab + off_ctr, 0, 16, s));

    // ---- generation ----
    std::vector<u64> init;
    for (auto &p : plans)
        if (p.steps > 0) init.insert(init.end(), p.initial.begin(), p.initial.end());
    std::sort(init.begin(), init.end());
    init.erase(std::unique(init.begin(), init.end()), init.end());
    int max_steps = 0;
    for (auto &p : plans) max_steps = std::max(max_steps, p.steps);
    BatchSink sink;
    sink.e = &e;
    sink.plans = &plans;
    sink.d_fid = d_tab;
    sink.d_active = d_tab + off_active;
    sink.active.assign(256, 0);
    sink.out = &out;
    sink.fn = b->layer_fn;
    sink.user = b->user;
    sink.ranges.resize(nf);
    sink.reserve_bytes = e.spill_reserve;
    sink.store.chunk_bytes = e.store_chunk;
    GenTimes tm;
    cudaEvent_t ev[3];
    for (auto &x : ev) cudaEventCreate(&x);
    cudaEventRecord(ev[0], s);
    if (ok) ok = sink.set_active(s);
    e.filter = FormationFilter{d_tab, d_tab + off_active};
    if (ok && max_steps > 0) ok = e.generate(init.data(), init.size(), 0, 2 * (max_steps - 1), sink, &tm);
    e.filter = FormationFilter{};
    cudaEventRecord(ev[1], s);
    st->gen_steps += max_steps;
    st->boards_generated += tm.boards;
    st->h2d_bytes += 8 * init.size();

    // ---- solve ----
    SolveRules rules = make_solve_rules(e.rules, (const u64 *)(d_tab + off_ws), (int)ws.size());
    rules.fid = d_tab;
    rules.ws_begin = (const u32 *)(d_tab + off_wsb);
    const int vbytes = b->precision == 32 ? 4 : 8;
    int max_tau = 0;
    for (auto &p : plans)
        for (int sum = p.end_gen; sum >= p.lo_solve && sum > 0; sum -= 2) max_tau = std::max(max_tau, (p.end_gen - sum) / 2 + 1);
    Solved t2, t4, cur;
    GraphRunner graph;
    if (ok) ok = solve_prepare();  // function attributes are set outside any capture
    for (int tau = 0; ok && tau < max_tau; tau++) {
        cur.parts.clear();
        cur.sums.clear();
        std::vector<std::pair<const u64 *, Range>> srcs;  // (store pointer of the block, range)
        u64 n = 0;
        for (int f = 0; ok && f < nf; f++) {
            const Plan &p = plans[f];
            const int sum = p.end_gen - 2 * tau;
            if (sum < p.lo_solve || sum <= 0) continue;
            Range src{-1, 0, 0};
            if (sum >= p.start && (sum - p.start) / 2 < (int)sink.ranges[f].size())
                src = sink.ranges[f][(sum - p.start) / 2];
            Range dst{-1, n, src.n};
            cur.parts.push_back({f, dst});
            cur.sums.push_back(sum);
            if (src.n) {
                const u64 *base = sink.store.ptr(sink.blocks[src.block].h, s);  // restores a spilled block
                if (!base) ok = false;
                srcs.push_back({base, src});
            }
            n += src.n;
        }
        if (!ok) break;
        // buffers before the capture: allocations are not part of the graph
        cur.n = n;
        const u64 cap = hash_capacity(n);
        ok = dev_alloc((void **)&cur.keys, 8 * n + 8, s) && dev_alloc(&cur.vals, (u64)vbytes * n + 8, s) &&
             dev_alloc(&cur.slots, 16 * cap + 16, s);
        if (!ok) break;
        const bool capture = b->use_graphs != 0;
        if (capture && !CGB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal))) {
            ok = false;
            break;
        }
        bool enq = true;
        u64 at = 0;
        for (auto &x : srcs) {
            // srcs follow cur.parts in order; empty ranges were skipped
            while (at < cur.parts.size() && cur.parts[at].second.n == 0) at++;
            enq = enq && CGB_CUDA(cudaMemcpyAsync(cur.keys + cur.parts[at].second.off, x.first + x.second.off,
                                                   8 * x.second.n, cudaMemcpyDeviceToDevice, s));
            at++;
        }
        enq = enq && solve_layer_enqueue(cur.keys, n, cur.vals, vbytes, t2.ix, t4.ix, rules, e.rt, d_probes, s);
        cur.ix.keys = cur.keys;
        cur.ix.vals = cur.vals;
        cur.ix.n = n;
        enq = enq && build_hash_enqueue(cur.ix, vbytes, cur.slots, cap, d_err, s);
        if (capture) ok = graph.finish(s, enq);
        else ok = enq;
        if (!ok) break;
        kstats().launches += 2;
        st->boards_solved += n;
        st->solve_steps++;
        const bool enqueued = b->table_fn != nullptr;  // this step's copy reads only cur
        if (b->table_fn) {
            // one copy of the step's union; the callback hands out each formation's range
            // (formations whose layer is empty at this step get an empty table)
            cgb_batch_table_fn tf = b->table_fn;
            void *u = b->user;
            auto parts = cur.parts;
            auto sums = cur.sums;
            std::vector<int> index(nf);
            for (int f = 0; f < nf; f++) index[f] = plans[f].index;
            const int prec = vbytes == 8 ? 64 : 32;
            const u64 total = n;
            ok = out.enqueue({{cur.keys, n * 8}, {cur.vals, n * (u64)vbytes}},
                             [tf, u, parts, sums, index, prec, total, vbytes](const char *h) {
                                 const uint64_t *keys = (const uint64_t *)h;
                                 const char *vals = h + 8 * total;
                                 for (size_t i = 0; i < parts.size(); i++) {
                                     const Range &r = parts[i].second;
                                     if (tf(u, index[parts[i].first], sums[i], keys + r.off, vals + r.off * vbytes,
                                            r.n, prec) != 0)
                                         return false;
                                 }
                                 return true;
                             });
            if (!ok) break;
        }
        // blocks whose every range has been gathered leave the store, t4 below.
        // When this step's table was enqueued, the copies still in flight are
        // this step's and the previous step's (an enqueue first completes the
        // copy it replaces), neither reading them; otherwise fence every copy
        if (!enqueued) ok = out.fence_main();
        for (auto &x : srcs) {
            auto &blk = sink.blocks[x.second.block];
            if (--blk.refs == 0 && blk.live) {
                sink.store.release(blk.h, s);
                blk.live = false;
            }
        }
        free_solved(t4, s);
        t4 = t2;
        t2 = cur;
        cur = Solved{};
    }
    if (ok) ok = out.drain();
    out.fence_main();
    free_solved(t2, s);
    free_solved(t4, s);
    free_solved(cur, s);
    sink.store.clear(s);
    u64 ctr[2] = {0, 0};
    if (ok) ok = CGB_CUDA(cudaMemcpyAsync(ctr, d_tab + off_ctr, 16, cudaMemcpyDeviceToHost, s)) && e.sync();
    if (ok && (u32)ctr[1]) {
        set_error("cgb_batch_run: device error " + err_string((u32)ctr[1]));
        ok = false;
    }
    dev_free(d_tab, s);
    cudaEventRecord(ev[2], s);
    cudaEventSynchronize(ev[2]);
    float gen_ms = 0, solve_ms = 0;
    cudaEventElapsedTime(&gen_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&solve_ms, ev[1], ev[2]);
    for (auto &x : ev) cudaEventDestroy(x);
    st->gen_ms += gen_ms;
    st->solve_ms += solve_ms;
    st->lookups += ctr[0];
    st->graph_launches += graph.launches;
    return ok;
}

// plans of every formation, in groups whose fixed-cell mask orbits are
// pairwise disjoint (greedy, first group that fits, at most 255 per group)
bool make_groups(const cgb_formation *fs, int n, std::vector<std::vector<Plan>> &groups, std::vector<int> *group_of)
{
    std::vector<Plan> all(n);
    for (int i = 0; i < n; i++) {
        const cgb_formation &f = fs[i];
        Plan &p = all[i];
        p.index = i;
        if (f.n_initial == 0 || !f.initial) {
            set_error("cgb_batch: formation " + std::to_string(i) + " has no initial boards");
            return false;
        }
        p.initial.assign(f.initial, f.initial + f.n_initial);
        p.start = tile_sum_host(p.initial[0]);
        p.mask = fixed_pattern(p.initial[0]);
        for (u64 x : p.initial)
            if (tile_sum_host(x) != p.start || fixed_pattern(x) != p.mask) {
                set_error("cgb_batch: formation " + std::to_string(i) +
                          ": initial boards must share one tile sum and one set of fixed cells");
                return false;
            }
        std::sort(p.initial.begin(), p.initial.end());
        p.initial.erase(std::unique(p.initial.begin(), p.initial.end()), p.initial.end());
        p.end_gen = f.end_gen;
        p.lo_solve = std::max(f.end_solve, 0);
        p.steps = f.end_gen >= p.start ? (f.end_gen - p.start) / 2 + 1 : 0;
        p.winstates = expand_winstates(f.winstates, f.n_winstates);
    }
    std::vector<std::vector<char>> taken;  // per group: masks used
    if (group_of) group_of->assign(n, -1);
    for (auto &p : all) {
        u32 orbit[8];
        mask_orbit(p.mask, orbit);
        size_t g = 0;
        for (; g < groups.size(); g++) {
            bool clash = groups[g].size() >= 255;
            for (u32 m : orbit) clash |= taken[g][m] != 0;
            if (!clash) break;
        }
        if (g == groups.size()) {
            groups.emplace_back();
            taken.emplace_back(65536, 0);
        }
        for (u32 m : orbit) taken[g][m] = 1;
        if (group_of) (*group_of)[p.index] = (int)g;
        groups[g].push_back(std::move(p));
    }
    return true;
}

}  // namespace

extern "C" int cgb_batch_plan(const cgb_formation *formations, int n_formations, int *group_of)
{
    std::vector<std::vector<Plan>> groups;
    std::vector<int> g;
    if (n_formations < 0 || !make_groups(formations, n_formations, groups, &g)) return -1;
    if (group_of)
        for (int i = 0; i < n_formations; i++) group_of[i] = g[i];
    return (int)groups.size();
}

extern "C" int cgb_batch_run(const cgb_batch *b, cgb_batch_stats *stats)
{
    if (!ensure_rules_for_api()) return -1;
    Engine &e = Engine::get();
    cgb_batch_stats st{};
    if (b->precision != 32 && b->precision != 64) {
        set_error("cgb_batch_run: precision must be 64 or 32");
        return -1;
    }
    if (e.rules.free_formation) {
        set_error("cgb_batch_run: needs free_formation off (fixed cells must not move)");
        return -1;
    }
    if (b->n_formations <= 0) {
        if (stats) *stats = st;
        return 0;
    }
    std::vector<std::vector<Plan>> groups;
    if (!make_groups(b->formations, b->n_formations, groups, nullptr)) return -1;
    AsyncOut out;
    if (!out.init(e.stream, e.io_stream, e.out_stage)) return -1;
    const KernelStats k0 = kstats();
    bool ok = true;
    for (auto &g : groups) {
        ok = run_group(e, b, g, &st, out);
        if (!ok) break;
    }
    st.groups = groups.size();
    st.total_ms = st.gen_ms + st.solve_ms;
    st.d2h_bytes = out.d2h;
    const KernelStats k1 = kstats();
    st.gpu_launches = k1.launches - k0.launches;
    if (stats) *stats = st;
    return ok ? 0 : -1;
}
