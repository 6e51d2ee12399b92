// engine.cu -- device runtime: memory, the generation sweep and the solve sweep.
//
// Generation (src/generate.c:409-615) keeps the rolling sets on the device:
//   S_s    boards of tile sum s still to move (the reference's n)
//   U4     sorted unique 4-spawns of the previous layer (the reference's n4,
//          carried to become part of n2)
// and per layer runs
//   moved = unique(sort(expand_moves(S_s)))           -> the layer s.boards
//   U2    = sort(spawn2(moved))                        (repeats kept)
//   U4'   = sort(spawn4(moved))                        (repeats kept)
//   S_s+2 = merge_unique(U2, U4)                       (src/generate.c:530-544)
// (the merge drops repeats inside its runs as well as across them; the unique
// pass of the move step also counts the spawns the next step will make)
// Layers go to a LayerSink: it keeps them in HBM (the resident gen+solve
// run) or copies them out (files through the C API).
//
// Solve (src/solve.c:172-224) walks the layers top-down with the s+2 and s+4
// tables resident.
#include "engine.h"
#include "cgb_engine.h"
#include <algorithm>
#include <mutex>
#include <unordered_map>

namespace cgb {

// ---- errors -----------------------------------------------------------------
static std::string g_last_error;
static std::mutex g_err_mu;

void set_error(const std::string &msg)
{
    std::lock_guard<std::mutex> g(g_err_mu);
    g_last_error = msg;
}
const char *last_error()
{
    std::lock_guard<std::mutex> g(g_err_mu);
    return g_last_error.c_str();
}
bool cuda_ok(cudaError_t e, const char *what, const char *file, int line)
{
    if (e == cudaSuccess) return true;
    char buf[512];
    snprintf(buf, sizeof buf, "%s:%d: %s failed: %s", file, line, what, cudaGetErrorString(e));
    set_error(buf);
    return false;
}
std::string err_string(u32 err)
{
    std::string s;
    if (err & ERR_LOOKBACK_TIMEOUT) s += "[look-back wait timed out]";
    if (err & ERR_CAPACITY) s += "[output capacity exceeded]";
    if (err & ERR_UNSORTED) s += "[input not sorted]";
    if (err & ERR_TOO_LARGE) s += "[size beyond 32-bit counters]";
    if (err & ERR_COPY_TIMEOUT) s += "[bulk copy wait timed out]";
    return s.empty() ? "[none]" : s;
}

// ---- kernel clocks ----------------------------------------------------------
KernelStats &kstats()
{
    static KernelStats k;
    return k;
}
KClock &kclock()
{
    static KClock c;
    return c;
}
cudaEvent_t KClock::take()
{
    if (free_.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    cudaEvent_t e = free_.back();
    free_.pop_back();
    return e;
}
void KClock::begin(cudaStream_t s, double *acc)
{
    open_ = take();
    open_acc_ = acc;
    cudaEventRecord(open_, s);
    kstats().launches++;
}
void KClock::end(cudaStream_t s)
{
    if (!open_) return;
    cudaEvent_t b = take();
    cudaEventRecord(b, s);
    pend_.push_back({open_, b, open_acc_});
    open_ = nullptr;
}
void KClock::flush()
{
    for (auto &p : pend_) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess && p.acc) *p.acc += ms;
        free_.push_back(p.a);
        free_.push_back(p.b);
    }
    pend_.clear();
}

// ---- memory -----------------------------------------------------------------
// Every engine allocation goes through dev_alloc/dev_free, which count the
// bytes held, so that a cap (option device_mem_cap_mb: a host whose allocator
// gives this library a fixed budget) turns into a clean allocation failure.
u64 g_dev_mem_cap = 0;
static std::mutex g_mem_mu;
static std::unordered_map<void *, u64> g_mem_blocks;
static u64 g_mem_held = 0;

bool dev_alloc(void **p, u64 bytes, cudaStream_t s)
{
    *p = nullptr;
    if (bytes == 0) bytes = 256;
    {
        std::lock_guard<std::mutex> g(g_mem_mu);
        if (g_dev_mem_cap && g_mem_held + bytes > g_dev_mem_cap) {
            char buf[200];
            snprintf(buf, sizeof buf, "device allocation of %.3f GB failed: over the cap of %.3f GB (%.3f GB held)",
                     bytes / 1e9, g_dev_mem_cap / 1e9, g_mem_held / 1e9);
            set_error(buf);
            return false;
        }
    }
    cudaError_t e = cudaMallocAsync(p, bytes, s);
    if (e == cudaErrorMemoryAllocation) {
        // freed blocks of other sizes may still sit in the pool: return them
        // to the device and retry once
        cudaGetLastError();
        cudaStreamSynchronize(s);
        int dev = 0;
        cudaGetDevice(&dev);
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
        kstats().pool_trims++;
        e = cudaMallocAsync(p, bytes, s);
    }
    if (e != cudaSuccess) {
        char buf[160];
        snprintf(buf, sizeof buf, "device allocation of %.3f GB failed: %s", bytes / 1e9, cudaGetErrorString(e));
        set_error(buf);
        cudaGetLastError();
        *p = nullptr;
        return false;
    }
    std::lock_guard<std::mutex> g(g_mem_mu);
    g_mem_blocks[*p] = bytes;
    g_mem_held += bytes;
    return true;
}
void dev_free(void *p, cudaStream_t s)
{
    if (!p) return;
    {
        std::lock_guard<std::mutex> g(g_mem_mu);
        auto it = g_mem_blocks.find(p);
        if (it != g_mem_blocks.end()) {
            g_mem_held -= it->second;
            g_mem_blocks.erase(it);
        }
    }
    cudaFreeAsync(p, s);
}

// free device memory plus what the stream-ordered pool holds cached but unused
u64 device_available_bytes(int dev)
{
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    cudaMemPool_t pool;
    u64 reserved = 0, used = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    }
    return (u64)free_b + (reserved > used ? reserved - used : 0);
}

// ---- resident layer store ---------------------------------------------------
bool LayerStore::push(u64 n, cudaStream_t s, Handle *h)
{
    const u64 need = n ? n : 1;
    if (chunks_.empty() || !chunks_.back().base || chunks_.back().top + need > chunks_.back().cap) {
        Chunk c;
        c.cap = std::max<u64>(need, chunk_bytes / 8);
        if (!dev_alloc((void **)&c.base, c.cap * 8, s)) return false;
        chunks_.push_back(std::move(c));
    }
    Chunk &c = chunks_.back();
    h->chunk = (int)chunks_.size() - 1;
    h->off = c.top;
    h->n = n;
    c.blocks.push_back({c.top, need, true});
    c.top += need;
    return true;
}

u64 *LayerStore::ptr(const Handle &h, cudaStream_t s)
{
    if (h.chunk < 0) return nullptr;
    Chunk &c = chunks_[h.chunk];
    if (!c.base) {  // spilled: bring the chunk back
        if (!dev_alloc((void **)&c.base, c.cap * 8, s)) return nullptr;
        if (!CGB_CUDA(cudaStreamWaitEvent(s, c.copied, 0))) return nullptr;
        if (c.top && !CGB_CUDA(cudaMemcpyAsync(c.base, c.host, c.top * 8, cudaMemcpyHostToDevice, s))) return nullptr;
        if (!CGB_CUDA(cudaStreamSynchronize(s))) return nullptr;
        cudaFreeHost(c.host);
        c.host = nullptr;
        restores++;
    }
    return c.base + h.off;
}

bool LayerStore::spill(u64 bytes, cudaStream_t s, cudaStream_t io)
{
    u64 done = 0;
    // never the last chunk: the generation appends to it
    for (size_t i = 0; i + 1 < chunks_.size() && done < bytes; i++) {
        Chunk &c = chunks_[i];
        if (!c.base || c.top == 0) continue;
        if (!CGB_CUDA(cudaMallocHost(&c.host, c.top * 8))) return false;
        if (!c.copied && !CGB_CUDA(cudaEventCreateWithFlags(&c.copied, cudaEventDisableTiming))) return false;
        cudaEvent_t written;  // the main stream's writes into the chunk
        if (!CGB_CUDA(cudaEventCreateWithFlags(&written, cudaEventDisableTiming))) return false;
        const bool ok = CGB_CUDA(cudaEventRecord(written, s)) && CGB_CUDA(cudaStreamWaitEvent(io, written, 0)) &&
                        CGB_CUDA(cudaMemcpyAsync(c.host, c.base, c.top * 8, cudaMemcpyDeviceToHost, io)) &&
                        CGB_CUDA(cudaEventRecord(c.copied, io));
        cudaEventDestroy(written);
        if (!ok) return false;
        dev_free(c.base, io);   // back to the pool once the copy has read it
        c.base = nullptr;
        done += c.cap * 8;
        spills++;
    }
    return done > 0;
}

void LayerStore::drop_chunk(Chunk &c, cudaStream_t s)
{
    if (c.base) dev_free(c.base, s);
    if (c.copied) {
        cudaEventSynchronize(c.copied);  // a spill copy may still be reading into c.host
        cudaEventDestroy(c.copied);
        c.copied = nullptr;
    }
    if (c.host) cudaFreeHost(c.host);
    c.base = nullptr;
    c.host = nullptr;
    c.blocks.clear();
    c.top = 0;
}

void LayerStore::release(const Handle &h, cudaStream_t s)
{
    if (h.chunk < 0 || h.chunk >= (int)chunks_.size()) return;
    Chunk &c = chunks_[h.chunk];
    for (auto &b : c.blocks)
        if (b.off == h.off) b.live = false;
    while (!c.blocks.empty() && !c.blocks.back().live) {
        c.top -= c.blocks.back().n;
        c.blocks.pop_back();
    }
    if (c.blocks.empty()) drop_chunk(c, s);
    // drop trailing empty chunks so push() starts a fresh one
    while (!chunks_.empty() && chunks_.back().blocks.empty()) {
        drop_chunk(chunks_.back(), s);
        chunks_.pop_back();
    }
}

void LayerStore::clear(cudaStream_t s)
{
    for (auto &c : chunks_) drop_chunk(c, s);
    chunks_.clear();
}

u64 LayerStore::bytes_in_use() const
{
    u64 b = 0;
    for (auto &c : chunks_)
        if (c.base) b += c.top * 8;
    return b;
}

u64 LayerStore::bytes_spilled() const
{
    u64 b = 0;
    for (auto &c : chunks_)
        if (c.host) b += c.top * 8;
    return b;
}

// ---- engine -----------------------------------------------------------------
Engine &Engine::get()
{
    static Engine e;
    return e;
}

bool Engine::init(int dev)
{
    if (ready && dev == device) return true;
    if (!CGB_CUDA(cudaSetDevice(dev))) return false;
    device = dev;
    if (!stream && !CGB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking))) return false;
    if (!io_stream && !CGB_CUDA(cudaStreamCreateWithFlags(&io_stream, cudaStreamNonBlocking))) return false;
    cudaMemPool_t pool;
    if (!CGB_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev))) return false;
    // keep freed blocks cached in the pool between layer steps; an allocation
    // that fails returns the cache to the device and retries (dev_alloc)
    u64 keep = ~0ull;
    if (!CGB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep))) return false;
    if (!h_spawn_check) {
        void *h = nullptr;
        if (!CGB_CUDA(cudaHostAlloc(&h, 2 * sizeof(u64), cudaHostAllocDefault))) return false;
        h_spawn_check = (u64 *)h;
        h_spawn_check[0] = h_spawn_check[1] = 0;
    }
    if (!spawn_check_ev && !CGB_CUDA(cudaEventCreateWithFlags(&spawn_check_ev, cudaEventDisableTiming))) return false;
    if (!ctr.d) {
        void *p;
        if (!CGB_CUDA(cudaMalloc(&p, 64 * sizeof(u64)))) return false;
        ctr.d = (u64 *)p;
        ctr.err = (u32 *)(ctr.d + 32);
        if (!CGB_CUDA(cudaMemset(p, 0, 64 * sizeof(u64)))) return false;
    }
    ready = true;
    return true;
}

bool Engine::set_rules(const cgb_rules &r)
{
    rules = r;
    return upload_row_table(rt, r.free_formation ? 1 : 0, r.ignore_f ? 1 : 0, stream);
}

PruneParams Engine::prune_params() const
{
    PruneParams p;
    p.enabled = rules.prune ? 1 : 0;
    p.stsl = rules.stsl;
    p.ltc = rules.ltc;
    p.smallest_large = rules.smallest_large;
    return p;
}

bool Engine::sync() { return CGB_CUDA(cudaStreamSynchronize(stream)); }

// grow-only device buffer with 25 % headroom, so layer after layer of slowly
// growing sizes reuses the same allocation
static bool reserve(DevBuf<u64> &b, u64 n, cudaStream_t s)
{
    if (b.p && b.cap >= n) return true;
    return grow(b, n + n / 4 + 1024, s);
}

// sort + unique of n raw keys in x (y = scratch); returns the buffer holding
// the unique keys (the other one is left free)
bool Engine::sort_unique_step(DevBuf<u64> &x, DevBuf<u64> &y, u64 n, u64 *nu, DevBuf<u64> **out, GenTimes *tm,
                              u64 *empties)
{
    cudaStream_t s = stream;
    u64 *sorted = x.p;
    SortStats st;
    if (!sort_keys(x.p, y.p, n, &sorted, ws, s, &st)) return false;
    if (tm) {
        tm->sorted_keys += n;
        tm->sort_passes += (u64)st.passes * n;
    }
    DevBuf<u64> &full = (sorted == x.p) ? x : y;
    DevBuf<u64> &dst = (sorted == x.p) ? y : x;
    if (!unique_keys(full.p, n, dst.p, nu, ws, s, empties)) return false;
    *out = &dst;
    return true;
}

// sort of n raw keys in x (y = scratch), repeats kept: the merge that takes the
// result drops them; returns the buffer holding the sorted keys
bool Engine::sort_step(DevBuf<u64> &x, DevBuf<u64> &y, u64 n, DevBuf<u64> **out, GenTimes *tm)
{
    u64 *sorted = x.p;
    SortStats st;
    if (!sort_keys(x.p, y.p, n, &sorted, ws, stream, &st)) return false;
    if (tm) {
        tm->sorted_keys += n;
        tm->sort_passes += (u64)st.passes * n;
    }
    *out = (sorted == x.p) ? &x : &y;
    return true;
}

// acc = acc u run (both sorted), through the scratch buffer t
bool Engine::merge_into(DevBuf<u64> &acc, const u64 *run, u64 n)
{
    cudaStream_t s = stream;
    GenBuffers &g = gen;
    if (!reserve(g.t, acc.n + n, s)) return false;
    u64 nm = 0;
    if (!merge_unique(acc.p, acc.n, run, n, g.t.p, &nm, ws, s)) return false;
    std::swap(acc, g.t);
    acc.n = nm;
    return true;
}

// moved = unique(sort(expand_moves(S))); an input whose raw moves exceed
// max_sort_keys is cut into slices whose sorted unique moves are merged
bool Engine::move_layer(const u64 *d_in, u64 n, GenTimes *tm)
{
    cudaStream_t s = stream;
    GenBuffers &g = gen;
    const u64 slice = std::max<u64>(1, max_sort_keys / 4);
    const bool chunked = n > slice;
    const u64 m0 = chunked ? slice : n;
    if (!reserve(g.a, 4 * m0, s) || !reserve(g.b, 4 * m0, s)) return false;
    if (chunked) g.moved.n = 0;
    g.moved_empties_known = false;
    for (u64 off = 0; off < n || (n == 0 && off == 0); off += m0) {
        const u64 m = std::min(m0, n - off);
        u64 nr = 0;
        if (!expand_moves(d_in + off, m, g.a.p, 4 * m, &nr, rt, prune_params(), ctr, s, filter, plan)) return false;
        u64 nu = 0, empties = 0;
        DevBuf<u64> *u = nullptr;
        if (!sort_unique_step(g.a, g.b, nr, &nu, &u, tm, chunked ? nullptr : &empties)) return false;
        if (!chunked) {
            std::swap(*u, g.moved);   // the layer; the old layer buffer becomes scratch
            g.moved.n = nu;
            g.moved_empties = empties;
            g.moved_empties_known = true;
            return true;
        }
        if (!merge_into(g.moved, u->p, nu)) return false;
        if (tm) tm->chunks++;
    }
    return true;
}

// U2 / U4: sorted canonical 2-spawns and 4-spawns of the moved layer (unique
// when unique_streams; else repeats stay for the next merge to drop);
// U2 lands in g.u2, U4 in g.u4_next.  Spawn streams longer than max_sort_keys
// are produced slice by slice and merged.
bool Engine::spawn_layer(GenTimes *tm, bool unique_streams)
{
    cudaStream_t s = stream;
    GenBuffers &g = gen;
    const u64 *d_moved = g.moved.p;
    const u64 n = g.moved.n;
    // the spawn total: counted by the move step's unique pass, else by a kernel
    u64 total = 0;
    if (g.moved_empties_known) total = g.moved_empties;
    else if (!count_spawns(d_moved, n, &total, ctr, s)) return false;
    g.moved_empties_known = false;  // it belongs to this layer only
    const bool chunked = total > max_sort_keys;
    const u64 cap = chunked ? max_sort_keys : total;
    for (auto &x : g.c)
        if (!reserve(x, cap, s)) return false;
    if (chunked) g.u2.n = g.u4_next.n = 0;
    // first guess of a slice that fits; halved while its count does not
    u64 step = chunked ? std::max<u64>(1, (u64)((double)n * 0.9 * (double)max_sort_keys / (double)total)) : n;
    for (u64 off = 0; off < n || (n == 0 && off == 0);) {
        u64 m = std::min(step, n - off);
        u64 t = total;
        if (chunked) {
            for (;;) {
                if (!count_spawns(d_moved + off, m, &t, ctr, s)) return false;
                if (t <= max_sort_keys || m == 1) break;
                m = (m + 1) / 2;
            }
            if (t > max_sort_keys) {
                set_error("spawn_layer: one board spawns more keys than max_sort_keys");
                return false;
            }
        }
        u64 ns = 0;
        // one slice: the streams hold exactly t keys each; the kernel's count and
        // error word are checked after the first sort below has waited on the
        // stream anyway.  Slices keep the synchronous check.
        const bool deferred = !chunked;
        if (deferred) {
            if (!expand_spawns_deferred(d_moved + off, m, g.c[0].p, g.c[1].p, t, ctr, s, plan, h_spawn_check,
                                        spawn_check_ev))
                return false;
            ns = t;
        } else if (!expand_spawns(d_moved + off, m, g.c[0].p, g.c[1].p, t, &ns, ctr, s, plan)) {
            return false;
        }
        // the 2-spawns sort c[0] with c[2] as scratch; the 4-spawns then sort
        // c[1] with the buffer the first sort left free.  Without unique_streams
        // the sorted streams keep their repeats: every later merge drops them
        DevBuf<u64> *u2 = nullptr, *u4 = nullptr;
        u64 n2 = ns, n4 = ns;
        if (unique_streams) {
            if (!sort_unique_step(g.c[0], g.c[2], ns, &n2, &u2, tm)) return false;
        } else if (!sort_step(g.c[0], g.c[2], ns, &u2, tm)) {
            return false;
        }
        if (deferred && !check_spawns_deferred(h_spawn_check, spawn_check_ev, t)) return false;
        DevBuf<u64> &spare = (u2 == &g.c[0]) ? g.c[2] : g.c[0];
        if (unique_streams) {
            if (!sort_unique_step(g.c[1], spare, ns, &n4, &u4, tm)) return false;
        } else if (!sort_step(g.c[1], spare, ns, &u4, tm)) {
            return false;
        }
        if (!chunked) {
            std::swap(g.u2, *u2);
            g.u2.n = n2;
            std::swap(g.u4_next, *u4);
            g.u4_next.n = n4;
            return true;
        }
        if (!merge_into(g.u2, u2->p, n2) || !merge_into(g.u4_next, u4->p, n4)) return false;
        if (tm) tm->chunks++;
        off += m;
    }
    return true;
}

bool Engine::generate(const u64 *h_initial, u64 n_init, int start, int end, LayerSink &sink, GenTimes *tm,
                      const u64 *h_carry, u64 n_carry)
{
    cudaStream_t s = stream;
    GenBuffers &g = gen;
    if (!reserve(g.S, n_init, s) || !reserve(g.u4, n_carry, s)) return false;
    if (n_init && !CGB_CUDA(cudaMemcpyAsync(g.S.p, h_initial, n_init * 8, cudaMemcpyHostToDevice, s))) return false;
    if (n_carry && !CGB_CUDA(cudaMemcpyAsync(g.u4.p, h_carry, n_carry * 8, cudaMemcpyHostToDevice, s))) return false;
    g.S.n = n_init;
    g.u4.n = n_carry;
    // canonical layer boards share the 0xf mask of the canonical first board (fixed
    // formation cells); the kernels check every board against it
    plan = (n_init && !filter.fid) ? make_canon_plan(canonical(h_initial[0]), rules.free_formation != 0) : CanonPlan{};
    bool ok = true;
    for (int layer = start; layer <= end && ok; layer += 2) {
        ok = move_layer(g.S.p, g.S.n, tm);
        if (!ok) break;
        ok = spawn_layer(tm);
        if (!ok) break;
        // S_{s+2} = U2 u U4(previous layer)
        if (!reserve(g.S, g.u2.n + g.u4.n, s)) {
            ok = false;
            break;
        }
        u64 nm = 0;
        ok = merge_unique(g.u2.p, g.u2.n, g.u4.p, g.u4.n, g.S.p, &nm, ws, s);
        if (!ok) break;
        g.S.n = nm;
        std::swap(g.u4, g.u4_next);
        if (tm) tm->boards += g.moved.n;
        bool kept = false;
        ok = sink.layer(layer, g.moved.p, g.moved.n, s, &kept);
        if (kept) {
            g.moved.p = nullptr;
            g.moved.cap = g.moved.n = 0;
        }
    }
    if (ok) ok = sync();
    return ok;
}

void Engine::release_buffers()
{
    GenBuffers &g = gen;
    for (DevBuf<u64> *b : {&g.a, &g.b, &g.c[0], &g.c[1], &g.c[2], &g.S, &g.u2, &g.u4, &g.u4_next, &g.moved, &g.t})
        drop(*b, stream);
}

}  // namespace cgb
