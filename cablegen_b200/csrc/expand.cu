// expand.cu -- the per-board work of one generation layer.
//
// expand_moves restates the move workers of the reference
// (src/generate.c:133-175, OpenCL move_kernel src/cl/generate.cl:249-282):
// optional prune of the input, the four moves, prune of each moved board,
// canonicalisation.  The left-move row table (128 KiB of u16, locked rows
// marked ROW_LOCKED) is staged into shared memory once per CTA of a
// persistent grid; right/up/down reuse it through the board views of
// board.cuh.  Canonical forms take the maximum over the images a CanonPlan
// names for the board's 0xf mask (all eight without a plan).  Repeated
// results of one CTA iteration are dropped through a shared-memory set, and
// the rest are appended with one atomic per CTA iteration after a block scan,
// so the output is compact (no 4N slot array + separate scan).
//
// expand_spawns restates src/generate.c:177-199: every empty cell receives a
// 2 (nibble 1) and a 4 (nibble 2); both boards are canonicalised.  The exact
// output size is counted first (no slot cap, unlike SPAWN_SLOTS=4 of the
// OpenCL path, src/cl/generate.cl:215-245).
#include "engine.h"

namespace cgb {

constexpr int EXP_THREADS = 1024;
constexpr int TABLE_BYTES = 65536 * 2;  // the left-move rows, ROW_LOCKED marking locked ones

void build_row_table(int free_formation, int ignore_f, unsigned short *move, u32 *ok)
{
    // One row = four cells, travel toward cell 0.  Restates move()
    // (src/board.c:62-98): slide the non-empty cells forward, merge equal
    // neighbours below 0xE once each from the front, slide again.  With
    // ignore_f, 0xF cells at the far end are walls.  A row is locked when a
    // cell that held 0xF no longer does (src/board.c:29-38), unless the
    // formation is free.
    for (u32 row = 0; row < 65536; row++) {
        int t[4], pre[4];
        for (int c = 0; c < 4; c++) pre[c] = t[c] = (row >> (12 - 4 * c)) & 0xF;
        int n = 4;
        if (ignore_f)
            while (n > 0 && t[n - 1] == 0xF) n--;
        auto slide = [&]() {
            int w = 0, tmp[4] = {0, 0, 0, 0};
            for (int i = 0; i < n; i++)
                if (t[i]) tmp[w++] = t[i];
            for (int i = 0; i < n; i++) t[i] = tmp[i];
        };
        slide();
        for (int i = 0; i + 1 < n; i++) {
            if (t[i] && t[i] == t[i + 1] && t[i] < 0xE) {
                for (int j = i + 1; j + 1 < n; j++) t[j] = t[j + 1];
                t[n - 1] = 0;
                t[i] += 1;
            }
        }
        slide();
        u32 out = (u32)((t[0] << 12) | (t[1] << 8) | (t[2] << 4) | t[3]);
        bool vacated = false;
        if (!free_formation)
            for (int c = 0; c < 4; c++)
                if (pre[c] == 0xF && t[c] != 0xF) vacated = true;
        move[row] = (unsigned short)out;
        if (row % 32 == 0) ok[row / 32] = 0;
        if (!vacated) ok[row / 32] |= 1u << (row % 32);
    }
    move[0] = 0;          // src/board.c:126-129
    move[0xFFFF] = 0xFFFF;
}

bool upload_row_table(DeviceRowTable &t, int free_formation, int ignore_f, cudaStream_t s)
{
    if (t.move && t.free_formation == free_formation && t.ignore_f == ignore_f) return true;
    std::vector<unsigned short> mv(65536);
    std::vector<u32> ok(2048);
    build_row_table(free_formation, ignore_f, mv.data(), ok.data());
    // the device table marks locked rows with ROW_LOCKED; no legal move yields it
    for (u32 row = 0; row < 65536; row++) {
        const bool legal = (ok[row >> 5] >> (row & 31)) & 1u;
        if (legal && mv[row] == ROW_LOCKED) {
            set_error("upload_row_table: a legal row move yields the locked-row marker");
            return false;
        }
        if (!legal) mv[row] = ROW_LOCKED;
    }
    if (!t.move) {
        void *p = nullptr;
        if (!CGB_CUDA(cudaMalloc(&p, TABLE_BYTES))) return false;
        t.move = (unsigned short *)p;
    }
    if (!CGB_CUDA(cudaMemcpyAsync(t.move, mv.data(), 65536 * 2, cudaMemcpyHostToDevice, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    t.free_formation = free_formation;
    t.ignore_f = ignore_f;
    return true;
}

__device__ __forceinline__ void stage_table(unsigned char *smem, const unsigned short *g_move)
{
    const uint4 *src = (const uint4 *)g_move;
    uint4 *dst = (uint4 *)smem;
    for (int i = threadIdx.x; i < TABLE_BYTES / 16; i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
}

// Set of the move results of one chunk of consecutive input boards (1 to 4
// CTA iterations of 1024 boards) in shared memory: open addressing over 8192
// u64 slots, 0 = empty (no canonical board is 0).  Neighbouring boards of a
// sorted layer often move to the same board (rows that differ only in where
// their tiles sit before a slide), so dropping the repeats here keeps most of
// the raw move stream out of the sort.  Measured on LL layers 144-150 (CPU
// count over the layer's raw moves): a chunk of 1024 boards keeps 51 % of its
// results, 2048 keep 48 %, 4096 keep 44 % (about 4600 set entries, 56 % of the
// slots); the whole layer would keep 17 %.
constexpr int MOVE_SET = 8192;
// boards (in units of 1024) that share one set, 1..4.  Default 1: on the LL
// sweep to tile sum 600 a window of 4 kept 10.5 % fewer moves (sort -44 ms
// per step) but the fuller set's longer probes cost the expansion 108 ms more
int g_move_window = 1;
constexpr int PRUNE_BYTES = ((int)sizeof(PruneTable) + 15) / 16 * 16;
constexpr int EXP_SMEM = TABLE_BYTES + MOVE_SET * 8 + PRUNE_BYTES;

// probes before a key is kept without a slot (a repeat that gets this far is
// kept too: the sort's unique drops it)
constexpr u32 MOVE_PROBES = 64;

__device__ __forceinline__ bool set_insert(unsigned long long *set, u64 key)
{
    u32 h = ((u32)(key >> 32) * 0x9E3779B1u) ^ ((u32)key * 0x85EBCA77u);
    h ^= h >> 15;
    for (u32 i = 0; i < MOVE_PROBES; i++) {
        const u32 slot = (h + i) & (MOVE_SET - 1);
        const unsigned long long prev = atomicCAS(set + slot, 0ull, (unsigned long long)key);
        if (prev == 0ull) return true;   // first copy
        if (prev == key) return false;   // a repeat
    }
    return true;
}

// the four moves of b, pruned, canonicalised (over the plan's images when
// PLANNED, chosen once per warp so that the choice is a uniform branch) and
// checked against the CTA's set; returns the mask of results to write
template <bool PLANNED>
__device__ __forceinline__ u32 board_moves(const RowTable &t, u64 b, const PruneParams &pp, const PruneTable &pt,
                                           const CanonPlan &plan, unsigned long long *set, u64 r[4], u32 *raw)
{
    u64 v[4];
    views(b, v);
    // a move that merges nothing keeps the multiset of tiles, so it keeps
    // the input's (passing) prune verdict; merges show as new empty cells
    const int empties = pp.enabled ? popc64(empty_mask(b)) : 0;
    u32 mask = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        u64 m;
        if (move_left(t, v[k], &m) == 2 && !(pp.enabled && popc64(empty_mask(m)) != empties && prune_by_table(m, pt))) {
            r[k] = PLANNED ? canon_cand(m, plan.cand(k)) : canonical(m);
            (*raw)++;
            if (set_insert(set, r[k])) mask |= 1u << k;
        }
    }
    return mask;
}

__global__ void __launch_bounds__(EXP_THREADS, 1) expand_moves_kernel(const u64 *__restrict__ in, u64 n,
                                                                      u64 *__restrict__ out, u64 cap,
                                                                      u64 *out_count, const unsigned short *g_move,
                                                                      PruneParams pp, const PruneTable *g_prune,
                                                                      u32 *err, FormationFilter ff, CanonPlan plan,
                                                                      u64 *raw_count, u32 window)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ u32 scan_scratch[33];
    __shared__ u64 base_sh;
    // the prune table next to the row table; both staged before the barrier in stage_table
    PruneTable *pt = (PruneTable *)(smem + TABLE_BYTES + MOVE_SET * 8);
    if (pp.enabled)
        for (int i = threadIdx.x; i < PRUNE_BYTES / 16; i += EXP_THREADS)
            ((uint4 *)pt)[i] = __ldg((const uint4 *)g_prune + i);
    stage_table(smem, g_move);
    const RowTable t{(const unsigned short *)smem};
    unsigned long long *set = (unsigned long long *)(smem + TABLE_BYTES);
    // a CTA takes chunks of `window` x 1024 consecutive boards; the set lives
    // for one chunk, so repeats among all of a chunk's moves are dropped
    const u64 chunk = (u64)window * EXP_THREADS;
    u32 raw = 0;  // legal, unpruned moves before the set drops repeats
    for (u64 c0 = (u64)blockIdx.x * chunk; c0 < n; c0 += (u64)gridDim.x * chunk)
    for (u64 first = c0; first < min(c0 + chunk, n); first += EXP_THREADS) {
        if (first == c0) {
            for (int i = threadIdx.x; i < MOVE_SET; i += EXP_THREADS) set[i] = 0ull;
            __syncthreads();
        }
        const u64 idx = first + threadIdx.x;
        u64 r[4] = {0, 0, 0, 0};
        u32 mask = 0;
        const u64 b = idx < n ? in[idx] : 0;
        // the images that can be canonical: the plan's when every board of the warp has its mask
        const bool planned = __all_sync(0xffffffffu, idx >= n || fixed_pattern(b) == plan.mask);
        if (idx < n) {
            // boards of a formation that has reached its last layer stop here
            const bool live = !ff.fid || __ldg(ff.active + __ldg(ff.fid + fixed_pattern(b)));
            if (live && !(pp.enabled && prune_by_table(b, *pt))) {
                if (planned) mask = board_moves<true>(t, b, pp, *pt, plan, set, r, &raw);
                else mask = board_moves<false>(t, b, pp, *pt, plan, set, r, &raw);
            }
        }
        const u32 cnt = __popc(mask);
        u32 total;
        const u32 excl = block_exclusive_scan<u32>(cnt, scan_scratch, &total);
        if (threadIdx.x == 0) base_sh = total ? (u64)atomicAdd((unsigned long long *)out_count, (unsigned long long)total) : 0;
        __syncthreads();
        u64 pos = base_sh + excl;
        if (pos + cnt > cap) {
            if (cnt) atomicOr(err, ERR_CAPACITY);
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (mask & (1u << k)) out[pos++] = r[k];
        }
    }
    const u32 w = __reduce_add_sync(0xffffffffu, raw);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd((unsigned long long *)raw_count, (unsigned long long)w);
}

__global__ void __launch_bounds__(256) count_spawns_kernel(const u64 *__restrict__ in, u64 n, u64 *total)
{
    __shared__ u32 scratch[33];
    u64 acc = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        acc += popc64(empty_mask(in[i]));
    u32 tot;
    block_exclusive_scan<u32>((u32)acc, scratch, &tot);
    if (threadIdx.x == 0 && tot) atomicAdd((unsigned long long *)total, (unsigned long long)tot);
}

// the canonical 2- and 4-spawn of one cell from the board's images: the
// maximum over the images in cand (all eight unless PLANNED)
template <bool PLANNED>
__device__ __forceinline__ void spawn_max(const u64 im[8], int cell, u32 cand, u64 *m2, u64 *m4)
{
#pragma unroll
    for (int k = 0; k < 8; k++) {
        if (PLANNED && !((cand >> k) & 1u)) continue;
        const int sh = 60 - 4 * image_cell(k, cell);
        *m2 = umax64(*m2, im[k] | (1ull << sh));
        *m4 = umax64(*m4, im[k] | (2ull << sh));
    }
}

__global__ void __launch_bounds__(256) expand_spawns_kernel(const u64 *__restrict__ in, u64 n,
                                                            u64 *__restrict__ out2, u64 *__restrict__ out4,
                                                            u64 cap, u64 *out_count, u32 *err, CanonPlan plan)
{
    __shared__ u32 scan_scratch[33];
    __shared__ u64 base_sh;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 first = (u64)blockIdx.x * blockDim.x; first < n; first += stride) {
        const u64 idx = first + threadIdx.x;
        const u64 b = idx < n ? in[idx] : ~0ull;
        u64 e = idx < n ? empty_mask(b) : 0;
        const bool planned = __all_sync(0xffffffffu, idx >= n || fixed_pattern(b) == plan.mask);
        const u32 cnt = popc64(e);
        u32 total;
        const u32 excl = block_exclusive_scan<u32>(cnt, scan_scratch, &total);
        if (threadIdx.x == 0) base_sh = total ? (u64)atomicAdd((unsigned long long *)out_count, (unsigned long long)total) : 0;
        __syncthreads();
        u64 pos = base_sh + excl;
        if (pos + cnt > cap) {
            if (cnt) atomicOr(err, ERR_CAPACITY);
        } else {
            // the images of b once; a spawn adds one nibble to each image.  A spawn
            // keeps b's 0xf cells, so only the plan's images of view 0 can be the
            // maximum when b has the plan's mask
            u64 im[8];
            images(b, im);
            while (e) {
                const int bit = 63 - __clzll(e);  // nibble's low bit
                e &= ~(1ull << bit);
                const int cell = (60 - bit) >> 2;
                u64 m2 = 0, m4 = 0;
                if (planned) spawn_max<true>(im, cell, plan.cand(0), &m2, &m4);
                else spawn_max<false>(im, cell, 0xFFu, &m2, &m4);
                out2[pos] = m2;
                out4[pos] = m4;
                pos++;
            }
        }
    }
}

static int sm_count()
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = NUM_SMS_B200;
    }
    return sms;
}

static bool read_word(u64 *dst, const u64 *src, cudaStream_t s)
{
    if (!CGB_CUDA(cudaMemcpyAsync(dst, src, sizeof(u64), cudaMemcpyDeviceToHost, s))) return false;
    return CGB_CUDA(cudaStreamSynchronize(s));
}

// one copy for a count word and the error word (Counters keeps the error word
// 32 words after the counts)
static bool read_count_checked(u64 *dst, Counters &c, int idx, cudaStream_t s, const char *what,
                               u64 *raw = nullptr)
{
    u64 words[33];
    if (!CGB_CUDA(cudaMemcpyAsync(words, c.d, sizeof words, cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    const u32 e = (u32)words[32];
    if (e) {
        set_error(std::string(what) + ": device error " + err_string(e));
        return false;
    }
    *dst = words[idx];
    if (raw) *raw = words[5];
    return true;
}

static bool check(Counters &c, cudaStream_t s, const char *what)
{
    u32 e = 0;
    if (!CGB_CUDA(cudaMemcpyAsync(&e, c.err, sizeof(u32), cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    if (e) {
        set_error(std::string(what) + ": device error " + err_string(e));
        return false;
    }
    return true;
}

bool expand_moves(const u64 *in, u64 n, u64 *out, u64 cap, u64 *n_out, const DeviceRowTable &t,
                  const PruneParams &p, Counters &c, cudaStream_t s, FormationFilter ff, const CanonPlan &plan)
{
    *n_out = 0;
    if (n == 0) return true;
    static bool attr = false;
    if (!attr) {
        if (!CGB_CUDA(cudaFuncSetAttribute(expand_moves_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           EXP_SMEM)))
            return false;
        attr = true;
    }
    if (!CGB_CUDA(cudaMemsetAsync(c.d, 0, sizeof(u64), s))) return false;
    if (!CGB_CUDA(cudaMemsetAsync(c.d + 5, 0, sizeof(u64), s))) return false;
    if (!CGB_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s))) return false;
    // the prune table of these parameters, in device memory until they change
    static PruneTable *d_prune = nullptr;
    static PruneParams have{-1, -1, -1, -1};
    if (p.enabled && (!d_prune || have.stsl != p.stsl || have.ltc != p.ltc || have.smallest_large != p.smallest_large)) {
        static PruneTable h;
        build_prune_table(p, &h);
        if (!d_prune && !CGB_CUDA(cudaMalloc((void **)&d_prune, PRUNE_BYTES))) return false;
        if (!CGB_CUDA(cudaMemcpyAsync(d_prune, &h, sizeof h, cudaMemcpyHostToDevice, s)) ||
            !CGB_CUDA(cudaStreamSynchronize(s)))
            return false;
        have = p;
    }
    // chunks of up to g_move_window x 1024 boards, no longer than keeps two
    // chunks per SM
    const u64 sms = (u64)sm_count();
    const u32 window = (u32)std::max<u64>(1, std::min<u64>((u64)g_move_window, n / (sms * EXP_THREADS * 2)));
    const u64 chunks = (n + (u64)window * EXP_THREADS - 1) / ((u64)window * EXP_THREADS);
    const int grid = (int)std::min<u64>(chunks, sms);
    kclock().begin(s, &kstats().expand_ms);
    expand_moves_kernel<<<grid, EXP_THREADS, EXP_SMEM, s>>>(in, n, out, cap, c.d, t.move, p, d_prune, c.err, ff,
                                                            plan, c.d + 5, window);
    kclock().end(s);
    if (!CGB_CUDA(cudaGetLastError())) return false;
    u64 raw = 0;
    if (!read_count_checked(n_out, c, 0, s, "expand_moves", &raw)) return false;
    kclock().flush();
    kstats().expand_bytes += 8 * (n + *n_out);
    kstats().moves_raw += raw;
    kstats().moves_kept += *n_out;
    return true;
}

bool count_spawns(const u64 *in, u64 n, u64 *total, Counters &c, cudaStream_t s)
{
    *total = 0;
    if (n == 0) return true;
    if (!CGB_CUDA(cudaMemsetAsync(c.d + 1, 0, sizeof(u64), s))) return false;
    const int grid = (int)std::min<u64>((n + 255) / 256, (u64)sm_count() * 8);
    kclock().begin(s, &kstats().spawn_ms);
    count_spawns_kernel<<<grid, 256, 0, s>>>(in, n, c.d + 1);
    kclock().end(s);
    if (!CGB_CUDA(cudaGetLastError())) return false;
    if (!read_word(total, c.d + 1, s)) return false;
    kclock().flush();
    kstats().spawn_bytes += 8 * n;
    return true;
}

// expand_spawns without the wait: the count and the error word are copied into
// h_check (pinned, two words) behind the kernel and `done` is recorded after the
// copy; check_spawns_deferred reads them once the caller has waited anyway
bool expand_spawns_deferred(const u64 *in, u64 n, u64 *out2, u64 *out4, u64 cap, Counters &c, cudaStream_t s,
                            const CanonPlan &plan, u64 *h_check, cudaEvent_t done)
{
    if (!CGB_CUDA(cudaMemsetAsync(c.d, 0, sizeof(u64), s))) return false;
    if (!CGB_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s))) return false;
    if (n) {
        const int grid = (int)std::min<u64>((n + 255) / 256, (u64)sm_count() * 8);
        kclock().begin(s, &kstats().spawn_ms);
        expand_spawns_kernel<<<grid, 256, 0, s>>>(in, n, out2, out4, cap, c.d, c.err, plan);
        kclock().end(s);
        if (!CGB_CUDA(cudaGetLastError())) return false;
    }
    if (!CGB_CUDA(cudaMemcpyAsync(h_check, c.d, sizeof(u64), cudaMemcpyDeviceToHost, s)) ||
        !CGB_CUDA(cudaMemcpyAsync(h_check + 1, c.err, sizeof(u32), cudaMemcpyDeviceToHost, s)) ||
        !CGB_CUDA(cudaEventRecord(done, s)))
        return false;
    kstats().spawn_bytes += 8 * n + 16 * cap;
    return true;
}

bool check_spawns_deferred(const u64 *h_check, cudaEvent_t done, u64 expect)
{
    if (!CGB_CUDA(cudaEventSynchronize(done))) return false;
    const u32 e = (u32)h_check[1];
    if (e) {
        set_error(std::string("expand_spawns: device error ") + err_string(e));
        return false;
    }
    if (h_check[0] != expect) {
        set_error("expand_spawns: " + std::to_string(h_check[0]) + " spawns written, " + std::to_string(expect) +
                  " expected");
        return false;
    }
    return true;
}

bool expand_spawns(const u64 *in, u64 n, u64 *out2, u64 *out4, u64 cap, u64 *n_out, Counters &c, cudaStream_t s,
                   const CanonPlan &plan)
{
    *n_out = 0;
    if (n == 0) return true;
    if (!CGB_CUDA(cudaMemsetAsync(c.d, 0, sizeof(u64), s))) return false;
    if (!CGB_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s))) return false;
    const int grid = (int)std::min<u64>((n + 255) / 256, (u64)sm_count() * 8);
    kclock().begin(s, &kstats().spawn_ms);
    expand_spawns_kernel<<<grid, 256, 0, s>>>(in, n, out2, out4, cap, c.d, c.err, plan);
    kclock().end(s);
    if (!CGB_CUDA(cudaGetLastError())) return false;
    if (!read_count_checked(n_out, c, 0, s, "expand_spawns")) return false;
    kclock().flush();
    kstats().spawn_bytes += 8 * n + 16 * *n_out;
    return true;
}

}  // namespace cgb
