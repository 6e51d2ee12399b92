// engine.h -- internal interfaces of the CUDA engine (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "common.cuh"
#include "board.cuh"
#include "hashidx.cuh"

namespace cgb {

// ---- sort / unique / merge (sort.cu) ------------------------------------
struct SortWorkspace {
    static constexpr int SMALL_WORDS = 8192;
    u32 *small = nullptr;       // histograms, tile counters, error word, counts
    u32 *lookback = nullptr;    // decoupled look-back state
    u64 lookback_bytes = 0;
    bool err_dirty = false;     // a sort left its errors in the word for unique to report
    bool reserve(u64 words, cudaStream_t s);
    void release(cudaStream_t s);
};

struct SortStats {
    int passes = 0;
    u64 n = 0;
};

int sort_plan(const u32 *hist_host, u64 n, int *digits);
// sorts keys[0,n) ascending using tmp[0,n); *sorted points at keys or tmp
bool sort_keys(u64 *keys, u64 *tmp, u64 n, u64 **sorted, SortWorkspace &ws, cudaStream_t s,
               SortStats *stats = nullptr);
// reports device errors a sort left behind (when no unique_keys follows)
bool sort_check(SortWorkspace &ws, cudaStream_t s);
// out must not alias in
// empties (optional): the number of empty cells over the kept keys
bool unique_keys(const u64 *in, u64 n, u64 *out, u64 *n_out, SortWorkspace &ws, cudaStream_t s,
                 u64 *empties = nullptr);
// sorted union of two sorted runs, without repeats (repeats inside a run are
// dropped as well)
bool merge_unique(const u64 *a, u64 na, const u64 *b, u64 nb, u64 *out, u64 *n_out, SortWorkspace &ws,
                  cudaStream_t s);

// ---- row table and expansion (expand.cu) ---------------------------------
struct DeviceRowTable {
    unsigned short *move = nullptr;  // 65536 rows, left move; ROW_LOCKED where a 0xf cell would move
    int free_formation = -1, ignore_f = -1;
};

// the left-move row table of the reference (src/board.c:62-132), host side
void build_row_table(int free_formation, int ignore_f, unsigned short *move, u32 *ok);
bool upload_row_table(DeviceRowTable &t, int free_formation, int ignore_f, cudaStream_t s);

struct Counters {
    u64 *d = nullptr;   // device words: [0] output count, [1] spawn total, [2..] scratch
    u32 *err = nullptr; // device error word
};

// move + prune + canonicalise every board; out needs room for 4n boards
// batched sweeps: stable partition by formation id (fid table of 65536
// entries, see fixed_pattern); counts[f] = boards of formation f
bool partition_by_formation(const u64 *in, u64 n, u64 *out, const unsigned char *fid, u32 counts[256],
                            SortWorkspace &ws, cudaStream_t s);
bool expand_moves(const u64 *in, u64 n, u64 *out, u64 cap, u64 *n_out, const DeviceRowTable &t,
                  const PruneParams &p, Counters &c, cudaStream_t s, FormationFilter ff = FormationFilter{},
                  const CanonPlan &plan = CanonPlan{});
// number of empty cells over all boards (exact size of the spawn streams)
bool count_spawns(const u64 *in, u64 n, u64 *total, Counters &c, cudaStream_t s);
// expand_spawns with cap = the exact spawn total and no wait: its count and error
// word land in h_check (pinned, 2 words) behind `done`, for check_spawns_deferred
bool expand_spawns_deferred(const u64 *in, u64 n, u64 *out2, u64 *out4, u64 cap, Counters &c, cudaStream_t s,
                            const CanonPlan &plan, u64 *h_check, cudaEvent_t done);
bool check_spawns_deferred(const u64 *h_check, cudaEvent_t done, u64 expect);
// canonical 2-spawn and 4-spawn of every empty cell of every board
bool expand_spawns(const u64 *in, u64 n, u64 *out2, u64 *out4, u64 cap, u64 *n_out, Counters &c,
                   cudaStream_t s, const CanonPlan &plan = CanonPlan{});

// ---- solve (solve.cu) ------------------------------------------------------
struct SolveRules {
    int nox = 0;       // char semantics already applied
    int score = 0;
    const u64 *winstates = nullptr;  // device, expanded x8
    int n_winstates = 0;
    // batched sweeps: formation f's winstates are winstates[ws_begin[f] ..
    // ws_begin[f+1]), f = fid[fixed_pattern(board)]
    const unsigned char *fid = nullptr;
    const u32 *ws_begin = nullptr;
};

// Lookup index over one solved layer (replaces the bisection of lookup(),
// src/solve.c:108-164; every kind returns the value of the key or 0.0).
enum IndexKind : int {
    INDEX_BISECT = 0,  // bisection over the sorted keys (the reference's search)
    INDEX_BUCKET = 1,  // top-bits bucket offsets after the common prefix, then bisection
    INDEX_HASH = 2,    // open addressing, key and value in one 16-byte slot
};

struct LayerIndex {
    int kind = INDEX_BISECT;
    const u64 *keys = nullptr;
    const void *vals = nullptr;   // double or float, aligned with keys
    u64 n = 0;
    // INDEX_BUCKET
    const u32 *bucket = nullptr;  // 2^bits + 1 offsets
    int prefix = 0;               // bucket = (key << prefix) >> (64 - bits)
    int bits = 0;
    u64 prefix_value = 0;         // the shared high bits (key >> (64 - prefix))
    // INDEX_HASH
    const void *slots = nullptr;  // cap slots of {u64 key, u64 value bits}; key 0 = empty
    u64 cap = 0;
    CompactHash ch;               // ch.on: cap (a power of two) 8-byte slots instead
};

// device storage owned by one index (reused across layers)
struct IndexStorage {
    void *p = nullptr;
    u64 bytes = 0;
};

// graph-capturable forms (no host round trip): the solve kernel, counting
// probes into *probes, and the hash index into caller-owned slots
// (hash_capacity(n) slots of 16 bytes); device errors accumulate in *err
bool solve_layer_enqueue(const u64 *keys, u64 n, void *out, int vbytes, const LayerIndex &t2, const LayerIndex &t4,
                         const SolveRules &r, const DeviceRowTable &rt, u64 *probes, cudaStream_t s);
u64 hash_capacity(u64 n);
bool solve_prepare();  // one-time kernel attributes (call before a capture)
bool build_hash_enqueue(LayerIndex &ix, int vbytes, void *slots, u64 cap, u32 *err, cudaStream_t s);

// builds ix (keys/vals/n already set) of the requested kind; vbytes = 8 or 4
bool build_index(LayerIndex &ix, int kind, int vbytes, IndexStorage &st, int bucket_bits, Counters &c,
                 cudaStream_t s);
// the value of each of m boards (canonicalised first when canon) in an indexed
// layer, widened to double; 0.0 for a board not in it
bool lookup_batch(const LayerIndex &ix, int vbytes, const u64 *boards, u64 m, bool canon, double *out,
                  cudaStream_t s);

// plan: images that can be canonical for the layer's 0xf mask (CanonPlan{}: all eight)
bool solve_layer_f64(const u64 *keys, u64 n, double *out, const LayerIndex &t2, const LayerIndex &t4,
                     const SolveRules &r, const DeviceRowTable &rt, Counters &c, cudaStream_t s,
                     const CanonPlan &plan = CanonPlan{});
bool solve_layer_f32(const u64 *keys, u64 n, float *out, const LayerIndex &t2, const LayerIndex &t4,
                     const SolveRules &r, const DeviceRowTable &rt, Counters &c, cudaStream_t s,
                     const CanonPlan &plan = CanonPlan{});

// ---- device memory --------------------------------------------------------
template <typename T>
struct DevBuf {
    T *p = nullptr;
    u64 n = 0;     // elements in use
    u64 cap = 0;   // elements allocated
};

bool dev_alloc(void **p, u64 bytes, cudaStream_t s);
void dev_free(void *p, cudaStream_t s);
template <typename T>
bool grow(DevBuf<T> &b, u64 n, cudaStream_t s)
{
    if (b.cap >= n && b.p) return true;
    if (b.p) dev_free(b.p, s);
    b.p = nullptr;
    b.cap = 0;
    u64 want = n < 64 ? 64 : n;
    if (!dev_alloc((void **)&b.p, want * sizeof(T), s)) return false;
    b.cap = want;
    return true;
}
template <typename T>
void drop(DevBuf<T> &b, cudaStream_t s)
{
    if (b.p) dev_free(b.p, s);
    b.p = nullptr;
    b.n = b.cap = 0;
}

// Resident layers of a sweep.  Layers are appended during generation and
// released top-down during the solve (last in, first out), so they are packed
// into a few large chunks instead of one allocation per layer; nothing is
// fragmented by the short-lived working buffers of each layer step.  When the
// device runs short, whole chunks of the oldest layers (the lowest tile sums,
// which the top-down solve needs last) are spilled to pinned host memory and
// brought back when a layer in them is needed again.  A spill copies on the
// I/O stream and frees the device chunk there, stream-ordered after the copy,
// so the layer loop on the main stream never waits for it.
u64 device_available_bytes(int dev);

class LayerStore {
  public:
    u64 chunk_bytes = 4ull << 30;   // device allocation unit of the store
    struct Handle {
        int chunk = -1;
        u64 off = 0, n = 0;
    };
    bool push(u64 n, cudaStream_t s, Handle *h);      // room for n boards
    u64 *ptr(const Handle &h, cudaStream_t s);         // device address (restores a spilled chunk)
    void release(const Handle &h, cudaStream_t s);     // frees a pushed block
    // spills oldest chunks (never the last) until `bytes` are on their way to
    // the host; false when nothing could be spilled
    bool spill(u64 bytes, cudaStream_t s, cudaStream_t io);
    void clear(cudaStream_t s);
    u64 bytes_in_use() const;
    size_t chunk_count() const { return chunks_.size(); }
    u64 bytes_spilled() const;
    u64 spills = 0, restores = 0;
  private:
    struct Block { u64 off, n; bool live; };
    struct Chunk {
        u64 *base = nullptr;   // device memory (null while spilled)
        void *host = nullptr;  // pinned copy while spilled
        cudaEvent_t copied = nullptr;  // the device-to-host copy of the spill is complete
        u64 cap = 0, top = 0;
        std::vector<Block> blocks;
    };
    std::vector<Chunk> chunks_;
    void drop_chunk(Chunk &c, cudaStream_t s);
};

}  // namespace cgb
