// cgb_engine.h -- the engine object behind the C ABI.
#pragma once
#include "engine.h"
#include "../../include/cablegen_b200.h"

namespace cgb {

// accumulates the device time of one phase into *acc (CUDA events)
struct Timer {
    cudaStream_t s;
    double *acc;
    cudaEvent_t a = nullptr, b = nullptr;
    Timer(cudaStream_t st, double *p) : s(st), acc(p)
    {
        if (acc) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, s);
        }
    }
    void stop()
    {
        if (!acc || !a) return;
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        *acc += ms;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        a = b = nullptr;
    }
    ~Timer() { stop(); }
};

struct GenTimes {
    double expand_ms = 0, sort_ms = 0, unique_ms = 0, merge_ms = 0;
    u64 boards = 0, sorted_keys = 0, sort_passes = 0;
    u64 chunks = 0;   // slices of layer steps cut at max_sort_keys
};

// receives each generated layer (device pointer, valid on stream s)
struct LayerSink {
    virtual ~LayerSink() {}
    // set *kept = true to take ownership of the device buffer (freed later by
    // the sink with dev_free on the engine stream)
    virtual bool layer(int sum, u64 *d_boards, u64 n, cudaStream_t s, bool *kept) = 0;
};

// pinned staging for device -> host copies of layers and tables
struct HostStage {
    void *p = nullptr;
    u64 bytes = 0;
    // grows with 50 % headroom: pinning memory is slow, so a sequence of
    // growing layers reallocates only a few times
    bool reserve(u64 b)
    {
        if (b <= bytes) return true;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        const u64 want = b + b / 2;
        if (!CGB_CUDA(cudaMallocHost(&p, want))) return false;
        bytes = want;
        return true;
    }
    ~HostStage()
    {
        if (p) cudaFreeHost(p);
    }
};

// Pinned host memory handed out in order and reset per sweep; its chunks are
// kept, so later sweeps pin nothing new.  Holds the host copies of a sweep's
// layers when the caller wants layers and tables both.
struct HostArena {
    struct Chunk {
        void *p = nullptr;
        u64 bytes = 0, top = 0;
    };
    std::vector<Chunk> chunks;
    size_t cur = 0;
    u64 used = 0;  // bytes handed out since the last reset
    void *take(u64 bytes)
    {
        bytes = (bytes + 15) & ~15ull;
        while (cur < chunks.size() && chunks[cur].top + bytes > chunks[cur].bytes) cur++;
        if (cur == chunks.size()) {
            Chunk c;
            c.bytes = bytes > (1ull << 30) ? bytes : (1ull << 30);
            if (cudaMallocHost(&c.p, c.bytes) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
            chunks.push_back(c);
        }
        Chunk &c = chunks[cur];
        void *r = (char *)c.p + c.top;
        c.top += bytes;
        used += bytes;
        return r;
    }
    void reset()
    {
        for (auto &c : chunks) c.top = 0;
        cur = 0;
        used = 0;
    }
};

// working buffers of the generation sweep, kept between layers and calls
struct GenBuffers {
    DevBuf<u64> a, b;          // raw move output and its sort scratch
    DevBuf<u64> c[3];          // raw spawn streams and their sort scratch
    DevBuf<u64> S;             // boards of the next layer to move
    DevBuf<u64> u2, u4, u4_next;
    DevBuf<u64> moved;         // the current layer
    DevBuf<u64> t;             // merge scratch of sliced layer steps
    // empty cells over the moved layer (the size of its spawn streams), counted by
    // the move step's unique pass; unknown after a sliced move step
    u64 moved_empties = 0;
    bool moved_empties_known = false;
};

struct Engine {
    int device = -1;
    bool ready = false;
    cudaStream_t stream = nullptr, io_stream = nullptr;
    DeviceRowTable rt;
    SortWorkspace ws;
    Counters ctr;
    // pinned words the spawn expansion's count and error word are copied into
    // without a wait, and the event after that copy (checked at a later wait)
    u64 *h_spawn_check = nullptr;
    cudaEvent_t spawn_check_ev = nullptr;
    cgb_rules rules{};
    int index_kind = INDEX_HASH;  // lookup structure of solved layers
    int bucket_bits = 22;         // INDEX_BUCKET: bucket count = 2^bits
    u64 spill_reserve = 24ull << 30;  // free device memory kept before spilling resident layers
    u64 max_sort_keys = 1ull << 28;   // larger layer steps are cut into chunks and merged
    u64 store_chunk = 4ull << 30;     // device allocation unit of the resident-layer store
    int fp64_top_layers = 4;          // FP32 sweeps: the highest layers solved in FP64
    FormationFilter filter;           // batched sweeps: formations that still generate
    CanonPlan plan;                   // images that can be canonical for the sweep's 0xf mask

    static Engine &get();
    bool init(int dev);
    bool set_rules(const cgb_rules &r);
    PruneParams prune_params() const;
    bool sync();

    GenBuffers gen;
    HostStage out_stage[2];     // pinned double buffer of the sweep's host copies
    HostArena host_layers;      // host copies of a sweep's layers (layers and tables both wanted)
    u64 host_layers_cap = 64ull << 30;  // bytes; beyond it tables carry their own key copy
    bool move_layer(const u64 *d_in, u64 n, GenTimes *tm);
    bool spawn_layer(GenTimes *tm, bool unique_streams = false);
    bool sort_step(DevBuf<u64> &x, DevBuf<u64> &y, u64 n, DevBuf<u64> **out, GenTimes *tm);
    bool sort_unique_step(DevBuf<u64> &x, DevBuf<u64> &y, u64 n, u64 *nu, DevBuf<u64> **out, GenTimes *tm,
                          u64 *empties = nullptr);
    bool merge_into(DevBuf<u64> &acc, const u64 *run, u64 n);
    // layers start..end from the input set of layer `start`; h_carry = the
    // 4-spawns of layer start-2 still to merge into layer start+2's input
    // (empty for a fresh sweep, the checkpointed set when resuming)
    bool generate(const u64 *h_initial, u64 n_init, int start, int end, LayerSink &sink, GenTimes *tm,
                  const u64 *h_carry = nullptr, u64 n_carry = 0);
    void release_buffers();
};

// ---- shared by the C ABI files (tablebase.cu, sweep.cu) ---------------------
std::vector<u64> expand_winstates(const u64 *w, int n);
SolveRules make_solve_rules(const cgb_rules &r, const u64 *d_ws, int nws);
void fill_stats(cgb_stats *st, const GenTimes &tm, const KernelStats &k0, const KernelStats &k1);

}  // namespace cgb

// initialises the engine and default rules if the caller has not
extern "C" bool ensure_rules_for_api();
