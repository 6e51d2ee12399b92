// async_out.h -- device -> pinned host copies on the engine's I/O stream.
//
// Layer and table callbacks get host arrays without stalling the layer loop:
// each request copies one or more device segments into one of two pinned
// buffers on the I/O stream (after an event on the main stream), and its
// callback runs when that slot is reused or drained.
#pragma once
#include "cgb_engine.h"
#include <functional>
#include <utility>
#include <vector>

namespace cgb {

// device -> pinned host copies on the I/O stream, two slots in flight
struct AsyncOut {
    cudaStream_t main = nullptr, io = nullptr;
    struct Slot {
        HostStage *buf = nullptr;
        cudaEvent_t ready = nullptr, done = nullptr;
        std::function<bool(const char *)> cb;
        bool busy = false;
    };
    Slot slot[2];
    int next = 0;
    u64 d2h = 0;
    bool failed = false;

    bool init(cudaStream_t m, cudaStream_t i, HostStage *stages)
    {
        main = m;
        io = i;
        slot[0].buf = &stages[0];
        slot[1].buf = &stages[1];
        for (auto &s : slot)
            if (!CGB_CUDA(cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming)) ||
                !CGB_CUDA(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming)))
                return false;
        return true;
    }
    ~AsyncOut()
    {
        for (auto &s : slot) {
            if (s.ready) cudaEventDestroy(s.ready);
            if (s.done) cudaEventDestroy(s.done);
        }
    }
    bool finish(Slot &s)
    {
        if (!s.busy) return true;
        s.busy = false;
        if (!CGB_CUDA(cudaEventSynchronize(s.done))) return false;
        if (!s.cb((const char *)s.buf->p)) {
            set_error("host callback failed");
            return false;
        }
        return true;
    }
    // copy the segments (device pointer, bytes) into one pinned buffer; cb
    // gets that buffer once the copy is complete
    bool enqueue(const std::vector<std::pair<const void *, u64>> &segs, std::function<bool(const char *)> cb)
    {
        Slot &s = slot[next];
        next ^= 1;
        if (!finish(s)) return false;
        u64 bytes = 16;
        for (auto &g : segs) bytes += g.second;
        if (!s.buf->reserve(bytes)) return false;
        if (!CGB_CUDA(cudaEventRecord(s.ready, main))) return false;
        if (!CGB_CUDA(cudaStreamWaitEvent(io, s.ready, 0))) return false;
        u64 off = 0;
        for (auto &g : segs) {
            if (g.second && !CGB_CUDA(cudaMemcpyAsync((char *)s.buf->p + off, g.first, g.second,
                                                      cudaMemcpyDeviceToHost, io)))
                return false;
            off += g.second;
            d2h += g.second;
        }
        if (!CGB_CUDA(cudaEventRecord(s.done, io))) return false;
        s.cb = std::move(cb);
        s.busy = true;
        return true;
    }
    // later frees on the main stream must not overtake copies still reading
    bool fence_main()
    {
        for (auto &s : slot)
            if (s.busy && !CGB_CUDA(cudaStreamWaitEvent(main, s.done, 0))) return false;
        return true;
    }
    bool drain() { return finish(slot[next]) && finish(slot[next ^ 1]); }
};

}  // namespace cgb
