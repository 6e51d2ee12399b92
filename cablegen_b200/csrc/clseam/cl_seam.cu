// cl_seam.cu -- the reference's GPU plug-in point (inc/cl_generate.h:16-63) on this engine.
//
// The reference's generate_layer (src/generate.c:303-548), built with
// -DUSE_OPENCL, hands each layer's moves and spawns to these functions and
// merges their sorted results with the carried n2/n4 on the CPU.  Here the
// same entry points run on the CUDA engine: a move is expand + sort + unique,
// a spawn the two sorted unique spawn streams, so an unmodified generate.c
// drives the GPU kernels and writes files identical to the CPU path's.
//
// Contracts kept from the header: results sorted ascending (here also free of
// duplicates); cl_spawn_dev and cl_darr_download consume their input handle
// whatever the outcome; a false / invalid return makes the caller fall back to
// its CPU path.  Host arrays are malloc'ed and freed by the caller (destroy_darr).
//
// This file is linked into libcablegen_b200_cl.so, which leaves out the
// library's own restatement of the reference API: the reference's objects
// provide it (settings come from its get_settings_min()).
#include "../cgb_engine.h"
#include "../../../include/cablegen.h"
#include "../../../include/cablegen_cl.h"
#include <algorithm>
#include <cstdlib>
#include <cstring>

using namespace cgb;

struct cl_darr {
    DevBuf<u64> buf;  // sorted unique boards on the device
};

namespace {

Engine &E() { return Engine::get(); }

u64 g_vram_peak = 0;

void note_vram()
{
    cudaMemPool_t pool;
    u64 high = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, E().device) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemHigh, &high) == cudaSuccess)
        g_vram_peak = std::max(g_vram_peak, high);
}

bool set_prune(bool prune, long stsl, long ltc, long smallest_large)
{
    cgb_rules r = E().rules;
    r.prune = prune;
    r.stsl = stsl;
    r.ltc = ltc;
    r.smallest_large = smallest_large;
    E().rules = r;  // prune parameters only: the row table stays as uploaded
    return true;
}

bool upload(const uint64_t *boards, size_t n, DevBuf<u64> &d)
{
    if (!grow(d, n + 1, E().stream)) return false;
    d.n = n;
    return n == 0 || CGB_CUDA(cudaMemcpyAsync(d.p, boards, n * 8, cudaMemcpyHostToDevice, E().stream));
}

bool download(const DevBuf<u64> &d, dynamic_arr_info *out)
{
    *out = dynamic_arr_info{false, nullptr, nullptr, 0};
    uint64_t *h = (uint64_t *)std::malloc(d.n ? d.n * 8 : 8);
    if (!h) return false;
    if (d.n && (!CGB_CUDA(cudaMemcpyAsync(h, d.p, d.n * 8, cudaMemcpyDeviceToHost, E().stream)) || !E().sync())) {
        std::free(h);
        return false;
    }
    *out = dynamic_arr_info{true, h, h + d.n, (size_t)d.n};
    return true;
}

// moves of n host boards: the engine's layer buffer, then moved out into *out
bool move_to(const uint64_t *boards, size_t n, bool prune, long stsl, long ltc, long sl, DevBuf<u64> *out)
{
    if (!E().ready || !E().rt.move) return false;
    set_prune(prune, stsl, ltc, sl);
    DevBuf<u64> in;
    if (!upload(boards, n, in)) return false;
    const bool ok = E().move_layer(in.p, n, nullptr);
    drop(in, E().stream);
    if (!ok) return false;
    std::swap(*out, E().gen.moved);
    E().gen.moved_empties_known = false;  // the count left with the layer
    note_vram();
    return E().sync();
}

// spawns of a device layer (consumed): two sorted unique streams
bool spawn_from(DevBuf<u64> &in, DevBuf<u64> *n2, DevBuf<u64> *n4)
{
    if (!E().ready) return false;
    std::swap(E().gen.moved, in);
    E().gen.moved_empties_known = false;  // a layer from outside: its spawns are counted
    drop(in, E().stream);  // the engine's previous layer buffer
    if (!E().spawn_layer(nullptr, true)) return false;  // the seam's contract: unique streams
    std::swap(*n2, E().gen.u2);
    std::swap(*n4, E().gen.u4_next);
    note_vram();
    return E().sync();
}

}  // namespace

extern "C" {

bool cl_init(void)
{
    if (E().ready) return true;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return false;
    }
    return E().init(0);
}

void cl_upload_luts(void)
{
    if (!E().ready) return;
    const min_settings_t *m = get_settings_min();
    cgb_rules r = E().rules;
    r.free_formation = m->free_formation;
    r.ignore_f = m->ignore_f;
    if (!E().set_rules(r)) E().rt = DeviceRowTable{};  // later calls report failure
}

void cl_shutdown(void)
{
    if (E().ready) {
        E().release_buffers();
        E().sync();
    }
}

dynamic_arr_info cl_move_boards(const uint64_t *boards, size_t n_boards, bool prune, long stsl, long ltc,
                                long smallest_large)
{
    dynamic_arr_info out{false, nullptr, nullptr, 0};
    DevBuf<u64> moved;
    if (move_to(boards, n_boards, prune, stsl, ltc, smallest_large, &moved)) download(moved, &out);
    drop(moved, E().stream);
    return out;
}

bool cl_spawn_boards(const uint64_t *boards, size_t n_boards, dynamic_arr_info *out_n2, dynamic_arr_info *out_n4)
{
    DevBuf<u64> in, n2, n4;
    bool ok = E().ready && upload(boards, n_boards, in) && spawn_from(in, &n2, &n4) && download(n2, out_n2);
    if (ok && !download(n4, out_n4)) {
        std::free(out_n2->bp);
        *out_n2 = dynamic_arr_info{false, nullptr, nullptr, 0};
        ok = false;
    }
    drop(in, E().stream);
    drop(n2, E().stream);
    drop(n4, E().stream);
    return ok;
}

bool cl_move_dev(const uint64_t *boards, size_t n, bool prune, long stsl, long ltc, long smallest_large,
                 cl_darr **out)
{
    *out = nullptr;
    cl_darr *d = new cl_darr;
    if (!move_to(boards, n, prune, stsl, ltc, smallest_large, &d->buf)) {
        cl_darr_release(d);
        return false;
    }
    *out = d;
    return true;
}

bool cl_spawn_dev(cl_darr *in, cl_darr **out_n2, cl_darr **out_n4)
{
    *out_n2 = *out_n4 = nullptr;
    if (!in) return false;
    cl_darr *a = new cl_darr, *b = new cl_darr;
    const bool ok = spawn_from(in->buf, &a->buf, &b->buf);
    cl_darr_release(in);
    if (!ok) {
        cl_darr_release(a);
        cl_darr_release(b);
        return false;
    }
    *out_n2 = a;
    *out_n4 = b;
    return true;
}

bool cl_darr_to_host(cl_darr *in, dynamic_arr_info *out)
{
    *out = dynamic_arr_info{false, nullptr, nullptr, 0};
    return in && download(in->buf, out);
}

bool cl_darr_download(cl_darr *in, dynamic_arr_info *out)
{
    const bool ok = cl_darr_to_host(in, out);
    cl_darr_release(in);
    return ok;
}

void cl_darr_release(cl_darr *in)
{
    if (!in) return;
    drop(in->buf, E().stream);
    delete in;
}

size_t cl_vram_bytes(void)
{
    note_vram();
    return (size_t)g_vram_peak;
}

}  // extern "C"
