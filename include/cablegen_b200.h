/*
 * cablegen_b200.h -- C ABI of the B200 engine below the cablegen API.
 *
 * Plain pointers and sizes only.  Functions return 0 on success and -1 on
 * failure; cgb_last_error() then describes the failure.  "d_" pointers are
 * device memory of the current CUDA device, "h_" pointers host memory.
 * Boards are u64 (nibble 0 = top-left cell, api/cablegen.h:9-12).
 *
 * The library is single-caller like the reference (global state: the row
 * table, settings); calls are serialised on one internal CUDA stream.
 */
#ifndef CABLEGEN_B200_H
#define CABLEGEN_B200_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Generation/solve knobs (src/settings.c:34-59, settings.h:15-31). */
typedef struct {
    int free_formation;        /* [Cablegen] free_formation */
    int ignore_f;              /* [Cablegen] ignore_f */
    int prune;                 /* [Generate] prune */
    long long stsl;            /* [Generate] stsl */
    long long ltc;             /* [Generate] ltc */
    long long smallest_large;  /* [Generate] smallest_large */
    int nox;                   /* [Cablegen] nox (char semantics: solve.c:18) */
    int score;                 /* [Solve] score */
} cgb_rules;

/* Initialise the engine on a device; idempotent. */
int cgb_init(int device);
const char *cgb_last_error(void);
/* Build and upload the row table for these rules (generate_lut, src/board.c:100-132). */
int cgb_set_rules(const cgb_rules *rules);
/* Tuning knobs: "index" = lookup structure of solved layers (0 bisection of the
 * sorted layer as in lookup(), src/solve.c:108-164; 1 top-bits buckets then
 * bisection; 2 open-addressing hash, the default), "bucket_bits" (buckets of
 * kind 1), "solve_variant" (0 one thread per board, 1 warp-compacted),
 * "sort_variant" (0 match ranking, 1 ballot ranking, 2 persistent CTAs with
 * bulk-copy prefetch of the next tile, 3 byte-digit passes over 4096-key tiles,
 * 4 byte-digit passes over 8192-key tiles, the default, 5 as 4 with one match
 * instruction per key in place of eight ballots), "spill_reserve_mb"
 * (free device memory kept before resident layers spill to host memory),
 * "max_sort_keys" (larger layer steps are cut into chunks and merged),
 * "store_chunk_mb" (device allocation unit of the resident-layer store),
 * "host_layers_mb" (pinned host memory a sweep may keep for its layers' host
 * copies when layer and table callbacks are both given, so table keys need no
 * second copy; default 65536),
 * "hash_load_pct" (target load factor of the hash index, 10..90, or 0, the
 * default: 25 up to 2^27 keys per table, 45 above),
 * "region_build" (1, the default: 16-byte-slot hash indexes of 2^16..2^28 keys
 * built region by region in shared memory; 0: atomic inserts into a zeroed table),
 * "hash_compact" (1, the default: FP32 tables in 8-byte slots where the keys allow),
 * "move_window" (1..4, default 1: the move expansion drops repeats among the
 * results of up to this many blocks of 1024 consecutive input boards at once),
 * "fp64_top_layers" (FP32 sweeps of cgb_sweep_run: the highest layers, solved
 * first, whose values come straight from the winstates, are solved in FP64 and
 * narrowed to FP32 for the layers below; default 4, 0 = none).
 * cgb_get_option returns -1 for an unknown name. */
int cgb_set_option(const char *name, long long value);
long long cgb_get_option(const char *name);

/* ---- device primitives of one layer step --------------------------------
 * Move + prune + canonicalise every board (the move workers,
 * src/generate.c:133-175; OpenCL move_kernel, src/cl/generate.cl:249-282).
 * d_out needs cap >= 4n slots; *n_out = boards written (unsorted).  Every
 * distinct result appears at least once; repeats among the results of the same
 * chunk of consecutive inputs (1024 x "move_window" boards at most) are
 * written once. */
int cgb_expand_moves(const uint64_t *d_in, uint64_t n, uint64_t *d_out, uint64_t cap, uint64_t *n_out);
/* Total number of empty cells (= size of each spawn stream). */
int cgb_count_spawns(const uint64_t *d_in, uint64_t n, uint64_t *total);
/* Canonical 2- and 4-spawns of every empty cell (src/generate.c:177-199). */
int cgb_expand_spawns(const uint64_t *d_in, uint64_t n, uint64_t *d_out2, uint64_t *d_out4, uint64_t cap,
                      uint64_t *n_out);
/* Ascending LSD radix sort of d_keys[0,n) with scratch d_tmp[0,n) (replaces
 * qs_sort_h/fluxsort_uint64, src/array.c:289-291).  *result_in_tmp tells which
 * buffer holds the result; *passes = digit passes executed. */
int cgb_sort(uint64_t *d_keys, uint64_t *d_tmp, uint64_t n, int *result_in_tmp, int *passes);
/* Drop repeats of a sorted array into d_out (must not alias d_in). */
int cgb_unique(const uint64_t *d_in, uint64_t n, uint64_t *d_out, uint64_t *n_out);
/* Sorted union without repeats of two sorted unique arrays
 * (deduplicate_threads with two runs, src/array.c:246-287). */
int cgb_merge_unique(const uint64_t *d_a, uint64_t na, const uint64_t *d_b, uint64_t nb, uint64_t *d_out,
                     uint64_t *n_out);
/* Canonical form of every board (canonicalize_b, src/board.c:314-337). */
int cgb_canonicalize(const uint64_t *d_in, uint64_t n, uint64_t *d_out);

/* Sort d_in[0,n) ascending and drop repeats into d_out (capacity n, must not
 * alias d_in); *n_out = number of distinct keys.  No counterpart in the
 * reference: this is cgb_sort + cgb_unique for callers that cannot let the
 * library allocate device memory (a host whose caching allocator owns the
 * GPU under a hard budget, or latency-sensitive code that cannot absorb
 * cudaMalloc's device-wide synchronisation).  Its scratch is one fixed
 * __device__ array (a little over 8 MiB), so n is limited to 2^20 keys;
 * larger n is rejected with an error.  The first call on a device is its
 * set-up: it looks up the array's address, and because the runtime loads
 * device code lazily, that is also when the driver places the array on the
 * GPU (an allocation that may synchronise the device).  A call with n = 0
 * does only the set-up: make it once per device outside any budgeted region
 * and before any stream capture; the array then stays until the process
 * exits.  Calls share the array: calls that overlap on the GPU race and must
 * be serialised.  stream may be 0.  Returns after the work on `stream` has
 * finished. */
int cgb_sort_unique_noalloc(const uint64_t *d_in, uint64_t n, uint64_t *d_out, uint64_t *n_out, void *stream);

/* ---- solve of one layer (solve_layer, src/solve.c:289-340) ---------------
 * precision 64: d_out/d_v2/d_v4 are double; 32: float (Kahan sums).
 * (d_k2,d_v2,n2) and (d_k4,d_v4,n4): the s+2 and s+4 tables, keys sorted.
 * h_winstates: winstate patterns, expanded to all 8 symmetries inside. */
int cgb_solve_layer(const uint64_t *d_keys, uint64_t n, void *d_out, int precision, const uint64_t *d_k2,
                    const void *d_v2, uint64_t n2, const uint64_t *d_k4, const void *d_v4, uint64_t n4,
                    const uint64_t *h_winstates, int n_winstates);

/* ---- lookup of many boards (lookup(), src/solve.c:108-164) ---------------
 * (d_keys, d_vals, n): one solved layer on the device, keys sorted; d_vals
 * double (precision 64) or float (32).  The layer gets the index the solve
 * builds (option "index"), then every board of d_boards[m] is looked up --
 * canonicalised first when canonicalize, as lookup() does -- and its value
 * written to d_out[m] as a double (0.0 for a board not in the layer).  For
 * consumers that look up many positions at once; lookup() itself stays the
 * host search over a table the caller holds. */
int cgb_lookup_batch(const uint64_t *d_keys, const void *d_vals, uint64_t n, int precision, const uint64_t *d_boards,
                     uint64_t m, int canonicalize, double *d_out);

/* ---- whole sweeps -------------------------------------------------------- */
typedef struct {
    uint64_t layers, boards_generated, boards_solved;
    double gen_ms, solve_ms, total_ms;         /* device time (CUDA events) */
    double expand_ms, sort_ms, unique_ms, merge_ms, solve_kernel_ms, index_ms;
    uint64_t sorted_keys, sort_key_passes;     /* keys through the sort, keys x passes */
    uint64_t lookups_bytes;                    /* algorithmic bytes of the solve kernels */
    uint64_t h2d_bytes, d2h_bytes;
    double max_abs_err;                        /* fp32 runs with check: max |fp32 - fp64| */
    uint64_t gpu_launches;                     /* kernels launched by the library */
    uint64_t spilled_chunks, restored_chunks;  /* resident-layer chunks moved to / from the host */
    uint64_t layer_slices;                     /* slices of layer steps cut at max_sort_keys */
} cgb_stats;

/* Device time (ms, CUDA events around every launch) and algorithmic bytes per
 * kernel family, accumulated since the last cgb_reset_kernel_stats().
 * Algorithmic bytes: sort pass 16 B/key, histogram 8 B/key, unique 8 B per key
 * in and out, merge 8 B per key in and out, move expansion 8 B in + 8 B per
 * output, spawns 8 B in + 16 B per output pair, solve (8 + value) B/board +
 * 64 B per table probe (one key sector + one value sector). */
typedef struct {
    uint64_t launches;
    double hist_ms, onesweep_ms, unique_ms, merge_ms, expand_ms, spawn_ms, solve_ms, index_ms;
    uint64_t hist_bytes, onesweep_bytes, unique_bytes, merge_bytes, expand_bytes, spawn_bytes, solve_bytes;
    uint64_t onesweep_launches, solve_launches, solve_boards, lookups;
    uint64_t index_builds, compact_index_builds;  /* hash indexes built; of them in 8-byte slots */
    uint64_t moves_raw, moves_kept;  /* move results before / after dropping repeats per chunk of
                                        1024 x "move_window" consecutive boards */
    uint64_t pool_trims;  /* device allocations that failed, returned the allocator's cached
                             blocks to the device and were retried */
} cgb_kernel_stats;
int cgb_get_kernel_stats(cgb_kernel_stats *out);
int cgb_reset_kernel_stats(void);

/* Layer callback: the layer `sum` as a host array (valid during the call). */
typedef int (*cgb_layer_fn)(void *user, int sum, const uint64_t *h_boards, uint64_t n);
/* Table callback: keys and values (double, or float for precision 32). */
typedef int (*cgb_table_fn)(void *user, int sum, const uint64_t *h_keys, const void *h_values, uint64_t n,
                            int precision);

/* Per-layer FP32-vs-FP64 report of a sweep run with precision 0. */
typedef int (*cgb_error_fn)(void *user, int sum, uint64_t n, double max_abs, double mean_abs);

/* A generation + solve sweep with every layer resident in HBM. */
typedef struct {
    const uint64_t *initial;   /* host boards, all of tile sum `start` */
    uint64_t n_initial;
    int start, end_gen, end_solve;
    const uint64_t *winstates; /* host winstate patterns (expanded to 8 images inside) */
    int n_winstates;
    int precision;             /* 64, 32, or 0: both, FP32 compared with FP64 layer by layer */
    cgb_layer_fn layer_fn;     /* optional: every layer copied to the host */
    cgb_table_fn table_fn;     /* optional: every table copied to the host (FP64 when precision 0) */
    cgb_error_fn error_fn;     /* optional, precision 0: per-layer max/mean |fp32 - fp64| */
    void *user;
} cgb_sweep;
/* Copies to the host run on a second stream into double-buffered pinned
 * memory and overlap the next layers' kernels; the callbacks run on the
 * calling thread. */
int cgb_sweep_run(const cgb_sweep *sweep, cgb_stats *stats);

/* Generation sweep from h_initial (all of tile sum `start`) up to `end`
 * (generate(), src/generate.c:551-615); every layer goes to fn. */
int cgb_generate(const uint64_t *h_initial, uint64_t n, int start, int end, cgb_layer_fn fn, void *user,
                 cgb_stats *stats);

/* Generation + solve with every layer resident in HBM (generate() then
 * solve(), src/solve.c:172-224, without files).  Layers are solved from
 * end_gen down to max(end_solve, start).  precision 64 or 32.  When
 * layer_fn / table_fn are non-null every layer / table is copied to the host
 * and handed to them (the end-to-end path). */
int cgb_tablebase(const uint64_t *h_initial, uint64_t n, int start, int end_gen, int end_solve,
                  const uint64_t *h_winstates, int n_winstates, int precision, cgb_layer_fn layer_fn,
                  cgb_table_fn table_fn, void *user, cgb_stats *stats);

/* ---- batched sweeps: many formations in one run --------------------------
 * No reference counterpart: the reference runs one formation per generate() /
 * solve() call.  Every formation of a batch advances one layer per step, all
 * formations' boards in the same kernels (one expansion, one sort, one merge,
 * one solve launch per step); the solve steps' launch sequences (gathers,
 * solve, index build) are captured as CUDA graphs.  Boards of different
 * formations must differ: formations whose fixed-cell masks are images of one
 * another under the board symmetries run in separate groups.  Requires
 * free_formation off (fixed cells never move). */
typedef struct {
    const uint64_t *initial;   /* host boards, one formation, one tile sum */
    uint64_t n_initial;
    int end_gen, end_solve;    /* layers start..end_gen; solved down to max(end_solve, 0) */
    const uint64_t *winstates; /* host winstate patterns (expanded to 8 images inside) */
    int n_winstates;
} cgb_formation;
/* formation = index into the batch's formation array */
typedef int (*cgb_batch_layer_fn)(void *user, int formation, int sum, const uint64_t *h_boards, uint64_t n);
typedef int (*cgb_batch_table_fn)(void *user, int formation, int sum, const uint64_t *h_keys,
                                  const void *h_values, uint64_t n, int precision);
typedef struct {
    const cgb_formation *formations;
    int n_formations;
    int precision;             /* 64 or 32 */
    int use_graphs;            /* 1: capture each solve step as a CUDA graph */
    cgb_batch_layer_fn layer_fn;
    cgb_batch_table_fn table_fn;
    void *user;
} cgb_batch;
typedef struct {
    uint64_t groups, gen_steps, solve_steps;
    uint64_t boards_generated, boards_solved;
    double gen_ms, solve_ms, total_ms;
    uint64_t graph_launches, gpu_launches, lookups;
    uint64_t h2d_bytes, d2h_bytes;
} cgb_batch_stats;
int cgb_batch_run(const cgb_batch *batch, cgb_batch_stats *stats);
/* Host only: the groups cgb_batch_run would form (group_of[i] for formation i);
 * returns the number of groups, or -1 on invalid formations. */
int cgb_batch_plan(const cgb_formation *formations, int n_formations, int *group_of);

#ifdef __cplusplus
}
#endif
#endif
