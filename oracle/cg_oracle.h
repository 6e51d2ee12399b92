/*
 * cg_oracle.h -- CPU restatement of cablegen's generation and solve hot paths.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU engine is compared
 * against: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * may load it.  The product (cablegen_b200/) never links or calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * golden vectors produced by the reference build itself (oracle/Makefile ->
 * oracle/_ref, tests/golden/make_golden.py).
 *
 * Every function cites the reference file:line whose behaviour it restates.
 * Board = u64 of 16 nibbles, nibble 0 (most significant) = top-left cell.
 */
#ifndef CG_ORACLE_H
#define CG_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint16_t move[2][65536];   /* [0]=left, [1]=right: row after the move   */
    uint8_t  locked[2][65536]; /* 1 = the move keeps every 0xf cell in place */
} orc_lut;

typedef struct {
    int free_formation, ignore_f;
    int prune;
    long stsl, ltc, smallest_large;
    int nox, score;
} orc_settings;

/* board.c:62-132 */
void orc_build_lut(orc_lut *lut, int free_formation, int ignore_f);

/* board.c:239-268, 376-393 */
uint64_t orc_rot_cw(uint64_t b);
uint64_t orc_rot_ccw(uint64_t b);
uint64_t orc_rot_180(uint64_t b);
uint64_t orc_flip(uint64_t b);
/* board.c:314-337 (scalar, unsigned max over the D4 orbit) */
uint64_t orc_canon(uint64_t b);
/* board.c:271-313 semantics (AVX-512 build): signed max over the orbit */
uint64_t orc_canon_signed(uint64_t b);
/* board.c:349-374 */
void orc_all_rots(uint64_t b, uint64_t out[8]);
/* board.c:340-347 */
int orc_get_sum(uint64_t b);

/* board.c:151-214: returns 1 when the move is legal and changed the board */
int orc_movedir_unstable(const orc_lut *lut, uint64_t *b, int dir);
int orc_movedir(const orc_lut *lut, uint64_t *b, int dir);

/* generate.c:98-131 */
int orc_prune(uint64_t b, long stsl, long ltc, long smallest_large);
/* generate.c:89-96: 1 when no cell holds exponent x */
int orc_checkx(uint64_t b, int x);

/*
 * One generation layer step (generate.c:133-199, 409-550) on host arrays.
 * in[n_in]: boards of tile sum s (any order, duplicates allowed).
 * moved: sorted unique moved+canonicalised boards (the s.boards content).
 * spawn2/spawn4: sorted unique canonical spawns of `moved`.
 * Output arrays are malloc'ed; caller frees.
 */
void orc_move_layer(const orc_lut *lut, const orc_settings *st,
                    const uint64_t *in, size_t n_in,
                    uint64_t **moved, size_t *n_moved);
void orc_spawn_layer(const uint64_t *moved, size_t n,
                     uint64_t **s2, size_t *n2, uint64_t **s4, size_t *n4);
/* array.c:246-287 restricted to two sorted runs: sorted union without duplicates */
size_t orc_merge_unique(const uint64_t *a, size_t na, const uint64_t *b, size_t nb,
                        uint64_t *out);
/* sort ascending + drop duplicates in place; returns the new length */
size_t orc_sort_unique(uint64_t *a, size_t n);

/* solve.c:226-231 */
int orc_cmpbrd(uint64_t board, uint64_t w);
/* solve.c:233-244 (winstates already expanded x8) */
int orc_satisfied(uint64_t board, const uint64_t *ws, size_t nws, int nox, int score);
/* solve.c:108-164: value of key (canonicalised when canon) or 0.0 */
double orc_lookup(uint64_t key, const uint64_t *keys, const double *vals, size_t n, int canon);
/* solve.c:257-281 */
double orc_expectimax(const orc_lut *lut, uint64_t board,
                      const uint64_t *k2, const double *v2, size_t n2,
                      const uint64_t *k4, const double *v4, size_t n4, int score);
/* solve.c:289-302 over a whole layer */
void orc_solve_layer(const orc_lut *lut, const orc_settings *st,
                     const uint64_t *keys, size_t n,
                     const uint64_t *k2, const double *v2, size_t n2,
                     const uint64_t *k4, const double *v4, size_t n4,
                     const uint64_t *ws, size_t nws, double *out);

/* Pure-CPU timing helpers for the CPU baseline: threads split boards in blocks. */
void orc_solve_layer_mt(const orc_lut *lut, const orc_settings *st,
                        const uint64_t *keys, size_t n,
                        const uint64_t *k2, const double *v2, size_t n2,
                        const uint64_t *k4, const double *v4, size_t n4,
                        const uint64_t *ws, size_t nws, double *out, int threads);

#ifdef __cplusplus
}
#endif
#endif
