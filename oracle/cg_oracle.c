/*
 * cg_oracle.c -- CPU restatement of cablegen's hot paths (see cg_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU engine, never shipped.
 * Written from the reference's behaviour, not copied: rotations are expressed
 * as cell-index maps, the row move as an operation on a 4-nibble array, the
 * sort as a plain LSD radix sort.  Parity with the reference is pinned by
 * tests/test_oracle.py against vectors the reference build itself produced.
 */
#include "cg_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <pthread.h>

static inline int tile(uint64_t b, int cell) { return (int)((b >> (60 - 4 * cell)) & 0xF); }
static inline uint64_t with_tile(uint64_t b, int cell, int v)
{
    int sh = 60 - 4 * cell;
    return (b & ~(0xFULL << sh)) | ((uint64_t)(v & 0xF) << sh);
}

/* ---- geometry (board.c:239-268, 376-393) --------------------------------
 * rotate_clockwise: the new cell (r, c) takes the old cell (3-c, r).
 * flip: reverses the order of the four rows (the reachable part of flip()). */
uint64_t orc_rot_cw(uint64_t b)
{
    uint64_t o = 0;
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++)
            o = with_tile(o, 4 * r + c, tile(b, 4 * (3 - c) + r));
    return o;
}
uint64_t orc_rot_ccw(uint64_t b) { return orc_rot_cw(orc_rot_cw(orc_rot_cw(b))); }
uint64_t orc_rot_180(uint64_t b)
{
    uint64_t o = 0;
    for (int c = 0; c < 16; c++) o = with_tile(o, c, tile(b, 15 - c));
    return o;
}
uint64_t orc_flip(uint64_t b)
{
    uint64_t o = 0;
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++)
            o = with_tile(o, 4 * r + c, tile(b, 4 * (3 - r) + c));
    return o;
}

/* board.c:349-374: e, a, a^2, a^3, b, ba, ba^2, ba^3 (a = clockwise, b = flip;
 * "ba" applies flip first, then the rotation). */
void orc_all_rots(uint64_t b, uint64_t out[8])
{
    out[0] = b;
    out[1] = orc_rot_cw(b);
    out[2] = orc_rot_180(b);
    out[3] = orc_rot_ccw(b);
    uint64_t f = orc_flip(b);
    out[4] = f;
    out[5] = orc_rot_cw(f);
    out[6] = orc_rot_180(f);
    out[7] = orc_rot_ccw(f);
}

/* board.c:314-337: the canonical board is the unsigned maximum of the orbit. */
uint64_t orc_canon(uint64_t b)
{
    uint64_t r[8];
    orc_all_rots(b, r);
    uint64_t m = r[0];
    for (int i = 1; i < 8; i++) if (r[i] > m) m = r[i];
    return m;
}

/* board.c:271-313 (AVX-512 VBMI build) takes a signed 64-bit maximum. */
uint64_t orc_canon_signed(uint64_t b)
{
    uint64_t r[8];
    orc_all_rots(b, r);
    int64_t m = (int64_t)r[0];
    for (int i = 1; i < 8; i++) if ((int64_t)r[i] > m) m = (int64_t)r[i];
    return (uint64_t)m;
}

/* board.c:340-347 */
int orc_get_sum(uint64_t b)
{
    int s = 0;
    for (int c = 0; c < 16; c++) {
        int t = tile(b, c);
        if (t != 0 && t != 0xE && t != 0xF) s += 1 << t;
    }
    return s;
}

/* ---- row LUT (board.c:29-132) -------------------------------------------
 * One row is four cells; `order` lists them in the direction of travel.  The
 * move slides tiles toward order[0], merges equal neighbours below 0xE once
 * each (greedy from order[0]), and slides again.  With ignore_f, fixed cells
 * at the far end of the travel order are walls and never move.  0xF cells
 * otherwise slide like tiles; `locked` rejects a move that vacates any cell
 * that held 0xF (unless the formation is free). */
static void slide(uint8_t *t, const int *order, int n)
{
    int w = 0;
    uint8_t tmp[4] = {0, 0, 0, 0};
    for (int i = 0; i < n; i++)
        if (t[order[i]]) tmp[w++] = t[order[i]];
    for (int i = 0; i < n; i++) t[order[i]] = tmp[i];
}

static void row_move(uint8_t *t, const int *order, int ignore_f)
{
    int n = 4;
    if (ignore_f)
        while (n > 0 && t[order[n - 1]] == 0xF) n--;
    slide(t, order, n);
    for (int i = 0; i + 1 < n; i++) {
        uint8_t v = t[order[i]];
        if (v && v == t[order[i + 1]] && v < 0xE) {
            /* absorb the neighbour: everything behind it moves up one cell */
            for (int j = i + 1; j + 1 < n; j++) t[order[j]] = t[order[j + 1]];
            t[order[n - 1]] = 0;
            t[order[i]] = (uint8_t)(v + 1);
        }
    }
    slide(t, order, n);
}

void orc_build_lut(orc_lut *lut, int free_formation, int ignore_f)
{
    static const int L[4] = {0, 1, 2, 3}, R[4] = {3, 2, 1, 0};
    for (uint32_t row = 0; row < 65536; row++) {
        for (int d = 0; d < 2; d++) {
            uint8_t pre[4], t[4];
            for (int c = 0; c < 4; c++) pre[c] = t[c] = (uint8_t)((row >> (12 - 4 * c)) & 0xF);
            row_move(t, d == 0 ? L : R, ignore_f);
            uint16_t out = (uint16_t)((t[0] << 12) | (t[1] << 8) | (t[2] << 4) | t[3]);
            int vacated = 0;
            if (!free_formation)
                for (int c = 0; c < 4; c++)
                    if (pre[c] == 0xF && t[c] != 0xF) vacated = 1;
            lut->move[d][row] = out;
            lut->locked[d][row] = (uint8_t)!vacated;
        }
    }
    /* board.c:126-129 pins these two rows to themselves */
    lut->move[0][0] = lut->move[1][0] = 0;
    lut->move[0][0xFFFF] = lut->move[1][0xFFFF] = 0xFFFF;
}

/* board.c:151-169: apply the row LUT to all four rows; any locked row makes
 * the whole move illegal (board restored, returns 0); else returns "changed". */
static int move_rows(const orc_lut *lut, uint64_t *b, int lr)
{
    uint64_t out = 0;
    int changed = 0;
    for (int i = 0; i < 4; i++) {
        uint16_t row = (uint16_t)(*b >> (16 * i));
        if (!lut->locked[lr][row]) return 0;
        uint16_t m = lut->move[lr][row];
        changed |= (m != row);
        out |= (uint64_t)m << (16 * i);
    }
    *b = out;
    return changed;
}

/* board.c:195-214: up = rotate clockwise then move right, down = rotate
 * clockwise then move left; the result stays rotated. */
int orc_movedir_unstable(const orc_lut *lut, uint64_t *b, int dir)
{
    switch (dir) {
    case 1: return move_rows(lut, b, 1);
    case 2: *b = orc_rot_cw(*b); return move_rows(lut, b, 1);
    case 3: *b = orc_rot_cw(*b); return move_rows(lut, b, 0);
    default: return move_rows(lut, b, 0);
    }
}

/* board.c:171-193: same moves, orientation restored. */
int orc_movedir(const orc_lut *lut, uint64_t *b, int dir)
{
    if (dir < 2) return orc_movedir_unstable(lut, b, dir);
    uint64_t t = orc_rot_cw(*b);
    int ch = move_rows(lut, &t, dir == 2 ? 1 : 0);
    *b = orc_rot_ccw(t);
    return ch;
}

/* ---- pruning (generate.c:98-131) -----------------------------------------
 * Large = smallest_large <= e < 0xE; small = e < smallest_large (an empty cell
 * counts as e = 0, adding 1).  Prune on a large value seen a third time (the
 * value smallest_large itself is allowed three extra copies first), when the
 * small-tile sum exceeds stsl + 64, or when more than ltc large tiles exist. */
int orc_prune(uint64_t b, long stsl, long ltc, long smallest_large)
{
    int large = 0, sl_count = 0;
    long small_sum = 0;
    unsigned once = 0, twice = 0;
    for (int c = 0; c < 16; c++) {
        int e = tile(b, c);
        if (e >= smallest_large && e < 0xE) {
            large++;
            if (e == smallest_large && sl_count < 3) { sl_count++; continue; }
            if (!(once & (1u << e))) once |= 1u << e;
            else if (!(twice & (1u << e))) twice |= 1u << e;
            else return 1;
        } else if (e < 0xE) {
            small_sum += 1L << e;
        }
    }
    if (small_sum > stsl + 64) return 1;
    if (large > ltc) return 1;
    return 0;
}

/* generate.c:89-96 */
int orc_checkx(uint64_t b, int x)
{
    int xc = (signed char)x;            /* the reference passes nox as a char */
    for (int c = 0; c < 16; c++) if (tile(b, c) == xc) return 0;
    return 1;
}

/* ---- sorting helpers -------------------------------------------------- */
static void radix_sort_u64(uint64_t *a, size_t n)
{
    if (n < 2) return;
    uint64_t *tmp = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint64_t *src = a, *dst = tmp;
    for (int pass = 0; pass < 4; pass++) {
        int sh = 16 * pass;
        size_t *cnt = (size_t *)calloc(65536, sizeof(size_t));
        for (size_t i = 0; i < n; i++) cnt[(src[i] >> sh) & 0xFFFF]++;
        size_t run = 0;
        int constant = 0;
        for (int d = 0; d < 65536; d++) { if (cnt[d] == n) constant = 1; size_t c = cnt[d]; cnt[d] = run; run += c; }
        if (!constant) {
            for (size_t i = 0; i < n; i++) dst[cnt[(src[i] >> sh) & 0xFFFF]++] = src[i];
            uint64_t *t = src; src = dst; dst = t;
        }
        free(cnt);
    }
    if (src != a) memcpy(a, src, n * sizeof(uint64_t));
    free(tmp);
}

size_t orc_sort_unique(uint64_t *a, size_t n)
{
    radix_sort_u64(a, n);
    size_t w = 0;
    for (size_t i = 0; i < n; i++)
        if (w == 0 || a[w - 1] != a[i]) a[w++] = a[i];
    return w;
}

size_t orc_merge_unique(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, uint64_t *out)
{
    size_t i = 0, j = 0, w = 0;
    while (i < na || j < nb) {
        uint64_t v;
        if (j >= nb || (i < na && a[i] <= b[j])) v = a[i++];
        else v = b[j++];
        if (w == 0 || out[w - 1] != v) out[w++] = v;
    }
    return w;
}

/* ---- one generation layer (generate.c:133-199, 409-550) ----------------- */
void orc_move_layer(const orc_lut *lut, const orc_settings *st,
                    const uint64_t *in, size_t n_in, uint64_t **moved, size_t *n_moved)
{
    uint64_t *out = (uint64_t *)malloc((4 * n_in + 1) * sizeof(uint64_t));
    size_t w = 0;
    for (size_t i = 0; i < n_in; i++) {
        uint64_t b = in[i];
        if (st->prune && orc_prune(b, st->stsl, st->ltc, st->smallest_large)) continue;
        for (int d = 0; d < 4; d++) {
            uint64_t t = b;
            if (!orc_movedir_unstable(lut, &t, d)) continue;
            if (st->prune && orc_prune(t, st->stsl, st->ltc, st->smallest_large)) continue;
            out[w++] = orc_canon(t);
        }
    }
    *n_moved = orc_sort_unique(out, w);
    *moved = out;
}

void orc_spawn_layer(const uint64_t *moved, size_t n, uint64_t **s2, size_t *n2, uint64_t **s4, size_t *n4)
{
    size_t cap = 16 * n + 1;
    uint64_t *a = (uint64_t *)malloc(cap * sizeof(uint64_t));
    uint64_t *b = (uint64_t *)malloc(cap * sizeof(uint64_t));
    size_t w = 0;
    for (size_t i = 0; i < n; i++)
        for (int c = 0; c < 16; c++)
            if (tile(moved[i], c) == 0) {
                a[w] = orc_canon(with_tile(moved[i], c, 1));
                b[w] = orc_canon(with_tile(moved[i], c, 2));
                w++;
            }
    *n2 = orc_sort_unique(a, w);
    *n4 = orc_sort_unique(b, w);
    *s2 = a;
    *s4 = b;
}

/* ---- solve (solve.c:108-302) ------------------------------------------ */
int orc_cmpbrd(uint64_t board, uint64_t w)
{
    uint64_t mask = 0;
    for (int c = 0; c < 16; c++)
        if (tile(w, c)) mask |= 0xFULL << (60 - 4 * c);
    return (board & mask) == w;
}

int orc_satisfied(uint64_t board, const uint64_t *ws, size_t nws, int nox, int score)
{
    nox = (signed char)nox;             /* solve.c:18 stores nox in a char */
    if (nox && !score) return !orc_checkx(board, nox);
    if (score) return 0;
    for (size_t i = 0; i < nws; i++)
        if (orc_cmpbrd(board, ws[i])) return 1;
    return 0;
}

/* solve.c:108-164: bisection that falls back to a linear scan once the
 * window is under 50 keys; a miss (or an empty table) gives 0.0. */
double orc_lookup(uint64_t key, const uint64_t *keys, const double *vals, size_t n, int canon)
{
    if (n == 0) return 0.0;
    if (canon) key = orc_canon(key);
    size_t lo = 0, hi = n, mid = n / 2;
    while (keys[mid] != key) {
        if (hi - lo < 50) {
            for (size_t i = lo; i < hi; i++)
                if (keys[i] == key) return vals[i];
            return 0.0;
        }
        if (keys[mid] < key) lo = mid; else hi = mid;
        mid = (lo + hi) / 2;
    }
    return vals[mid];
}

static double best_move(const orc_lut *lut, uint64_t b, const uint64_t *k, const double *v, size_t n)
{
    double p[4] = {0, 0, 0, 0};
    for (int d = 0; d < 4; d++) {
        uint64_t t = b;
        if (orc_movedir_unstable(lut, &t, d)) p[d] = orc_lookup(t, k, v, n, 1);
    }
    return fmax(fmax(p[0], p[1]), fmax(p[2], p[3]));
}

double orc_expectimax(const orc_lut *lut, uint64_t board,
                      const uint64_t *k2, const double *v2, size_t n2,
                      const uint64_t *k4, const double *v4, size_t n4, int score)
{
    int spaces = 0;
    double s2 = 0, s4 = 0;
    for (int c = 0; c < 16; c++) {
        if (tile(board, c)) continue;
        spaces++;
        s2 += best_move(lut, with_tile(board, c, 1), k2, v2, n2);
        s4 += best_move(lut, with_tile(board, c, 2), k4, v4, n4);
    }
    double res = 0;
    if (spaces) {
        volatile double a = 0.9 * s2;   /* keep the reference's evaluation order */
        volatile double b = 0.1 * s4;
        res = a / spaces + b / spaces;
    }
    if (score && res == 0) res = orc_get_sum(board);
    return res;
}

void orc_solve_layer(const orc_lut *lut, const orc_settings *st,
                     const uint64_t *keys, size_t n,
                     const uint64_t *k2, const double *v2, size_t n2,
                     const uint64_t *k4, const double *v4, size_t n4,
                     const uint64_t *ws, size_t nws, double *out)
{
    for (size_t i = 0; i < n; i++)
        out[i] = orc_satisfied(keys[i], ws, nws, st->nox, st->score)
                     ? 1.0
                     : orc_expectimax(lut, keys[i], k2, v2, n2, k4, v4, n4, st->score);
}

typedef struct {
    const orc_lut *lut; const orc_settings *st;
    const uint64_t *keys; size_t lo, hi;
    const uint64_t *k2; const double *v2; size_t n2;
    const uint64_t *k4; const double *v4; size_t n4;
    const uint64_t *ws; size_t nws; double *out;
} solve_job;

static void *solve_job_run(void *p)
{
    solve_job *j = (solve_job *)p;
    orc_solve_layer(j->lut, j->st, j->keys + j->lo, j->hi - j->lo, j->k2, j->v2, j->n2,
                    j->k4, j->v4, j->n4, j->ws, j->nws, j->out + j->lo);
    return NULL;
}

void orc_solve_layer_mt(const orc_lut *lut, const orc_settings *st,
                        const uint64_t *keys, size_t n,
                        const uint64_t *k2, const double *v2, size_t n2,
                        const uint64_t *k4, const double *v4, size_t n4,
                        const uint64_t *ws, size_t nws, double *out, int threads)
{
    if (threads < 1) threads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    solve_job *jobs = (solve_job *)malloc(sizeof(solve_job) * threads);
    for (int t = 0; t < threads; t++) {
        solve_job j = {lut, st, keys, n * t / threads, n * (t + 1) / threads,
                       k2, v2, n2, k4, v4, n4, ws, nws, out};
        jobs[t] = j;
        pthread_create(&th[t], NULL, solve_job_run, &jobs[t]);
    }
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    free(th);
    free(jobs);
}
