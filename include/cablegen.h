/*
 * cablegen.h -- the reference's public C API, served by libcablegen_b200.so.
 *
 * Every declaration here has the name, argument meaning, return convention
 * and ownership rules of the function it replaces in clepdn/cablegen's
 * api/cablegen.h (cited per entry), so the reference CLI
 * (frontends/cli/main.c) and any other caller links against this library
 * unchanged.  Host buffers returned by the library are malloc()ed and freed
 * by the caller with free(), as in the reference.  The functions are
 * single-caller and not re-entrant (global settings and row table), like the
 * reference.  The board macros and types are restated because callers use
 * them; they must stay byte-identical with the reference's.
 */
#ifndef CABLEGEN_H
#define CABLEGEN_H
#include <stdbool.h>
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* api/cablegen.h:6-12 -- nibble access, nibble 0 = most significant = top-left */
#define SETBIT(x, y) (x |= (1 << y))
#define CLEARBIT(x, y) (x &= ~(1 << y))
#define GETBIT(x, y) (x & (1 << y))
#define BIT_MASK (0xf000000000000000)
#define OFFSET(x) (x * 4)
#define GET_TILE(b, x) (uint8_t)(((b << OFFSET(x)) & BIT_MASK) >> OFFSET(15))
#define SET_TILE(b, x, v) ( b = (~(~b | (BIT_MASK >> OFFSET(x))) | ((BIT_MASK & ((uint64_t)v << OFFSET(15))) >> OFFSET(x)) ))

#ifndef REMOVE_STRUCT_DECL
/* api/cablegen.h:15-20 */
typedef struct {
    bool valid;
    uint64_t *bp;
    uint64_t *sp;
    size_t size;
} dynamic_arr_info;

/* api/cablegen.h:22-26 */
typedef struct {
    bool valid;
    uint64_t *bp;
    size_t size;
} static_arr_info;

/* api/cablegen.h:28-31: N keys, N values (f64 bit patterns) */
typedef struct {
    static_arr_info key;
    static_arr_info value;
} table;

/* api/cablegen.h:33-38 */
typedef enum { left, right, up, down } dir;
#endif

/* api/cablegen.h:41 -- move in place, orientation kept; false if illegal or unchanged */
bool movedir(uint64_t *, dir);
/* api/cablegen.h:42 -- build the row table for the current settings */
void generate_lut(void);
/* api/cablegen.h:43-44 -- whole file of u64 boards; valid=false on failure */
static_arr_info read_boards(const char *dir);
void read_boards2(static_arr_info *b, const char *dir);
/* api/cablegen.h:45 -- use this INI file from now on (re-read lazily) */
void change_config(char *cfg);
/* api/cablegen.h:46 -- value of key (canonicalised first if asked) or 0.0 */
double lookup(uint64_t key, table *t, bool canonicalize);

/* api/cablegen.h:47-59 -- must stay the first member of the full settings */
typedef struct {
    bool free_formation;
    bool ignore_f;
    long long cores;
    long long nox;
    char *bdir;
    char *initial;
    long long end_gen;
    char *tdir;
    char *winstates;
    long long end_solve;
    bool delete_boards;
} min_settings_t;

/* api/cablegen.h:61-62 */
min_settings_t *get_settings_min(void);
void init_settings(void);
/* api/cablegen.h:63 -- layers start..end (step 2) written to sprintf(fmt, sum) */
void generate(const int start, const int end, const char *fmt, const static_arr_info *initial);
/* api/cablegen.h:64 -- tables start..end (step 2, top-down) from posfmt to tablefmt */
void solve(unsigned start, unsigned end, char *posfmt, char *tablefmt, const static_arr_info *winstates);
/* api/cablegen.h:65-72 -- host array helpers */
void *malloc_errcheck(size_t size);
dynamic_arr_info init_darr(bool zero, size_t size);
static_arr_info init_sarr(bool zero, size_t size);
static_arr_info shrink_darr(dynamic_arr_info *info);
dynamic_arr_info concat(dynamic_arr_info *arr1, dynamic_arr_info *arr2);
void destroy_darr(dynamic_arr_info *arr);
void destroy_sarr(static_arr_info *arr);
bool push_back(dynamic_arr_info *, uint64_t);
/* api/cablegen.h:73-74 */
void write_boards(const static_arr_info n, const char *fmt, const int layer);
void read_table(table *t, const char *path);
/* api/cablegen.h:75-79 */
double pun_uint64(uint64_t);
bool test(void);
int get_sum(uint64_t board);
void output_board(uint64_t);
char *get_version(void);

#ifdef __cplusplus
}
#endif
#endif
