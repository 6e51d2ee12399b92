/*
 * ref_q1_wrap.c -- linked into the reference build (oracle/_ref) only.
 *
 * TEST INFRASTRUCTURE: lets the reference's own CPU generation run pruned
 * workloads.  The reference's init_threads() (src/generate.c:215-241) never
 * assigns arguments.smallest_large, and generate() allocates the worker
 * array with malloc_errcheck (src/generate.c:570), so the pruning workers
 * (src/generate.c:160,166) read an uninitialised field; on this toolchain it
 * reads 0 and every board is pruned.  The OpenCL path passes the configured
 * value (src/generate.c:321,433).  Instead of editing the reference sources,
 * the link wraps malloc_errcheck (-Wl,--wrap=malloc_errcheck) and gives the
 * field of a worker array its configured value at allocation time.  Nothing
 * else of the reference changes.
 */
#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>
#include <pthread.h>
#include "settings.h"

/* Field layout of `arguments` (src/generate.c:23-36). */
typedef struct {
    static_arr_info n;
    dynamic_arr_info nret, n2, n4;
    size_t start, end;
    long stsl, smallest_large, ltc;
    char nox;
    long layer;
    pthread_t thread;
} ref_arguments;

void *__real_malloc_errcheck(size_t size);

void *__wrap_malloc_errcheck(size_t size)
{
    void *p = __real_malloc_errcheck(size);
    settings_t *st = get_settings();
    long long cores = st->min.cores;
    if (p && cores > 0 && size == sizeof(ref_arguments) * (size_t)cores) {
        ref_arguments *a = (ref_arguments *)p;
        for (long long i = 0; i < cores; i++) a[i].smallest_large = (long)st->smallest_large;
    }
    return p;
}
