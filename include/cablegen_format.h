/*
 * cablegen_format.h -- string helpers that the reference library exports to
 * its CLI (src/format.c); the CLI declares them in frontends/cli/format.h.
 * libcablegen_b200.so exports the same symbols so the unmodified CLI links.
 */
#ifndef CABLEGEN_FORMAT_H
#define CABLEGEN_FORMAT_H
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* frontends/cli/format.h:4-15 */
typedef struct {
    long res;
    int status;
} atoi_res;
typedef struct {
    long res;
    int status;
} atoi_res_ll;
char *format_str(const char *fmt, ...);
atoi_res safe_atoi(const char *input);
atoi_res_ll safe_atoi_ll(const char *input, const int radix);
bool isdigit_radix(const char input, const unsigned int radix);

#ifdef __cplusplus
}
#endif
#endif
