/* cablegen_cl.h -- the reference's GPU plug-in seam (inc/cl_generate.h:16-63), implemented on
 * the CUDA engine by libcablegen_b200_cl.so (cablegen_b200/csrc/clseam/cl_seam.cu).
 *
 * The reference's generate_layer (src/generate.c:303-548), compiled with -DUSE_OPENCL, calls
 * these for each layer's moves and spawns and merges the sorted results on the CPU.  The
 * names, arguments and ownership follow the reference header: results are sorted ascending
 * (here also unique); cl_spawn_dev and cl_darr_download release their input handle whatever
 * the outcome; a false return (or an invalid array) sends the caller to its CPU path; host
 * arrays are malloc'ed and released by the caller with destroy_darr. */
#ifndef CABLEGEN_CL_H
#define CABLEGEN_CL_H
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include "cablegen.h" /* dynamic_arr_info */

#ifdef __cplusplus
extern "C" {
#endif

bool cl_init(void);                 /* inc/cl_generate.h:16 -- false without a CUDA device */
void cl_upload_luts(void);          /* :20 -- row table for the current free_formation/ignore_f */
void cl_shutdown(void);             /* :22 */
dynamic_arr_info cl_move_boards(const uint64_t *boards, size_t n_boards, bool prune, long stsl, long ltc,
                                long smallest_large);                       /* :24-29 */
bool cl_spawn_boards(const uint64_t *boards, size_t n_boards, dynamic_arr_info *out_n2,
                     dynamic_arr_info *out_n4);                             /* :31-34 */
typedef struct cl_darr cl_darr;     /* :39 -- device-resident sorted board array */
bool cl_move_dev(const uint64_t *boards, size_t n, bool prune, long stsl, long ltc, long smallest_large,
                 cl_darr **out);                                            /* :41-45 */
bool cl_spawn_dev(cl_darr *in, cl_darr **out_n2, cl_darr **out_n4);        /* :50-52 */
bool cl_darr_download(cl_darr *in, dynamic_arr_info *out);                 /* :55 */
bool cl_darr_to_host(cl_darr *in, dynamic_arr_info *out);                  /* :58 */
void cl_darr_release(cl_darr *in);                                         /* :60 */
size_t cl_vram_bytes(void);                                                /* :63 -- peak device bytes */

#ifdef __cplusplus
}
#endif
#endif
