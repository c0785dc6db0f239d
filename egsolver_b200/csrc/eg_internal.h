/*
 * eg_internal.h -- declarations shared by the library's C and CUDA sources.
 */
#ifndef EG_INTERNAL_H
#define EG_INTERNAL_H

#include "../../include/egsolver_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Records a message for eg_last_error() and returns st. */
eg_status eg_set_error(eg_status st, const char *fmt, ...);

eg_owned_game *eg_owned_game_alloc(int32_t n, int64_t m);

/* Owner-sorted internal CSR from a CSR in file order (see eg_host.c). */
eg_status eg_owner_sort(int32_t n, int64_t m, const int64_t *ptr, const int32_t *succ,
                        const int32_t *w, const uint8_t *owner, const int32_t *ext_of_file,
                        eg_owned_game **out);

#ifdef __cplusplus
}
#endif

#endif
