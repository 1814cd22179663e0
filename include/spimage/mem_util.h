/* Allocation wrappers of the phasing path: plain malloc/free, as the
 * reference's default build maps them (include/spimage/mem_util.h,
 * SP_MEM_DEBUG off). */
#ifndef SPB_MEM_UTIL_H
#define SPB_MEM_UTIL_H 1
#include <stdlib.h>
#define sp_malloc(n) malloc(n)
#define sp_calloc(nmemb, size) calloc(nmemb, size)
#define sp_realloc(p, n) realloc(p, n)
#define sp_free(p) free(p)
#endif
