/*
 * ORACLE — test infrastructure only. Force-included (-include) when the
 * reference's CPU sources are compiled for oracle/_ref.
 *
 * The reference writes up to naux doubles *before* its pqA buffer whenever a
 * basis-function pair is screened inside a shell pair that survives
 * (build_DF_tensor.c:36-43 uses bf_pair_mask == -1 as a row index). Those
 * integrals are meant to be dropped; the writes are out of bounds. To run the
 * reference unchanged, every allocation of 1 MiB or more made through
 * _mm_malloc gets a 1 MiB guard zone in front, where those stray writes land.
 * The reference's arithmetic is untouched.
 */
#ifndef ORACLE_GUARD_MALLOC_H
#define ORACLE_GUARD_MALLOC_H
#include <stdlib.h>
#include <mm_malloc.h>

#define ORACLE_GUARD_BYTES ((size_t) 1 << 20)
#define ORACLE_GUARD_SLOTS 1024

/* One table for the whole program, defined in mkl_shim.c. */
extern void *oracle_guard_tab[ORACLE_GUARD_SLOTS];

static inline void *oracle_guarded_malloc(size_t size, size_t align)
{
    (void) align;
    void *base = NULL;
    if (size < ORACLE_GUARD_BYTES)
    {
        if (posix_memalign(&base, 64, size ? size : 64)) return NULL;
        return base;
    }
    if (posix_memalign(&base, 64, size + ORACLE_GUARD_BYTES)) return NULL;
    char *p = (char *) base + ORACLE_GUARD_BYTES;
    for (int i = 0; i < ORACLE_GUARD_SLOTS; i++)
        if (__sync_bool_compare_and_swap(&oracle_guard_tab[i], (void *) 0, (void *) p)) return p;
    abort();
}

static inline void oracle_guarded_free(void *p)
{
    if (p == NULL) return;
    for (int i = 0; i < ORACLE_GUARD_SLOTS; i++)
        if (oracle_guard_tab[i] == p)
        {
            oracle_guard_tab[i] = NULL;
            free((char *) p - ORACLE_GUARD_BYTES);
            return;
        }
    free(p);
}

#define _mm_malloc(s, a) oracle_guarded_malloc((s), (a))
#define _mm_free(p)      oracle_guarded_free(p)
#endif
