/*
 * Force-included (-include) into kd_api.c by the host tests: routes the host
 * library's allocations through an allocator that can be told to fail its
 * n-th call, so that every allocation failure path is exercised.
 */
#ifndef FAKE_ALLOC_H
#define FAKE_ALLOC_H
#include <stdlib.h>

extern int fake_alloc_countdown; /* > 0: the countdown-th allocation from now fails */
void *fake_malloc(size_t n);
void *fake_calloc(size_t count, size_t size);
int fake_posix_memalign(void **p, size_t align, size_t n);

#define malloc fake_malloc
#define calloc fake_calloc
#define posix_memalign fake_posix_memalign
#endif
