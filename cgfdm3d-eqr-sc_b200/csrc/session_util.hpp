// Allocation and error macros for Session member functions (they use the
// members alloc, cuda_fail and err).
#pragma once

#define ALLOC(ptr, type, count)                                                                                  \
    do {                                                                                                         \
        ptr = (type *)alloc(sizeof(type) * (size_t)(count));                                                    \
        if (!ptr) {                                                                                              \
            err = "cannot allocate device memory for " #ptr;                                                     \
            return ST_ALLOC;                                                                                     \
        }                                                                                                        \
    } while (0)
#define CU(x)                                                                                                    \
    do {                                                                                                         \
        cudaError_t e__ = (x);                                                                                   \
        if (e__ != cudaSuccess) return cuda_fail(e__, #x);                                                       \
    } while (0)
