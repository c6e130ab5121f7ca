/*
 * ref_kernel_entry.cpp -- compiles the reference's device arithmetic,
 * libRpack/kernel_entry.cl, unchanged as host C++ (the OpenCL keywords it uses are
 * mapped to nothing below) and exports its p32_add / p32_mul under plain C names.
 * The file is included from the reference tree at build time; nothing of it is
 * copied into this repository.  Test infrastructure only (oracle/_ref).
 */
#include <stdint.h>
#include <sys/types.h> /* uint, ulong, ushort */

#define __kernel
#define __global
#define __local
#define restrict __restrict__
#define CLK_LOCAL_MEM_FENCE 0
#ifndef TS
#define TS 8
#endif
static inline void barrier(int) {}
static inline int get_local_id(int) { return 0; }
static inline int get_group_id(int) { return 0; }
static inline int get_global_id(int) { return 0; }

#include "kernel_entry.cl"

extern "C" uint32_t ref_p32_add(uint32_t a, uint32_t b)
{
    posit32_t x, y;
    x.v = a;
    y.v = b;
    return p32_add(x, y).v;
}

extern "C" uint32_t ref_p32_mul(uint32_t a, uint32_t b)
{
    posit32_t x, y;
    x.v = a;
    y.v = b;
    return p32_mul(x, y).v;
}

extern "C" void ref_p32_add_n(const uint32_t *a, const uint32_t *b, uint32_t *out, int64_t n)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++)
        out[i] = ref_p32_add(a[i], b[i]);
}

extern "C" void ref_p32_mul_n(const uint32_t *a, const uint32_t *b, uint32_t *out, int64_t n)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++)
        out[i] = ref_p32_mul(a[i], b[i]);
}
