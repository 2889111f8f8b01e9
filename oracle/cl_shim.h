/*
 * cl_shim.h -- lets the reference's OpenCL C kernel file (FibreNet/kernel.cl)
 * compile unmodified as C11 with gcc, so its ten kernels can run on the host
 * as the parity checker.  TEST INFRASTRUCTURE ONLY: nothing in the product
 * links this.
 *
 * Semantic choices (each maps one OpenCL built-in used by kernel.cl):
 *   kernel / global / __global   -> nothing (plain C functions and pointers)
 *   get_global_id(0)             -> a thread-local work-item index set by the
 *                                   driver before each kernel call
 *   mad(a,b,c)                   -> a*b + c, unfused (built with
 *                                   -ffp-contract=off); OpenCL allows either
 *   native_sqrt(double)          -> sqrt (OpenCL defines native_* for float
 *                                   only; the reference applies it to double
 *                                   at kernel.cl:384, 880, 924, 964)
 *   atomic_add(int*, int)        -> relaxed __atomic_fetch_add
 *   atomic_cmpxchg / atom_cmpxchg-> relaxed compare-exchange returning the old
 *                                   value (kernel.cl:168, 192)
 *   inline                       -> static inline (C99 inline would need an
 *                                   external definition)
 *   ulong                        -> uint64_t
 */
#ifndef FIBRENET_CL_SHIM_H
#define FIBRENET_CL_SHIM_H

#include <math.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdlib.h>

typedef uint64_t ulong;

#define kernel
#define global
#define __global
#define inline static inline

extern _Thread_local int fn_cl_global_id;
#define get_global_id(dim) (fn_cl_global_id)

#define mad(a, b, c) ((a) * (b) + (c))
#define native_sqrt(x) sqrt(x)

static __attribute__((unused)) int atomic_add(volatile int* p, int v) {
    return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}

static __attribute__((unused)) unsigned int atomic_cmpxchg(volatile unsigned int* p,
                                                           unsigned int cmp,
                                                           unsigned int val) {
    __atomic_compare_exchange_n(p, &cmp, val, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
    return cmp;
}

static __attribute__((unused)) ulong atom_cmpxchg(volatile ulong* p, ulong cmp, ulong val) {
    __atomic_compare_exchange_n(p, &cmp, val, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
    return cmp;
}

#endif
