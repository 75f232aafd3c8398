/*
 * Prelude for compiling the reference's OpenCL C kernels (cvrp_ocl/gpu/kernel.cl)
 * as C++ on the CPU.  TEST INFRASTRUCTURE ONLY.
 *
 * The work-item built-ins read the current work-item from the fake runtime
 * (fakecl.cpp), barrier() yields to the work-group scheduler, and NUM_NODE /
 * N_ANTS -- which the reference injects as #defines when it builds the program
 * (g_type.cpp:193-200) -- become runtime values, so the kernels' private arrays
 * turn into variable-length arrays.  The OpenCL `pow` on floats follows the
 * oracle's rule: exact products for small integer exponents.
 */
#ifndef KERNEL_SHIM_H
#define KERNEL_SHIM_H

#include <math.h>
#include <stdio.h>
#include <stddef.h>

extern int fcl_num_node;
extern int fcl_n_ants;
size_t fcl_get_global_id(unsigned d);
size_t fcl_get_local_id(unsigned d);
size_t fcl_get_group_id(unsigned d);
size_t fcl_get_local_size(unsigned d);
void fcl_barrier(void);
unsigned fcl_atomic_cmpxchg(volatile unsigned *p, unsigned cmp, unsigned val);
float fcl_pow(float x, float e);

#define NUM_NODE fcl_num_node
#define N_ANTS fcl_n_ants
#define __kernel
#define __global
#define global
#define __local
#define CLK_LOCAL_MEM_FENCE 1
#define barrier(x) fcl_barrier()
#define get_global_id(d) fcl_get_global_id(d)
#define get_local_id(d) fcl_get_local_id(d)
#define get_group_id(d) fcl_get_group_id(d)
#define get_local_size(d) fcl_get_local_size(d)
#define atomic_cmpxchg(p, c, v) fcl_atomic_cmpxchg((p), (c), (v))
#define pow(x, e) fcl_pow((x), (e))

#endif
