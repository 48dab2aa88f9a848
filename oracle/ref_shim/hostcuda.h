/* Test infrastructure (oracle). Lets the reference's CUDA kernel sources
 * (GPU_program1.cu and the GPU_*.h headers it includes) compile as host C++,
 * so the reference's own per-cell kernel bodies can be executed on the CPU by
 * oracle/ref_kernels.cpp, which walks the launch grid thread by thread.
 * Nothing here is product code. */
#ifndef HAMR_REF_HOSTCUDA_H
#define HAMR_REF_HOSTCUDA_H
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#define __device__
#define __global__
#define __host__
#define __shared__ static
#define __forceinline__ inline
struct hc_dim3 { unsigned x, y, z; };
extern struct hc_dim3 threadIdx, blockIdx, blockDim;
#define __syncthreads()
/* Declared before use: GPU_bounds.h:1336 calls it before its definition at
 * GPU_bounds.h:1606 (only reachable in neutron-star builds). */
double omega_star(double t);
#endif
