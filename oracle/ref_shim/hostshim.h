/* Test infrastructure (oracle). Types that the reference's host headers
 * (decs.h:293) expect from the CUDA/HIP runtime, which the host-only oracle
 * build of metric.c / coord.c / lu.c does not include. */
#ifndef HAMR_REF_HOSTSHIM_H
#define HAMR_REF_HOSTSHIM_H
typedef void *gpuStream_t;
typedef void *gpuEvent_t;
typedef int gpuError_t;
/* copy kinds named by the reference's restart.c (its device paths are never
 * called in the host builds) */
#define gpuMemcpyHostToDevice 1
#define gpuMemcpyDeviceToHost 2
#endif
