/* Minimal OpenCL host API surface used by the reference task sources, backed by
 * the CPU runtime in ref_runtime.cpp (test infrastructure only). */
#ifndef REFSHIM_CL_H
#define REFSHIM_CL_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef uint64_t cl_ulong;
typedef float cl_float;
typedef double cl_double;
typedef uint64_t cl_mem_flags;
typedef struct refshim_mem *cl_mem;
typedef struct refshim_kernel *cl_kernel;
typedef void *cl_context;
typedef void *cl_command_queue;
typedef void *cl_event;
typedef void *cl_sampler;
typedef struct { cl_float s[2]; } cl_float2;
typedef struct { cl_double s[2]; } cl_double2;
#define CL_SUCCESS 0
#define CL_MEM_READ_WRITE (1 << 0)
#define CL_MEM_WRITE_ONLY (1 << 1)
#define CL_MEM_READ_ONLY (1 << 2)
#define CL_MEM_COPY_HOST_PTR (1 << 5)
cl_mem clCreateBuffer(cl_context ctx, cl_mem_flags flags, size_t size, void *host_ptr, cl_int *err);
cl_int clSetKernelArg(cl_kernel k, cl_uint index, size_t size, const void *value);
cl_int clRetainKernel(cl_kernel k);
cl_int clReleaseKernel(cl_kernel k);
cl_int clRetainContext(cl_context c);
cl_int clReleaseContext(cl_context c);
cl_int clReleaseMemObject(cl_mem m);
#ifdef __cplusplus
}
#endif
#endif
