/* Minimal OpenCL host API surface used by the reference task sources, backed by
 * the CPU runtime in ref_runtime.cpp / ref_clc_jit.cpp (test infrastructure
 * only).  Enumerant values follow the OpenCL 1.2 headers, because the
 * reference stores some of them in its own enums (common/ufo-addressing.h). */
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
typedef uint16_t cl_half;
typedef uint8_t cl_uchar;
typedef uint16_t cl_ushort;
typedef cl_uint cl_bool;
typedef float cl_float;
typedef double cl_double;
typedef uint64_t cl_mem_flags;
typedef cl_uint cl_addressing_mode;
typedef cl_uint cl_filter_mode;
typedef cl_uint cl_channel_order;
typedef cl_uint cl_channel_type;
typedef cl_uint cl_mem_object_type;
typedef struct refshim_mem *cl_mem;
typedef struct refshim_kernel *cl_kernel;
typedef struct refshim_sampler *cl_sampler;
typedef void *cl_context;
typedef void *cl_command_queue;
typedef void *cl_event;
typedef struct { cl_float s[2]; } cl_float2;
typedef struct { cl_float s[4]; } cl_float3; /* OpenCL 3-vectors have the size of 4-vectors */
typedef struct { cl_float s[4]; } cl_float4;
typedef struct { cl_float s[8]; } cl_float8;
typedef struct { cl_float s[16]; } cl_float16;
typedef struct { cl_double s[2]; } cl_double2;
typedef struct { cl_double s[4]; } cl_double3;
typedef struct { cl_int s[4]; } cl_int3;
typedef struct { cl_uint s[4]; } cl_uint4;
typedef struct { cl_channel_order image_channel_order; cl_channel_type image_channel_data_type; } cl_image_format;
typedef struct {
    cl_mem_object_type image_type;
    size_t image_width, image_height, image_depth, image_array_size, image_row_pitch, image_slice_pitch;
    cl_uint num_mip_levels, num_samples;
    cl_mem buffer;
} cl_image_desc;
#define CL_SUCCESS 0
#define CL_MEM_READ_WRITE (1 << 0)
#define CL_MEM_WRITE_ONLY (1 << 1)
#define CL_MEM_READ_ONLY (1 << 2)
#define CL_MEM_COPY_HOST_PTR (1 << 5)
#define CL_R 0x10B0
#define CL_RG 0x10B2
#define CL_RGBA 0x10B5
#define CL_INTENSITY 0x10B8
#define CL_UNSIGNED_INT8 0x10DA
#define CL_HALF_FLOAT 0x10DD
#define CL_FLOAT 0x10DE
#define CL_MEM_OBJECT_IMAGE2D 0x10F1
#define CL_MEM_OBJECT_IMAGE2D_ARRAY 0x10F3
#define CL_ADDRESS_NONE 0x1130
#define CL_ADDRESS_CLAMP_TO_EDGE 0x1131
#define CL_ADDRESS_CLAMP 0x1132
#define CL_ADDRESS_REPEAT 0x1133
#define CL_ADDRESS_MIRRORED_REPEAT 0x1134
#define CL_FILTER_NEAREST 0x1140
#define CL_FILTER_LINEAR 0x1141
cl_mem clCreateBuffer(cl_context ctx, cl_mem_flags flags, size_t size, void *host_ptr, cl_int *err);
cl_mem clCreateImage2D(cl_context ctx, cl_mem_flags flags, const cl_image_format *fmt, size_t width, size_t height,
                       size_t row_pitch, void *host_ptr, cl_int *err);
cl_mem clCreateImage(cl_context ctx, cl_mem_flags flags, const cl_image_format *fmt, const cl_image_desc *desc,
                     void *host_ptr, cl_int *err);
cl_sampler clCreateSampler(cl_context ctx, cl_bool normalized, cl_addressing_mode addressing, cl_filter_mode filter,
                           cl_int *err);
cl_int clReleaseSampler(cl_sampler s);
cl_int clSetKernelArg(cl_kernel k, cl_uint index, size_t size, const void *value);
cl_int clRetainKernel(cl_kernel k);
cl_int clReleaseKernel(cl_kernel k);
cl_int clRetainContext(cl_context c);
cl_int clReleaseContext(cl_context c);
cl_int clReleaseMemObject(cl_mem m);
cl_int clWaitForEvents(cl_uint n, const cl_event *events);
cl_int clReleaseEvent(cl_event e);
cl_int clEnqueueCopyBufferToImage(cl_command_queue q, cl_mem src, cl_mem dst, size_t src_offset,
                                  const size_t *dst_origin, const size_t *region, cl_uint n, const cl_event *wait,
                                  cl_event *event);
cl_int clEnqueueCopyImage(cl_command_queue q, cl_mem src, cl_mem dst, const size_t *src_origin,
                          const size_t *dst_origin, const size_t *region, cl_uint n, const cl_event *wait,
                          cl_event *event);
cl_int clEnqueueCopyBufferRect(cl_command_queue q, cl_mem src, cl_mem dst, const size_t *src_origin,
                               const size_t *dst_origin, const size_t *region, size_t src_row_pitch,
                               size_t src_slice_pitch, size_t dst_row_pitch, size_t dst_slice_pitch, cl_uint n,
                               const cl_event *wait, cl_event *event);
#ifdef __cplusplus
}
#endif
#endif
