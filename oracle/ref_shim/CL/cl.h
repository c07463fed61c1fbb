// Minimal stand-in for <CL/cl.h>: the OpenCL types, constants and entry points that the
// reference's host sources (LabelingAlgs.cpp, LabelingTools.cpp, TOCLBuffer_impl.hpp) name, so
// that its OpenMP CPU labelers compile without an OpenCL SDK.  The entry points are defined in
// ref_cpu.cpp and fail with CL_INVALID_OPERATION; the OpenCL classes are never run.
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include <stddef.h>
#include <stdint.h>

typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef uint32_t cl_bool;
typedef uint64_t cl_ulong;
typedef cl_ulong cl_bitfield;
typedef cl_bitfield cl_mem_flags;
typedef cl_bitfield cl_device_type;
typedef struct _cl_mem *cl_mem;
typedef struct _cl_kernel *cl_kernel;
typedef struct _cl_context *cl_context;
typedef struct _cl_command_queue *cl_command_queue;
typedef struct _cl_program *cl_program;
typedef struct _cl_device_id *cl_device_id;
typedef struct _cl_platform_id *cl_platform_id;
typedef struct _cl_event *cl_event;

#define CL_SUCCESS 0
#define CL_INVALID_OPERATION (-59)
#define CL_FALSE 0u
#define CL_TRUE 1u
#define CL_MEM_READ_WRITE (1 << 0)
#define CL_MEM_WRITE_ONLY (1 << 1)
#define CL_MEM_READ_ONLY (1 << 2)
#define CL_DEVICE_TYPE_CPU (1 << 1)
#define CL_DEVICE_TYPE_GPU (1 << 2)

#ifdef __cplusplus
extern "C" {
#endif
cl_mem clCreateBuffer(cl_context, cl_mem_flags, size_t, void *, cl_int *);
cl_int clReleaseMemObject(cl_mem);
cl_kernel clCreateKernel(cl_program, const char *, cl_int *);
cl_int clReleaseKernel(cl_kernel);
cl_int clSetKernelArg(cl_kernel, cl_uint, size_t, const void *);
cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel, cl_uint, const size_t *, const size_t *,
                              const size_t *, cl_uint, const cl_event *, cl_event *);
cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, void *, cl_uint,
                           const cl_event *, cl_event *);
cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, const void *, cl_uint,
                            const cl_event *, cl_event *);
cl_int clFinish(cl_command_queue);
#ifdef __cplusplus
}
#endif
