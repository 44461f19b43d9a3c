/* Type-only stand-in for <CL/cl.h>: the reference's CPU files include
 * KernelDefs.h, which needs these handle types but never an OpenCL call
 * (the calls live in Kernels.c, which the oracle does not build). */
#ifndef ST_CL_STUB_H
#define ST_CL_STUB_H
#include <stddef.h>
typedef struct st_cl_kernel *cl_kernel;
typedef struct st_cl_mem *cl_mem;
typedef struct st_cl_program *cl_program;
typedef struct st_cl_platform *cl_platform_id;
typedef struct st_cl_context *cl_context;
typedef struct st_cl_device *cl_device_id;
typedef struct st_cl_queue *cl_command_queue;
typedef unsigned int cl_uint;
typedef int cl_int;
typedef unsigned long cl_mem_flags;
#endif
