/*
 * Macro shim that lets the reference's OpenCL-C kernel files compile as C11
 * (TEST INFRASTRUCTURE ONLY; used by oracle/ref_driver.c).
 *
 * The reference kernels (opencl_fdtd_solver/kernels/{precision,yee_update,
 * sources}.cl) use only scalar OpenCL C: address-space qualifiers, the
 * work-item id and the float2/double2 vector types named in precision.cl.
 * Mapping those onto C lets the reference's own kernel arithmetic run on the
 * host: each kernel becomes a static function called once per work-item.
 */
#ifndef FDTD_REF_SHIM_H
#define FDTD_REF_SHIM_H
#include <stddef.h>

#define __kernel static
#define __global
#define __local
#define cl_khr_fp64 1
#define cl_khr_int64_base_atomics 1

typedef struct { float x, y; } float2;
typedef struct { double x, y; } double2;

/* Work-item id of the calling host thread (set by the driver loop). */
static __thread size_t ref_gid[3];
#define get_global_id(d) (ref_gid[(d)])

#endif
