/*
 * TEST INFRASTRUCTURE ONLY (oracle). Never linked into the product library.
 *
 * Shim that lets the reference's OpenCL C source (pyqrackising/kernels.cl,
 * v9.16.6) compile unmodified as C11 with gcc, so that the reference's own
 * kernels can run on the host under the ND-range emulator in ref_launch.c.
 *
 * It maps the OpenCL address-space qualifiers to nothing, the scalar type
 * names to their C99 fixed-width equivalents, real1 to float (the
 * reference's default PYQRACKISING_FPPOW=5 build, maxcut_tfim_util.py:86-94),
 * and the work-item built-ins to thread-local state set by the emulator.
 * barrier() becomes a pthread barrier over the work-group's threads.
 */
#ifndef PQI_REF_SHIM_H
#define PQI_REF_SHIM_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <math.h>

typedef unsigned int uint;
typedef unsigned long ulong;

#define __kernel
#define __global
#define __constant const
#define __local

/* Precision macros of the default float build (maxcut_tfim_util.py:86-94). */
#define real1 float
#define qint int
#define EPSILON FLT_EPSILON
#define ZERO_R1 0.0f
#define ONE_R1 1.0f
#define TWO_R1 2.0f

#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2

size_t pqi_ref_get_global_id(uint dim);
size_t pqi_ref_get_global_size(uint dim);
size_t pqi_ref_get_local_id(uint dim);
size_t pqi_ref_get_local_size(uint dim);
size_t pqi_ref_get_group_id(uint dim);
void pqi_ref_barrier(int flags);

#define get_global_id(d) pqi_ref_get_global_id(d)
#define get_global_size(d) pqi_ref_get_global_size(d)
#define get_local_id(d) pqi_ref_get_local_id(d)
#define get_local_size(d) pqi_ref_get_local_size(d)
#define get_group_id(d) pqi_ref_get_group_id(d)
#define barrier(f) pqi_ref_barrier(f)

#endif
