/*
 * ref_prelude.h -- TEST INFRASTRUCTURE (oracle A). Never linked into the product.
 *
 * Lets the reference's OpenCL C pair kernels (the string literals `kernelfull`,
 * `kernelint`, `kernelfullsafe`, `kernelintsafe` in src/EpiOpenCL.c:45-963) compile
 * unmodified as host C99. The kernels use no barriers and no atomics, so running the
 * work-items one after another reproduces each work-item exactly.
 *
 * The OpenCL address-space qualifiers become nothing, `float4`/`vload4` become a plain
 * struct and loader, and the work-item query functions read thread-local variables that
 * the NDRange emulator (ndrange_emu.c) sets before each work-item call.
 */
#ifndef EPI_REF_PRELUDE_H
#define EPI_REF_PRELUDE_H
#include <math.h>
#include <stddef.h>

#define __kernel
#define __global
#define __local

typedef struct { float x, y, z, w; } float4;

static inline float4 vload4(size_t offset, const float *p)
{
    float4 v;
    p += 4 * offset;
    v.x = p[0]; v.y = p[1]; v.z = p[2]; v.w = p[3];
    return v;
}

/* dimension d of the current work-item, set by the emulator */
extern __thread size_t epi_emu_global_id[2];
extern __thread size_t epi_emu_local_id[2];
extern __thread size_t epi_emu_local_size[2];
extern __thread size_t epi_emu_global_size[2];

#define get_global_id(d)   (epi_emu_global_id[(d)])
#define get_local_id(d)    (epi_emu_local_id[(d)])
#define get_local_size(d)  (epi_emu_local_size[(d)])
#define get_global_size(d) (epi_emu_global_size[(d)])

#endif
