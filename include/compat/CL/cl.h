/*
 * CL/cl.h -- stand-in for the OpenCL header, for building epiGPU's own host sources against
 * libepigpu.so.
 *
 * The reference's src/epiopencl.h includes <CL/cl.h> (src/epiopencl.h:1-5). Once
 * src/EpiOpenCL.c is replaced by epigpu_b200/host/scan_driver.c no OpenCL type or call is
 * left in the program (src/main.c, src/readplink.c and src/timing.c use none), so this
 * header declares nothing; it only lets that include resolve on a machine without an OpenCL
 * SDK. Put its directory (include/compat) on the include path.
 */
#ifndef EPIGPU_COMPAT_CL_CL_H
#define EPIGPU_COMPAT_CL_CL_H
#endif
