/*
 * Host-only stand-in for the small part of the cuFFT API that GO-Ferro's
 * reference sources call, so that the reference compiles and runs on a
 * machine with no GPU and no FFT library.
 *
 * TEST INFRASTRUCTURE: this header and host_fft.cpp are used only to build
 * the CPU oracle under oracle/_ref.  They are never linked into the product.
 *
 * Semantics follow cuFFT's documented behaviour for the calls the reference
 * makes (magnetostatic_solver.cpp:149-151,183-185; magnetic_initialize.cpp:
 * 114-115,1103-1111; ferroelectric_initialize.cpp:351-352,510;
 * elastic_initialize.cpp:224-225):
 *   - cufftPlan3d(plan, nx, ny, nz, type): row-major nx*ny*nz, z fastest;
 *   - D2Z: unnormalised forward transform (exp(-i...)), output is the
 *     non-redundant half spectrum nx*ny*(nz/2+1);
 *   - Z2D: unnormalised inverse transform (exp(+i...)) of a Hermitian half
 *     spectrum back to nx*ny*nz reals.
 * Pointers are host pointers (the reference's OpenACC host_data regions are
 * no-ops when compiled without OpenACC).
 */
#ifndef GOFERRO_ORACLE_CUFFT_SHIM_H
#define GOFERRO_ORACLE_CUFFT_SHIM_H

/* The real cufft.h includes cuComplex.h, which includes <math.h>; with
 * libstdc++ that makes the global abs(double) overload visible.  The
 * reference's Newell-kernel code calls unqualified abs() on doubles
 * (magnetic_initialize.cpp:1440-1553) and silently truncates to int without
 * it, so the shim keeps the same transitive include. */
#include <math.h>

typedef int cufftHandle;
typedef int cufftResult;
typedef enum { CUFFT_R2C = 0x2a, CUFFT_C2R = 0x2c, CUFFT_C2C = 0x29,
               CUFFT_D2Z = 0x6a, CUFFT_Z2D = 0x6c, CUFFT_Z2Z = 0x69 } cufftType;
typedef struct { double x, y; } cufftDoubleComplex;
typedef double cufftDoubleReal;

#define CUFFT_SUCCESS 0
#define CUFFT_INVALID_PLAN 1
#define CUFFT_INVALID_VALUE 4

cufftResult cufftPlan3d(cufftHandle* plan, int nx, int ny, int nz, cufftType type);
cufftResult cufftExecD2Z(cufftHandle plan, cufftDoubleReal* idata, cufftDoubleComplex* odata);
cufftResult cufftExecZ2D(cufftHandle plan, cufftDoubleComplex* idata, cufftDoubleReal* odata);
cufftResult cufftDestroy(cufftHandle plan);

#endif
