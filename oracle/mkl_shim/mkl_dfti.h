/*
 * Oracle infrastructure (test-only; never linked into the product).
 *
 * A project-written stand-in for the small part of Intel MKL's DFTI interface
 * that the reference CPU platform calls (MklFFT1D/2D/3D.cpp:
 * DftiCreateDescriptor, DftiSetValue x4, DftiCommitDescriptor,
 * DftiComputeForward/Backward, DftiFreeDescriptor).  The names and argument
 * conventions have to match MKL's public API so the reference sources compile
 * unchanged; the transform behind them is this project's own FP64 FFT
 * (dfti_shim.cpp).  Only what the reference uses is supported: double
 * precision, real domain, 1-3 dimensions, out-of-place, COMPLEX_COMPLEX
 * conjugate-even storage, contiguous row-major strides.
 */
#ifndef LFTS_ORACLE_MKL_DFTI_SHIM_H_
#define LFTS_ORACLE_MKL_DFTI_SHIM_H_

typedef long MKL_LONG;

enum DFTI_CONFIG_PARAM {
    DFTI_PLACEMENT = 11,
    DFTI_CONJUGATE_EVEN_STORAGE = 18,
    DFTI_INPUT_STRIDES = 12,
    DFTI_OUTPUT_STRIDES = 13
};

enum DFTI_CONFIG_VALUE {
    DFTI_SINGLE = 35,
    DFTI_DOUBLE = 36,
    DFTI_COMPLEX = 32,
    DFTI_REAL = 33,
    DFTI_INPLACE = 43,
    DFTI_NOT_INPLACE = 44,
    DFTI_COMPLEX_COMPLEX = 39
};

struct lfts_dfti_descriptor;
typedef struct lfts_dfti_descriptor *DFTI_DESCRIPTOR_HANDLE;

#ifdef __cplusplus
extern "C" {
#endif

/* dimension == 1: the variadic argument is one MKL_LONG length;
 * dimension  > 1: it is a pointer to `dimension` MKL_LONG lengths. */
MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *handle,
                              enum DFTI_CONFIG_VALUE precision,
                              enum DFTI_CONFIG_VALUE domain,
                              MKL_LONG dimension, ...);
MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE handle, enum DFTI_CONFIG_PARAM param, ...);
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE handle);
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE handle, void *in, ...);
MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE handle, void *in, ...);
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *handle);

#ifdef __cplusplus
}
#endif

#endif
