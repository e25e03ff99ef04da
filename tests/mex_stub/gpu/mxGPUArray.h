/* Declarations of the MATLAB GPU array C API calls used by mex/fame_mex.c (syntax check only;
 * not MATLAB's header). */
#pragma once
#include "mex.h"
typedef struct mxGPUArray_tag mxGPUArray;
typedef enum { MX_GPU_InitializeValues, MX_GPU_DoNotInitialize } mxGPUInitialize;
int mxInitGPU(void);
const mxGPUArray* mxGPUCreateFromMxArray(const mxArray* a);
mxGPUArray* mxGPUCopyFromMxArray(const mxArray* a);
const mwSize* mxGPUGetDimensions(const mxGPUArray* g);
mwSize mxGPUGetNumberOfDimensions(const mxGPUArray* g);
mwSize mxGPUGetNumberOfElements(const mxGPUArray* g);
mxClassID mxGPUGetClassID(const mxGPUArray* g);
mxComplexity mxGPUGetComplexity(const mxGPUArray* g);
const void* mxGPUGetDataReadOnly(const mxGPUArray* g);
void* mxGPUGetData(mxGPUArray* g);
mxGPUArray* mxGPUCreateGPUArray(mwSize nd, const mwSize* dims, mxClassID c, mxComplexity x, mxGPUInitialize init);
mxArray* mxGPUCreateMxArrayOnGPU(const mxGPUArray* g);
void mxGPUDestroyGPUArray(const mxGPUArray* g);
