/* Declarations of the MATLAB C API calls used by mex/fame_mex.c, written for a syntax check
 * of the gateway against include/fame.h where MATLAB is not installed.  Not MATLAB's header. */
#pragma once
#include <stddef.h>
#include <stdint.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxUNKNOWN_CLASS, mxDOUBLE_CLASS, mxSINGLE_CLASS, mxUINT32_CLASS, mxUINT64_CLASS } mxClassID;
typedef enum { mxREAL, mxCOMPLEX } mxComplexity;
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
void* mxMalloc(size_t n);
void mxFree(void* p);
void mexMakeMemoryPersistent(void* p);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x);
void* mxGetData(const mxArray* a);
int mxIsUint64(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
mxArray* mxGetField(const mxArray* s, size_t i, const char* name);
double mxGetScalar(const mxArray* a);
int mxGetString(const mxArray* a, char* buf, mwSize n);
double* mxGetDoubles(const mxArray* a);
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names);
void mxSetField(mxArray* s, size_t i, const char* name, mxArray* v);
mxArray* mxCreateDoubleScalar(double v);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity x);
mxArray* mxCreateLogicalScalar(int v);
double mxGetNaN(void);
void mxDestroyArray(mxArray* a);
