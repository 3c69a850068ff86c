/*
 * mex.h -- project-written stand-in for MATLAB's MEX API, declaring only the
 * subset the reference's src/CUDA code calls (and mxFree).  Together with
 * mex_shim.cpp it lets the reference's own CUDA path (mex_main.cu, mset.cu,
 * utility.cu, mex_tools.cpp) be compiled unchanged and driven from C, and
 * drives this library's MEX gateway (mset_b200/mex/mset_cuda_kernel.cpp) the
 * same way.  TEST INFRASTRUCTURE ONLY: the results, oracle/_ref/libmset_ref.so
 * and oracle/_gw/libmset_gateway.so, are checkers and a timed baseline.
 */
#ifndef MSET_TEST_MEX_SHIM_H
#define MSET_TEST_MEX_SHIM_H
#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

typedef size_t mwSize;
typedef size_t mwIndex;
typedef bool mxLogical;
typedef struct mxArray_tag mxArray;

typedef enum {
    mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS,
    mxVOID_CLASS, mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS,
    mxINT16_CLASS, mxUINT16_CLASS, mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS,
    mxUINT64_CLASS, mxFUNCTION_CLASS
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

typedef struct { float real, imag; } mxComplexSingle;

#ifdef __cplusplus
extern "C" {
#endif
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
void mexErrMsgTxt(const char *msg);
mxArray *mxGetCell(const mxArray *pm, mwIndex index);
float *mxGetSingles(const mxArray *pm);
mxComplexSingle *mxGetComplexSingles(const mxArray *pm);
double *mxGetDoubles(const mxArray *pm);
uint8_t *mxGetUint8s(const mxArray *pm);
int32_t *mxGetInt32s(const mxArray *pm);
mxLogical *mxGetLogicals(const mxArray *pm);
void *mxGetData(const mxArray *pm);
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid, mxComplexity flag);
mxClassID mxGetClassID(const mxArray *pm);
size_t mxGetNumberOfElements(const mxArray *pm);
mwSize mxGetNumberOfDimensions(const mxArray *pm);
const mwSize *mxGetDimensions(const mxArray *pm);
int mxGetNumberOfFields(const mxArray *pm);
const char *mxGetFieldNameByNumber(const mxArray *pm, int n);
mxArray *mxGetFieldByNumber(const mxArray *pm, mwIndex index, int n);
bool mxIsStruct(const mxArray *pm);
bool mxIsChar(const mxArray *pm);
char *mxArrayToString(const mxArray *pm);
void mxFree(void *ptr);
#ifdef __cplusplus
}
#endif
#endif
