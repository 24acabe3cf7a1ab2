/*
 * A minimal stand-in for MATLAB's C MEX API, enough to build and drive the shims under
 * mex/ without MATLAB or Octave (test infrastructure only).  Arrays are column-major with
 * MATLAB's separate real/imaginary storage; mexErrMsgIdAndTxt unwinds to sim_call.
 */
#ifndef MEXSIM_MEX_H
#define MEXSIM_MEX_H
#include <stddef.h>

typedef size_t mwSize;
typedef struct mxArray_tag mxArray;
typedef enum { mxUNKNOWN_CLASS = 0, mxCELL_CLASS = 1, mxSTRUCT_CLASS = 2, mxDOUBLE_CLASS = 6,
               mxSINGLE_CLASS = 7, mxINT32_CLASS = 12 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
size_t mxGetNumberOfElements(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
int mxIsSingle(const mxArray* a);
int mxIsDouble(const mxArray* a);
int mxIsComplex(const mxArray* a);
int mxIsStruct(const mxArray* a);
int mxIsCell(const mxArray* a);
mxArray* mxGetCell(const mxArray* a, mwSize i);
void mxSetCell(mxArray* a, mwSize i, mxArray* v);
mxArray* mxCreateCellMatrix(mwSize m, mwSize n);
void* mxGetData(const mxArray* a);
double* mxGetPr(const mxArray* a);
double* mxGetPi(const mxArray* a);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x);
mxArray* mxCreateNumericArray(mwSize nd, const mwSize* dims, mxClassID c, mxComplexity x);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity x);
mxArray* mxCreateDoubleScalar(double v);
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names);
void mxSetField(mxArray* s, mwSize i, const char* name, mxArray* v);
mxArray* mxGetField(const mxArray* s, mwSize i, const char* name);
void mxDestroyArray(mxArray* a);
void* mxMalloc(size_t n);
void mxFree(void* p);

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);
#endif
