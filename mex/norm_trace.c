/* data_out = norm_trace(data_in) (core/norm_trace.m:1-22) on libswd.so: each column of the
 * nt x ng gather over its largest magnitude (a dead trace becomes NaN, as 0/0 there).  The
 * output is double, as the reference's zeros(size(data_in)); single input is divided in single
 * as MATLAB does (the FP64 quotient rounded to single is that quotient). */
#include "swd_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 1) mexErrMsgIdAndTxt("swd:nrhs", "norm_trace takes 1 input (data_in)");
  if (nlhs > 1) mexErrMsgIdAndTxt("swd:nlhs", "norm_trace returns one output");
  const int nt = (int)mxGetM(prhs[0]), ng = (int)mxGetN(prhs[0]);
  double* owned;
  const double* in = swd_as_double(prhs[0], "data_in", 0, &owned);
  mxArray* out = mxCreateDoubleMatrix((mwSize)nt, (mwSize)ng, mxREAL);
  const int rc = nt > 0 && ng > 0 ? swd_norm_trace(in, nt, ng, mxGetPr(out)) : SWD_OK;
  if (owned) mxFree(owned);
  if (rc != SWD_OK) mxDestroyArray(out);
  swd_mex_fail(rc, "norm_trace");
  if (mxIsSingle(prhs[0])) {
    double* o = mxGetPr(out);
    for (size_t i = 0; i < (size_t)nt * ng; ++i) o[i] = (double)(float)o[i];
  }
  plhs[0] = out;
}
