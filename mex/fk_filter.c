/* [dfk] = fk_filter(d, dt, dx) (core/fk_filter.m:1-302) on libswd.so: the f-k dip filter that
 * the field drivers apply to a gather before the Radon transform.  d: ns x ntr; the output is
 * double, as the reference's real(ifft2(...)); single input is filtered in double and returned
 * rounded to single, as MATLAB's fft2 of single data computes in single precision. */
#include "swd_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 3) mexErrMsgIdAndTxt("swd:nrhs", "fk_filter takes 3 inputs (d, dt, dx)");
  if (nlhs > 1) mexErrMsgIdAndTxt("swd:nlhs", "fk_filter returns one output");
  const int ns = (int)mxGetM(prhs[0]), ntr = (int)mxGetN(prhs[0]);
  const double dt = swd_scalar(prhs[1], "dt"), dx = swd_scalar(prhs[2], "dx");
  double* owned;
  const double* in = swd_as_double(prhs[0], "d", 0, &owned);
  mxArray* out = mxCreateDoubleMatrix((mwSize)ns, (mwSize)ntr, mxREAL);
  const int rc = ns > 0 && ntr > 0 ? swd_fk_filter(in, ns, ntr, dt, dx, mxGetPr(out)) : SWD_OK;
  if (owned) mxFree(owned);
  if (rc != SWD_OK) mxDestroyArray(out);
  swd_mex_fail(rc, "fk_filter");
  if (mxIsSingle(prhs[0])) {
    double* o = mxGetPr(out);
    for (size_t i = 0; i < (size_t)ns * ntr; ++i) o[i] = (double)(float)o[i];
  }
  plhs[0] = out;
}
