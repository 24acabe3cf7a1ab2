/*
 * [res, cr_pre] = LHDispPick(ml, vmin, cr_0, method, ini) (core/LHDispPick.m:2-13) on libswd.so.
 * method 1: the guided picker pickFDC1(ml, ini, 2, 4); cr_pre is npair x 1 (idx' + vmin).
 * Otherwise: argmax per column; cr_pre is 1 x npair as max() returns it.  res is the mean
 * squared difference to cr_0 taken element by element.
 */
#include "swd_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 5) mexErrMsgIdAndTxt("swd:nrhs", "LHDispPick takes 5 inputs (ml,vmin,cr_0,method,ini)");
  if (nlhs > 2) mexErrMsgIdAndTxt("swd:nlhs", "LHDispPick returns at most 2 outputs");
  const int np = (int)mxGetM(prhs[0]), npair = (int)mxGetN(prhs[0]);
  double* ml_owned;
  const double* ml = swd_as_double(prhs[0], "ml", 0, &ml_owned);
  const double vmin = swd_scalar(prhs[1], "vmin");
  double* cr0_owned;
  const double* cr0 = swd_as_double(prhs[2], "cr_0", 0, &cr0_owned);
  const int method = (int)swd_scalar(prhs[3], "method");
  const int ini = (int)swd_scalar(prhs[4], "ini");
  double* cr0b = NULL;
  if (swd_numel(prhs[2]) == 1) { /* scalar cr_0 broadcasts */
    cr0b = (double*)mxMalloc((size_t)(npair > 0 ? npair : 1) * sizeof(double));
    for (int i = 0; i < npair; ++i) cr0b[i] = cr0[0];
    cr0 = cr0b;
  } else if (swd_numel(prhs[2]) != (size_t)npair) {
    mexErrMsgIdAndTxt("swd:size", "cr_0 has %zu elements, ml has %d columns", swd_numel(prhs[2]), npair);
  }
  mxArray* cr = method == 1 ? mxCreateDoubleMatrix((mwSize)npair, 1, mxREAL)
                            : mxCreateDoubleMatrix(1, (mwSize)npair, mxREAL);
  double res = 0.0;
  const int rc = swd_pick(ml, np, npair, vmin, cr0, method, ini, &res, mxGetPr(cr));
  if (ml_owned) mxFree(ml_owned);
  if (cr0_owned) mxFree(cr0_owned);
  if (cr0b) mxFree(cr0b);
  if (rc != SWD_OK) mxDestroyArray(cr);
  swd_mex_fail(rc, "LHDispPick");
  plhs[0] = mxCreateDoubleScalar(res);
  if (nlhs >= 2) plhs[1] = cr;
  else mxDestroyArray(cr);
}
