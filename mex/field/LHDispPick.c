/*
 * [res, cr_pre] = LHDispPick(ml, vmin, cr_0, method, saveForBackward) of the outcrop field
 * driver (fieldexamples/outcrop/core/LHDispPick.m:2-25) on libswd.so: the guided pick starts at
 * the global maximum of saveForBackward.mlr (or .mll for a left-side spectrum), seeded with its
 * row (pickFDCValue(ml,ini,iniP,2,4), fieldexamples/outcrop/core/pickFDCValue.m:1-131) for
 * method 1, argmax per column otherwise; res is the mean squared difference over rows
 * 15..end-15.  cr_pre is npair x 1 for method 1, 1 x npair otherwise (as the reference's
 * idx' + vmin and p_max + vmin).  saveForBackward must come from the RTrAD / RTlAD shims.
 */
#include "swd_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 5) mexErrMsgIdAndTxt("swd:nrhs", "LHDispPick takes 5 inputs (ml,vmin,cr_0,method,saveForBackward)");
  if (nlhs > 2) mexErrMsgIdAndTxt("swd:nlhs", "LHDispPick returns at most 2 outputs");
  const int np = (int)mxGetM(prhs[0]), npair = (int)mxGetN(prhs[0]);
  const mxArray* S = prhs[4];
  const mxArray* rawa = mxIsStruct(S) ? mxGetField(S, 0, mxGetField(S, 0, "uxtposr") ? "mlr" : "mll") : NULL;
  if (!rawa) mexErrMsgIdAndTxt("swd:sfb", "saveForBackward needs mlr (with uxtposr) or mll");
  double* ml_owned;
  const double* ml = swd_as_double(prhs[0], "ml", 0, &ml_owned);
  const double* raw = swd_in_double(rawa, "saveForBackward.mlr/mll", (size_t)np * npair);
  const double vmin = swd_scalar(prhs[1], "vmin");
  double* cr0_owned;
  const double* cr0 = swd_as_double(prhs[2], "cr_0", (size_t)npair, &cr0_owned);
  const int method = (int)swd_scalar(prhs[3], "method");
  mxArray* cr = method == 1 ? mxCreateDoubleMatrix((mwSize)npair, 1, mxREAL)
                            : mxCreateDoubleMatrix(1, (mwSize)npair, mxREAL);
  double res = 0.0;
  const int rc = swd_pick_field(ml, raw, np, npair, vmin, cr0, method, 1, &res, mxGetPr(cr));
  if (ml_owned) mxFree(ml_owned);
  if (cr0_owned) mxFree(cr0_owned);
  if (rc != SWD_OK) mxDestroyArray(cr);
  swd_mex_fail(rc, "LHDispPick");
  plhs[0] = mxCreateDoubleScalar(res);
  if (nlhs >= 2) plhs[1] = cr;
  else mxDestroyArray(cr);
}
