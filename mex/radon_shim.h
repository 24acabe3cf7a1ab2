/*
 * Body of the RTrAD / RTlAD / RTr / RTl shims, included with SWD_SIDE (0 right, 1 left),
 * SWD_AD (1: also return saveForBackward) and SWD_NAME defined.
 *
 * [ml, dataLen, saveForBackward] = RTrAD(seismo_v1,is,df,dt,np,vmin,vmax,fmin,fmax,a,b,ds,offset,m,M)
 * (core/RTrAD.m:2-35, core/RTlAD.m:2-36; RTr/RTl return [ml, dataLen], core/RTr.m:2-32).
 * The velocity axis is vmin:vmax in 1 m/s steps as in the reference (np = vmax-vmin+1).
 * saveForBackward carries the reference's fields (mm, ll0, lf, nf, ccn, mlr|mll,
 * uxtposr|uxtposl) plus swd_params, which the ADWDgrad_1 shim reads back.
 */
#include <math.h>

#include "swd_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 15)
    mexErrMsgIdAndTxt("swd:nrhs", "%s takes 15 inputs (seismo_v1,is,df,dt,np,vmin,vmax,fmin,fmax,a,b,ds,offset,m,M)",
                      SWD_NAME);
  if (nlhs > 2 + SWD_AD) mexErrMsgIdAndTxt("swd:nlhs", "%s returns at most %d outputs", SWD_NAME, 2 + SWD_AD);
  swd_radon_params p;
  memset(&p, 0, sizeof(p));
  const int is = (int)swd_scalar(prhs[1], "is");
  p.df = swd_scalar(prhs[2], "df");
  p.dt = swd_scalar(prhs[3], "dt");
  const int np_arg = (int)swd_scalar(prhs[4], "np");
  p.vmin = swd_scalar(prhs[5], "vmin");
  p.vmax = swd_scalar(prhs[6], "vmax");
  p.fmin = swd_scalar(prhs[7], "fmin");
  p.fmax = swd_scalar(prhs[8], "fmax");
  p.nt = (int)swd_scalar(prhs[9], "a");
  p.ng = (int)swd_scalar(prhs[10], "b");
  p.ds = swd_scalar(prhs[11], "ds");
  p.offset = (int)swd_scalar(prhs[12], "offset");
  p.m = (int)swd_scalar(prhs[13], "m");
  p.M = (int)swd_scalar(prhs[14], "M");
  p.dv = 1.0;
  p.precision = SWD_PREC_FP64;
  int np = 0, npair = 0, lf = 0, nf = 0, ccn = 0;
  swd_mex_fail(swd_radon_sizes(&p, &np, &npair, &lf, &nf, &ccn), SWD_NAME);
  if (np_arg != np) mexErrMsgIdAndTxt("swd:np", "%s: np (%d) must be vmax-vmin+1 (%d)", SWD_NAME, np_arg, np);
  double* seis_owned;
  const double* seis = swd_as_double(prhs[0], "seismo_v1", (size_t)p.nt * (size_t)p.ng, &seis_owned);
  mxArray* ml = mxCreateDoubleMatrix((mwSize)np, (mwSize)npair, mxREAL);
  mxArray* raw = SWD_AD ? mxCreateDoubleMatrix((mwSize)np, (mwSize)npair, mxREAL) : NULL;
  double* mm = SWD_AD ? (double*)mxMalloc((size_t)2 * np * nf * sizeof(double)) : NULL;
  int* pos = SWD_AD ? (int*)mxMalloc((size_t)(p.offset > 0 ? p.offset : 1) * sizeof(int)) : NULL;
  int len = 0;
  const int rc = swd_radon(&p, SWD_SIDE, is, seis, mxGetPr(ml), raw ? mxGetPr(raw) : NULL, mm, &len, pos);
  if (seis_owned) mxFree(seis_owned);
  if (rc != SWD_OK) {
    if (mm) mxFree(mm);
    if (pos) mxFree(pos);
    swd_mex_fail(rc, SWD_NAME);
  }
  plhs[0] = ml;
  if (nlhs >= 2) plhs[1] = mxCreateDoubleScalar((double)len);
  if (SWD_AD && nlhs >= 3) {
    static const char* fields[8] = {"mm", "ll0", "lf", "nf", "ccn", SWD_SIDE ? "mll" : "mlr",
                                    SWD_SIDE ? "uxtposl" : "uxtposr", "swd_params"};
    mxArray* S = mxCreateStructMatrix(1, 1, 8, fields);
    mxArray* amm = mxCreateDoubleMatrix((mwSize)np, (mwSize)nf, mxCOMPLEX);
    double *re = mxGetPr(amm), *im = mxGetPi(amm);
    for (size_t i = 0; i < (size_t)np * nf; ++i) { re[i] = mm[2 * i]; im[i] = mm[2 * i + 1]; }
    /* ll0 = 1i*2*pi*df*(pp*x), pp = 1./(vmin:vmax)', x = (m + (0:dataLen-1))*ds (RTrAD.m:11,20-21) */
    mxArray* all0 = mxCreateDoubleMatrix((mwSize)np, (mwSize)len, mxCOMPLEX);
    double* lim = mxGetPi(all0);
    const double w = 2.0 * M_PI * p.df;
    for (int j = 0; j < len; ++j)
      for (int k = 0; k < np; ++k) lim[(size_t)j * np + k] = w * ((1.0 / (p.vmin + k)) * ((p.m + j) * p.ds));
    mxArray* apos = mxCreateDoubleMatrix(1, (mwSize)len, mxREAL);
    for (int j = 0; j < len; ++j) mxGetPr(apos)[j] = pos[j];
    mxArray* prm = mxCreateDoubleMatrix(1, 13, mxREAL);
    const double pv[13] = {p.df, p.dt, p.fmin, p.fmax, p.vmin, p.vmax, p.dv, p.ds, p.nt, p.ng, p.offset, p.m, p.M};
    memcpy(mxGetPr(prm), pv, sizeof(pv));
    mxSetField(S, 0, "mm", amm);
    mxSetField(S, 0, "ll0", all0);
    mxSetField(S, 0, "lf", mxCreateDoubleScalar(lf));
    mxSetField(S, 0, "nf", mxCreateDoubleScalar(nf));
    mxSetField(S, 0, "ccn", mxCreateDoubleScalar(ccn));
    mxSetField(S, 0, fields[5], raw);
    mxSetField(S, 0, fields[6], apos);
    mxSetField(S, 0, "swd_params", prm);
    plhs[2] = S;
  } else if (raw) {
    mxDestroyArray(raw);
  }
  if (mm) mxFree(mm);
  if (pos) mxFree(pos);
}
