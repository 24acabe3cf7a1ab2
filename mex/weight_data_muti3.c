/*
 * seismo_v_d1 = weight_data_muti3(seismo_v_d,seismo_v,is,dt,df,offset,dg,F1,w,M,m,ns,refsx,win,
 *                                 fmin,fmax,cr_0,cr_0l,cr_pre_r,cr_pre_l,ind)
 * (core/weight_data_muti3.m:1-122, the WD adjoint source of SWD.m:188) on libswd.so.
 * The seismograms may be single or double; pick vectors that do not hold
 * floor((fmax-fmin)/df+1) entries are passed as missing, and the library rejects them
 * for a side it computes (the reference fails there with a size mismatch).
 */
#include <math.h>

#include "swd_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 21) mexErrMsgIdAndTxt("swd:nrhs", "weight_data_muti3 takes 21 inputs");
  if (nlhs > 1) mexErrMsgIdAndTxt("swd:nlhs", "weight_data_muti3 returns one output here (deta_c is never set)");
  const int nt = (int)mxGetM(prhs[0]), ng = (int)mxGetN(prhs[0]);
  if (nt < 1 || ng < 1) mexErrMsgIdAndTxt("swd:size", "seismo_v_d must be a non-empty nt x ng array");
  const int is = (int)swd_scalar(prhs[2], "is");
  const double dt = swd_scalar(prhs[3], "dt"), df = swd_scalar(prhs[4], "df");
  const int offset = (int)swd_scalar(prhs[5], "offset");
  const double dg = swd_scalar(prhs[6], "dg");
  const int F1 = (int)swd_scalar(prhs[7], "F1"), w = (int)swd_scalar(prhs[8], "w");
  const double M = swd_scalar(prhs[9], "M");
  const int m = (int)swd_scalar(prhs[10], "m"), ns = (int)swd_scalar(prhs[11], "ns");
  const double* refsx = swd_in_double(prhs[12], "refsx", ns > 0 ? (size_t)ns : 1);
  const int win = (int)swd_scalar(prhs[13], "win");
  const double fmin = swd_scalar(prhs[14], "fmin"), fmax = swd_scalar(prhs[15], "fmax");
  const double indd = swd_scalar(prhs[20], "ind");
  if (indd != floor(indd)) mexErrMsgIdAndTxt("swd:ind", "ind must be an integer index");
  const size_t npair = df > 0 ? (size_t)floor((fmax - fmin) / df + 1) : 0;
  const double* cr[4];
  for (int k = 0; k < 4; ++k) {
    const mxArray* a = prhs[16 + k];
    cr[k] = (mxIsDouble(a) && !mxIsComplex(a) && swd_numel(a) == npair) ? (const double*)mxGetData(a) : NULL;
  }
  const int src = F1 == 1 ? 0 : 1;
  if ((int)mxGetM(prhs[src]) != nt || (int)mxGetN(prhs[src]) != ng)
    mexErrMsgIdAndTxt("swd:size", "seismo_v must have the size of seismo_v_d");
  double* owned = NULL;
  const double* seis = swd_as_double(prhs[src], src ? "seismo_v" : "seismo_v_d", (size_t)nt * ng, &owned);
  plhs[0] = mxCreateDoubleMatrix((mwSize)nt, (mwSize)ng, mxREAL);
  const int rc = swd_wd_residual(nt, ng, src ? NULL : seis, src ? seis : NULL, is, dt, df, offset, dg, F1, w, M, m,
                                 ns, refsx, win, fmin, fmax, cr[0], cr[1], cr[2], cr[3], (int)indd,
                                 mxGetPr(plhs[0]));
  if (owned) mxFree(owned);
  swd_mex_fail(rc, "weight_data_muti3");
}
