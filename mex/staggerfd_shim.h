/*
 * Body of the eigen_staggerfd_single / eigen_staggerfd_double shims, included once per
 * precision with SWD_T, SWD_CLASS, SWD_IN, SWD_IV, SWD_FD and SWD_NAME defined.
 *
 * [seismo_u, seismo_w, www] = eigen_staggerfd_*(input_vector, temp, ca, cl, cm, cm1, b, b1, s)
 * as called at core/staggerfd_eigen.m:139 (arguments and outputs of
 * core/eigen_staggerfd_single.cpp:98-152 and :359-383).  www.{fux,fuz,bwx,bwz} are
 * nz x nx x (nt/nt_wf) for format 3 and nz x (nx*nt/nt_wf) for format 2.  When the caller
 * asks for fewer than three outputs the snapshots are not computed at all.
 */
#include "swd_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  static const char* names[8] = {"temp", "ca", "cl", "cm", "cm1", "b", "b1", "s"};
  static const char* fields[4] = {"fux", "fuz", "bwx", "bwz"};
  if (nrhs != 9) mexErrMsgIdAndTxt("swd:nrhs", "%s takes 9 inputs (input_vector,temp,ca,cl,cm,cm1,b,b1,s)", SWD_NAME);
  if (nlhs > 3) mexErrMsgIdAndTxt("swd:nlhs", "%s returns at most 3 outputs", SWD_NAME);
  SWD_T ivbuf[16];
  const SWD_T* iv = SWD_IV(prhs[0], 16, ivbuf, 16);
  const int n_iv = swd_numel(prhs[0]) < 16 ? (int)swd_numel(prhs[0]) : 16;
  const int nt = (int)iv[0], nzbc = (int)iv[1], nxbc = (int)iv[2], ng = (int)iv[4];
  const int nt_wf = (int)iv[12], nz = (int)iv[13], nx = (int)iv[14], fmt = (int)iv[15];
  if (nt < 1 || nzbc < 1 || nxbc < 1 || ng < 1 || nt_wf < 1 || nz < 1 || nx < 1)
    mexErrMsgIdAndTxt("swd:iv", "%s: input_vector sizes must be positive", SWD_NAME);
  const size_t cells = (size_t)nzbc * (size_t)nxbc;
  const SWD_T* f[8];
  for (int k = 0; k < 7; ++k) f[k] = SWD_IN(prhs[1 + k], names[k], cells);
  f[7] = SWD_IN(prhs[8], names[7], (size_t)nt);
  plhs[0] = swd_new((mwSize)nt, (mwSize)ng, SWD_CLASS);
  mxArray* w = swd_new((mwSize)nt, (mwSize)ng, SWD_CLASS);
  if (nlhs >= 2) plhs[1] = w;
  SWD_T* snap[4] = {NULL, NULL, NULL, NULL};
  if (nlhs >= 3) {
    mxArray* S = mxCreateStructMatrix(1, 1, 4, fields);
    const mwSize nrec = (mwSize)(nt / nt_wf);
    mwSize d3[3] = {(mwSize)nz, (mwSize)nx, nrec};
    mwSize d2[2] = {(mwSize)nz, (mwSize)nx * nrec};
    for (int k = 0; k < 4; ++k) {
      mxArray* a = fmt == 2 ? mxCreateNumericArray(2, d2, SWD_CLASS, mxREAL)
                            : mxCreateNumericArray(3, d3, SWD_CLASS, mxREAL);
      mxSetField(S, 0, fields[k], a);
      snap[k] = (SWD_T*)mxGetData(a);
    }
    plhs[2] = S;
  }
  const int rc = SWD_FD(iv, n_iv, f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], (SWD_T*)mxGetData(plhs[0]),
                        (SWD_T*)mxGetData(w), snap[0], snap[1], snap[2], snap[3]);
  if (nlhs < 2) mxDestroyArray(w);
  swd_mex_fail(rc, SWD_NAME);
}
