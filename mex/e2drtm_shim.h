/*
 * Body of the eigen_e2drtm_single / eigen_e2drtm_double shims, included once per
 * precision with SWD_T, SWD_CLASS, SWD_IN, SWD_IV, SWD_RTM and SWD_NAME defined.
 *
 * [cl_img, cm_img, illum_div] = eigen_e2drtm_*(input_vector, temp, ca, cl, cm, cm1, b, b1,
 *                                              seismo_w, fux, fuz, bwx, bwz)
 * as called at core/e2drtm_eigen.m:122 (core/eigen_e2drtm_single.cpp:69-136, :288-296).
 */
#include "swd_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  static const char* names[12] = {"temp", "ca", "cl", "cm", "cm1", "b", "b1", "seismo_w", "fux", "fuz", "bwx", "bwz"};
  if (nrhs != 13)
    mexErrMsgIdAndTxt("swd:nrhs", "%s takes 13 inputs (input_vector,temp,ca,cl,cm,cm1,b,b1,seismo_w,fux,fuz,bwx,bwz)",
                      SWD_NAME);
  if (nlhs > 3) mexErrMsgIdAndTxt("swd:nlhs", "%s returns at most 3 outputs", SWD_NAME);
  SWD_T ivbuf[14];
  const SWD_T* iv = SWD_IV(prhs[0], 14, ivbuf, 14);
  const int n_iv = swd_numel(prhs[0]) < 14 ? (int)swd_numel(prhs[0]) : 14;
  const int nt = (int)iv[0], nzbc = (int)iv[1], nxbc = (int)iv[2], ng = (int)iv[4];
  const int nt_wf = (int)iv[10], nz = (int)iv[11], nx = (int)iv[12];
  if (nt < 1 || nzbc < 1 || nxbc < 1 || ng < 1 || nt_wf < 1 || nz < 1 || nx < 1)
    mexErrMsgIdAndTxt("swd:iv", "%s: input_vector sizes must be positive", SWD_NAME);
  const size_t cells = (size_t)nzbc * (size_t)nxbc;
  const size_t snap = (size_t)nz * (size_t)nx * (size_t)(nt / nt_wf);
  const SWD_T* f[12];
  for (int k = 0; k < 7; ++k) f[k] = SWD_IN(prhs[1 + k], names[k], cells);
  f[7] = SWD_IN(prhs[8], names[7], (size_t)nt * (size_t)ng);
  for (int k = 8; k < 12; ++k) f[k] = SWD_IN(prhs[1 + k], names[k], snap);
  mxArray* out[3];
  for (int k = 0; k < 3; ++k) out[k] = swd_new((mwSize)nz, (mwSize)nx, SWD_CLASS);
  const int rc = SWD_RTM(iv, n_iv, f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[10], f[11],
                         (SWD_T*)mxGetData(out[0]), (SWD_T*)mxGetData(out[1]), (SWD_T*)mxGetData(out[2]));
  for (int k = 0; k < 3; ++k) {
    if (k < (nlhs > 0 ? nlhs : 1)) plhs[k] = out[k];
    else mxDestroyArray(out[k]);
  }
  swd_mex_fail(rc, SWD_NAME);
}
