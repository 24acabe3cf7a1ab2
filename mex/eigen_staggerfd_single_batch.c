/* [seismo_u, seismo_w, www] = eigen_staggerfd_single_batch(input_vectors, temps, cas, cls, cms, cm1s,
 *                                                          bs, b1s, ss)
 * on libswd.so: several eigen_staggerfd_single calls (core/staggerfd_eigen.m:139) at once.  Every
 * input is a cell array with one entry per job, each entry what eigen_staggerfd_single takes; the
 * outputs are cell arrays of the jobs' seismograms (and www structs) in job order.  The jobs may
 * have grids of different sizes; one launch per time step advances all of them, and each job's
 * outputs are those of its own call, bit for bit.  It has no counterpart in the reference, which
 * makes one MEX call per shot and model. */
#include "swd_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  static const char* names[8] = {"temp", "ca", "cl", "cm", "cm1", "b", "b1", "s"};
  static const char* fields[4] = {"fux", "fuz", "bwx", "bwz"};
  if (nrhs != 9)
    mexErrMsgIdAndTxt("swd:nrhs", "eigen_staggerfd_single_batch takes 9 cell arrays (input_vectors, temps, cas, "
                      "cls, cms, cm1s, bs, b1s, ss)");
  if (nlhs > 3) mexErrMsgIdAndTxt("swd:nlhs", "eigen_staggerfd_single_batch returns at most 3 outputs");
  for (int i = 0; i < 9; ++i)
    if (!mxIsCell(prhs[i])) mexErrMsgIdAndTxt("swd:class", "input %d must be a cell array (one entry per job)", i + 1);
  const size_t n = swd_numel(prhs[0]);
  if (n < 1) mexErrMsgIdAndTxt("swd:size", "no jobs");
  for (int i = 1; i < 9; ++i)
    if (swd_numel(prhs[i]) != n) mexErrMsgIdAndTxt("swd:size", "input %d has %zu entries, the first %zu", i + 1,
                                                   swd_numel(prhs[i]), n);
  swd_staggerfd_job* jobs = (swd_staggerfd_job*)mxMalloc(n * sizeof(swd_staggerfd_job));
  float* ivs = (float*)mxMalloc(n * 16 * sizeof(float));
  mxArray* out[3];
  out[0] = mxCreateCellMatrix(1, (mwSize)n);
  out[1] = mxCreateCellMatrix(1, (mwSize)n);
  out[2] = nlhs >= 3 ? mxCreateCellMatrix(1, (mwSize)n) : NULL;
  for (size_t j = 0; j < n; ++j) {
    const mxArray* ivj = mxGetCell(prhs[0], (mwSize)j);
    if (!ivj) mexErrMsgIdAndTxt("swd:size", "job %zu has no input_vector", j + 1);
    const float* iv = swd_iv_single(ivj, 16, ivs + 16 * j, 16);
    if (iv != ivs + 16 * j)
      for (int k = 0; k < 16; ++k) ivs[16 * j + k] = iv[k];
    const float* v = ivs + 16 * j;
    const int nt = (int)v[0], nzbc = (int)v[1], nxbc = (int)v[2], ng = (int)v[4];
    const int nt_wf = (int)v[12], nz = (int)v[13], nx = (int)v[14], fmt = (int)v[15];
    if (nt < 1 || nzbc < 1 || nxbc < 1 || ng < 1 || nt_wf < 1 || nz < 1 || nx < 1)
      mexErrMsgIdAndTxt("swd:iv", "job %zu: input_vector sizes must be positive", j + 1);
    const size_t cells = (size_t)nzbc * (size_t)nxbc;
    const float* f[8];
    for (int k = 0; k < 8; ++k) {
      const mxArray* a = mxGetCell(prhs[1 + k], (mwSize)j);
      if (!a) mexErrMsgIdAndTxt("swd:size", "job %zu has no %s", j + 1, names[k]);
      f[k] = swd_in_single(a, names[k], k < 7 ? cells : (size_t)nt);
    }
    mxArray* su = swd_new((mwSize)nt, (mwSize)ng, mxSINGLE_CLASS);
    mxArray* sw = swd_new((mwSize)nt, (mwSize)ng, mxSINGLE_CLASS);
    mxSetCell(out[0], (mwSize)j, su);
    mxSetCell(out[1], (mwSize)j, sw);
    float* snap[4] = {NULL, NULL, NULL, NULL};
    if (out[2]) {
      mxArray* S = mxCreateStructMatrix(1, 1, 4, fields);
      const mwSize nrec = (mwSize)(nt / nt_wf);
      mwSize d3[3] = {(mwSize)nz, (mwSize)nx, nrec};
      mwSize d2[2] = {(mwSize)nz, (mwSize)nx * nrec};
      for (int k = 0; k < 4; ++k) {
        mxArray* a = fmt == 2 ? mxCreateNumericArray(2, d2, mxSINGLE_CLASS, mxREAL)
                              : mxCreateNumericArray(3, d3, mxSINGLE_CLASS, mxREAL);
        mxSetField(S, 0, fields[k], a);
        snap[k] = (float*)mxGetData(a);
      }
      mxSetCell(out[2], (mwSize)j, S);
    }
    swd_staggerfd_job q = {v, 16, f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7],
                           (float*)mxGetData(su), (float*)mxGetData(sw), snap[0], snap[1], snap[2], snap[3]};
    jobs[j] = q;
  }
  const int rc = swd_staggerfd_single_batch((int)n, jobs);
  mxFree(jobs);
  mxFree(ivs);
  if (rc != SWD_OK)
    for (int i = 0; i < 3; ++i) mxDestroyArray(out[i]);
  swd_mex_fail(rc, "eigen_staggerfd_single_batch");
  plhs[0] = out[0];
  if (nlhs >= 2) plhs[1] = out[1];
  else mxDestroyArray(out[1]);
  if (nlhs >= 3) plhs[2] = out[2];
}
