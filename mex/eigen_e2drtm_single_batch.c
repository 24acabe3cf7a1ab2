/* [cl_imgs, cm_imgs, illum_divs] = eigen_e2drtm_single_batch(input_vectors, temps, cas, cls, cms, cm1s,
 *                                                            bs, b1s, seismo_ws, fuxs, fuzs, bwxs, bwzs)
 * on libswd.so: several eigen_e2drtm_single calls (core/e2drtm_eigen.m:122) at once.  Every input
 * is a cell array with one entry per job, each entry what eigen_e2drtm_single takes; the outputs
 * are cell arrays of the jobs' nz x nx images in job order.  The jobs may have grids of different
 * sizes and different nt; one launch per time step advances all of them, each job counting its
 * steps back from its own nt, and each job's images are those of its own call, bit for bit.  It
 * has no counterpart in the reference, which makes one MEX call per shot and model. */
#include "swd_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  static const char* names[12] = {"temp", "ca", "cl", "cm", "cm1", "b", "b1", "seismo_w", "fux", "fuz", "bwx", "bwz"};
  if (nrhs != 13)
    mexErrMsgIdAndTxt("swd:nrhs", "eigen_e2drtm_single_batch takes 13 cell arrays (input_vectors, temps, cas, cls, "
                      "cms, cm1s, bs, b1s, seismo_ws, fuxs, fuzs, bwxs, bwzs)");
  if (nlhs > 3) mexErrMsgIdAndTxt("swd:nlhs", "eigen_e2drtm_single_batch returns at most 3 outputs");
  for (int i = 0; i < 13; ++i)
    if (!mxIsCell(prhs[i])) mexErrMsgIdAndTxt("swd:class", "input %d must be a cell array (one entry per job)", i + 1);
  const size_t n = swd_numel(prhs[0]);
  if (n < 1) mexErrMsgIdAndTxt("swd:size", "no jobs");
  for (int i = 1; i < 13; ++i)
    if (swd_numel(prhs[i]) != n) mexErrMsgIdAndTxt("swd:size", "input %d has %zu entries, the first %zu", i + 1,
                                                   swd_numel(prhs[i]), n);
  swd_e2drtm_job* jobs = (swd_e2drtm_job*)mxMalloc(n * sizeof(swd_e2drtm_job));
  float* ivs = (float*)mxMalloc(n * 14 * sizeof(float));
  mxArray* out[3];
  for (int k = 0; k < 3; ++k) out[k] = mxCreateCellMatrix(1, (mwSize)n);
  for (size_t j = 0; j < n; ++j) {
    const mxArray* ivj = mxGetCell(prhs[0], (mwSize)j);
    if (!ivj) mexErrMsgIdAndTxt("swd:size", "job %zu has no input_vector", j + 1);
    const float* iv = swd_iv_single(ivj, 14, ivs + 14 * j, 14);
    if (iv != ivs + 14 * j)
      for (int k = 0; k < 14; ++k) ivs[14 * j + k] = iv[k];
    const float* v = ivs + 14 * j;
    const int nt = (int)v[0], nzbc = (int)v[1], nxbc = (int)v[2], ng = (int)v[4];
    const int nt_wf = (int)v[10], nz = (int)v[11], nx = (int)v[12];
    if (nt < 1 || nzbc < 1 || nxbc < 1 || ng < 1 || nt_wf < 1 || nz < 1 || nx < 1)
      mexErrMsgIdAndTxt("swd:iv", "job %zu: input_vector sizes must be positive", j + 1);
    const size_t cells = (size_t)nzbc * (size_t)nxbc;
    const size_t snap = (size_t)nz * (size_t)nx * (size_t)(nt / nt_wf);
    const float* f[12];
    for (int k = 0; k < 12; ++k) {
      const mxArray* a = mxGetCell(prhs[1 + k], (mwSize)j);
      if (!a) mexErrMsgIdAndTxt("swd:size", "job %zu has no %s", j + 1, names[k]);
      f[k] = swd_in_single(a, names[k], k < 7 ? cells : k == 7 ? (size_t)nt * (size_t)ng : snap);
    }
    float* img[3];
    for (int k = 0; k < 3; ++k) {
      mxArray* a = swd_new((mwSize)nz, (mwSize)nx, mxSINGLE_CLASS);
      mxSetCell(out[k], (mwSize)j, a);
      img[k] = (float*)mxGetData(a);
    }
    swd_e2drtm_job q = {v, 14, f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[10], f[11],
                        img[0], img[1], img[2]};
    jobs[j] = q;
  }
  const int rc = swd_e2drtm_single_batch((int)n, jobs);
  mxFree(jobs);
  mxFree(ivs);
  if (rc != SWD_OK)
    for (int k = 0; k < 3; ++k) mxDestroyArray(out[k]);
  swd_mex_fail(rc, "eigen_e2drtm_single_batch");
  for (int k = 0; k < 3; ++k) {
    if (k < (nlhs > 0 ? nlhs : 1)) plhs[k] = out[k];
    else mxDestroyArray(out[k]);
  }
}
