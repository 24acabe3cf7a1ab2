/*
 * Shared body of the ADWDgrad_1 / ADWDgrad_norm MEX shims:
 * a_data_res = NAME(nt,ng,ns,npair,is,w,m,M,SoftArgNorm,grad_outputr,grad_outputl,
 *                   space_M,saveForBackwardr,saveForBackwardl)
 * The saveForBackward structs must come from the RTrAD / RTlAD shims (their swd_params field
 * holds the transform's parameters); a side the reference skips for this shot
 * (ADWDgrad_1.m:13, :46) is not read, as in the reference.  With SWD_ADWD_NORM set, the
 * structs also carry cr_r / cr_l (the picks minus vmin, SWD.m:178, :184), around which
 * ADWDgrad_norm.m weights the spectrum with normpdf(1:np, cr, 16).  With SWD_ADWD_LIMBAND set,
 * the call is ADWDgradlimband (core/ADWDgradlimband.m); with SWD_ADWD_MAXNORM set, the field
 * drivers' ADWDgrad_1 (the adjoint source over its largest magnitude).
 */
#include <math.h>
#include <string.h>

#include "swd_mex.h"

static const mxArray* field(const mxArray* S, const char* name, const char* side) {
  const mxArray* f = mxIsStruct(S) ? mxGetField(S, 0, name) : NULL;
  if (!f)
    mexErrMsgIdAndTxt("swd:sfb", "saveForBackward%s has no field %s (it must come from the RTrAD/RTlAD shims)", side,
                      name);
  return f;
}

/* mm (np x nf, complex in MATLAB's separate storage or real) as interleaved re/im. */
static double* interleave(const mxArray* a, size_t n, const char* side) {
  if (!mxIsDouble(a) || swd_numel(a) != n)
    mexErrMsgIdAndTxt("swd:sfb", "saveForBackward%s.mm must be a double np x nf array", side);
  double* out = (double*)mxMalloc(2 * n * sizeof(double));
  const double* re = mxGetPr(a);
  const double* im = mxIsComplex(a) ? mxGetPi(a) : NULL;
  for (size_t i = 0; i < n; ++i) { out[2 * i] = re[i]; out[2 * i + 1] = im ? im[i] : 0.0; }
  return out;
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 14) mexErrMsgIdAndTxt("swd:nrhs", SWD_NAME " takes 14 inputs");
  if (nlhs > 1) mexErrMsgIdAndTxt("swd:nlhs", SWD_NAME " returns one output");
  const int nt = (int)swd_scalar(prhs[0], "nt"), ng = (int)swd_scalar(prhs[1], "ng");
  const int ns = (int)swd_scalar(prhs[2], "ns"), npair = (int)swd_scalar(prhs[3], "npair");
  const int is = (int)swd_scalar(prhs[4], "is"), w = (int)swd_scalar(prhs[5], "w");
  const int m = (int)swd_scalar(prhs[6], "m"), M = (int)swd_scalar(prhs[7], "M");
  const double beta = swd_scalar(prhs[8], "SoftArgNorm");
  if (M < 1) mexErrMsgIdAndTxt("swd:M", "M must be >= 1");
  const int on[2] = {is <= ns - (int)floor((double)m / M) - swd_round((double)w / M),
                     is >= swd_round((double)w / M) + (int)floor((double)m / M) + 1};
  static const char* sname[2] = {"r", "l"};
  static const char* rawname[2] = {"mlr", "mll"};
  static const char* crname[2] = {"cr_r", "cr_l"};
  swd_radon_params p;
  int have_p = 0;
  const double* go[2] = {NULL, NULL};
  const double* raw[2] = {NULL, NULL};
  const double* cr[2] = {NULL, NULL};
  double* mm[2] = {NULL, NULL};
  int np = 0, np2 = 0, lf = 0, nf = 0, ccn = 0;
  for (int s = 0; s < 2; ++s) {
    if (!on[s]) continue;
    const mxArray* S = prhs[12 + s];
    const mxArray* prm = field(S, "swd_params", sname[s]);
    const double* v = swd_in_double(prm, "swd_params", 13);
    swd_radon_params q;
    memset(&q, 0, sizeof(q));
    q.df = v[0]; q.dt = v[1]; q.fmin = v[2]; q.fmax = v[3]; q.vmin = v[4]; q.vmax = v[5]; q.dv = v[6]; q.ds = v[7];
    q.nt = (int)v[8]; q.ng = (int)v[9]; q.offset = (int)v[10]; q.m = (int)v[11]; q.M = (int)v[12];
    q.precision = SWD_PREC_FP64;
    if (q.nt != nt || q.ng != ng || q.m != m || q.M != M)
      mexErrMsgIdAndTxt("swd:sfb", "saveForBackward%s was computed for other nt/ng/m/M", sname[s]);
    p = q;
    have_p = 1;
    swd_mex_fail(swd_radon_sizes(&p, &np, &np2, &lf, &nf, &ccn), SWD_NAME);
    if (np2 != npair) mexErrMsgIdAndTxt("swd:npair", "npair (%d) differs from the spectrum's (%d)", npair, np2);
    go[s] = swd_in_double(prhs[9 + s], s ? "grad_outputl" : "grad_outputr", (size_t)npair);
    raw[s] = swd_in_double(field(S, rawname[s], sname[s]), rawname[s], (size_t)np * npair);
    if (SWD_ADWD_NORM) cr[s] = swd_in_double(field(S, crname[s], sname[s]), crname[s], (size_t)npair);
    mm[s] = interleave(field(S, "mm", sname[s]), (size_t)np * nf, sname[s]);
  }
  plhs[0] = mxCreateDoubleMatrix((mwSize)nt, (mwSize)ng, mxREAL);
  if (!have_p) return; /* neither side runs: zeros(nt,ng) as the reference returns */
  const double* space = swd_in_double(prhs[11], "space_M", (size_t)np * npair);
#ifndef SWD_ADWD_LIMBAND
#define SWD_ADWD_LIMBAND 0
#endif
#ifndef SWD_ADWD_MAXNORM
#define SWD_ADWD_MAXNORM 0
#endif
  const int rc = SWD_ADWD_NORM ? swd_adwdgrad_norm(&p, ns, is, w, beta, go[0], go[1], space, mm[0], raw[0], cr[0],
                                                  mm[1], raw[1], cr[1], mxGetPr(plhs[0]))
                 : SWD_ADWD_MAXNORM ? swd_adwdgrad_maxnorm(&p, ns, is, w, beta, go[0], go[1], space, mm[0], raw[0],
                                                           mm[1], raw[1], mxGetPr(plhs[0]))
                 : SWD_ADWD_LIMBAND ? swd_adwdgrad_limband(&p, ns, is, w, beta, go[0], go[1], space, mm[0], raw[0],
                                                           mm[1], raw[1], mxGetPr(plhs[0]))
                                    : swd_adwdgrad(&p, ns, is, w, beta, go[0], go[1], space, mm[0], raw[0], mm[1],
                                                   raw[1], mxGetPr(plhs[0]));
  for (int s = 0; s < 2; ++s)
    if (mm[s]) mxFree(mm[s]);
  swd_mex_fail(rc, SWD_NAME);
}
