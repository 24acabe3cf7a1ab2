/*
 * swd_mex.h -- helpers shared by the C MEX shims that put libswd.so behind the
 * reference's MEX/function names.  The shims use only the C MEX API, so both
 * MATLAB (`mex`) and Octave (`mkoctfile --mex`) build them:
 *
 *   mkoctfile --mex -I../include eigen_staggerfd_single.c -L../swd_b200/lib -lswd
 *
 * Every shim validates class and size of its inputs and reports errors through
 * mexErrMsgIdAndTxt (the reference's MEX files check nothing).
 */
#ifndef SWD_MEX_H
#define SWD_MEX_H

#include <stddef.h>
#include <stdlib.h>

#include "mex.h"
#include "swd.h"

static void swd_mex_fail(int rc, const char* fn) {
  if (rc != SWD_OK) mexErrMsgIdAndTxt("swd:call", "%s: %s", fn, swd_last_error());
}

static size_t swd_numel(const mxArray* a) { return (size_t)mxGetNumberOfElements(a); }

/* Real single array with at least `need` elements (need 0: any size). */
static const float* swd_in_single(const mxArray* a, const char* what, size_t need) {
  if (!mxIsSingle(a) || mxIsComplex(a)) mexErrMsgIdAndTxt("swd:class", "%s must be a real single array", what);
  if (need && swd_numel(a) < need)
    mexErrMsgIdAndTxt("swd:size", "%s has %zu elements, needs %zu", what, swd_numel(a), need);
  return (const float*)mxGetData(a);
}

/* Real double array with at least `need` elements (need 0: any size). */
static const double* swd_in_double(const mxArray* a, const char* what, size_t need) {
  if (!mxIsDouble(a) || mxIsComplex(a)) mexErrMsgIdAndTxt("swd:class", "%s must be a real double array", what);
  if (need && swd_numel(a) < need)
    mexErrMsgIdAndTxt("swd:size", "%s has %zu elements, needs %zu", what, swd_numel(a), need);
  return (const double*)mxGetData(a);
}

/* A real scalar of class single or double, as a double. */
static double swd_scalar(const mxArray* a, const char* what) {
  if (mxIsComplex(a) || swd_numel(a) < 1 || !(mxIsDouble(a) || mxIsSingle(a)))
    mexErrMsgIdAndTxt("swd:class", "%s must be a real numeric scalar", what);
  return mxIsDouble(a) ? ((const double*)mxGetData(a))[0] : (double)((const float*)mxGetData(a))[0];
}

/* input_vector as float: the single path builds it in single (staggerfd_eigen.m:70), but a
 * double vector is accepted and rounded the way MATLAB's single() would. */
static const float* swd_iv_single(const mxArray* a, size_t need, float* buf, size_t cap) {
  if (mxIsSingle(a)) return swd_in_single(a, "input_vector", need);
  const double* d = swd_in_double(a, "input_vector", need);
  size_t n = swd_numel(a) < cap ? swd_numel(a) : cap;
  for (size_t i = 0; i < n; ++i) buf[i] = (float)d[i];
  return buf;
}

/* input_vector as double (the double path builds it in double, staggerfd_eigend.m:70). */
static const double* swd_iv_double(const mxArray* a, size_t need, double* buf, size_t cap) {
  if (mxIsDouble(a)) return swd_in_double(a, "input_vector", need);
  const float* f = swd_in_single(a, "input_vector", need);
  size_t n = swd_numel(a) < cap ? swd_numel(a) : cap;
  for (size_t i = 0; i < n; ++i) buf[i] = (double)f[i];
  return buf;
}

/* Real numeric array (single or double) as doubles: the data itself when it is double,
 * else a converted copy in *owned (mxFree it). */
static const double* swd_as_double(const mxArray* a, const char* what, size_t need, double** owned) {
  *owned = NULL;
  if (mxIsDouble(a)) return swd_in_double(a, what, need);
  const float* f = swd_in_single(a, what, need);
  size_t n = swd_numel(a);
  double* d = (double*)mxMalloc((n ? n : 1) * sizeof(double));
  for (size_t i = 0; i < n; ++i) d[i] = (double)f[i];
  *owned = d;
  return d;
}

/* MATLAB round() of a non-negative ratio (half away from zero). */
static int swd_round(double x) { return (int)(x >= 0 ? (long)(x + 0.5) : -(long)(-x + 0.5)); }

static mxArray* swd_new(mwSize m, mwSize n, mxClassID c) { return mxCreateNumericMatrix(m, n, c, mxREAL); }

#endif
