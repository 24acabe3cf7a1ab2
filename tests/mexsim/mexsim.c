/* Implementation of the MEX API stand-in in mex.h plus the sim_* calls the tests use. */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

#define MAXF 16
struct mxArray_tag {
  mxClassID cls;
  int cplx;
  size_t nd, dims[8], n, esz;
  void *re, *im;
  int nf;
  char* fname[MAXF];
  mxArray* fval[MAXF];
  mxArray** cells; /* cell arrays: n elements (NULL = empty) */
};

static jmp_buf g_jmp;
static int g_in_call = 0;
static char g_err[1024];

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int k = snprintf(g_err, sizeof(g_err), "%s: ", id);
  vsnprintf(g_err + k, sizeof(g_err) - k, fmt, ap);
  va_end(ap);
  if (g_in_call) longjmp(g_jmp, 1);
  fprintf(stderr, "%s\n", g_err);
  abort();
}

static size_t esz_of(mxClassID c) { return c == mxDOUBLE_CLASS ? 8 : (c == mxSINGLE_CLASS || c == mxINT32_CLASS) ? 4 : 0; }

static mxArray* make(mxClassID c, mwSize nd, const mwSize* dims, int cplx) {
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = c;
  a->cplx = cplx;
  a->nd = nd < 2 ? 2 : nd;
  a->dims[0] = a->dims[1] = 1;
  a->n = 1;
  for (size_t i = 0; i < nd; ++i) { a->dims[i] = dims[i]; a->n *= dims[i]; }
  a->esz = esz_of(c);
  if (c == mxCELL_CLASS) a->cells = (mxArray**)calloc(a->n ? a->n : 1, sizeof(mxArray*));
  if (a->esz) {
    a->re = calloc(a->n ? a->n : 1, a->esz);
    if (cplx) a->im = calloc(a->n ? a->n : 1, a->esz);
  }
  return a;
}

size_t mxGetNumberOfElements(const mxArray* a) { return a->n; }
size_t mxGetM(const mxArray* a) { return a->dims[0]; }
size_t mxGetN(const mxArray* a) { size_t n = 1; for (size_t i = 1; i < a->nd; ++i) n *= a->dims[i]; return n; }
int mxIsSingle(const mxArray* a) { return a->cls == mxSINGLE_CLASS; }
int mxIsDouble(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }
int mxIsComplex(const mxArray* a) { return a->cplx; }
int mxIsStruct(const mxArray* a) { return a->cls == mxSTRUCT_CLASS; }
int mxIsCell(const mxArray* a) { return a->cls == mxCELL_CLASS; }
mxArray* mxGetCell(const mxArray* a, mwSize i) { return a->cls == mxCELL_CLASS && i < a->n ? a->cells[i] : NULL; }
void mxSetCell(mxArray* a, mwSize i, mxArray* v) {
  if (a->cls == mxCELL_CLASS && i < a->n) { mxDestroyArray(a->cells[i]); a->cells[i] = v; }
}
mxArray* mxCreateCellMatrix(mwSize m, mwSize n) {
  mwSize d[2] = {m, n};
  return make(mxCELL_CLASS, 2, d, 0);
}
void* mxGetData(const mxArray* a) { return a->re; }
double* mxGetPr(const mxArray* a) { return a->cls == mxDOUBLE_CLASS ? (double*)a->re : NULL; }
double* mxGetPi(const mxArray* a) { return a->cls == mxDOUBLE_CLASS ? (double*)a->im : NULL; }
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x) {
  mwSize d[2] = {m, n};
  return make(c, 2, d, x == mxCOMPLEX);
}
mxArray* mxCreateNumericArray(mwSize nd, const mwSize* dims, mxClassID c, mxComplexity x) {
  return make(c, nd, dims, x == mxCOMPLEX);
}
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity x) { return mxCreateNumericMatrix(m, n, mxDOUBLE_CLASS, x); }
mxArray* mxCreateDoubleScalar(double v) {
  mxArray* a = mxCreateDoubleMatrix(1, 1, mxREAL);
  ((double*)a->re)[0] = v;
  return a;
}
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names) {
  mwSize d[2] = {m, n};
  mxArray* a = make(mxSTRUCT_CLASS, 2, d, 0);
  for (int i = 0; i < nfields && i < MAXF; ++i) a->fname[a->nf++] = strdup(names[i]);
  return a;
}
void mxSetField(mxArray* s, mwSize i, const char* name, mxArray* v) {
  (void)i;
  for (int k = 0; k < s->nf; ++k)
    if (!strcmp(s->fname[k], name)) { s->fval[k] = v; return; }
  if (s->nf < MAXF) { s->fname[s->nf] = strdup(name); s->fval[s->nf++] = v; }
}
mxArray* mxGetField(const mxArray* s, mwSize i, const char* name) {
  (void)i;
  for (int k = 0; k < s->nf; ++k)
    if (!strcmp(s->fname[k], name)) return s->fval[k];
  return NULL;
}
void mxDestroyArray(mxArray* a) {
  if (!a) return;
  for (int k = 0; k < a->nf; ++k) { free(a->fname[k]); mxDestroyArray(a->fval[k]); }
  if (a->cells) {
    for (size_t i = 0; i < a->n; ++i) mxDestroyArray(a->cells[i]);
    free(a->cells);
  }
  free(a->re);
  free(a->im);
  free(a);
}
void* mxMalloc(size_t n) { return malloc(n ? n : 1); }
void mxFree(void* p) { free(p); }

/* ---- calls used by the Python side ---- */
mxArray* sim_numeric(int cls, int nd, const size_t* dims, const void* re, const void* im) {
  mxArray* a = make((mxClassID)cls, (mwSize)nd, dims, im != NULL);
  if (re) memcpy(a->re, re, a->n * a->esz);
  if (im) memcpy(a->im, im, a->n * a->esz);
  return a;
}
mxArray* sim_struct(void) { return mxCreateStructMatrix(1, 1, 0, NULL); }
void sim_set_field(mxArray* s, const char* name, mxArray* v) { mxSetField(s, 0, name, v); }
int sim_class(const mxArray* a) { return (int)a->cls; }
int sim_complex(const mxArray* a) { return a->cplx; }
int sim_ndim(const mxArray* a) { return (int)a->nd; }
size_t sim_dim(const mxArray* a, int i) { return a->dims[i]; }
void* sim_re(const mxArray* a) { return a->re; }
void* sim_im(const mxArray* a) { return a->im; }
int sim_nfields(const mxArray* a) { return a->nf; }
const char* sim_field_name(const mxArray* a, int k) { return a->fname[k]; }
mxArray* sim_field_value(const mxArray* a, int k) { return a->fval[k]; }
void sim_destroy(mxArray* a) { mxDestroyArray(a); }
mxArray* sim_cell(size_t n) { return mxCreateCellMatrix(1, n); }
void sim_set_cell(mxArray* a, size_t i, mxArray* v) { mxSetCell(a, i, v); }
mxArray* sim_get_cell(const mxArray* a, size_t i) { return mxGetCell(a, i); }
size_t sim_numel(const mxArray* a) { return a->n; }
const char* sim_error(void) { return g_err; }

/* Run mexFunction; 0 on success, 1 if it raised an error (message in sim_error()). */
int sim_call(int nlhs, mxArray** plhs, int nrhs, mxArray** prhs) {
  g_err[0] = 0;
  for (int i = 0; i < nlhs; ++i) plhs[i] = NULL;
  g_in_call = 1;
  if (setjmp(g_jmp)) { g_in_call = 0; return 1; }
  mexFunction(nlhs, plhs, nrhs, (const mxArray**)prhs);
  g_in_call = 0;
  return 0;
}
