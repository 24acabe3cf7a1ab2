/*
 * swd.h -- C ABI of the B200-native SWD gradient hot path (libswd.so).
 *
 * Every entry point takes plain pointers and sizes, returns an SWD_* status
 * code, and records a message for swd_last_error() on failure.  Host-pointer
 * entry points use MATLAB's column-major layout so that a C MEX shim can pass
 * mxArray data straight through; they allocate their own device memory.
 * Each declaration names the reference interface it replaces (paths are
 * relative to the zhangchang271/SWD tree).
 */
#ifndef SWD_H
#define SWD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SWD_OK = 0,
  SWD_ERR_INVALID = 1,      /* bad argument; see swd_last_error() */
  SWD_ERR_UNSUPPORTED = 2,  /* accepted by the reference, not built here (fd_order 24/26/28) */
  SWD_ERR_CUDA = 3,         /* CUDA runtime error */
  SWD_ERR_OOM = 4,          /* device allocation failed or over the HBM budget */
  SWD_ERR_CANCELLED = 5,    /* a served request was cancelled */
  SWD_ERR_NUMERIC = 6       /* NaN spectrum column, or interp1 with fewer than two picks */
};

/* Precision of the Radon transform (DFT + contraction). */
enum {
  SWD_PREC_FP64 = 0,   /* double, like the reference's MATLAB .m path */
  SWD_PREC_FP32 = 1,   /* float CUDA cores */
  SWD_PREC_BF16X2 = 2, /* tcgen05 tensor cores, split-BF16 hi+lo, FP32 accumulate */
  SWD_PREC_BF16X3 = 3  /* tcgen05 tensor cores, split-BF16 hi+mid+lo, FP32 accumulate */
};

/* Message of the last failed call on this thread ("" if none). */
const char* swd_last_error(void);
/* Library version, major*10000 + minor*100 + patch. */
int swd_version(void);
/* Number of this library's kernels launched so far in this process. */
uint64_t swd_kernel_launches(void);

/* ------------------------------------------------------------------------
 * FD kernels, MEX calling convention (host pointers, MATLAB column-major).
 * ------------------------------------------------------------------------ */

/* Replaces eigen_staggerfd_single(iv,temp,ca,cl,cm,cm1,b,b1,s)
 * (core/eigen_staggerfd_single.cpp:68-383, called at core/staggerfd_eigen.m:139).
 * iv: the 16-entry input_vector of core/staggerfd_eigen.m:138.
 * temp..b1: nzbc x nxbc.  s: nt.  seismo_u, seismo_w: nt x ng (out).
 * fux..bwz: nz x nx x (nt/nt_wf) strain snapshots (out; all four NULL = not kept).
 * fd_order must be 22 (the only order SWD.m uses); nt must be a multiple of nt_wf. */
int swd_staggerfd_single(const float* iv, int n_iv, const float* temp, const float* ca,
                         const float* cl, const float* cm, const float* cm1, const float* b,
                         const float* b1, const float* s, float* seismo_u, float* seismo_w,
                         float* fux, float* fuz, float* bwx, float* bwz);

/* Replaces eigen_staggerfd_double (binary-only in the reference; interface at
 * core/staggerfd_eigend.m:139).  Same arguments in double precision. */
int swd_staggerfd_double(const double* iv, int n_iv, const double* temp, const double* ca,
                         const double* cl, const double* cm, const double* cm1, const double* b,
                         const double* b1, const double* s, double* seismo_u, double* seismo_w,
                         double* fux, double* fuz, double* bwx, double* bwz);

/* Replaces eigen_e2drtm_single(iv,temp,ca,cl,cm,cm1,b,b1,seismo_w,fux,fuz,bwx,bwz)
 * (core/eigen_e2drtm_single.cpp:67-296, called at core/e2drtm_eigen.m:122).
 * iv: the 14-entry input_vector of core/e2drtm_eigen.m:121.  seismo_w: nt x ng
 * adjoint source.  Outputs nz x nx.  The images accumulate in FP64 on the GPU and
 * are rounded to float on return (the reference accumulates in float). */
int swd_e2drtm_single(const float* iv, int n_iv, const float* temp, const float* ca,
                      const float* cl, const float* cm, const float* cm1, const float* b,
                      const float* b1, const float* seismo_w, const float* fux, const float* fuz,
                      const float* bwx, const float* bwz, float* cl_img, float* cm_img,
                      float* illum_div);

/* As swd_e2drtm_single, returning the FP64 accumulators unrounded. */
int swd_e2drtm_single_f64out(const float* iv, int n_iv, const float* temp, const float* ca,
                             const float* cl, const float* cm, const float* cm1, const float* b,
                             const float* b1, const float* seismo_w, const float* fux,
                             const float* fuz, const float* bwx, const float* bwz,
                             double* cl_img, double* cm_img, double* illum_div);

/* Replaces eigen_e2drtm_double (binary-only; interface at core/e2drtm_eigend.m:122). */
int swd_e2drtm_double(const double* iv, int n_iv, const double* temp, const double* ca,
                      const double* cl, const double* cm, const double* cm1, const double* b,
                      const double* b1, const double* seismo_w, const double* fux,
                      const double* fuz, const double* bwx, const double* bwz, double* cl_img,
                      double* cm_img, double* illum_div);

#ifdef __cplusplus
}
#endif
#endif /* SWD_H */
