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
  SWD_ERR_CANCELLED = 5,    /* a served request or an engine call was cancelled */
  SWD_ERR_NUMERIC = 6,      /* NaN spectrum column, or interp1 with fewer than two picks */
  SWD_ERR_TIMEOUT = 7       /* swd_server_wait: the request has not finished yet */
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

/* Several eigen_staggerfd_single calls, on grids of any sizes, advanced together: one launch per
 * time step covers the tiles of every job (each CTA finds its job from the jobs' running tile
 * counts and reads that job's geometry, materials, state, source, receivers and snapshot
 * buffer).  It has no counterpart in the reference, where each shot and model is a separate MEX
 * call (core/staggerfd_eigen.m:138-140).  A job is one call's arguments and outputs as for
 * swd_staggerfd_single; its outputs are the same, bit for bit.  Jobs may differ in grid, nt,
 * nt_wf, source and receivers; a job with fewer steps idles after them. */
typedef struct {
  const float* iv;      /* input_vector (16 entries) */
  int n_iv;
  const float *temp, *ca, *cl, *cm, *cm1, *b, *b1; /* nzbc x nxbc */
  const float* s;       /* wavelet, nt */
  float* seismo_u;      /* nt x ng, may be NULL */
  float* seismo_w;      /* nt x ng */
  float *fux, *fuz, *bwx, *bwz; /* nz x nx x nt/nt_wf each, or all NULL */
} swd_staggerfd_job;
int swd_staggerfd_single_batch(int n_jobs, const swd_staggerfd_job* jobs);

/* The adjoint counterpart: several eigen_e2drtm_single calls, on grids of any sizes, advanced
 * together by one launch per time step; each job counts its steps back from its own nt
 * (core/eigen_e2drtm_single.cpp:181) and images on its own nt_wf steps.  No counterpart in the
 * reference.  A job is one call's arguments and outputs as for swd_e2drtm_single; its images
 * are the same, bit for bit. */
typedef struct {
  const float* iv;      /* input_vector (14 entries) */
  int n_iv;
  const float *temp, *ca, *cl, *cm, *cm1, *b, *b1; /* nzbc x nxbc */
  const float* seismo_w;                            /* adjoint source, nt x ng */
  const float *fux, *fuz, *bwx, *bwz;               /* nz x nx x nt/nt_wf each */
  float *cl_img, *cm_img, *illum_div;               /* nz x nx each */
} swd_e2drtm_job;
int swd_e2drtm_single_batch(int n_jobs, const swd_e2drtm_job* jobs);

/* A forward batch whose strain snapshots stay on the device for an adjoint batch of the same
 * jobs, so that they need not go to the host and back (no counterpart in the reference, where
 * the snapshots are MEX outputs and inputs).  swd_staggerfd_single_batch_keep runs the forward
 * as swd_staggerfd_single_batch, recording every job's snapshots on the device even where fux..bwz
 * are NULL (where they are given they are also returned), and fills *kept.
 * swd_e2drtm_single_batch_kept runs the adjoint as swd_e2drtm_single_batch with job j reading
 * forward job j's snapshots in place of its fux..bwz (ignored; job j must have forward job j's
 * nz, nx and nt / nt_wf).  Its images equal those of the adjoint batch given the forward's
 * returned snapshots, bit for bit.  kept may serve several adjoint batches; swd_fd_batch_free
 * releases it. */
typedef struct swd_fd_batch swd_fd_batch;
int swd_staggerfd_single_batch_keep(int n_jobs, const swd_staggerfd_job* jobs, swd_fd_batch** kept);
int swd_e2drtm_single_batch_kept(int n_jobs, const swd_e2drtm_job* jobs, const swd_fd_batch* kept);
void swd_fd_batch_free(swd_fd_batch* kept);

/* Replaces eigen_staggerfd_double (binary-only in the reference; interface at
 * core/staggerfd_eigend.m:139).  Same arguments in double precision. */
int swd_staggerfd_double(const double* iv, int n_iv, const double* temp, const double* ca,
                         const double* cl, const double* cm, const double* cm1, const double* b,
                         const double* b1, const double* s, double* seismo_u, double* seismo_w,
                         double* fux, double* fuz, double* bwx, double* bwz);

/* Replaces eigen_e2drtm_single(iv,temp,ca,cl,cm,cm1,b,b1,seismo_w,fux,fuz,bwx,bwz)
 * (core/eigen_e2drtm_single.cpp:67-296, called at core/e2drtm_eigen.m:122).
 * iv: the 14-entry input_vector of core/e2drtm_eigen.m:121.  seismo_w: nt x ng
 * adjoint source.  Outputs nz x nx.  The images are summed over time steps in FP32, as the
 * reference's single MEX sums them (core/eigen_e2drtm_single.cpp:274-279), and equal its
 * images bit for bit. */
int swd_e2drtm_single(const float* iv, int n_iv, const float* temp, const float* ca,
                      const float* cl, const float* cm, const float* cm1, const float* b,
                      const float* b1, const float* seismo_w, const float* fux, const float* fuz,
                      const float* bwx, const float* bwz, float* cl_img, float* cm_img,
                      float* illum_div);

/* As swd_e2drtm_single, with the images summed over time steps in FP64 and returned unrounded. */
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

/* Padded FD inputs from (vp, vs), as core/staggerfd_eigen.m:37-107 builds them
 * (calparam, pad, damp_circle, free-surface row edits), computed on the GPU.
 * vp, vs: nz x nx (double).  Outputs: nzbc x nxbc with nzbc = nz+pad_top+nbc,
 * nxbc = nx+2*nbc, pad_top = (fd_order-20)/2+1.  isfs must be 1. */
int swd_prep_model_single(int nz, int nx, int nbc, int isfs, int fd_order, double dx, double dt, double dtx,
                          const double* vp, const double* vs, float* temp, float* ca, float* cl, float* cm,
                          float* cm1, float* b, float* b1);
int swd_prep_model_double(int nz, int nx, int nbc, int isfs, int fd_order, double dx, double dt, double dtx,
                          const double* vp, const double* vs, double* temp, double* ca, double* cl, double* cm,
                          double* cm1, double* b, double* b1);

/* ------------------------------------------------------------------------
 * Dispersion spectrum, picking and SoftMax gradient (host pointers).
 * ------------------------------------------------------------------------ */

/* Arguments shared by RTr/RTl/RTrAD/RTlAD (core/RTrAD.m:2) and ADWDgrad_1. */
typedef struct {
  double df, dt;       /* frequency step, time step */
  double fmin, fmax;   /* kept band: bins round(fmin/df)+1 .. round(fmax/df)+1 */
  double vmin, vmax;   /* phase-velocity axis vmin:dv:vmax */
  double dv;           /* 1 in the reference (pp=1./(vmin:vmax)') */
  double ds;           /* trace spacing in metres */
  int nt, ng;          /* seismogram size (a, b) */
  int offset, m, M;    /* window length, minimum offset, shot spacing in traces */
  int precision;       /* SWD_PREC_*; the per-shot entry points compute in FP64 */
} swd_radon_params;

/* np (velocities), npair (kept bins), lf, nf and ccn = fix(1/df/dt) for p. */
int swd_radon_sizes(const swd_radon_params* p, int* np, int* npair, int* lf, int* nf, int* ccn);

/* Replaces RTrAD (side 0, core/RTrAD.m:2-35) and RTlAD (side 1, core/RTlAD.m:2-36);
 * ml is also the output of RTr/RTl (core/RTr.m:2-32, core/RTl.m:2-32).
 * seismo: nt x ng.  ml, ml_raw: np x npair (ml_raw = saveForBackward.mlr/mll).
 * mm: np x nf complex, interleaved re/im (saveForBackward.mm).  uxtpos: data_len
 * 1-based trace columns, ascending (uxtposr/uxtposl).  ml_raw, mm, data_len and
 * uxtpos may be NULL. */
int swd_radon(const swd_radon_params* p, int side, int is, const double* seismo, double* ml, double* ml_raw,
              double* mm, int* data_len, int* uxtpos);

/* Replaces LHDispPick(ml,vmin,cr_0,method,ini) (core/LHDispPick.m:2-13) with the
 * guided picker pickFDC1(ml,ini,2,4) (core/pickFDC1.m:1-131) for method 1.
 * ml: np x npair; cr_0, cr_pre: npair; res: scalar misfit (may be NULL). */
int swd_pick(const double* ml, int np, int npair, double vmin, const double* cr_0, int method, int ini,
             double* res, double* cr_pre);

/* Allocation-free variant of swd_pick; it has no counterpart in the reference.
 * For callers that cannot allocate device memory: it calls no cudaMalloc, cudaFree or other
 * allocating routine.  All arrays are caller-owned DEVICE memory: d_ml np x npair, d_cr_0 and
 * d_cr_pre npair, d_res one double (may be NULL).  stream is a cudaStream_t (NULL: the legacy
 * default stream); the call synchronises it to read the pick status.  The scratch lives in one
 * static device array of libswd.so (16 KiB, held by every GPU that loads the library until the
 * process exits), which limits npair to SWD_PICK_NOALLOC_MAX_NPAIR.  The first call on a device
 * looks up the array's device address; make that call before any stream capture.  Later calls
 * outside a capture look it up again, so a cudaDeviceReset leaves no stale address.  Every call
 * shares the array: calls that overlap on the GPU race. */
#define SWD_PICK_NOALLOC_MAX_NPAIR 2047
int swd_pick_noalloc(const double* d_ml, int np, int npair, double vmin, const double* d_cr_0, int method,
                     int ini, double* d_res, double* d_cr_pre, void* stream);

/* Replaces ADWDgrad_1(nt,ng,ns,npair,is,w,m,M,SoftArgNorm,grad_outputr,grad_outputl,
 * space_M,saveForBackwardr,saveForBackwardl) (core/ADWDgrad_1.m:1-81).
 * grad_output_*: npair; space_m: np x npair (NULL = 1..np per column, SWD.m:133-136);
 * mm_*: np x nf interleaved complex; ml_raw_*: np x npair; a side the reference
 * skips for this shot may pass NULLs.  a_data_res: nt x ng (out). */
int swd_adwdgrad(const swd_radon_params* p, int ns, int is, int w, double soft_arg_norm,
                 const double* grad_output_r, const double* grad_output_l, const double* space_m,
                 const double* mm_r, const double* ml_raw_r, const double* mm_l, const double* ml_raw_l,
                 double* a_data_res);

/* Replaces ADWDgradlimband(...) (core/ADWDgradlimband.m:1-102, same arguments as ADWDgrad_1):
 * the weights are mlr.^SoftArgNorm normalised by their column sum (its derivative weights
 * SoftArgNorm*(mlr.^SoftArgNorm).^(SoftArgNorm-1) over the same sum), without the SoftArgNorm
 * factor of ADWDgrad_1, and the adjoint spectrum is extended by linear ramps over the 25 bins
 * below lf and above nf.  Needs lf >= 26.  The reference has no caller for it; with
 * SoftArgNorm = 1e4 (SWD.m:114) mlr.^SoftArgNorm overflows there as it does here. */
int swd_adwdgrad_limband(const swd_radon_params* p, int ns, int is, int w, double soft_arg_norm,
                         const double* grad_output_r, const double* grad_output_l, const double* space_m,
                         const double* mm_r, const double* ml_raw_r, const double* mm_l, const double* ml_raw_l,
                         double* a_data_res);

/* ---- field-data variants (fieldexamples/outcrop, fieldexamples/QadimahFault) ---- */

/* Replaces the field-data LHDispPick variants, which start the guided pick at the global
 * maximum of the unnormalised spectrum ml_raw (saveForBackward.mlr / .mll):
 *   variant 1: fieldexamples/outcrop/core/LHDispPick.m:2-25 -> pickFDCValue(ml,ini,iniP,2,4)
 *              (fieldexamples/outcrop/core/pickFDCValue.m:1-131) for method 1, argmax picks
 *              otherwise; misfit over rows 15..npair-15;
 *   variant 2: fieldexamples/QadimahFault/core/LHDispPick.m:2-41 (its mode 1) -> pickFDC1(ml,ini,
 *              2,4) for any method; misfit over rows 50..npair-30 (NaN when that range is empty).
 * ini = the first column holding the maximum of ml_raw, iniP = its first row of that value.
 * ml, ml_raw: np x npair; cr_0, cr_pre: npair; res: scalar (may be NULL). */
int swd_pick_field(const double* ml, const double* ml_raw, int np, int npair, double vmin, const double* cr_0,
                   int method, int variant, double* res, double* cr_pre);

/* Replaces fieldexamples/outcrop/core/ADWDgrad_1.m:1-81 (same arguments as ADWDgrad_1): the
 * adjoint source divided by its largest magnitude (:79). */
int swd_adwdgrad_maxnorm(const swd_radon_params* p, int ns, int is, int w, double soft_arg_norm,
                         const double* grad_output_r, const double* grad_output_l, const double* space_m,
                         const double* mm_r, const double* ml_raw_r, const double* mm_l, const double* ml_raw_l,
                         double* a_data_res);

/* Replaces norm_trace(data_in) (core/norm_trace.m:1-22; fieldexamples/outcrop/outcrop.m:174 applies
 * it to every predicted gather): each column of the nt x ng array divided by its largest
 * magnitude (an all-zero trace becomes NaN, 0/0, as in the reference). */
int swd_norm_trace(const double* data_in, int nt, int ng, double* data_out);

/* Replaces [dfk]=fk_filter(d,dt,dx) (core/fk_filter.m:1-302; the same file in the
 * fieldexamples drivers' core folders): the dip filter that the field drivers apply to a gather before the
 * Radon transform when FK == 1 (fieldexamples/QadimahFault/core/RTrAD.m:14-16, RTlAD.m:15-17).
 * d, dfk: ns x ntr (column-major, host).  The gather is zero-padded to 2ns x 2ntr; of its f-k
 * spectrum the quadrants with frequency and wavenumber of the same sign (in fftshift order) are
 * removed; the result is the leading ns x ntr block of the real part.  dt and dx only set axes
 * that fk_filter.m computes and never uses; they are accepted for the same call. */
int swd_fk_filter(const double* d, int ns, int ntr, double dt, double dx, double* dfk);

/* Replaces ADWDgrad_norm(...) (core/ADWDgrad_norm.m:1-102, same arguments as ADWDgrad_1):
 * the SoftMax weights are replaced by normpdf(1:np, cr, 16) around the picks
 * (core/paddingMl_norm.m:1-9).  cr_r / cr_l: npair, saveForBackward.cr_r / cr_l = cr_pre - vmin
 * (SWD.m:178, 184). */
int swd_adwdgrad_norm(const swd_radon_params* p, int ns, int is, int w, double soft_arg_norm,
                      const double* grad_output_r, const double* grad_output_l, const double* space_m,
                      const double* mm_r, const double* ml_raw_r, const double* cr_r, const double* mm_l,
                      const double* ml_raw_l, const double* cr_l, double* a_data_res);

/* Replaces weight_data_muti3(seismo_v_d,seismo_v,is,dt,df,offset,dg,F1,w,M,m,ns,refsx,win,
 * fmin,fmax,cr_0,cr_0l,cr_pre_r,cr_pre_l,ind) (core/weight_data_muti3.m:1-122), the WD adjoint
 * source of SWD.m:188.  seismo_v_d / seismo_v: nt x ng (F1 = 1 reads seismo_v_d, F1 = 0
 * seismo_v; the other may be NULL); refsx: ns receiver indices floor(sx/dg)+1 (SWD.m:96);
 * dg: receiver spacing in metres; cr_*: npair = floor((fmax-fmin)/df+1) picks (a side the
 * reference skips may pass NULL).  Needs nt <= floor(1/dt/df), 2*win < floor(1/dt/df) and
 * ind+npair-1 <= win (SWD.m:124-127 gives win = npair+2*ind).  seismo_v_d1: nt x ng (out). */
int swd_wd_residual(int nt, int ng, const double* seismo_v_d, const double* seismo_v, int is, double dt, double df,
                    int offset, double dg, int F1, int w, double M, int m, int ns, const double* refsx, int win,
                    double fmin, double fmax, const double* cr_0, const double* cr_0l, const double* cr_pre_r,
                    const double* cr_pre_l, int ind, double* seismo_v_d1);

/* ------------------------------------------------------------------------
 * Batched gradient engine: the per-iteration shot loops of SWD.m run as one
 * batched GPU pipeline (replaces the parfor loops SWD.m:155-162 observed curves,
 * SWD.m:171-201 gradient, SWD.m:215-304 forward-only misfits).
 * ------------------------------------------------------------------------ */

typedef struct swd_engine swd_engine;

/* Survey of one inversion (the top-of-file variables of SWD.m:73-116).
 * Positions are the reference's 1-based model coordinates. */
typedef struct {
  int nz, nx, nbc, nt, nt_wf, fd_order, isfs, source_type; /* source_type 1..5 ('w' = 5) */
  double dx, dt;
  int ns;
  const int* sx; /* ns shot columns */
  const int* sz; /* ns shot rows */
  int ng, gx0, dgx, gz; /* receivers gx0, gx0+dgx, ... on row gz */
  double df, fmin, fmax, vmin, vmax, dv; /* Radon axes (dv = 1 in the reference) */
  int offset, m, M, w, ini, pick_method;
  double soft_arg_norm;  /* SoftArgNorm, 1e4 in SWD.m:114 */
  int smooth_z, smooth_x;
  /* Shots of a larger survey (one rank's share of the parfor of SWD.m:171): shot_no holds the
   * 1-based shot numbers `is` of these ns shots in that survey and ns_total its shot count; both
   * set the Radon windows and the side rules (RTrAD.m:4-9, ADWDgrad_1.m:15,47).
   * shot_no NULL: 1..ns.  ns_total 0: ns. */
  const int* shot_no;
  int ns_total;
} swd_survey;

typedef struct {
  size_t hbm_budget;  /* bytes the engine may allocate (0: 92% of free memory) */
  int max_batch;      /* shots per batch (0: as many as fit) */
  int snapshot_mode;  /* 0 auto, 1 keep every strain snapshot, 2 checkpoint + recompute */
  int ckpt_interval;  /* steps between forward checkpoints (mode 2; rounded to nt_wf; 0: the
                         interval that minimises checkpoint + snapshot memory per shot) */
  int use_graphs;     /* capture the time loops in CUDA graphs */
  int chunk_rows;     /* rows per CTA in the FD kernels (0: heuristic; at most 60 for the warp
                         schedules 0, 2, 3 and 5) */
  int device;
  int warps, cells;   /* FD kernels: warps per CTA and output columns per thread; (w,c) in
                         (1,2), (1,3), (2,1), (3,1), (4,1); others: (3,1) */
  int ring_fwd, ring_adj; /* rows in the forward / adjoint shared-memory ring: 4, 6 or 8 (6 at most
                             for (1,3)); anything else: 4 */
  int autotune;       /* 1: at create, time the FD step kernels of each schedule, CTA shape, ring
                         depth and chunk height on this survey's buffers and keep the fastest
                         (overrides warps, cells, ring_*, chunk_rows, fd_schedule) */
  int radon_precision; /* forward Radon contraction: SWD_PREC_FP64 (0, default, as the reference)
                          or SWD_PREC_BF16X2 / _BF16X3 (tcgen05 split-BF16, see swd_contract_*) */
  int fd_schedule;    /* FD kernels, all giving the same bits: 0 (default) or 3 warp streaming
                         with two time steps per launch, 2 warp streaming with one step per launch
                         (both: warps = 2, 4 or 8 per CTA, ring_* = 4, 6 or 8 staged rows), 1 one
                         CTA barrier per row with the velocities a row ahead (shapes (2,1), (3,1),
                         (4,1) ring 4, (3,1) ring 6), 4 two CTA barriers per row (shared-memory
                         ring; the shapes of warps/cells/ring_*), 5 as 3 with two shots per warp
                         in packed FP32 pairs (warps = 2 or 4, ring_* = 4 or 6) */
  int adjoint_weight; /* adjoint source: 0 ADWDgrad_1 (SoftMax weights, SWD.m:190), 1 ADWDgrad_norm
                         (Gaussian weights around the picks, core/ADWDgrad_norm.m), 2 the WD residual
                         weight_data_muti3 with F1 = 0 (SWD.m:188; ind = fmin/df+1, win = npair+2*ind,
                         refsx = floor(sx/dgx)+1, dg = dgx*dx as SWD.m:96-97,124-127 set them) */
  int image_precision; /* per-shot imaging sums: 0 (default) FP32, as the reference's single MEX
                          accumulates them (core/eigen_e2drtm_single.cpp:274-279), 1 FP64; the
                          sum over shots is FP64 in shot order either way */
} swd_engine_opts;

typedef struct {
  int batch, nbatch, mode, ckpt_interval;
  size_t bytes;
  int npair, np, ccn, nzbc, nxbc, chunk_rows, warps, cells, ring_fwd, ring_adj;
  double tuned_fwd_us, tuned_adj_us; /* autotune: the chosen variants' step times (0 if not tuned) */
  int fd_schedule;
} swd_engine_info_t;

/* Gradient outputs (host pointers, nz x nx column-major; NULL entries skipped). */
typedef struct {
  double* g_cl;      /* sum over shots of cl_img (SWD.m:193) */
  double* g_cm;      /* sum over shots of cm_img */
  double* g_illum;   /* sum over shots of illum_div */
  double* dk_vs;     /* smooth2a(-4 vs g_cl/g_illum + 2 vs g_cm/g_illum) (SWD.m:199-201) */
  double* res_r;     /* ns: right-side misfits (NaN where skipped) */
  double* res_l;     /* ns: left-side misfits */
  double* cr_pre_r;  /* npair x ns predicted picks */
  double* cr_pre_l;
  double residual;   /* mean(res_r) over the right-side shots (SWD.m:196) */
} swd_gradient_out;

int swd_engine_create(const swd_survey* survey, const swd_engine_opts* opts, swd_engine** out);
int swd_engine_destroy(swd_engine* e);
/* The plan swd_engine_create would make for (s, o): batch, mode and device bytes, without
 * allocating anything (o->hbm_budget 0 plans against the device's free memory). */
int swd_engine_plan(const swd_survey* s, const swd_engine_opts* o, swd_engine_info_t* info);
int swd_engine_info(const swd_engine* e, swd_engine_info_t* info);
/* Source wavelet s (nt samples), rounded to float as SWD_single.m:92 does. */
int swd_engine_set_source(swd_engine* e, const double* s);
/* Observed picks cr_0 / cr_0l (npair x ns), as SWD.m:155-162 computes them. */
int swd_engine_set_observed(swd_engine* e, const double* cr0_r, const double* cr0_l);
/* Observed curves of a model (SWD.m:155-162): forward, RTr/RTl, LHDispPick. */
int swd_engine_observed_curves(swd_engine* e, const double* vp, const double* vs, double* cr0_r, double* cr0_l);
/* Forward-only misfits of a model (the line-search passes, SWD.m:215-228). */
int swd_engine_misfit(swd_engine* e, const double* vp, const double* vs, double* res_r, double* res_l,
                      double* cr_pre_r, double* cr_pre_l, double* residual);
/* One gradient of SWD.m:171-201 for model (vp, vs) (host pointers, nz x nx). */
int swd_engine_gradient(swd_engine* e, const double* vp, const double* vs, swd_gradient_out* out);
/* As swd_engine_gradient with device-resident vp, vs and dk_vs (device pointers). */
int swd_engine_gradient_device(swd_engine* e, const double* d_vp, const double* d_vs, double* d_dk_vs,
                               double* residual);
/* The engine's CUDA stream (a cudaStream_t). */
/* Cancel the engine's call in flight (callable from any host thread; returns at once).  The
 * call's remaining FD launches return as soon as they start, and the call returns
 * SWD_ERR_CANCELLED without results; the engine is ready for the next call.  A cancel raised
 * while no call runs cancels the next call.  No counterpart in the reference (its parfor has no
 * cancellation). */
int swd_engine_cancel(swd_engine* e);
/* Withdraw a cancel that no call has taken yet (e.g. one that arrived after its call finished),
 * so that it does not cancel the next call.  No counterpart in the reference. */
int swd_engine_cancel_clear(swd_engine* e);
/* With radon_precision SWD_PREC_BF16X2 / _BF16X3 the spectra come from the tensor cores and the
 * picker certifies each gather: a gather with any pick decision whose compared spectrum values
 * differ by less than 1e-4 (of the column maximum) is recomputed in FP64 and picked again, so the
 * picks are those of the FP64 spectrum.  gathers: gathers picked so far; recomputed: how many of
 * them were recomputed.  No counterpart in the reference. */
int swd_engine_radon_stats(swd_engine* e, uint64_t* gathers, uint64_t* recomputed);
int swd_engine_stream(const swd_engine* e, void** stream);
/* Split form of the gradient for several GPUs (shots sharded across ranks; the
 * parfor sum of SWD.m:193 becomes one all-reduce): the shot sums g_cl, g_cm,
 * g_illum of this engine's shots go to d_gsum (3*nz*nx doubles, opaque layout)
 * with the right-side misfit sum and count; after the caller has summed d_gsum
 * over ranks, swd_engine_assemble_device forms dk_vs (SWD.m:199-201). */
int swd_engine_shot_sums_device(swd_engine* e, const double* d_vp, const double* d_vs, double* d_gsum,
                                double* res_sum, int* res_count);
int swd_engine_assemble_device(swd_engine* e, const double* d_gsum, double* d_dk_vs);
/* Per-phase CUDA-event timing of later calls (forward, spectra+picks+adjoint
 * sources, adjoint+imaging), summed over batches, in milliseconds. */
int swd_engine_set_timing(swd_engine* e, int on);
int swd_engine_phase_times(const swd_engine* e, double* fwd_ms, double* spec_ms, double* adj_ms);

/* ------------------------------------------------------------------------
 * Batched Radon contraction with general axes (the slant stack of RTrAD.m:20-26
 * for many shots at once): mm[s][f][p] = sum_x exp(i*2*pi*freq[f]*offset[x]/vel[p])
 * * spec[s][f][x].  spec and mm are DEVICE arrays of interleaved complex doubles,
 * [ns][nf][nx] and [ns][nf][np].  precision: SWD_PREC_FP64 / _FP32 (CUDA cores)
 * or _BF16X2 / _BF16X3 (tcgen05 tensor cores, split-BF16 operands, FP32 accumulate).
 * The kernel table is built once at create time.
 * ------------------------------------------------------------------------ */

typedef struct swd_contract swd_contract;

int swd_contract_create(int nf, const double* freq, int np, const double* vel, int nx, const double* offset,
                        int ns, int precision, int device, swd_contract** out);
/* Enqueue one contraction on `stream` (a cudaStream_t; NULL: legacy default stream). */
int swd_contract_run(swd_contract* c, const double* d_spec, double* d_mm, void* stream);
/* 1 in *timed_out when a tensor-core launch gave up waiting on its MMAs (results invalid). */
int swd_contract_status(swd_contract* c, int* timed_out);
/* Useful FLOPs (8 per complex multiply-add) and the FLOPs the tensor cores execute
 * (padded tiles x split products; equal to useful on CUDA cores). */
int swd_contract_flops(const swd_contract* c, double* useful, double* issued);
int swd_contract_destroy(swd_contract* c);

/* ------------------------------------------------------------------------
 * Served request loop (one GPU): misfit and gradient requests of any survey size
 * are admitted in arrival order by the HBM footprint of their engines and run
 * concurrently, each on its own stream.  Engines stay resident between requests
 * with the same nonzero survey_key (device memory, Radon tables, checkpoint
 * buffers and captured time loops are reused).  No counterpart in the reference,
 * whose SWD.m runs one inversion at a time.
 * ------------------------------------------------------------------------ */

typedef struct swd_server swd_server;

enum { SWD_REQ_GRADIENT = 0, SWD_REQ_MISFIT = 1 };

typedef struct {
  size_t hbm_budget; /* bytes all engines together may hold (0: 85% of free memory) */
  int max_inflight;  /* requests on the GPU at once (0: 4); each may plan up to budget/max_inflight */
  int device;
  int keep_engines;  /* keep finished engines resident for their survey_key */
} swd_server_opts;

typedef struct {
  const swd_survey* survey; /* copied at submit */
  uint64_t survey_key;      /* nonzero: reuse a resident engine of the same key and survey */
  int kind;                 /* SWD_REQ_GRADIENT or SWD_REQ_MISFIT */
  int npair;                /* kept frequency bins (rows of cr0_r / cr0_l) */
  const double* wavelet;    /* nt samples */
  const double* vp;         /* nz x nx, column-major */
  const double* vs;
  const double* cr0_r;      /* npair x ns observed curves */
  const double* cr0_l;
} swd_request;

typedef struct {
  int status;               /* the request's own SWD_* status */
  double residual;          /* mean right-side misfit (SWD.m:196) */
  double queue_ms, run_ms, total_ms; /* submit -> start -> done */
  int reused_engine;        /* 1 when a resident engine served it */
  size_t engine_bytes;
  double* dk_vs;            /* outputs, caller buffers (NULL skipped): nz x nx (gradient only) */
  double* res_r;            /* ns */
  double* res_l;            /* ns */
  double* cr_pre_r;         /* npair x ns */
  double* cr_pre_l;         /* npair x ns */
} swd_request_result;

typedef struct {
  uint64_t submitted, admitted, completed, cancelled, waits_for_memory;
  int peak_inflight, idle_engines;
  size_t peak_bytes, bytes_in_use, budget;
} swd_server_stats_t;

int swd_server_create(const swd_server_opts* opts, swd_server** out);
/* Queue a request (inputs are copied); *id names it for swd_server_wait / _cancel. */
int swd_server_submit(swd_server* s, const swd_request* req, uint64_t* id);
/* Wait up to timeout_ms (< 0: forever) for request id; copies its outputs into out's buffers
 * and releases it.  SWD_ERR_TIMEOUT leaves it pending; otherwise returns its status. */
int swd_server_wait(swd_server* s, uint64_t id, int timeout_ms, swd_request_result* out);
/* Cancel a request: one still queued never starts; one already running has its engine's call
 * cancelled (swd_engine_cancel).  Either way its wait returns SWD_ERR_CANCELLED.  A request that
 * has finished cannot be cancelled (SWD_ERR_INVALID). */
int swd_server_cancel(swd_server* s, uint64_t id);
int swd_server_stats(swd_server* s, swd_server_stats_t* out);
/* Cancel queued requests, wait for running ones, free every engine. */
int swd_server_destroy(swd_server* s);

#ifdef __cplusplus
}
#endif
#endif /* SWD_H */
