// WD adjoint source (core/weight_data_muti3.m): a per-trace low-bin filter of the data,
// for batches of (shot, side) gathers.
#pragma once
#include "radon.cuh"

namespace swd {

// Static description of the filter.  `dft` drives the DFT of the kept bins 1..win
// (lf = 2, npair = win, ccn = ntpad = floor(1/dt/df), ntd = nt) with the Radon DFT kernel.
struct WdGeom {
  RadonGeom dft;
  int win;      // bins 1..win are filtered (weight_data_muti3.m:48)
  int ind;      // 1-based bin of the first pick frequency (SWD.m:124)
  int nfre;     // pick frequencies, linspace(fmin, fmax, (fmax-fmin)/df+1) (weight_data_muti3.m:4)
  int npair;    // row stride of the pick arrays (nfre)
  int m, F1;    // F1 = 1: observed-data form of the weights (weight_data_muti3.m:37-38)
  double dg;    // receiver spacing in metres (SWD.m:97)
};

// nt, ng, dt, df, offset, m, win, ind, fmin, fmax, dg, F1 -> geometry; checks nt <= ntpad,
// 2*win < ntpad and 1 <= ind, ind+nfre-1 <= win (the cases the reference's bin loop handles).
int wd_geom(int nt, int ng, double dt, double df, int offset, int m, int win, int ind, double fmin, double fmax,
            double dg, int F1, WdGeom& g);
// 2 pi * linspace(fmin, fmax, nfre) as MATLAB evaluates it.
void wd_fre(double fmin, double fmax, int nfre, double* fre);
// Gather of shot `is` (1-based) and side with refsx = the shot's receiver index (SWD.m:96):
// right columns refsx+m .. min(refsx+m+offset-1, ng), left refsx-m down to max(refsx-offset-m,0)+1;
// the left side runs only for is > round(w/M)+floor(m/M)+1 (weight_data_muti3.m:74).
// valid = -1 marks an active side with an empty window (the reference fails there).
Gather make_wd_gather(const WdGeom& g, int is, int side, int shot_index, int ns, int w, double M, int refsx);

// out[shot][t][col] = seis + (2/ntpad) Re sum_k (fac_k - 1) X_k exp(2 pi i k t / ntpad) for the
// gathers' columns (other columns untouched), X = DFT of the gather's traces at bins 1..win.
// cr0 / crp: [g][npair] observed and predicted picks of gather g; X: [G][win][offset] scratch.
template <typename S, typename O>
int wd_adjoint(const WdGeom& g, const Gather* d_gath, int G, const S* seis, size_t sstride, const double2* W,
               const double* fre, const double* cr0, const double* crp, double2* X, O* out, size_t ostride,
               cudaStream_t st);

}  // namespace swd
