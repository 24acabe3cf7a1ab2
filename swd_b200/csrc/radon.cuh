// Linear Radon dispersion transform, guided picker and SoftMax misfit gradient
// for batches of (shot, side) gathers.
#pragma once
#include "swd_common.cuh"

namespace swd {

// Static description of the transform (RTrAD.m / RTlAD.m / ADWDgrad_1.m).
struct RadonGeom {
  int nt, ng;          // seismogram samples and traces (a, b of SWD.m:142)
  int ccn;             // FFT length fix(1/df/dt) (RTrAD.m:15)
  int ntd;             // samples entering the DFT: min(nt, ccn)
  int lf, nf, npair;   // 1-based frequency bins lf..nf (RTrAD.m:18-19)
  int np;              // phase velocities
  int offset, m, M;
  double df, dt, ds, vmin, dv;
};

// One (shot, side) gather: trace columns c0, c0+dir, ..., c0+dir*(noff-1) (0-based).
struct Gather {
  int shot;   // index into the seismogram / adjoint-source batch
  int side;   // 0 right (RTrAD), 1 left (RTlAD)
  int c0;     // 0-based column of offset x = 0
  int dir;    // +1 right, -1 left (fliplr)
  int noff;   // traces in the window (dataLen)
  int valid;  // 1 when the reference computes this side for the shot
};

int radon_geom(const swd_radon_params* p, RadonGeom& g);
// Gather for shot `is` (1-based) and side (0 right / 1 left), reference window rules.
Gather make_gather(const RadonGeom& g, int is, int side, int shot_index, int ns, int w);
bool side_active(int is, int side, int ns, int m, int M, int w);

// W[f][t] = exp(-2 pi i (lf-1+f) t / ccn);  K[f][x][p] = exp(i 2 pi df (j-1) pp_p x_x)
int radon_tables(const RadonGeom& g, double2* W, double2* K, cudaStream_t st);

// D[g][f][x] = sum_t W[f][t] * seis(t, trace(g,x));  seis element (t, j) of shot s at seis[s*sstride + t*ng + j]
template <typename S>
int radon_dft(const RadonGeom& g, const Gather* d_gath, int G, const S* seis, size_t sstride, const double2* W,
              double2* D, cudaStream_t st);
// MM[g][f][p] = sum_x K[f][x][p] D[g][f][x]; mlraw = |MM|; ml = mlraw / max_p mlraw
// only (nullable, [G]): gathers with only[g] == 0 are left as they are
int radon_contract(const RadonGeom& g, const Gather* d_gath, int G, const double2* K, const double2* D, double2* MM,
                   double* mlraw, double* ml, cudaStream_t st, const int* only = nullptr);
// mlraw = |MM|, ml = mlraw / max_p mlraw for an MM computed elsewhere (valid gathers only)
int radon_amplitudes(const RadonGeom& g, const Gather* d_gath, int G, const double2* MM, double* mlraw, double* ml,
                     cudaStream_t st);
// pickFDC1 + LHDispPick per gather: cr_pre = picks + vmin, res = mean((cr_pre-cr0)^2), dc = cr_pre - cr0.
// Gathers with valid <= 0 are skipped (res = NaN); d_gath may be null (all gathers picked).
// Options of the guided picker.
//  * Field-data variants: raw ([g][npair][np], the unnormalised spectrum) picks the seed column as
//    the first one holding its global maximum, and the seed row from raw (value_from_raw,
//    pickFDCValue) or from ml (pickFDC1); r0 > 0 restricts the misfit to rows r0..npair-r1_from_end.
//  * Certification (split-BF16 spectra): with cert set, every hard decision records its margin
//    (the gap between the compared spectrum values: top two of each argmax, adjacent samples of
//    each local-minimum scan) and a gather with a margin below delta gets cert[g] = 1 (and
//    cert_count is incremented); with only set, gathers whose only[g] is 0 are skipped.
struct PickSeed {
  const double* raw = nullptr;
  int value_from_raw = 0;
  int r0 = 0, r1_from_end = 0;
  int* cert = nullptr;
  double delta = 0.0;
  unsigned long long* cert_count = nullptr;
  const int* only = nullptr;
};
int pick_batch(int np, int npair, int G, int ini, int method, double vmin, const Gather* d_gath, const double* ml,
               const double* cr0, double* cr_pre, double* dc, double* res, int* status, cudaStream_t st,
               PickSeed seed = PickSeed{});
// SoftMax gradient + adjoint Radon: Gx[g][f][x] = sum_p conj(K[f][x][p]) * gm[g][f][p];
// with `pick` ([g][f]) the weights are ADWDgrad_norm's Gaussian around pick - pick_off (= cr_pre - vmin);
// with `limband` they are ADWDgradlimband's power weights, mlr.^beta normalised per column
int softmax_adjoint(const RadonGeom& g, const Gather* d_gath, int G, const double* mlraw, const double2* MM,
                    const double* dc, const double* space_m, double beta, const double2* K, double2* Gx,
                    cudaStream_t st, const double* pick = nullptr, double pick_off = 0.0, int limband = 0);
// real(ifft(Gx, ccn))(1:nt) written into out[shot][t][col] (right: all x; left: x >= 1), ADWDgrad_1.m:42-44, 76
template <typename O>
int radon_idft_scatter(const RadonGeom& g, const Gather* d_gath, int G, const double2* Gx, const double2* W, O* out,
                       size_t ostride, cudaStream_t st,
                       const double2* TA = nullptr, const double2* TB = nullptr);

}  // namespace swd
