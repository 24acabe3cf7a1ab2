// The f-k dip filter of core/fk_filter.m (the same file in the field drivers' core folders),
// which the field drivers apply to a gather before the Radon transform when FK == 1
// (fieldexamples/QadimahFault/core/RTrAD.m:14-16, RTlAD.m:15-17).
//
// fk_filter.m zero-pads the ns x ntr gather to nf x nk = 2ns x 2ntr (:49-51), takes fft2 and
// fftshift (:52-53), zeroes the shifted quadrants (i <= nf/2, j <= nk/2) and (i > nf/2, j > nk/2)
// (:283-289), and returns the leading ns x ntr block of real(ifft2) of the re-shifted spectrum
// (:293-296).  In unshifted bins (u_f, u_k) the kept bins are those with exactly one of
// u_f >= nf/2, u_k >= nk/2.  dt and dx only set axes that the live code never uses.
//
// Here, in FP64:
//   T[x][u_f]  = DFT over time of each zero-padded trace (length nf), as a four-step transform
//                nf = L1 * L2 of two direct DFTs of sizes L1 and L2 (nf * (L1 + L2) products
//                per trace instead of nf^2);
//   R[x'][u_f] = sum_x T[x][u_f] h(x' - x mod nk), with h = h_plus (the bins u_k >= nk/2) for
//                u_f < nf/2 and h_minus (u_k < nk/2) otherwise: the wavenumber DFT, the mask and
//                the inverse wavenumber DFT in one pass, whose outputs x' < ntr are the only ones
//                kept (h(m) = 1/nk * sum over the kept u_k of exp(2 pi i u_k m / nk));
//   out        = real part of the inverse time DFT of R / nf (the same four-step transform),
//                rows t < ns.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fd_host.cuh"

namespace swd {
namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 conj_if(double2 w, bool c) { return c ? make_double2(w.x, -w.y) : w; }

// Step 1 of the four-step DFT of length nf = L1 * L2 (input index n = L2 n1 + n2, output index
// k = k1 + L1 k2): Y[tr][n2 L1 + k1] = W_nf^(n2 k1) * sum_n1 in[tr][L2 n1 + n2] W_L1^(n1 k1), with
// W_N = exp(-2 pi i / N) (INV: conjugated).  Inputs past `valid` are zero (the padding).
template <bool REAL_IN, bool INV>
__global__ void fk_step1(const void* __restrict__ in, int ld_in, int valid, int L1, int L2, int nf,
                         const double2* __restrict__ WL1, const double2* __restrict__ Wnf, double2* __restrict__ Y) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x, tr = blockIdx.y;
  if (idx >= nf) return;
  const int n2 = idx / L1, k1 = idx % L1;
  double2 acc = make_double2(0.0, 0.0);
  for (int n1 = 0; n1 < L1; ++n1) {
    const int n = L2 * n1 + n2;
    if (n >= valid) break;  // n grows with n1
    double2 v;
    if (REAL_IN) v = make_double2(static_cast<const double*>(in)[(size_t)tr * ld_in + n], 0.0);
    else v = static_cast<const double2*>(in)[(size_t)tr * ld_in + n];
    const double2 w = conj_if(WL1[(n1 * k1) % L1], INV);
    acc.x += v.x * w.x - v.y * w.y;
    acc.y += v.x * w.y + v.y * w.x;
  }
  Y[(size_t)tr * nf + idx] = cmul(acc, conj_if(Wnf[(int)(((long long)n2 * k1) % nf)], INV));
}

// Step 2: out[tr][k1 + L1 k2] = scale * sum_n2 Y[tr][n2 L1 + k1] W_L2^(n2 k2), for outputs k < need
// (REAL_OUT: the real part only, as real(ifft2)).
template <bool INV, bool REAL_OUT>
__global__ void fk_step2(const double2* __restrict__ Y, int L1, int L2, int nf, const double2* __restrict__ WL2,
                         void* __restrict__ out, int ld_out, int need, double scale) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x, tr = blockIdx.y;
  if (k >= nf || k >= need) return;
  const int k1 = k % L1, k2 = k / L1;
  double2 acc = make_double2(0.0, 0.0);
  for (int n2 = 0; n2 < L2; ++n2) {
    const double2 v = Y[(size_t)tr * nf + n2 * L1 + k1];
    const double2 w = conj_if(WL2[(int)(((long long)n2 * k2) % L2)], INV);
    acc.x += v.x * w.x - v.y * w.y;
    acc.y += v.x * w.y + v.y * w.x;
  }
  if (REAL_OUT) static_cast<double*>(out)[(size_t)tr * ld_out + k] = scale * acc.x;
  else static_cast<double2*>(out)[(size_t)tr * ld_out + k] = make_double2(scale * acc.x, scale * acc.y);
}

// The wavenumber pass: R[x'][u] = sum_{x < ntr} T[x][u] h(x' - x mod nk), h = hp for u < nf/2,
// hm otherwise.
__global__ void fk_offset(const double2* __restrict__ T, int nf, int ntr, int nk, const double2* __restrict__ hp,
                          const double2* __restrict__ hm, double2* __restrict__ R) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x, xo = blockIdx.y;
  if (u >= nf) return;
  const double2* h = u < nf / 2 ? hp : hm;
  double2 acc = make_double2(0.0, 0.0);
  for (int x = 0; x < ntr; ++x) {
    const double2 v = T[(size_t)x * nf + u], w = h[(xo - x + nk) % nk];
    acc.x += v.x * w.x - v.y * w.y;
    acc.y += v.x * w.y + v.y * w.x;
  }
  R[(size_t)xo * nf + u] = acc;
}

// exp(-2 pi i j / n), j < n, from the reduced fraction j / n
std::vector<double2> roots(int n) {
  std::vector<double2> w(n);
  for (int j = 0; j < n; ++j) {
    const double a = 2.0 * M_PI * (double)j / (double)n;
    w[j] = make_double2(std::cos(a), -std::sin(a));
  }
  return w;
}

}  // namespace
}  // namespace swd

using namespace swd;

extern "C" int swd_fk_filter(const double* d, int ns, int ntr, double dt, double dx, double* dfk) {
  (void)dt;  // fk_filter.m:56-67: only the unused frequency and wavenumber axes depend on them
  (void)dx;
  clear_error();
  SWD_CHECK(d && dfk && ns >= 1 && ntr >= 1, "bad fk_filter arguments (ns %d, ntr %d)", ns, ntr);
  SWD_CHECK(ntr <= 65535 && ns <= (1 << 29), "fk_filter gather too large (ns %d, ntr %d; traces index the grid's "
            "y dimension, at most 65535)", ns, ntr);
  const int nf = 2 * ns, nk = 2 * ntr;
  int L1 = 1;
  for (int q = 1; (long long)q * q <= nf; ++q)
    if (nf % q == 0) L1 = q;
  const int L2 = nf / L1;
  // h_plus / h_minus: 1/nk * sum over u_k >= nk/2 (resp. < nk/2) of exp(2 pi i u_k m / nk)
  std::vector<double2> hp(nk), hm(nk);
  for (int m = 0; m < nk; ++m) {
    double pr = 0, pi = 0, mr = 0, mi = 0;
    for (int u = 0; u < nk; ++u) {
      const double a = 2.0 * M_PI * (double)(((long long)u * m) % nk) / (double)nk;
      if (u >= nk / 2) { pr += std::cos(a); pi += std::sin(a); }
      else { mr += std::cos(a); mi += std::sin(a); }
    }
    hp[m] = make_double2(pr / nk, pi / nk);
    hm[m] = make_double2(mr / nk, mi / nk);
  }
  const std::vector<double2> w1 = roots(L1), w2 = roots(L2), wn = roots(nf);
  const size_t nd = (size_t)ns * ntr, nc = (size_t)ntr * nf;
  const size_t n_tab = (size_t)(L1 + L2 + nf + 2 * nk) * sizeof(double2);
  SlabPlan sl;
  const size_t o_d = sl.add(nd * sizeof(double)), o_x = sl.add(nc * sizeof(double2));
  const size_t o_y = sl.add(nc * sizeof(double2)), o_r = sl.add(nc * sizeof(double2)), o_t = sl.add(n_tab);
  DevBuf slab;
  SWD_TRY(slab.alloc(sl.bytes));
  const DevView bd(slab, o_d, nd * sizeof(double)), bx(slab, o_x, nc * sizeof(double2));
  const DevView by(slab, o_y, nc * sizeof(double2)), br(slab, o_r, nc * sizeof(double2)), bt(slab, o_t, n_tab);
  double2* W1 = bt.as<double2>();
  double2* W2 = W1 + L1;
  double2* Wn = W2 + L2;
  double2* Hp = Wn + nf;
  double2* Hm = Hp + nk;
  cudaStream_t st = 0;
  SWD_CUDA(cudaMemcpyAsync(bd.p, d, nd * sizeof(double), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(W1, w1.data(), L1 * sizeof(double2), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(W2, w2.data(), L2 * sizeof(double2), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(Wn, wn.data(), nf * sizeof(double2), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(Hp, hp.data(), nk * sizeof(double2), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(Hm, hm.data(), nk * sizeof(double2), cudaMemcpyHostToDevice, st));
  const dim3 blk(256), grd((nf + 255) / 256, ntr);
  double2* X = bx.as<double2>();
  double2* Y = by.as<double2>();
  double2* R = br.as<double2>();
  fk_step1<true, false><<<grd, blk, 0, st>>>(bd.p, ns, ns, L1, L2, nf, W1, Wn, Y);
  fk_step2<false, false><<<grd, blk, 0, st>>>(Y, L1, L2, nf, W2, X, nf, nf, 1.0);
  fk_offset<<<grd, blk, 0, st>>>(X, nf, ntr, nk, Hp, Hm, R);
  fk_step1<false, true><<<grd, blk, 0, st>>>(R, nf, nf, L1, L2, nf, W1, Wn, Y);
  fk_step2<true, true><<<grd, blk, 0, st>>>(Y, L1, L2, nf, W2, bd.p, ns, ns, 1.0 / nf);
  count_launch(5);
  SWD_CUDA(cudaGetLastError());
  SWD_CUDA(cudaMemcpyAsync(dfk, bd.p, nd * sizeof(double), cudaMemcpyDeviceToHost, st));
  SWD_CUDA(cudaStreamSynchronize(st));
  return SWD_OK;
}
