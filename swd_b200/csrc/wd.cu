// WD adjoint source: core/weight_data_muti3.m:1-122 (the wave-equation dispersion residual
// that SWD.m:188 offers in place of ADWDgrad_1).
//
// For each gather the reference zero-pads the traces to ntpad = floor(1/dt/df) samples,
// Fourier transforms them, multiplies bins 2..win+1 by a factor fac(k, y), mirrors them into
// bins ntpad-win+1..ntpad, leaves the other bins as they are and transforms back.  Only win
// bins change, so the result is the trace plus a low-bin correction:
//     out(t) = x(t) + (2/ntpad) Re sum_{k=1..win} (fac_k - 1) X_k exp(2 pi i k t / ntpad),
// X_k the trace's DFT at bin k.  The DFT of the win bins reuses the Radon DFT kernel; the
// correction, the factors and the scatter into the adjoint-source columns are one kernel.
// All arithmetic is FP64.
#include <cmath>
#include <vector>

#include "fd_host.cuh"
#include "wd.cuh"

namespace swd {

static int mround(double x) {  // MATLAB round: half away from zero
  double r = std::floor(std::fabs(x));
  if (std::fabs(x) - r >= 0.5) r += 1;
  return (int)std::copysign(r, x);
}

int wd_geom(int nt, int ng, double dt, double df, int offset, int m, int win, int ind, double fmin, double fmax,
            double dg, int F1, WdGeom& g) {
  SWD_CHECK(nt >= 1 && ng >= 1, "seismogram must be non-empty");
  SWD_CHECK(dt > 0 && df > 0 && dg > 0, "dt, df and dg must be positive");
  SWD_CHECK(offset >= 1 && m >= 0, "offset >= 1 and m >= 0 required");
  SWD_CHECK(F1 == 0 || F1 == 1, "F1 must be 0 (predicted data) or 1 (observed data)");
  const double np_ = std::floor(1.0 / dt / df);  // weight_data_muti3.m:10
  SWD_CHECK(np_ >= 1 && np_ < 2147483647.0, "ntpad = floor(1/dt/df) out of range");
  const int ntpad = (int)np_;
  const double nf = std::floor((fmax - fmin) / df + 1);  // linspace count (weight_data_muti3.m:4)
  SWD_CHECK(nf >= 1 && nf < 1e7, "no pick frequencies in fmin:df:fmax");
  g.nfre = (int)nf;
  g.npair = g.nfre;
  SWD_CHECK(nt <= ntpad, "weight_data_muti3 needs nt (%d) <= ntpad = floor(1/dt/df) (%d)", nt, ntpad);
  SWD_CHECK(win >= 1 && 2 * (long)win < ntpad, "win (%d) must satisfy 1 <= win and 2*win < ntpad (%d)", win, ntpad);
  SWD_CHECK(ind >= 1 && ind + g.nfre - 1 <= win, "bins ind..ind+npair-1 (%d..%d) must lie in 1..win (%d)", ind,
            ind + g.nfre - 1, win);
  g.win = win;
  g.ind = ind;
  g.m = m;
  g.F1 = F1;
  g.dg = dg;
  RadonGeom& r = g.dft;
  r = RadonGeom{};
  r.nt = nt; r.ng = ng; r.ccn = ntpad; r.ntd = nt;
  r.lf = 2; r.nf = win + 1; r.npair = win;
  r.np = 1;
  r.offset = offset; r.m = m; r.M = 1;
  r.df = df; r.dt = dt; r.ds = dg; r.vmin = 1; r.dv = 1;
  return SWD_OK;
}

void wd_fre(double fmin, double fmax, int nfre, double* fre) {
  // 2*pi*linspace(fmin, fmax, n): fmin + i*(fmax-fmin)/(n-1), the last point fmax
  const double pi2 = 2.0 * 3.141592653589793;
  for (int i = 0; i < nfre; ++i) {
    const double v = (nfre == 1 || i == nfre - 1) ? fmax : fmin + (double)i * (fmax - fmin) / (nfre - 1);
    fre[i] = pi2 * v;
  }
}

Gather make_wd_gather(const WdGeom& g, int is, int side, int shot_index, int ns, int w, double M, int refsx) {
  Gather r{};
  r.shot = shot_index;
  r.side = side;
  const int fm = (int)std::floor((double)g.m / M), rw = mround((double)w / M);
  const int ng = g.dft.ng, offset = g.dft.offset;
  if (side == 0) {  // weight_data_muti3.m:21-29
    r.valid = is <= ns - fm - rw ? 1 : 0;
    const int nend = std::min(g.m + offset - 1 + refsx, ng);
    r.c0 = refsx + g.m - 1;
    r.dir = 1;
    r.noff = nend - (refsx + g.m) + 1;
  } else {          // weight_data_muti3.m:74-82
    r.valid = is > rw + fm + 1 ? 1 : 0;
    const int nend = std::max(refsx - offset - g.m, 0);
    r.c0 = refsx - g.m - 1;
    r.dir = -1;
    r.noff = refsx - g.m - nend;
  }
  if (r.noff < 1 || r.c0 < 0 || r.c0 >= ng || r.c0 + r.dir * (r.noff - 1) < 0 || r.c0 + r.dir * (r.noff - 1) >= ng)
    r.valid = r.valid ? -1 : 0;
  return r;
}

constexpr int kWdT = 64;   // samples per block (8 warps x 8)
constexpr int kWdK = 32;   // bins per shared-memory chunk

// One block: 32 traces (lanes) x 64 samples of one gather.  The corrections D_k = (fac_k-1) X_k
// of a chunk of bins go through shared memory; each warp sums them for its 8 samples.
template <typename S, typename O>
__global__ void __launch_bounds__(256) wd_scatter_kernel(WdGeom g, const Gather* gs, const S* __restrict__ seis,
                                                         size_t sstride, const double2* __restrict__ X,
                                                         const double2* __restrict__ W,
                                                         const double* __restrict__ fre,
                                                         const double* __restrict__ cr0,
                                                         const double* __restrict__ crp, O* out, size_t ostride) {
  __shared__ double2 sd[kWdK][32];
  const int gi = blockIdx.z;
  const Gather gg = gs[gi];
  if (gg.valid <= 0) return;
  const int x0 = blockIdx.y * 32;
  if (x0 >= gg.noff) return;
  const RadonGeom& r = g.dft;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int t0 = blockIdx.x * kWdT;
  double acc[kWdT / 8];
#pragma unroll
  for (int i = 0; i < kWdT / 8; ++i) acc[i] = 0.0;
  const double* c0 = cr0 + (size_t)gi * g.npair;
  const double* cp = crp + (size_t)gi * g.npair;
  for (int k0 = 0; k0 < g.win; k0 += kWdK) {
    for (int i = threadIdx.x; i < kWdK * 32; i += blockDim.x) {
      const int kk = i >> 5, xx = i & 31, k = k0 + kk + 1, x = x0 + xx;
      double2 d = make_double2(0.0, 0.0);
      if (k <= g.win && x < gg.noff) {
        const double2 Xk = X[((size_t)gi * r.npair + (k - 1)) * r.offset + x];
        // deta_cc2(ind:ind+npair-1) = fre'.*(cr_0-cr_pre)./(cr_0.*cr_pre) (:23), 0 elsewhere
        const int j = k - g.ind;
        const double dk = (j >= 0 && j < g.nfre) ? (fre[j] * (c0[j] - cp[j])) / (c0[j] * cp[j]) : 0.0;
        const double y = (double)(g.m + x) * g.dg;  // (m + linspace(...))*dg (:30, :85)
        const double th = -(dk * y);                 // imaginary part of -1i*y1*y
        double fr, fi;
        if (g.F1) {  // (-1i*y1*y).*exp(-1i*y1*y)/pi/2 (:37)
          double s, c;
          sincos(th, &s, &c);
          fr = ((-(th * s)) / 3.141592653589793) / 2.0;
          fi = ((th * c) / 3.141592653589793) / 2.0;
        } else {     // (-1i*y1*y)/pi/2 (:39)
          fr = 0.0;
          fi = (th / 3.141592653589793) / 2.0;
        }
        // bin .* fac (:50) minus the bin itself
        const double yr = Xk.x * fr - Xk.y * fi, yi = Xk.x * fi + Xk.y * fr;
        d = make_double2(yr - Xk.x, yi - Xk.y);
      }
      sd[kk][xx] = d;
    }
    __syncthreads();
    const int kn = min(kWdK, g.win - k0);
#pragma unroll
    for (int i = 0; i < kWdT / 8; ++i) {
      const int t = t0 + wp + 8 * i;
      if (t >= r.nt) break;
      const double2* Wt = W + (size_t)k0 * r.ntd + t;
      double a = acc[i];
      for (int kk = 0; kk < kn; ++kk) {
        const double2 w = Wt[(size_t)kk * r.ntd];  // exp(-i th); the inverse uses exp(+i th)
        const double2 v = sd[kk][lane];
        a += v.x * w.x + v.y * w.y;
      }
      acc[i] = a;
    }
    __syncthreads();
  }
  const int x = x0 + lane;
  if (x >= gg.noff) return;
  const int col = gg.c0 + gg.dir * x;
  const S* src = seis + (size_t)gg.shot * sstride;
  O* o = out + (size_t)gg.shot * ostride;
  const double scale = 2.0 / (double)r.ccn;
#pragma unroll
  for (int i = 0; i < kWdT / 8; ++i) {
    const int t = t0 + wp + 8 * i;
    if (t >= r.nt) break;
    const size_t e = (size_t)t * r.ng + col;
    o[e] = (O)((double)src[e] + acc[i] * scale);
  }
}

template <typename S, typename O>
int wd_adjoint(const WdGeom& g, const Gather* d_gath, int G, const S* seis, size_t sstride, const double2* W,
               const double* fre, const double* cr0, const double* crp, double2* X, O* out, size_t ostride,
               cudaStream_t st) {
  SWD_TRY(radon_dft<S>(g.dft, d_gath, G, seis, sstride, W, X, st));
  dim3 grid((g.dft.nt + kWdT - 1) / kWdT, (g.dft.offset + 31) / 32, G);
  wd_scatter_kernel<S, O><<<grid, 256, 0, st>>>(g, d_gath, seis, sstride, X, W, fre, cr0, crp, out, ostride);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}
template int wd_adjoint<float, float>(const WdGeom&, const Gather*, int, const float*, size_t, const double2*,
                                      const double*, const double*, const double*, double2*, float*, size_t,
                                      cudaStream_t);
template int wd_adjoint<double, double>(const WdGeom&, const Gather*, int, const double*, size_t, const double2*,
                                        const double*, const double*, const double*, double2*, double*, size_t,
                                        cudaStream_t);

}  // namespace swd

// ====================================================================== C ABI (host pointers)

using namespace swd;

extern "C" int swd_wd_residual(int nt, int ng, const double* seismo_v_d, const double* seismo_v, int is, double dt,
                               double df, int offset, double dg, int F1, int w, double M, int m, int ns,
                               const double* refsx, int win, double fmin, double fmax, const double* cr_0,
                               const double* cr_0l, const double* cr_pre_r, const double* cr_pre_l, int ind,
                               double* seismo_v_d1) {
  clear_error();
  WdGeom g{};
  SWD_TRY(wd_geom(nt, ng, dt, df, offset, m, win, ind, fmin, fmax, dg, F1, g));
  SWD_CHECK(M > 0, "M must be positive");
  SWD_CHECK(is >= 1 && is <= ns && refsx, "shot %d outside 1..ns (%d) or null refsx", is, ns);
  SWD_CHECK(seismo_v_d1 && (F1 ? seismo_v_d : seismo_v), "null seismogram or output");
  const double rs = refsx[is - 1];
  SWD_CHECK(rs == std::floor(rs) && std::fabs(rs) < 1e9, "refsx(%d) must be an integer", is);
  Gather gg[2];
  const double* c0[2] = {cr_0, cr_0l};
  const double* cp[2] = {cr_pre_r, cr_pre_l};
  for (int s = 0; s < 2; ++s) {
    gg[s] = make_wd_gather(g, is, s, 0, ns, w, M, (int)rs);
    SWD_CHECK(gg[s].valid >= 0, "shot %d: the %s WD window is empty or leaves the receiver line", is,
              s ? "left" : "right");
    SWD_CHECK(!gg[s].valid || (c0[s] && cp[s]), "missing %s-side picks", s ? "left" : "right");
  }
  const size_t nsz = (size_t)nt * ng, np2 = (size_t)g.npair;
  const size_t n_seis = nsz * sizeof(double), n_W = (size_t)g.win * nt * sizeof(double2);
  const size_t n_X = 2 * (size_t)g.win * offset * sizeof(double2);
  SlabPlan sl;
  const size_t o_in = sl.add(n_seis), o_t = sl.add(n_seis), o_out = sl.add(n_seis), o_W = sl.add(n_W);
  const size_t o_X = sl.add(n_X), o_fre = sl.add(np2 * sizeof(double)), o_cr = sl.add(4 * np2 * sizeof(double));
  const size_t o_g = sl.add(2 * sizeof(Gather));
  DevBuf slab;
  SWD_TRY(slab.alloc(sl.bytes));
  const DevView b_in(slab, o_in, n_seis), b_t(slab, o_t, n_seis), b_out(slab, o_out, n_seis), b_W(slab, o_W, n_W);
  const DevView b_X(slab, o_X, n_X), b_fre(slab, o_fre, np2 * sizeof(double));
  const DevView b_cr(slab, o_cr, 4 * np2 * sizeof(double)), b_g(slab, o_g, 2 * sizeof(Gather));
  std::vector<double> fre(np2);
  wd_fre(fmin, fmax, g.nfre, fre.data());
  cudaStream_t st = 0;
  SWD_CUDA(cudaMemcpyAsync(b_in.p, F1 ? seismo_v_d : seismo_v, nsz * sizeof(double), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(b_fre.p, fre.data(), np2 * sizeof(double), cudaMemcpyHostToDevice, st));
  // pick arrays laid out [gather][npair]: observed r, l, then predicted r, l
  double* d_cr = b_cr.as<double>();
  for (int s = 0; s < 2; ++s) {
    if (gg[s].valid != 1) continue;
    SWD_CUDA(cudaMemcpyAsync(d_cr + s * np2, c0[s], np2 * sizeof(double), cudaMemcpyHostToDevice, st));
    SWD_CUDA(cudaMemcpyAsync(d_cr + (2 + s) * np2, cp[s], np2 * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  SWD_CUDA(cudaMemcpyAsync(b_g.p, gg, 2 * sizeof(Gather), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemsetAsync(b_out.p, 0, nsz * sizeof(double), st));
  // MATLAB nt x ng -> [nt][ng]
  SWD_TRY(transpose<double, double>(b_in.as<double>(), 0, b_t.as<double>(), 0, 1, ng, nt, st));
  SWD_TRY(radon_tables(g.dft, b_W.as<double2>(), nullptr, st));
  // right side then left side, as the reference writes them (both write the same values to a
  // shared column when m = 0)
  for (int s = 0; s < 2; ++s) {
    if (gg[s].valid != 1) continue;
    SWD_TRY(wd_adjoint<double, double>(g, b_g.as<Gather>() + s, 1, b_t.as<double>(), 0, b_W.as<double2>(),
                                       b_fre.as<double>(), d_cr + s * np2, d_cr + (2 + s) * np2,
                                       b_X.as<double2>() + (size_t)s * g.win * offset, b_out.as<double>(), 0, st));
  }
  SWD_TRY(transpose<double, double>(b_out.as<double>(), 0, b_t.as<double>(), 0, 1, nt, ng, st));
  SWD_CUDA(cudaMemcpyAsync(seismo_v_d1, b_t.p, nsz * sizeof(double), cudaMemcpyDeviceToHost, st));
  SWD_CUDA(cudaStreamSynchronize(st));
  return SWD_OK;
}
