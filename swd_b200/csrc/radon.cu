// Radon dispersion spectrum, guided picker and SoftMax misfit gradient (FP64 path).
//
// Reference:  core/RTrAD.m:2-35, core/RTlAD.m:2-36 (spectrum and saved state),
//             core/LHDispPick.m:2-13 + core/pickFDC1.m:1-131 (picker),
//             core/ADWDgrad_1.m:1-81 (SoftMax gradient, adjoint Radon, inverse FFT).
// All gathers of a batch run in one launch per stage.  The DFT evaluates only
// the bins lf..nf that the reference keeps; the Radon sum runs in double like
// MATLAB; the SoftMax uses a max-shifted FP64 log-sum-exp.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "fd_host.cuh"
#include "radon.cuh"

namespace swd {

static int mround(double x) {  // MATLAB round: half away from zero
  double r = std::floor(std::fabs(x));
  if (std::fabs(x) - r >= 0.5) r += 1;
  return (int)std::copysign(r, x);
}

int radon_geom(const swd_radon_params* p, RadonGeom& g) {
  SWD_CHECK(p != nullptr, "null radon params");
  SWD_CHECK(p->df > 0 && p->dt > 0 && p->ds > 0, "df, dt and ds must be positive");
  SWD_CHECK(p->nt >= 1 && p->ng >= 1, "seismogram must be non-empty");
  SWD_CHECK(p->offset >= 1 && p->M >= 1 && p->m >= 0, "offset >= 1, M >= 1, m >= 0 required");
  SWD_CHECK(p->dv > 0 && p->vmax >= p->vmin && p->vmin > 0, "velocity axis vmin:dv:vmax must be positive");
  g.nt = p->nt; g.ng = p->ng;
  const double cc = std::trunc(1.0 / p->df / p->dt);  // fix(1./df./dt)
  SWD_CHECK(cc >= 1 && cc < 2147483647.0, "ccn = fix(1/df/dt) out of range");
  g.ccn = (int)cc;
  g.ntd = std::min(g.nt, g.ccn);
  g.lf = mround(p->fmin / p->df) + 1;
  g.nf = mround(p->fmax / p->df) + 1;
  SWD_CHECK(g.lf >= 1 && g.nf >= g.lf && g.nf <= g.ccn, "frequency bins %d..%d outside 1..ccn (%d)", g.lf, g.nf, g.ccn);
  g.npair = g.nf - g.lf + 1;
  g.np = (int)std::floor((p->vmax - p->vmin) / p->dv + 1e-9) + 1;
  g.offset = p->offset; g.m = p->m; g.M = p->M;
  g.df = p->df; g.dt = p->dt; g.ds = p->ds; g.vmin = p->vmin; g.dv = p->dv;
  return SWD_OK;
}

bool side_active(int is, int side, int ns, int m, int M, int w) {
  // ADWDgrad_1.m:15 (right) and :47 (left); SWD.m:175, 181
  if (side == 0) return is <= ns - (int)std::floor((double)m / M) - mround((double)w / M);
  return is >= mround((double)w / M) + (int)std::floor((double)m / M) + 1;
}

Gather make_gather(const RadonGeom& g, int is, int side, int shot_index, int ns, int w) {
  Gather r{};
  r.shot = shot_index;
  r.side = side;
  r.valid = side_active(is, side, ns, g.m, g.M, w) ? 1 : 0;
  if (side == 0) {  // RTrAD.m:4-9
    const int c0 = g.M * is - g.M + 1 + g.m;
    const int nend = std::min(g.m + g.offset - 1 + g.M * is - g.M + 1, g.ng);
    r.c0 = c0 - 1;
    r.dir = 1;
    r.noff = nend - c0 + 1;
  } else {          // RTlAD.m:4-9: fliplr(seismo(:, nend+1 : M*is-M+1-m))
    int nend = g.M * is - g.M + 1 - g.offset - g.m;
    if (nend < 1) nend = 0;
    const int last = g.M * is - g.M + 1 - g.m;
    r.c0 = last - 1;
    r.dir = -1;
    r.noff = last - nend;
  }
  if (r.noff < 1 || r.c0 < 0 || r.c0 >= g.ng || r.c0 + r.dir * (r.noff - 1) < 0 ||
      r.c0 + r.dir * (r.noff - 1) >= g.ng)
    r.valid = r.valid ? -1 : 0;  // empty or out-of-range window where the reference would compute one
  return r;
}

// ------------------------------------------------------------------ tables

__global__ void w_table_kernel(RadonGeom g, double2* W) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x, f = blockIdx.y;
  if (t >= g.ntd) return;
  const long long k = g.lf - 1 + f;
  const long long r = (k * (long long)t) % g.ccn;
  double s, c;
  sincospi(2.0 * (double)r / (double)g.ccn, &s, &c);
  W[(size_t)f * g.ntd + t] = make_double2(c, -s);
}

__global__ void k_table_kernel(RadonGeom g, double2* K) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y, f = blockIdx.z;
  if (p >= g.np) return;
  // RTrAD.m:13,20-21: x=(m+(0:off-1))*ds, pp=1./v, ll0 = 1i*2*pi*df*(pp*x), l = exp(ll0*(j-1))
  const double v = g.vmin + g.dv * p;
  const double pp = 1.0 / v;
  const double xx = (g.m + x) * g.ds;
  const double w0 = 2.0 * 3.141592653589793 * g.df;
  const double th = (w0 * (pp * xx)) * (double)(g.lf - 1 + f);
  double s, c;
  sincos(th, &s, &c);
  K[((size_t)f * g.offset + x) * g.np + p] = make_double2(c, s);
}

int radon_tables(const RadonGeom& g, double2* W, double2* K, cudaStream_t st) {
  if (W) {
    dim3 grid((g.ntd + 255) / 256, g.npair);
    w_table_kernel<<<grid, 256, 0, st>>>(g, W);
    count_launch(1);
  }
  if (K) {
    dim3 grid((g.np + 127) / 128, g.offset, g.npair);
    k_table_kernel<<<grid, 128, 0, st>>>(g, K);
    count_launch(1);
  }
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}

// ------------------------------------------------------------------ DFT at the kept bins

constexpr int kDftF = 8, kDftT = 64;

template <typename S>
__global__ void __launch_bounds__(256) dft_kernel(RadonGeom g, const Gather* gs, const S* seis, size_t sstride,
                                                  const double2* __restrict__ W, double2* D) {
  __shared__ double su[kDftT][33];
  __shared__ double2 sw[kDftF][kDftT];
  const Gather gg = gs[blockIdx.z];
  if (gg.valid <= 0) return;
  const int f0 = blockIdx.x * kDftF, x0 = blockIdx.y * 32;
  if (x0 >= gg.noff) return;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const S* src = seis + (size_t)gg.shot * sstride;
  double2 acc = make_double2(0.0, 0.0);
  const int f = f0 + wp, x = x0 + lane;
  for (int t0 = 0; t0 < g.ntd; t0 += kDftT) {
    for (int i = threadIdx.x; i < kDftT * 32; i += 256) {
      const int tt = i >> 5, xx = i & 31, t = t0 + tt, xg = x0 + xx;
      double v = 0.0;
      if (t < g.ntd && xg < gg.noff) v = (double)src[(size_t)t * g.ng + (gg.c0 + gg.dir * xg)];
      su[tt][xx] = v;
    }
    for (int i = threadIdx.x; i < kDftF * kDftT; i += 256) {
      const int ff = i / kDftT, tt = i % kDftT, t = t0 + tt, fg = f0 + ff;
      sw[ff][tt] = (t < g.ntd && fg < g.npair) ? W[(size_t)fg * g.ntd + t] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll 8
    for (int tt = 0; tt < kDftT; ++tt) {
      const double u = su[tt][lane];
      const double2 w = sw[wp][tt];
      acc.x += w.x * u;
      acc.y += w.y * u;
    }
    __syncthreads();
  }
  if (f < g.npair && x < gg.noff) D[((size_t)blockIdx.z * g.npair + f) * g.offset + x] = acc;
}

template <typename S>
int radon_dft(const RadonGeom& g, const Gather* d_gath, int G, const S* seis, size_t sstride, const double2* W,
              double2* D, cudaStream_t st) {
  dim3 grid((g.npair + kDftF - 1) / kDftF, (g.offset + 31) / 32, G);
  dft_kernel<S><<<grid, 256, 0, st>>>(g, d_gath, seis, sstride, W, D);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}
template int radon_dft<float>(const RadonGeom&, const Gather*, int, const float*, size_t, const double2*, double2*,
                              cudaStream_t);
template int radon_dft<double>(const RadonGeom&, const Gather*, int, const double*, size_t, const double2*,
                               double2*, cudaStream_t);

// ------------------------------------------------------------------ Radon sum, |mm|, column normalisation

__device__ double block_max(double v, double* sm) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  v = threadIdx.x < nw ? sm[threadIdx.x] : -1.0 / 0.0;
  if (threadIdx.x < 32)
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (threadIdx.x == 0) sm[32] = v;
  __syncthreads();
  v = sm[32];
  __syncthreads();
  return v;
}

__device__ double block_sum(double v, double* sm) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  v = threadIdx.x < nw ? sm[threadIdx.x] : 0.0;
  if (threadIdx.x < 32)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (threadIdx.x == 0) sm[32] = v;
  __syncthreads();
  v = sm[32];
  __syncthreads();
  return v;
}

__global__ void __launch_bounds__(256) contract_kernel(RadonGeom g, const Gather* gs, const double2* __restrict__ K,
                                                       const double2* __restrict__ D, double2* MM, double* mlraw,
                                                       double* ml, const int* only) {
  extern __shared__ double2 sd[];
  __shared__ double red[33];
  const int f = blockIdx.x, gi = blockIdx.y;
  const Gather gg = gs[gi];
  if (gg.valid <= 0 || (only && !only[gi])) return;  // the whole block returns
  const size_t col = ((size_t)gi * g.npair + f);
  for (int x = threadIdx.x; x < gg.noff; x += blockDim.x) sd[x] = D[col * g.offset + x];
  __syncthreads();
  const double2* Kf = K + (size_t)f * g.offset * g.np;
  double mx = -1.0 / 0.0;
  for (int p = threadIdx.x; p < g.np; p += blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int x = 0; x < gg.noff; ++x) {
      const double2 k = Kf[(size_t)x * g.np + p];
      const double2 d = sd[x];
      re += k.x * d.x - k.y * d.y;
      im += k.x * d.y + k.y * d.x;
    }
    MM[col * g.np + p] = make_double2(re, im);
    const double a = hypot(re, im);
    mlraw[col * g.np + p] = a;
    mx = fmax(mx, a);
  }
  mx = block_max(mx, red);
  for (int p = threadIdx.x; p < g.np; p += blockDim.x) ml[col * g.np + p] = mlraw[col * g.np + p] / mx;
}

// mlraw = |MM| and ml = mlraw / max_p mlraw per (gather, bin), for an MM computed elsewhere
// (the tensor-core contraction); the same amplitude and normalisation as contract_kernel.
__global__ void __launch_bounds__(256) amplitude_kernel(RadonGeom g, const Gather* gs, const double2* __restrict__ MM,
                                                        double* mlraw, double* ml) {
  __shared__ double red[33];
  const int f = blockIdx.x, gi = blockIdx.y;
  if (gs[gi].valid <= 0) return;
  const size_t col = ((size_t)gi * g.npair + f) * g.np;
  double mx = -1.0 / 0.0;
  for (int p = threadIdx.x; p < g.np; p += blockDim.x) {
    const double2 v = MM[col + p];
    const double a = hypot(v.x, v.y);
    mlraw[col + p] = a;
    mx = fmax(mx, a);
  }
  mx = block_max(mx, red);
  for (int p = threadIdx.x; p < g.np; p += blockDim.x) ml[col + p] = mlraw[col + p] / mx;
}

int radon_amplitudes(const RadonGeom& g, const Gather* d_gath, int G, const double2* MM, double* mlraw, double* ml,
                     cudaStream_t st) {
  amplitude_kernel<<<dim3(g.npair, G), 256, 0, st>>>(g, d_gath, MM, mlraw, ml);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}

int radon_contract(const RadonGeom& g, const Gather* d_gath, int G, const double2* K, const double2* D, double2* MM,
                   double* mlraw, double* ml, cudaStream_t st, const int* only) {
  dim3 grid(g.npair, G);
  const size_t smem = (size_t)g.offset * sizeof(double2);
  if (smem > 48 * 1024) SWD_CUDA(cudaFuncSetAttribute(contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  contract_kernel<<<grid, 256, smem, st>>>(g, d_gath, K, D, MM, mlraw, ml, only);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}

// ------------------------------------------------------------------ guided picker (one warp per gather)

// First q in (s, e) (1-based, inclusive segment [s, e]) where y has a findpeaks(-y) peak; 0 if none.
__device__ int first_local_min(const double* y, int s, int e, int lane) {
  for (int base = s + 1; base < e; base += 32) {
    const int q = base + lane;
    bool ok = false;
    if (q < e) {
      const double yq = y[q - 1];
      if (yq < y[q - 2]) {
        int r = q + 1;
        while (r <= e && y[r - 1] == yq) ++r;
        ok = (r <= e) && (y[r - 1] > yq);
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (m) return base + __ffs(m) - 1;
  }
  return 0;
}

// Last such q in (1, e) for the segment [1, e]; 0 if none.
__device__ int last_local_min(const double* y, int e, int lane) {
  for (int top = e - 1; top >= 2; top -= 32) {
    const int q = top - lane;
    bool ok = false;
    if (q >= 2) {
      const double yq = y[q - 1];
      if (yq < y[q - 2]) {
        int r = q + 1;
        while (r <= e && y[r - 1] == yq) ++r;
        ok = (r <= e) && (y[r - 1] > yq);
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (m) return top - (__ffs(m) - 1);
  }
  return 0;
}

// MATLAB [~,i]=max(y(lo:hi)): first index of the maximum, returned 1-based absolute.
__device__ int warp_argmax(const double* y, int lo, int hi, int lane) {
  double bv = -1.0 / 0.0;
  int bi = 0x7fffffff;
  for (int q = lo + lane; q <= hi; q += 32) {
    const double v = y[q - 1];
    if (v > bv || (v == bv && q < bi)) { bv = v; bi = q; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
  }
  return bi;
}

// Margins of the picker's decisions (certification of a split-BF16 spectrum).
// Adjacent samples compared by a findpeaks scan over y(lo:hi): min |y(q) - y(q-1)|, q = lo+1..hi.
__device__ double warp_adjacent_gap(const double* y, int lo, int hi, int lane) {
  double m = 1.0 / 0.0;
  for (int q = lo + 1 + lane; q <= hi; q += 32) m = fmin(m, fabs(y[q - 1] - y[q - 2]));
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  return m;
}
// An argmax over y(lo:hi): the largest value minus the next largest (0 for a tie, inf for one sample).
__device__ double warp_top2_gap(const double* y, int lo, int hi, int lane) {
  double t1 = -1.0 / 0.0, t2 = -1.0 / 0.0;
  for (int q = lo + lane; q <= hi; q += 32) {
    const double v = y[q - 1];
    if (v > t1) { t2 = t1; t1 = v; }
    else if (v > t2) t2 = v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double a1 = __shfl_xor_sync(0xffffffffu, t1, o), a2 = __shfl_xor_sync(0xffffffffu, t2, o);
    const double n1 = fmax(t1, a1), n2 = fmax(fmin(t1, a1), fmax(t2, a2));
    t1 = n1;
    t2 = n2;
  }
  return t1 - t2;
}

// MATLAB [~,ini] = max(max(raw)) over a np x npair column-major spectrum: the first column
// holding the largest value, 1-based (every lane returns it).
__device__ int warp_colmax_argmax(const double* raw, int np, int npair, int lane) {
  double bv = -1.0 / 0.0;
  int bi = 0x7fffffff;
  for (int i = 1 + lane; i <= npair; i += 32) {
    const double* c = raw + (size_t)(i - 1) * np;
    double m = -1.0 / 0.0;
    for (int q = 0; q < np; ++q) m = fmax(m, c[q]);
    if (m > bv || (m == bv && i < bi)) { bv = m; bi = i; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
  }
  return bi;
}

__global__ void pick_kernel(int np, int npair, int G, int lp, int method, double fg, double lfg, double vmin,
                            const Gather* gs, const double* ml, const double* cr0, double* cr_pre, double* dc,
                            double* res, int* status, PickSeed seed) {
  extern __shared__ int psm[];
  const int gi = blockIdx.x;
  const int lane = threadIdx.x;
  if (seed.only) {  // re-pick pass: only the flagged gathers, whose status starts over
    if (!seed.only[gi]) return;
    if (lane == 0) status[gi] = 0;
    __syncwarp();
  }
  if (gs && gs[gi].valid <= 0) {  // side not computed for this shot
    if (lane == 0) res[gi] = 0.0 / 0.0;
    return;
  }
  const bool cert = seed.cert != nullptr;
  double mg = 1.0 / 0.0;  // smallest decision margin (certification)
  int* idx = psm;                  // 1-based column arrays, entry 0 unused
  int* dvmin = idx + (npair + 1);
  int* dvmax = dvmin + (npair + 1);
  int* chazhi = dvmax + (npair + 1);
  double* qj = (double*)(psm + 4 * (npair + 1));  // 16*(npair+1) bytes in: 8-byte aligned
  const double* mlg = ml + (size_t)gi * npair * np;
  auto col = [&](int i) { return mlg + (size_t)(i - 1) * np; };
  const int a = np, b = npair;
  // NaN columns are not supported (findpeaks semantics would need them)
  bool bad = false;
  for (int i = lane; i < np * npair; i += 32) bad |= isnan(mlg[i]);
  if (__any_sync(0xffffffffu, bad)) {
    if (lane == 0) {
      status[gi] = 1;
      if (seed.cert) seed.cert[gi] = 1;  // let the FP64 spectrum decide
    }
    return;
  }
  double* crp = cr_pre + (size_t)gi * npair;
  if (method != 1) {  // LHDispPick.m:8-9: plain argmax per column
    for (int i = 1; i <= b; ++i) {
      const int q = warp_argmax(col(i), 1, a, lane);
      if (cert) mg = fmin(mg, warp_top2_gap(col(i), 1, a, lane));
      if (lane == 0) crp[i - 1] = q + vmin;
    }
  } else {
    for (int i = lane; i <= b; i += 32) { idx[i] = 0; dvmin[i] = 0; dvmax[i] = 0; chazhi[i] = 1; qj[i] = 0.0 / 0.0; }
    __syncwarp();
    const double nanv = 0.0 / 0.0;
    int cur;
    if (seed.raw) {  // field variants: start at the global maximum of the unnormalised spectrum
      const double* rg = seed.raw + (size_t)gi * npair * np;
      lp = warp_colmax_argmax(rg, np, npair, lane);  // [~,ini] = max(max(mlr))
      cur = seed.value_from_raw ? warp_argmax(rg + (size_t)(lp - 1) * np, 1, a, lane)  // pickFDCValue.m:20
                                : warp_argmax(col(lp), 1, a, lane);
    } else {
      cur = warp_argmax(col(lp), 1, a, lane);  // pickFDC1.m:19
      if (cert) mg = fmin(mg, warp_top2_gap(col(lp), 1, a, lane));
    }
    if (lane == 0) idx[lp] = cur;
    for (int i = lp - 1; i >= 1; --i) {          // pickFDC1.m:21-77
      __syncwarp();
      const int prev = idx[i + 1];
      if (prev == a) {
        if (lane == 0) { idx[i] = a; dvmax[i] = dvmax[i + 1]; dvmin[i] = dvmin[i + 1]; qj[i] = nanv; }
        continue;
      }
      int vmx, vmn;
      if (prev > a - 3) vmx = a;
      else {
        const int q = first_local_min(col(i), prev, a, lane);
        vmx = q ? q + 1 : a;
        if (cert) mg = fmin(mg, warp_adjacent_gap(col(i), prev, q ? min(q + 1, a) : a, lane));
      }
      if (prev < 3) vmn = 1;
      else {
        const int q = last_local_min(col(i), prev, lane);
        vmn = q ? q : 1;
        if (cert) mg = fmin(mg, warp_adjacent_gap(col(i), q ? q - 1 : 1, prev, lane));
      }
      const double qi = (double)(vmx - vmn);
      const double qn = qj[i + 1];
      int newidx;
      if (qi > qn * lfg) {  // NaN compares false
        newidx = prev;
        vmx = dvmax[i + 1];
        vmn = dvmin[i + 1];
        if (lane == 0) { chazhi[i] = 0; }
      } else {
        newidx = warp_argmax(col(i), vmn, vmx, lane);
        if (cert) mg = fmin(mg, warp_top2_gap(col(i), vmn, vmx, lane));
      }
      __syncwarp();
      if (lane == 0) { idx[i] = newidx; dvmax[i] = vmx; dvmin[i] = vmn; qj[i] = (double)(vmx - vmn); }
    }
    for (int i = lp + 1; i <= b; ++i) {          // pickFDC1.m:79-128
      __syncwarp();
      const int prev = idx[i - 1];
      int vmx, vmn;
      if (prev > a - 3) vmx = a;
      else {
        const int q = first_local_min(col(i), prev, a, lane);
        vmx = q ? q + 1 : a;
        if (cert) mg = fmin(mg, warp_adjacent_gap(col(i), prev, q ? min(q + 1, a) : a, lane));
      }
      if (prev < 3) vmn = 1;
      else {
        const int q = last_local_min(col(i), prev, lane);
        vmn = q ? q : 1;
        if (cert) mg = fmin(mg, warp_adjacent_gap(col(i), q ? q - 1 : 1, prev, lane));
      }
      const double qi = (double)(vmx - vmn);
      const double qp = qj[i - 1];
      int newidx;
      if (qi > fg * qp) {
        newidx = prev;
        vmx = dvmax[i - 1];
        vmn = dvmin[i - 1];
        if (lane == 0) chazhi[i] = 0;
      } else {
        newidx = warp_argmax(col(i), vmn, vmx, lane);
        if (cert) mg = fmin(mg, warp_top2_gap(col(i), vmn, vmx, lane));
      }
      __syncwarp();
      if (lane == 0) { idx[i] = newidx; dvmax[i] = vmx; dvmin[i] = vmn; qj[i] = (double)(vmx - vmn); }
    }
    __syncwarp();
    if (lane == 0) {  // pickFDC1.m:129-131: linear interp over held columns, then nearest + extrap
      int nq = 0, qfirst = 0, qlast = 0;
      for (int i = 1; i <= b; ++i)
        if (chazhi[i] == 1) { if (!nq) qfirst = i; qlast = i; ++nq; }
      if (nq < 2) {
        status[gi] = 2;
      } else {
        int k0 = qfirst;
        for (int t = 1; t <= b; ++t) {
          double v;
          if (t <= qfirst) v = idx[qfirst];
          else if (t >= qlast) v = idx[qlast];
          else {
            while (true) {  // advance to the retained sample interval [k0, k1] containing t
              int k1 = k0 + 1;
              while (chazhi[k1] != 1) ++k1;
              if (t < k1) break;
              k0 = k1;
            }
            int k1 = k0 + 1;
            while (chazhi[k1] != 1) ++k1;
            if (t == k0) v = idx[k0];
            else {
              const double x0 = k0, x1 = k1, y0 = idx[k0], y1 = idx[k1];
              v = y0 + ((double)t - x0) * ((y1 - y0) / (x1 - x0));
            }
          }
          crp[t - 1] = v + vmin;
        }
      }
    }
  }
  __syncwarp();
  if (lane == 0 && status[gi] == 0) {
    // misfit over rows r0..r1 (1-based; all rows unless a field variant trims them), mean([]) = NaN
    const int r0 = seed.r0 > 0 ? seed.r0 : 1, r1 = seed.r0 > 0 ? b - seed.r1_from_end : b;
    double s = 0.0;
    for (int i = 0; i < b; ++i) {
      const double d = crp[i] - cr0[(size_t)gi * npair + i];
      dc[(size_t)gi * npair + i] = d;
      if (i + 1 >= r0 && i + 1 <= r1) s += d * d;
    }
    res[gi] = r1 >= r0 ? s / (r1 - r0 + 1) : 0.0 / 0.0;
  }
  if (cert && lane == 0 && !(mg >= seed.delta)) {  // a decision within delta (or NaN): recompute in FP64
    seed.cert[gi] = 1;
    if (seed.cert_count) atomicAdd(seed.cert_count, 1ull);
  }
}

int pick_batch(int np, int npair, int G, int ini, int method, double vmin, const Gather* d_gath, const double* ml,
               const double* cr0, double* cr_pre, double* dc, double* res, int* status, cudaStream_t st,
               PickSeed seed) {
  SWD_CHECK(seed.raw || (ini >= 1 && ini <= npair), "ini (%d) must lie in 1..npair (%d)", ini, npair);
  const size_t smem = (size_t)(npair + 1) * (4 * sizeof(int) + sizeof(double));
  if (!seed.only) SWD_CUDA(cudaMemsetAsync(status, 0, G * sizeof(int), st));
  pick_kernel<<<G, 32, smem, st>>>(np, npair, G, ini, method, 2.0, 4.0, vmin, d_gath, ml, cr0, cr_pre, dc, res,
                                   status, seed);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}

// ------------------------------------------------------------------ SoftMax gradient + adjoint Radon

__global__ void __launch_bounds__(256) softmax_adjoint_kernel(RadonGeom g, const Gather* gs,
                                                              const double* __restrict__ mlraw,
                                                              const double2* __restrict__ MM,
                                                              const double* __restrict__ dc,
                                                              const double* __restrict__ space_m, double beta,
                                                              const double2* __restrict__ K, double2* Gx,
                                                              const double* __restrict__ pick, double pick_off,
                                                              int limband) {
  extern __shared__ double2 sgm[];
  __shared__ double red[33];
  const int f = blockIdx.x, gi = blockIdx.y;
  const Gather gg = gs[gi];
  if (gg.valid <= 0) return;
  const size_t col = (size_t)gi * g.npair + f;
  const double* mr = mlraw + col * g.np;
  // Weights over p.  ADWDgrad_1.m:22-23: E = softmax(beta * mlr.^(1/40)), max-shifted in FP64.
  // ADWDgrad_norm.m:22-23 (pick != null): E = normpdf(1:np, cr, 16) around the pick cr =
  // cr_pre - vmin (paddingMl_norm.m:5-7), not normalised.
  // ADWDgradlimband.m:20-24 (limband): P = mlr.^beta normalised by its column sum S; the
  // derivative weights are N = beta*P.^(beta-1)/S, the mean is taken with N1 = P/S.
  double zmax = 0.0, se = 1.0, mu = 0.0;
  if (pick) {
    mu = pick[(size_t)gi * g.npair + f] - pick_off;
  } else if (limband) {
    se = 0.0;
    for (int p = threadIdx.x; p < g.np; p += blockDim.x) se += pow(mr[p], beta);
    se = block_sum(se, red);
  } else {
    zmax = -1.0 / 0.0;
    for (int p = threadIdx.x; p < g.np; p += blockDim.x) zmax = fmax(zmax, pow(mr[p], 1.0 / 40.0) * beta);
    zmax = block_max(zmax, red);
    se = 0.0;
    for (int p = threadIdx.x; p < g.np; p += blockDim.x) se += exp(pow(mr[p], 1.0 / 40.0) * beta - zmax);
    se = block_sum(se, red);
  }
  auto weight = [&](int p) -> double {
    if (limband) return (beta * pow(pow(mr[p], beta), beta - 1.0)) / se;
    if (pick) {
      const double z = ((double)(p + 1) - mu) / 16.0;
      return exp(-0.5 * (z * z)) / (2.5066282746310002 * 16.0);  // sqrt(2*pi) * sigma
    }
    return exp(pow(mr[p], 1.0 / 40.0) * beta - zmax) / se;
  };
  double sm = 0.0;
  for (int p = threadIdx.x; p < g.np; p += blockDim.x) {
    const double E = limband ? pow(mr[p], beta) / se : weight(p);  // N1 for limband
    const double s = space_m ? space_m[(size_t)f * g.np + p] : (double)(p + 1);
    sm += s * E;
  }
  sm = block_sum(sm, red);
  double d = dc[(size_t)gi * g.npair + f];
  if (d == 0.0) d = 1.0;  // grad_output(grad_output==0)=1 (ADWDgrad_1.m:26)
  for (int p = threadIdx.x; p < g.np; p += blockDim.x) {
    const double E = weight(p);
    const double s = space_m ? space_m[(size_t)f * g.np + p] : (double)(p + 1);
    const double gml = (((E * s - sm * E) * 2.0) * d) * (limband ? 1.0 : beta);   // :28-31 (limband :29-31)
    const double2 m = MM[col * g.np + p];
    const double mag = hypot(m.x, m.y);
    double2 ph = make_double2(m.x / mag, m.y / mag);              // :32-33
    if (isnan(ph.x) || isnan(ph.y)) ph = make_double2(0.0, 0.0);
    sgm[p] = make_double2(ph.x * gml, ph.y * gml);
  }
  __syncthreads();
  // G(x) = sum_p conj(K_f(p,x)) gm(p)   (:36-40)
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double2* Kf = K + (size_t)f * g.offset * g.np;
  for (int x = wp; x < gg.noff; x += nw) {
    double re = 0.0, im = 0.0;
    for (int p = lane; p < g.np; p += 32) {
      const double2 k = Kf[(size_t)x * g.np + p];
      const double2 v = sgm[p];
      re += k.x * v.x + k.y * v.y;
      im += k.x * v.y - k.y * v.x;
    }
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_xor_sync(0xffffffffu, re, o);
      im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0) Gx[col * g.offset + x] = make_double2(re, im);
  }
}

int softmax_adjoint(const RadonGeom& g, const Gather* d_gath, int G, const double* mlraw, const double2* MM,
                    const double* dc, const double* space_m, double beta, const double2* K, double2* Gx,
                    cudaStream_t st, const double* pick, double pick_off, int limband) {
  dim3 grid(g.npair, G);
  const size_t smem = (size_t)g.np * sizeof(double2);
  if (smem > 48 * 1024)
    SWD_CUDA(cudaFuncSetAttribute(softmax_adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  softmax_adjoint_kernel<<<grid, 256, smem, st>>>(g, d_gath, mlraw, MM, dc, space_m, beta, K, Gx, pick, pick_off,
                                                  limband);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}

// ------------------------------------------------------------------ inverse DFT into the adjoint source

constexpr int kIdftT = 64;

// TA / TB (nullable, [ntd]): sum_i w_i exp(+i th_i t) over the taper bins below lf / above nf
// (ADWDgradlimband.m:41-48), which carry copies of the bins lf / nf scaled by w_i.
template <typename O>
__global__ void __launch_bounds__(256) idft_kernel(RadonGeom g, const Gather* gs, const double2* __restrict__ Gx,
                                                   const double2* __restrict__ W, O* out, size_t ostride,
                                                   const double2* __restrict__ TA, const double2* __restrict__ TB) {
  extern __shared__ double2 sg[];  // [npair][32]
  const Gather gg = gs[blockIdx.z];
  if (gg.valid <= 0) return;
  const int x0 = blockIdx.y * 32;
  if (x0 >= gg.noff) return;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int x = x0 + lane;
  for (int i = threadIdx.x; i < g.npair * 32; i += blockDim.x) {
    const int f = i >> 5, xx = x0 + (i & 31);
    sg[i] = xx < gg.noff ? Gx[((size_t)blockIdx.z * g.npair + f) * g.offset + xx] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const int t0 = blockIdx.x * kIdftT;
  const double inv = (double)g.ccn;
  // ADWDgrad_1.m:76 writes the left side without its source trace (x = 0)
  const bool write = x < gg.noff && !(gg.side == 1 && x == 0);
  const int colx = gg.c0 + gg.dir * x;
  O* o = out + (size_t)gg.shot * ostride;
  for (int tt = wp; tt < kIdftT; tt += 8) {
    const int t = t0 + tt;
    if (t >= g.nt) break;
    double acc = 0.0;
    for (int f = 0; f < g.npair; ++f) {
      const double2 w = W[(size_t)f * g.ntd + t];  // exp(-i th); ifft uses exp(+i th) = conj(w)
      const double2 v = sg[f * 32 + lane];
      acc += v.x * w.x + v.y * w.y;
    }
    if (TA) {
      const double2 vl = sg[lane], vn = sg[(g.npair - 1) * 32 + lane], a = TA[t], b = TB[t];
      acc += (vl.x * a.x - vl.y * a.y) + (vn.x * b.x - vn.y * b.y);
    }
    if (write) o[(size_t)t * g.ng + colx] = (O)(acc / inv);
  }
}

template <typename O>
int radon_idft_scatter(const RadonGeom& g, const Gather* d_gath, int G, const double2* Gx, const double2* W, O* out,
                       size_t ostride, cudaStream_t st, const double2* TA, const double2* TB) {
  SWD_CHECK(g.ccn >= g.nt, "ADWDgrad_1 needs ccn = fix(1/df/dt) (%d) >= nt (%d)", g.ccn, g.nt);
  dim3 grid((g.nt + kIdftT - 1) / kIdftT, (g.offset + 31) / 32, G);
  const size_t smem = (size_t)g.npair * 32 * sizeof(double2);
  if (smem > 48 * 1024)
    SWD_CUDA(cudaFuncSetAttribute(idft_kernel<O>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  idft_kernel<O><<<grid, 256, smem, st>>>(g, d_gath, Gx, W, out, ostride, TA, TB);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}
template int radon_idft_scatter<float>(const RadonGeom&, const Gather*, int, const double2*, const double2*, float*,
                                       size_t, cudaStream_t, const double2*, const double2*);
template int radon_idft_scatter<double>(const RadonGeom&, const Gather*, int, const double2*, const double2*,
                                        double*, size_t, cudaStream_t, const double2*, const double2*);

}  // namespace swd

// ====================================================================== C ABI (host pointers)

using namespace swd;

extern "C" {

int swd_radon_sizes(const swd_radon_params* p, int* np_out, int* npair, int* lf, int* nf, int* ccn) {
  clear_error();
  RadonGeom g{};
  SWD_TRY(radon_geom(p, g));
  if (np_out) *np_out = g.np;
  if (npair) *npair = g.npair;
  if (lf) *lf = g.lf;
  if (nf) *nf = g.nf;
  if (ccn) *ccn = g.ccn;
  return SWD_OK;
}

int swd_radon(const swd_radon_params* p, int side, int is, const double* seismo, double* ml, double* ml_raw,
              double* mm, int* data_len, int* uxtpos) {
  clear_error();
  RadonGeom g{};
  SWD_TRY(radon_geom(p, g));
  SWD_CHECK(side == 0 || side == 1, "side must be 0 (right, RTrAD) or 1 (left, RTlAD)");
  SWD_CHECK(seismo && ml, "null seismo/ml");
  Gather gg = make_gather(g, is, side, 0, 1 << 30, 0);
  SWD_CHECK(gg.noff >= 1 && gg.c0 >= 0 && gg.c0 < g.ng && gg.c0 + gg.dir * (gg.noff - 1) >= 0 &&
                gg.c0 + gg.dir * (gg.noff - 1) < g.ng,
            "shot %d has an empty or out-of-range %s window", is, side ? "left" : "right");
  gg.valid = 1;
  const size_t nsz = (size_t)g.nt * g.ng, spec = (size_t)g.npair * g.np;
  SlabPlan sp;
  const size_t o_seis = sp.add(nsz * sizeof(double)), o_seis_t = sp.add(nsz * sizeof(double));
  const size_t o_W = sp.add((size_t)g.npair * g.ntd * sizeof(double2));
  const size_t o_K = sp.add((size_t)g.npair * g.offset * g.np * sizeof(double2));
  const size_t o_D = sp.add((size_t)g.npair * g.offset * sizeof(double2));
  const size_t o_MM = sp.add(spec * sizeof(double2)), o_raw = sp.add(spec * sizeof(double));
  const size_t o_ml = sp.add(spec * sizeof(double)), o_g = sp.add(sizeof(Gather));
  DevBuf slab;
  SWD_TRY(slab.alloc(sp.bytes));
  double* d_seis = SlabPlan::at<double>(slab, o_seis);
  double* d_seis_t = SlabPlan::at<double>(slab, o_seis_t);
  double2* d_W = SlabPlan::at<double2>(slab, o_W);
  double2* d_K = SlabPlan::at<double2>(slab, o_K);
  double2* d_D = SlabPlan::at<double2>(slab, o_D);
  double2* d_MM = SlabPlan::at<double2>(slab, o_MM);
  double* d_raw = SlabPlan::at<double>(slab, o_raw);
  double* d_ml = SlabPlan::at<double>(slab, o_ml);
  Gather* d_g = SlabPlan::at<Gather>(slab, o_g);
  cudaStream_t st = 0;
  SWD_CUDA(cudaMemcpyAsync(d_seis, seismo, nsz * sizeof(double), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(d_g, &gg, sizeof(Gather), cudaMemcpyHostToDevice, st));
  SWD_TRY(transpose<double, double>(d_seis, 0, d_seis_t, 0, 1, g.ng, g.nt, st));
  SWD_TRY(radon_tables(g, d_W, d_K, st));
  SWD_TRY(radon_dft<double>(g, d_g, 1, d_seis_t, 0, d_W, d_D, st));
  SWD_TRY(radon_contract(g, d_g, 1, d_K, d_D, d_MM, d_raw, d_ml, st));
  SWD_CUDA(cudaMemcpyAsync(ml, d_ml, spec * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (ml_raw) SWD_CUDA(cudaMemcpyAsync(ml_raw, d_raw, spec * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (mm) {  // np x nf interleaved complex, columns before lf are zero (RTrAD.m:22)
    std::memset(mm, 0, (size_t)(g.lf - 1) * g.np * 2 * sizeof(double));
    SWD_CUDA(cudaMemcpyAsync(mm + (size_t)(g.lf - 1) * g.np * 2, d_MM, spec * sizeof(double2),
                             cudaMemcpyDeviceToHost, st));
  }
  SWD_CUDA(cudaStreamSynchronize(st));
  if (data_len) *data_len = gg.noff;
  if (uxtpos) {  // RTrAD.m:33 / RTlAD.m:34, ascending 1-based
    for (int x = 0; x < gg.noff; ++x) {
      const int c = gg.c0 + gg.dir * x + 1;
      uxtpos[side == 0 ? x : gg.noff - 1 - x] = c;
    }
  }
  return SWD_OK;
}

int swd_pick(const double* ml, int np_, int npair, double vmin, const double* cr_0, int method, int ini, double* res,
             double* cr_pre) {
  clear_error();
  SWD_CHECK(ml && cr_0 && cr_pre && np_ >= 1 && npair >= 1, "bad pick arguments");
  const size_t spec = (size_t)np_ * npair;
  DevBuf b;
  SWD_TRY(b.alloc((spec + 3 * (size_t)npair + 1) * sizeof(double) + sizeof(int)));
  double* d_ml = b.as<double>();
  double* d_cr0 = d_ml + spec;
  double* d_crp = d_cr0 + npair;
  double* d_dc = d_crp + npair;
  double* d_res = d_dc + npair;
  int* d_st = (int*)(d_res + 1);
  cudaStream_t st = 0;
  SWD_CUDA(cudaMemcpyAsync(d_ml, ml, spec * sizeof(double), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(d_cr0, cr_0, npair * sizeof(double), cudaMemcpyHostToDevice, st));
  SWD_TRY(pick_batch(np_, npair, 1, ini, method, vmin, nullptr, d_ml, d_cr0, d_crp, d_dc, d_res, d_st, st));
  int status = 0;
  SWD_CUDA(cudaMemcpyAsync(&status, d_st, sizeof(int), cudaMemcpyDeviceToHost, st));
  SWD_CUDA(cudaMemcpyAsync(cr_pre, d_crp, npair * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (res) SWD_CUDA(cudaMemcpyAsync(res, d_res, sizeof(double), cudaMemcpyDeviceToHost, st));
  SWD_CUDA(cudaStreamSynchronize(st));
  if (status == 1) { set_error("NaN in the dispersion spectrum"); return SWD_ERR_NUMERIC; }
  if (status == 2) { set_error("interp1 needs at least two retained picks (pickFDC1.m:129)"); return SWD_ERR_NUMERIC; }
  return SWD_OK;
}

int swd_pick_field(const double* ml, const double* ml_raw, int np_, int npair, double vmin, const double* cr_0,
                   int method, int variant, double* res, double* cr_pre) {
  clear_error();
  SWD_CHECK(ml && ml_raw && cr_0 && cr_pre && np_ >= 1 && npair >= 1, "bad pick arguments");
  SWD_CHECK(variant == 1 || variant == 2, "variant must be 1 (outcrop) or 2 (QadimahFault)");
  const size_t spec = (size_t)np_ * npair;
  DevBuf b;
  SWD_TRY(b.alloc((2 * spec + 3 * (size_t)npair + 1) * sizeof(double) + sizeof(int)));
  double* d_ml = b.as<double>();
  double* d_raw = d_ml + spec;
  double* d_cr0 = d_raw + spec;
  double* d_crp = d_cr0 + npair;
  double* d_dc = d_crp + npair;
  double* d_res = d_dc + npair;
  int* d_st = (int*)(d_res + 1);
  cudaStream_t st = 0;
  SWD_CUDA(cudaMemcpyAsync(d_ml, ml, spec * sizeof(double), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(d_raw, ml_raw, spec * sizeof(double), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(d_cr0, cr_0, npair * sizeof(double), cudaMemcpyHostToDevice, st));
  PickSeed seed;
  seed.raw = d_raw;
  seed.value_from_raw = variant == 1;  // pickFDCValue seeds from mlr; pickFDC1 from ml
  seed.r0 = variant == 1 ? 15 : 50;    // misfit rows 15:end-15 / 50:end-30
  seed.r1_from_end = variant == 1 ? 15 : 30;
  SWD_TRY(pick_batch(np_, npair, 1, 1, variant == 2 ? 1 : method, vmin, nullptr, d_ml, d_cr0, d_crp, d_dc, d_res,
                     d_st, st, seed));
  int status = 0;
  SWD_CUDA(cudaMemcpyAsync(&status, d_st, sizeof(int), cudaMemcpyDeviceToHost, st));
  SWD_CUDA(cudaMemcpyAsync(cr_pre, d_crp, npair * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (res) SWD_CUDA(cudaMemcpyAsync(res, d_res, sizeof(double), cudaMemcpyDeviceToHost, st));
  SWD_CUDA(cudaStreamSynchronize(st));
  if (status == 1) { set_error("NaN in the dispersion spectrum"); return SWD_ERR_NUMERIC; }
  if (status == 2) { set_error("interp1 needs at least two retained picks (pickFDC1.m:129)"); return SWD_ERR_NUMERIC; }
  return SWD_OK;
}

}  // extern "C"

// each trace (a column of the MATLAB nt x ng array, contiguous) divided by its largest magnitude
__global__ void norm_trace_kernel(const double* __restrict__ in, double* __restrict__ out, int nt) {
  __shared__ unsigned long long wm[32];
  const double* c = in + (size_t)blockIdx.x * nt;
  unsigned long long m = 0;
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    const double v = fabs(c[t]);
    if (!isnan(v)) m = max(m, (unsigned long long)__double_as_longlong(v));
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : 0ull;
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) wm[0] = m;
  }
  __syncthreads();
  const double d = __longlong_as_double((long long)wm[0]);
  for (int t = threadIdx.x; t < nt; t += blockDim.x) out[(size_t)blockIdx.x * nt + t] = c[t] / d;
}

extern "C" int swd_norm_trace(const double* data_in, int nt, int ng, double* data_out) {
  clear_error();
  SWD_CHECK(data_in && data_out && nt >= 1 && ng >= 1, "bad norm_trace arguments");
  const size_t n = (size_t)nt * ng;
  DevBuf b;
  SWD_TRY(b.alloc(2 * n * sizeof(double)));
  cudaStream_t st = 0;
  SWD_CUDA(cudaMemcpyAsync(b.p, data_in, n * sizeof(double), cudaMemcpyHostToDevice, st));
  norm_trace_kernel<<<ng, 256, 0, st>>>(b.as<double>(), b.as<double>() + n, nt);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  SWD_CUDA(cudaMemcpyAsync(data_out, b.as<double>() + n, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  SWD_CUDA(cudaStreamSynchronize(st));
  return SWD_OK;
}

// max |x| over n values, NaN skipped as MATLAB's max skips it: non-negative doubles order as their
// bit patterns, so an atomic max on the bits of |x| finds it (0 when every value is NaN or 0).
__global__ void maxabs_kernel(const double* __restrict__ x, size_t n, unsigned long long* out) {
  unsigned long long m = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double v = fabs(x[i]);
    if (!isnan(v)) m = max(m, (unsigned long long)__double_as_longlong(v));
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}
__global__ void scale_by_kernel(double* x, size_t n, const unsigned long long* m) {
  const double d = __longlong_as_double((long long)*m);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = x[i] / d;  // 0/0 = NaN when the array is all zero, as in MATLAB
}
// x ./ max(abs(x(:))) in place (fieldexamples/outcrop/core/ADWDgrad_1.m:79); m: one device word
static int divide_by_maxabs(double* x, size_t n, unsigned long long* m, cudaStream_t st) {
  SWD_CUDA(cudaMemsetAsync(m, 0, sizeof(unsigned long long), st));
  const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 1184);
  maxabs_kernel<<<blocks, 256, 0, st>>>(x, n, m);
  scale_by_kernel<<<blocks, 256, 0, st>>>(x, n, m);
  count_launch(2);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}

// ADWDgrad_1 (mode 0), ADWDgrad_norm (mode 1, picks cr_r / cr_l) or ADWDgradlimband (mode 2) of one
// shot; maxnorm divides the adjoint source by its largest magnitude (the field-data ADWDgrad_1).
static int adwdgrad_impl(const swd_radon_params* p, int ns, int is, int w, double soft_arg_norm,
                         const double* grad_output_r, const double* grad_output_l, const double* space_m,
                         const double* mm_r, const double* ml_raw_r, const double* mm_l, const double* ml_raw_l,
                         const double* cr_r, const double* cr_l, int mode, double* a_data_res, bool maxnorm = false) {
  const bool gauss = mode == 1;
  RadonGeom g{};
  SWD_TRY(radon_geom(p, g));
  SWD_CHECK(a_data_res, "null a_data_res");
  SWD_CHECK(g.ccn >= g.nt, "ADWDgrad_1 needs ccn = fix(1/df/dt) (%d) >= nt (%d)", g.ccn, g.nt);
  // ADWDgradlimband.m:41-48 writes bins lf-25 .. nf+25 (1-based); the first must exist
  SWD_CHECK(mode != 2 || g.lf - 25 >= 1, "ADWDgradlimband needs lf - 25 >= 1 (lf = %d)", g.lf);
  Gather gg[2];
  const double* mm[2] = {mm_r, mm_l};
  const double* raw[2] = {ml_raw_r, ml_raw_l};
  const double* go[2] = {grad_output_r, grad_output_l};
  const double* cr[2] = {cr_r, cr_l};
  for (int s = 0; s < 2; ++s) {
    gg[s] = make_gather(g, is, s, 0, ns, w);
    if (gg[s].valid) {
      SWD_CHECK(gg[s].valid == 1, "shot %d: %s window is empty", is, s ? "left" : "right");
      SWD_CHECK(mm[s] && raw[s] && go[s], "missing saved state for the %s side", s ? "left" : "right");
      SWD_CHECK(!gauss || cr[s], "missing picks cr_%s for the %s side", s ? "l" : "r", s ? "left" : "right");
    }
  }
  const size_t spec = (size_t)g.npair * g.np, nsz = (size_t)g.nt * g.ng;
  SlabPlan sp;
  const size_t o_max = sp.add(maxnorm ? sizeof(unsigned long long) : 0);
  const size_t o_cr = sp.add(gauss ? 2 * (size_t)g.npair * sizeof(double) : 0);
  const size_t o_W = sp.add((size_t)g.npair * g.ntd * sizeof(double2));
  const size_t o_K = sp.add((size_t)g.npair * g.offset * g.np * sizeof(double2));
  const size_t o_MM = sp.add(2 * spec * sizeof(double2)), o_raw = sp.add(2 * spec * sizeof(double));
  const size_t o_dc = sp.add(2 * (size_t)g.npair * sizeof(double));
  const size_t o_Gx = sp.add(2 * (size_t)g.npair * g.offset * sizeof(double2));
  const size_t o_out = sp.add(nsz * sizeof(double)), o_out_t = sp.add(nsz * sizeof(double));
  const size_t o_g = sp.add(2 * sizeof(Gather));
  const size_t o_sm = sp.add(space_m ? spec * sizeof(double) : 0);
  const size_t o_tab = sp.add(mode == 2 ? 2 * (size_t)g.ntd * sizeof(double2) : 0);
  DevBuf slab;
  SWD_TRY(slab.alloc(sp.bytes));
  unsigned long long* d_max = SlabPlan::at<unsigned long long>(slab, o_max);
  double* d_cr = SlabPlan::at<double>(slab, o_cr);
  double2* d_W = SlabPlan::at<double2>(slab, o_W);
  double2* d_K = SlabPlan::at<double2>(slab, o_K);
  double2* d_MM = SlabPlan::at<double2>(slab, o_MM);
  double* d_raw = SlabPlan::at<double>(slab, o_raw);
  double* d_dc = SlabPlan::at<double>(slab, o_dc);
  double2* d_Gx = SlabPlan::at<double2>(slab, o_Gx);
  double* d_out = SlabPlan::at<double>(slab, o_out);
  double* d_out_t = SlabPlan::at<double>(slab, o_out_t);
  Gather* d_g = SlabPlan::at<Gather>(slab, o_g);
  double* d_sm = SlabPlan::at<double>(slab, o_sm);
  double2* d_tab = SlabPlan::at<double2>(slab, o_tab);
  cudaStream_t st = 0;
  if (mode == 2) {
    // taper tables: bins i = lf-25 .. lf-1 carry bin lf times (i-lf+25)/25, bins nf+1 .. nf+25
    // carry bin nf times (nf-i+25)/25; ifft(.., ccn) drops bins past ccn (ADWDgradlimband.m:41-50)
    std::vector<double2> tab(2 * (size_t)g.ntd);
    const double two_pi = 2.0 * 3.141592653589793;
    for (int t = 0; t < g.ntd; ++t) {
      double ar = 0, ai = 0, br = 0, bi = 0;
      for (int i = g.lf - 25; i <= g.lf - 1; ++i) {
        const double wgt = (double)(i - g.lf + 25) / 25.0;
        const double th = two_pi * (double)(((long long)(i - 1) * t) % g.ccn) / (double)g.ccn;
        ar += wgt * std::cos(th);
        ai += wgt * std::sin(th);
      }
      for (int i = g.nf + 1; i <= std::min(g.nf + 25, g.ccn); ++i) {
        const double wgt = (double)(g.nf - i + 25) / 25.0;
        const double th = two_pi * (double)(((long long)(i - 1) * t) % g.ccn) / (double)g.ccn;
        br += wgt * std::cos(th);
        bi += wgt * std::sin(th);
      }
      tab[t] = make_double2(ar, ai);
      tab[(size_t)g.ntd + t] = make_double2(br, bi);
    }
    SWD_CUDA(cudaMemcpy(d_tab, tab.data(), tab.size() * sizeof(double2), cudaMemcpyHostToDevice));
  }
  for (int s = 0; s < 2; ++s) {
    if (gg[s].valid != 1) continue;
    SWD_CUDA(cudaMemcpyAsync(d_MM + s * spec, mm[s] + (size_t)(g.lf - 1) * g.np * 2, spec * sizeof(double2),
                             cudaMemcpyHostToDevice, st));
    SWD_CUDA(cudaMemcpyAsync(d_raw + s * spec, raw[s], spec * sizeof(double), cudaMemcpyHostToDevice, st));
    SWD_CUDA(cudaMemcpyAsync(d_dc + s * g.npair, go[s], g.npair * sizeof(double), cudaMemcpyHostToDevice, st));
    if (gauss)
      SWD_CUDA(cudaMemcpyAsync(d_cr + s * g.npair, cr[s], g.npair * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  if (space_m) SWD_CUDA(cudaMemcpyAsync(d_sm, space_m, spec * sizeof(double), cudaMemcpyHostToDevice, st));
  gg[0].shot = 0;
  gg[1].shot = 0;
  SWD_CUDA(cudaMemcpyAsync(d_g, gg, 2 * sizeof(Gather), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemsetAsync(d_out, 0, nsz * sizeof(double), st));
  SWD_TRY(radon_tables(g, d_W, d_K, st));
  SWD_TRY(softmax_adjoint(g, d_g, 2, d_raw, d_MM, d_dc, space_m ? d_sm : nullptr, soft_arg_norm, d_K, d_Gx, st,
                          gauss ? d_cr : nullptr, 0.0, mode == 2));
  SWD_TRY(radon_idft_scatter<double>(g, d_g, 2, d_Gx, d_W, d_out, 0, st, mode == 2 ? d_tab : nullptr,
                                     mode == 2 ? d_tab + g.ntd : nullptr));
  if (maxnorm) SWD_TRY(divide_by_maxabs(d_out, nsz, d_max, st));
  // [nt][ng] -> MATLAB nt x ng
  SWD_TRY(transpose<double, double>(d_out, 0, d_out_t, 0, 1, g.nt, g.ng, st));
  SWD_CUDA(cudaMemcpyAsync(a_data_res, d_out_t, nsz * sizeof(double), cudaMemcpyDeviceToHost, st));
  SWD_CUDA(cudaStreamSynchronize(st));
  return SWD_OK;
}

extern "C" {

int swd_adwdgrad(const swd_radon_params* p, int ns, int is, int w, double soft_arg_norm, const double* grad_output_r,
                 const double* grad_output_l, const double* space_m, const double* mm_r, const double* ml_raw_r,
                 const double* mm_l, const double* ml_raw_l, double* a_data_res) {
  clear_error();
  return adwdgrad_impl(p, ns, is, w, soft_arg_norm, grad_output_r, grad_output_l, space_m, mm_r, ml_raw_r, mm_l,
                       ml_raw_l, nullptr, nullptr, 0, a_data_res);
}

int swd_adwdgrad_maxnorm(const swd_radon_params* p, int ns, int is, int w, double soft_arg_norm,
                         const double* grad_output_r, const double* grad_output_l, const double* space_m,
                         const double* mm_r, const double* ml_raw_r, const double* mm_l, const double* ml_raw_l,
                         double* a_data_res) {
  clear_error();
  return adwdgrad_impl(p, ns, is, w, soft_arg_norm, grad_output_r, grad_output_l, space_m, mm_r, ml_raw_r, mm_l,
                       ml_raw_l, nullptr, nullptr, 0, a_data_res, true);
}

int swd_adwdgrad_limband(const swd_radon_params* p, int ns, int is, int w, double soft_arg_norm,
                         const double* grad_output_r, const double* grad_output_l, const double* space_m,
                         const double* mm_r, const double* ml_raw_r, const double* mm_l, const double* ml_raw_l,
                         double* a_data_res) {
  clear_error();
  return adwdgrad_impl(p, ns, is, w, soft_arg_norm, grad_output_r, grad_output_l, space_m, mm_r, ml_raw_r, mm_l,
                       ml_raw_l, nullptr, nullptr, 2, a_data_res);
}

int swd_adwdgrad_norm(const swd_radon_params* p, int ns, int is, int w, double soft_arg_norm,
                      const double* grad_output_r, const double* grad_output_l, const double* space_m,
                      const double* mm_r, const double* ml_raw_r, const double* cr_r, const double* mm_l,
                      const double* ml_raw_l, const double* cr_l, double* a_data_res) {
  clear_error();
  return adwdgrad_impl(p, ns, is, w, soft_arg_norm, grad_output_r, grad_output_l, space_m, mm_r, ml_raw_r, mm_l,
                       ml_raw_l, cr_r, cr_l, 1, a_data_res);
}

}  // extern "C"
