// Elastic staggered-grid FD time steps (forward, adjoint + imaging) for B200.
//
// One launch advances every shot of a batch by one time step.  Each warp owns a
// strip of 30 output columns (lanes 1..30; lanes 0 and 31 carry the x halo)
// over a chunk of rows and streams down z, keeping the rows it still needs in
// registers: x neighbours come from warp shuffles, z neighbours from the
// previous/next row registers, and the next row's loads are issued one
// iteration ahead.  Velocity and stress updates, the damping taper (temp), the
// free-surface row, the source, receiver extraction and strain snapshots are
// fused into that single pass, so the state is read once and written once per
// step (ping-pong buffers).  This file must be compiled with -fmad=false: the
// arithmetic is written in exactly the order of the reference's Eigen
// expressions and no multiply-add may be contracted, which makes the FP32
// results bit-identical to the reference's single-precision MEX.
//
// Reference loops:  core/eigen_staggerfd_single.cpp:207-357 (forward),
//                   core/eigen_e2drtm_single.cpp:181-283 (adjoint + imaging).
#pragma once
#include "swd_common.cuh"

namespace swd {

constexpr int kStrip = 30;            // output columns per warp
constexpr unsigned kFull = 0xffffffffu;

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };

// Geometry of one padded grid plus the warp decomposition of a launch.
struct FdGeom {
  int NZ, NX, pitch;         // padded grid (nzbc x nxbc), row pitch in elements
  int nz, nx, nbc;           // model interior: rows pad_top+1.., cols nbc..
  int pad_top;               // free-surface row (1 for fd_order 22)
  int nt, nt_wf, nrec;       // time steps, snapshot interval, snapshots per shot
  int ng, gz, gx, dg;        // receivers (0-based padded coordinates)
  int n_strips, n_chunks, chunk;
  size_t field;              // NZ * pitch
};

template <typename T>
struct FwdArgs {
  FdGeom g;
  const typename Vec4<T>::type* m1;   // {temp, b, b1, 0}     [NZ][pitch]
  const typename Vec4<T>::type* m2;   // {ca, cl, cm1, 0}     [NZ][pitch]
  const T* in;                        // state at t   [shot][uu,ww,xx,zz,xz][NZ][pitch]
  T* out;                             // state at t+1
  const int2* src;                    // per shot (sz, sx), 0-based padded
  int src_type;                       // 1..5 as in core/staggerfd_eigen.m:126-136
  const T* s;                         // wavelet [nt]
  T dtx;
  T* seis_u;                          // [shot][nt][ng] (may be null)
  T* seis_w;                          // [shot][nt][ng] (may be null)
  T* snap;                            // [shot][nrec][NF][nz][nx] (may be null)
  int rec0;                           // snapshot it/nt_wf is stored at index it/nt_wf - rec0
  int n_shots;
};

template <typename T>
struct AdjArgs {
  FdGeom g;
  const typename Vec4<T>::type* m1;
  const typename Vec4<T>::type* m2;
  const T* in;
  T* out;
  const T* res;                       // adjoint source [shot][nt][ng]
  const T* snap;                      // forward strain snapshots [shot][nrec][NF][nz][nx]
  double* img;                        // [shot][cl,cm,illum][nz][nx]
  T dtx, dt;
  int rec0;                           // snapshot it/nt_wf is read from index it/nt_wf - rec0
  int n_shots;
};

template <typename T>
__device__ __forceinline__ T ldz(const T* f, int z, int x, const FdGeom& g, bool xin) {
  return (xin && z < g.NZ) ? f[(size_t)z * g.pitch + x] : T(0);
}
template <typename V>
__device__ __forceinline__ V ldv(const V* f, int z, int x, const FdGeom& g, bool xin) {
  V r;
  if (xin && z < g.NZ) {
    r = f[(size_t)z * g.pitch + x];
  } else {
    r.x = 0; r.y = 0; r.z = 0; r.w = 0;
  }
  return r;
}

// ---------------------------------------------------------------- forward

// uu at (z,x) after the velocity update and the source (eigen_staggerfd_single.cpp:225-226, 286-300).
template <typename T, typename V>
__device__ __forceinline__ T fwd_vel_u(int z, int x, bool xint, const FdGeom& g, T uu, T xx, T xx_r,
                                       T xz, T xz_u, const V& m1, int st, int2 sp, T sv) {
  T r = uu;
  if (xint && z >= 1 && z <= g.NZ - 2) r = m1.x * uu + m1.y * (((xx_r - xx) + xz) - xz_u);
  if (x == sp.y) {
    if (z == sp.x && (st == 2 || st == 3)) r = r + sv;
    if (z == sp.x - 1 && st == 2) r = r - sv;
  }
  return r;
}

// ww at (z,x) after the velocity update and the source (:227-228, 286-300).
template <typename T, typename V>
__device__ __forceinline__ T fwd_vel_w(int z, int x, bool xint, const FdGeom& g, T ww, T xz, T xz_l,
                                       T zz, T zz_d, const V& m1, int st, int2 sp, T sv) {
  T r = ww;
  if (xint && z >= 1 && z <= g.NZ - 2) r = m1.x * ww + m1.z * (((xz - xz_l) + zz_d) - zz);
  if (z == sp.x) {
    if (x == sp.y) {
      if (st == 5) r = sv;
      else if (st == 2 || st == 3) r = r + sv;
    } else if (x == sp.y + 1 && st == 2) {
      r = r + sv;
    }
  }
  return r;
}

template <typename T, int NF, int WPB>
__global__ void __launch_bounds__(WPB * 32)
fd_fwd_step(FwdArgs<T> a, int it) {
  using V = typename Vec4<T>::type;
  const FdGeom& g = a.g;
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * WPB + (threadIdx.x >> 5);
  const int strip = gw % g.n_strips;
  const int rest = gw / g.n_strips;
  const int chunk = rest % g.n_chunks;
  const int shot = rest / g.n_chunks;
  if (shot >= a.n_shots) return;  // whole warp
  const int x = strip * kStrip + lane;   // lane 0 is column x0-1 of x0 = 30*strip+1
  const bool xin = x < g.NX;
  const bool xint = x >= 1 && x <= g.NX - 2;
  const bool outl = lane >= 1 && lane <= kStrip && xint;
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const size_t F = g.field;
  const T* uu_i = a.in + (size_t)shot * 5 * F;
  const T* ww_i = uu_i + F;
  const T* xx_i = ww_i + F;
  const T* zz_i = xx_i + F;
  const T* xz_i = zz_i + F;
  T* uu_o = a.out + (size_t)shot * 5 * F;
  T* ww_o = uu_o + F;
  T* xx_o = ww_o + F;
  T* zz_o = xx_o + F;
  T* xz_o = zz_o + F;
  const int st = a.src_type;
  const int2 sp = a.src[shot];
  const T sv = a.s[it];
  const T dtx = a.dtx;
  const bool snap = a.snap != nullptr && (it % g.nt_wf) == 0;
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const bool ximg = x >= g.nbc && x < g.nbc + g.nx;
  int recj = -1;
  if (x >= g.gx && (x - g.gx) % g.dg == 0 && (x - g.gx) / g.dg < g.ng) recj = (x - g.gx) / g.dg;

  // prologue: rows zs-1 and zs
  const int za = zs - 1;
  T ww_a = ldz(ww_i, za, x, g, xin), xz_a = ldz(xz_i, za, x, g, xin), zz_a = ldz(zz_i, za, x, g, xin);
  V m1_a = ldv(a.m1, za, x, g, xin);
  T uu_c = ldz(uu_i, zs, x, g, xin), ww_c = ldz(ww_i, zs, x, g, xin), xx_c = ldz(xx_i, zs, x, g, xin);
  T zz_c = ldz(zz_i, zs, x, g, xin), xz_c = ldz(xz_i, zs, x, g, xin);
  V m1_c = ldv(a.m1, zs, x, g, xin);
  T wn_prev = fwd_vel_w(za, x, xint, g, ww_a, xz_a, __shfl_up_sync(kFull, xz_a, 1), zz_a, zz_c, m1_a, st, sp, sv);
  T un_cur = fwd_vel_u(zs, x, xint, g, uu_c, xx_c, __shfl_down_sync(kFull, xx_c, 1), xz_c, xz_a, m1_c, st, sp, sv);
  // row zs+1 and the stress materials of row zs
  T uu_n = ldz(uu_i, zs + 1, x, g, xin), ww_n = ldz(ww_i, zs + 1, x, g, xin);
  T xx_n = ldz(xx_i, zs + 1, x, g, xin), zz_n = ldz(zz_i, zs + 1, x, g, xin);
  T xz_n = ldz(xz_i, zs + 1, x, g, xin);
  V m1_n = ldv(a.m1, zs + 1, x, g, xin);
  V m2_c = ldv(a.m2, zs, x, g, xin);

  for (int k = zs; k < ze; ++k) {
    // prefetch row k+2 (and the stress materials of row k+1)
    const int kp = k + 2;
    T uu_p = ldz(uu_i, kp, x, g, xin), ww_p = ldz(ww_i, kp, x, g, xin);
    T xx_p = ldz(xx_i, kp, x, g, xin), zz_p = ldz(zz_i, kp, x, g, xin);
    T xz_p = ldz(xz_i, kp, x, g, xin);
    V m1_p = ldv(a.m1, kp, x, g, xin);
    V m2_p = ldv(a.m2, k + 1, x, g, xin);

    // velocities: ww at row k, uu at row k+1
    const T wn = fwd_vel_w(k, x, xint, g, ww_c, xz_c, __shfl_up_sync(kFull, xz_c, 1), zz_c, zz_n, m1_c, st, sp, sv);
    const T un_next = fwd_vel_u(k + 1, x, xint, g, uu_n, xx_n, __shfl_down_sync(kFull, xx_n, 1), xz_n, xz_c,
                                m1_n, st, sp, sv);
    // strains at row k (:302-306)
    const T un_l = __shfl_up_sync(kFull, un_cur, 1);
    const T wn_r = __shfl_down_sync(kFull, wn, 1);
    const T fux = un_cur - un_l;
    const T fuz = un_next - un_cur;
    const T bwx = wn_r - wn;
    const T bwz = wn - wn_prev;
    // stresses at row k (:334-336), source types 1/4 first (:286-298), free surface (:340)
    T xo = xx_c, zo = zz_c;
    if (k == sp.x && x == sp.y) {
      if (st == 1) { xo = xo + sv; zo = zo + sv; }
      else if (st == 4) { zo = zo + sv; }
    }
    const T te = m1_c.x;
    const T xxn = te * xo + (m2_c.x * fux + m2_c.y * bwz) * dtx;
    T zzn = te * zo + (m2_c.x * bwz + m2_c.y * fux) * dtx;
    const T xzn = te * xz_c + (m2_c.z * (fuz + bwx)) * dtx;
    if (k == g.pad_top) zzn = T(0);
    if (outl) {
      const size_t o = (size_t)k * g.pitch + x;
      uu_o[o] = un_cur;
      ww_o[o] = wn;
      xx_o[o] = xxn;
      zz_o[o] = zzn;
      xz_o[o] = xzn;
      if (k == g.gz && recj >= 0 && a.seis_w) {  // :342-345
        const size_t r = ((size_t)shot * g.nt + it) * g.ng + recj;
        a.seis_w[r] = wn;
        if (a.seis_u) a.seis_u[r] = un_cur;
      }
      if (snap && ximg && k >= z_img0 && k < z_img1) {  // :346-351
        const size_t plane = (size_t)g.nz * g.nx;
        T* sp0 = a.snap + ((size_t)shot * g.nrec + (it / g.nt_wf - a.rec0)) * NF * plane +
                 (size_t)(k - z_img0) * g.nx + (x - g.nbc);
        if (NF == 4) {
          sp0[0] = fux; sp0[plane] = fuz; sp0[2 * plane] = bwx; sp0[3 * plane] = bwz;
        } else {  // the adjoint needs fux, bwz and fuz+bwx only
          sp0[0] = fux; sp0[plane] = bwz; sp0[2 * plane] = fuz + bwx;
        }
      }
    }
    // rotate
    wn_prev = wn;
    un_cur = un_next;
    ww_c = ww_n; xx_c = xx_n; zz_c = zz_n; xz_c = xz_n; m1_c = m1_n;
    uu_n = uu_p; ww_n = ww_p; xx_n = xx_p; zz_n = zz_p; xz_n = xz_p; m1_n = m1_p;
    m2_c = m2_p;
  }
}

// ---------------------------------------------------------------- adjoint

template <typename T, int NF, int WPB>
__global__ void __launch_bounds__(WPB * 32)
fd_adj_step(AdjArgs<T> a, int it) {
  using V = typename Vec4<T>::type;
  const FdGeom& g = a.g;
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * WPB + (threadIdx.x >> 5);
  const int strip = gw % g.n_strips;
  const int rest = gw / g.n_strips;
  const int chunk = rest % g.n_chunks;
  const int shot = rest / g.n_chunks;
  if (shot >= a.n_shots) return;
  const int x = strip * kStrip + lane;
  const bool xin = x < g.NX;
  const bool xint = x >= 1 && x <= g.NX - 2;
  const bool outl = lane >= 1 && lane <= kStrip && xint;
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const size_t F = g.field;
  const T* uu_i = a.in + (size_t)shot * 5 * F;
  const T* ww_i = uu_i + F;
  const T* xx_i = ww_i + F;
  const T* zz_i = xx_i + F;
  const T* xz_i = zz_i + F;
  T* uu_o = a.out + (size_t)shot * 5 * F;
  T* ww_o = uu_o + F;
  T* xx_o = ww_o + F;
  T* zz_o = xx_o + F;
  T* xz_o = zz_o + F;
  const T dtx = a.dtx;
  const bool img = (it % g.nt_wf) == 0;
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const bool ximg = x >= g.nbc && x < g.nbc + g.nx;
  T inj = T(0);  // dt*res at this column if it holds a receiver (:238-242)
  bool has_rec = false;
  if (x >= g.gx && (x - g.gx) % g.dg == 0 && (x - g.gx) / g.dg < g.ng) {
    has_rec = true;
    inj = a.dt * a.res[((size_t)shot * g.nt + it) * g.ng + (x - g.gx) / g.dg];
  }

  // adjoint velocities (:182-187); du/dw are formed from products at each cell
  auto vel_u = [&](int z, T uu, T P1, T P1l, T P2, T P2l, T P3, T P3u, const V& m1) -> T {
    if (xint && z >= 1 && z <= g.NZ - 2) {
      const T du = ((P1 - P1l) + (P2 - P2l)) + (P3 - P3u);
      return m1.x * uu - m1.y * du;
    }
    return uu;
  };
  auto vel_w = [&](int z, T ww, T Q1d, T Q1, T Q2d, T Q2, T P3r, T P3, const V& m1) -> T {
    T r = ww;
    if (xint && z >= 1 && z <= g.NZ - 2) {
      const T dw = ((Q1d - Q1) + (Q2d - Q2)) + (P3r - P3);
      r = m1.x * ww - m1.z * dw;
    }
    if (has_rec && z == g.gz) r = r + inj;
    return r;
  };

  // prologue: rows zs-1 (a) and zs (c)
  const int za = zs - 1;
  T xx_a = ldz(xx_i, za, x, g, xin), zz_a = ldz(zz_i, za, x, g, xin), xz_a = ldz(xz_i, za, x, g, xin);
  T ww_a = ldz(ww_i, za, x, g, xin);
  V m1_a = ldv(a.m1, za, x, g, xin), m2_a = ldv(a.m2, za, x, g, xin);
  T xx_c = ldz(xx_i, zs, x, g, xin), zz_c = ldz(zz_i, zs, x, g, xin), xz_c = ldz(xz_i, zs, x, g, xin);
  T uu_c = ldz(uu_i, zs, x, g, xin), ww_c = ldz(ww_i, zs, x, g, xin);
  V m1_c = ldv(a.m1, zs, x, g, xin), m2_c = ldv(a.m2, zs, x, g, xin);
  const T P3a = m2_a.z * xz_a, Q1a = m2_a.y * xx_a, Q2a = m2_a.x * zz_a;
  T P1c = m2_c.x * xx_c, P2c = m2_c.y * zz_c, P3c = m2_c.z * xz_c;
  T Q1c = m2_c.y * xx_c, Q2c = m2_c.x * zz_c;
  T wn_prev = vel_w(za, ww_a, Q1c, Q1a, Q2c, Q2a, __shfl_down_sync(kFull, P3a, 1), P3a, m1_a);
  T un_cur = vel_u(zs, uu_c, P1c, __shfl_up_sync(kFull, P1c, 1), P2c, __shfl_up_sync(kFull, P2c, 1), P3c, P3a, m1_c);
  T xx_n = ldz(xx_i, zs + 1, x, g, xin), zz_n = ldz(zz_i, zs + 1, x, g, xin), xz_n = ldz(xz_i, zs + 1, x, g, xin);
  T uu_n = ldz(uu_i, zs + 1, x, g, xin), ww_n = ldz(ww_i, zs + 1, x, g, xin);
  V m1_n = ldv(a.m1, zs + 1, x, g, xin), m2_n = ldv(a.m2, zs + 1, x, g, xin);

  for (int k = zs; k < ze; ++k) {
    const int kp = k + 2;
    T xx_p = ldz(xx_i, kp, x, g, xin), zz_p = ldz(zz_i, kp, x, g, xin), xz_p = ldz(xz_i, kp, x, g, xin);
    T uu_p = ldz(uu_i, kp, x, g, xin), ww_p = ldz(ww_i, kp, x, g, xin);
    V m1_p = ldv(a.m1, kp, x, g, xin), m2_p = ldv(a.m2, kp, x, g, xin);

    const T P1n = m2_n.x * xx_n, P2n = m2_n.y * zz_n, P3n = m2_n.z * xz_n;
    const T Q1n = m2_n.y * xx_n, Q2n = m2_n.x * zz_n;
    const T wn = vel_w(k, ww_c, Q1n, Q1c, Q2n, Q2c, __shfl_down_sync(kFull, P3c, 1), P3c, m1_c);
    const T un_next = vel_u(k + 1, uu_n, P1n, __shfl_up_sync(kFull, P1n, 1), P2n, __shfl_up_sync(kFull, P2n, 1),
                            P3n, P3c, m1_n);
    // adjoint stresses at row k (:245-248), free surface (:270)
    const T un_r = __shfl_down_sync(kFull, un_cur, 1);
    const T wn_l = __shfl_up_sync(kFull, wn, 1);
    const T te = m1_c.x;
    const T xxn = te * xx_c - dtx * (un_r - un_cur);
    T zzn = te * zz_c - dtx * (wn - wn_prev);
    const T xzn = (te * xz_c - dtx * (un_next - un_cur)) - dtx * (wn - wn_l);
    if (k == g.pad_top) zzn = T(0);
    if (outl) {
      const size_t o = (size_t)k * g.pitch + x;
      uu_o[o] = un_cur;
      ww_o[o] = wn;
      xx_o[o] = xxn;
      zz_o[o] = zzn;
      xz_o[o] = xzn;
      if (img && ximg && k >= z_img0 && k < z_img1) {  // imaging condition (:274-279)
        const size_t plane = (size_t)g.nz * g.nx;
        const size_t cell = (size_t)(k - z_img0) * g.nx + (x - g.nbc);
        const T* s0 = a.snap + ((size_t)shot * g.nrec + (it / g.nt_wf - a.rec0)) * NF * plane + cell;
        T fx, bz, sg;
        if (NF == 4) {
          fx = s0[0]; bz = s0[3 * plane]; sg = s0[plane] + s0[2 * plane];
        } else {
          fx = s0[0]; bz = s0[plane]; sg = s0[2 * plane];
        }
        const T Fs = fx + bz;
        const T tcl = Fs * (xxn + zzn);
        const T tcm = T(2) * ((xxn * fx + zzn * bz) + T(0.5) * (xzn * sg));
        const T til = Fs * Fs;
        double* im = a.img + (size_t)shot * 3 * plane + cell;
        im[0] += (double)tcl;
        im[plane] += (double)tcm;
        im[2 * plane] += (double)til;
      }
    }
    wn_prev = wn;
    un_cur = un_next;
    P3c = P3n; Q1c = Q1n; Q2c = Q2n;
    xx_c = xx_n; zz_c = zz_n; xz_c = xz_n; ww_c = ww_n; m1_c = m1_n;
    xx_n = xx_p; zz_n = zz_p; xz_n = xz_p; uu_n = uu_p; ww_n = ww_p; m1_n = m1_p; m2_n = m2_p;
  }
}

}  // namespace swd
