// FD time steps with one CTA barrier per row ("lead" schedule).
//
// Same arithmetic, ring staging and CTA shapes as fd_smem.cuh; only the order of the work
// within a CTA differs.  The kernels in fd_smem.cuh compute the new velocities of row k
// (ww of row k, uu of row k+1), exchange them through shared memory behind a barrier, then
// compute the stresses of row k behind a second barrier.  Here iteration k computes the
// velocities one row ahead (ww of row k+1, uu of row k+2) into the next buffers while it
// computes the stresses of row k from velocities published by the previous iterations, so
// one barrier per row separates producers from consumers.  The stresses of row k need that
// row's old xx, zz, xz and materials at the thread's own column only; they are carried in
// registers from the iteration before, which lets row k's ring slot be refilled at once.
//
// Velocity buffers in shared memory: uu of row k in su[(k - zs) % D] (D buffers: rows k,
// k+1, k+2 live, one free), ww of row k in sw[(k - zs) & 1].  With the row loop unrolled by
// the even ring depth D these indices are compile-time constants.
//
// Reference loops:  core/eigen_staggerfd_single.cpp:207-357 (forward),
//                   core/eigen_e2drtm_single.cpp:181-283 (adjoint + imaging).
#pragma once
#include "fd_smem.cuh"

namespace swd {

template <typename T, int W, int C, int D, bool GB>
constexpr size_t lead_smem_bytes() {
  using R = SRow<T, 32 * W * C, GB>;
  return sizeof(R) * D + (D + 2) * R::kWin * sizeof(T);
}

// ---------------------------------------------------------------- forward

template <typename T, int NF, int W, int C, int D, bool GB, bool SNAP>
__global__ void __launch_bounds__(32 * W)
fd_fwd_lead(FwdArgs<T> a, int it) {
  if (cta_cancelled(a.cancel)) return;  // every thread of the CTA reaches this first
  static_assert(D >= 4 && D % 2 == 0, "rows k+1, k+2 in use, rows in flight, even depth for static slots");
  constexpr int NT = 32 * W;
  using R = SRow<T, NT * C, GB>;
  using V4 = typename Vec4<T>::type;
  constexpr int kCols = R::kCols, kWin = R::kWin;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* ring = reinterpret_cast<R*>(smem_raw);
  T* su = reinterpret_cast<T*>(ring + D);  // [D][kWin]
  T* sw = su + D * kWin;                    // [2][kWin]
  const unsigned ring_addr = (unsigned)__cvta_generic_to_shared(ring);
  const FdGeom& g = a.g;
  const int strip = blockIdx.x % g.n_strips;
  const int rest = blockIdx.x / g.n_strips;
  const int chunk = rest % g.n_chunks;
  const int shot = rest / g.n_chunks;
  const int tid = threadIdx.x;
  const int c0 = strip * kCols;
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const size_t F = g.field;
  const T* sbase = a.in + (size_t)shot * 5 * F;
  const int st = a.src_type;
  const int2 sp = a.src[shot];
  const T sv = a.s[it];
  const T dtx = a.dtx;
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  T* snap_base = SNAP ? a.snap + ((size_t)shot * g.nrec + (it / g.nt_wf - a.rec0)) * NF * plane : nullptr;
  int xl[C], x[C], recj[C];
  bool xint[C], s_w[C], s_wr[C], s_u[C], s_um[C], s_xz[C], snapc[C];
  T* ob[C];
  bool src_any = false, rec_any = false;
#pragma unroll
  for (int h = 0; h < C; ++h) {
    xl[h] = tid + 1 + h * NT;
    x[h] = c0 + xl[h];
    xint[h] = x[h] >= 1 && x[h] <= g.NX - 2;
    const bool sc = x[h] == sp.y, sr = x[h] == sp.y + 1;
    s_w[h] = sc && st != 1 && st != 4;
    s_wr[h] = sr && st == 2;
    s_u[h] = sc && (st == 2 || st == 3);
    s_um[h] = sc && st == 2;
    s_xz[h] = sc && (st == 1 || st == 4);
    src_any = src_any || sc || sr;
    recj[h] = (a.seis_w != nullptr && xint[h] && x[h] >= g.gx && (x[h] - g.gx) % g.dg == 0 &&
               (x[h] - g.gx) / g.dg < g.ng) ? (x[h] - g.gx) / g.dg : -1;
    rec_any = rec_any || recj[h] >= 0;
    snapc[h] = SNAP && xint[h] && x[h] >= g.nbc && x[h] < g.nbc + g.nx;
    ob[h] = a.out + (size_t)shot * 5 * F + (xint[h] ? x[h] : 0);
  }
  Stager<T, kCols, GB, NT> stg;
  stg.init(sbase, F, a.mat, a.mb, c0, zs - 1, g);

  auto vel_w = [&](bool inner, T ww, T xz, T xzl, T zz, T zzd, T te, T b1) -> T {
    return inner ? te * ww + b1 * (((xz - xzl) + zzd) - zz) : ww;
  };
  auto vel_u = [&](bool inner, T uu, T xx, T xxr, T xz, T xzu, T te, T b) -> T {
    return inner ? te * uu + b * (((xxr - xx) + xz) - xzu) : uu;
  };
  auto src_w = [&](int z, T r, bool here, bool right) -> T {
    if (z == sp.x) {
      if (here) r = (st == 5) ? sv : r + sv;
      else if (right) r = r + sv;
    }
    return r;
  };
  auto src_u = [&](int z, T r, bool here, bool minus) -> T {
    if (here && z == sp.x) r = r + sv;
    if (minus && z == sp.x - 1) r = r - sv;
    return r;
  };
  // ww at window column j of row z (rows Rz = z, Rd = z+1)
  auto ww_at = [&](const R& Rz, const R& Rd, int j, int z, bool inner) -> T {
    const auto b = bvals<T, GB>(Rz.mb, j, z, g, dtx);
    return vel_w(inner, Rz.f[1][j], Rz.f[4][j], Rz.f[4][j - 1], Rz.f[3][j], Rd.f[3][j], Rz.mat[j].x, b.y);
  };
  // uu at window column j of row z (rows Rz = z, Ru = z-1)
  auto uu_at = [&](const R& Rz, const R& Ru, int j, int z, bool inner) -> T {
    const auto b = bvals<T, GB>(Rz.mb, j, z, g, dtx);
    return vel_u(inner, Rz.f[0][j], Rz.f[2][j], Rz.f[2][j + 1], Rz.f[4][j], Ru.f[4][j], Rz.mat[j].x, b.x);
  };

  // prologue: rows zs-1 .. zs+D-2 in flight; rows zs-1, zs, zs+1 needed now
#pragma unroll
  for (int r = 0; r < D; ++r) {
    stg.issue(ring_addr + r * (unsigned)sizeof(R), zs - 1 + r, g);
    cp_async_commit();
  }
  cp_async_wait<D - 3>();
  cta_sync<W>();
  T wn_prev[C], wn_cur[C], un_cur[C], un_next[C];
  T a2[C], a3[C], a4[C];  // old xx, zz, xz of row k at the thread's column
  V4 am[C];               // materials of row k
  {
    const R& A = ring[0];   // row zs-1
    const R& B = ring[1];   // row zs
    const R& Cc = ring[2];  // row zs+1
    const bool in1 = zs + 1 <= g.NZ - 2;
#pragma unroll
    for (int h = 0; h < C; ++h) {
      const int j = xl[h];
      wn_prev[h] = ww_at(A, B, j, zs - 1, xint[h] && zs - 1 >= 1);
      un_cur[h] = uu_at(B, A, j, zs, xint[h]);
      wn_cur[h] = ww_at(B, Cc, j, zs, xint[h]);
      un_next[h] = uu_at(Cc, B, j, zs + 1, xint[h] && in1);
      if (src_any) {
        wn_prev[h] = src_w(zs - 1, wn_prev[h], s_w[h], s_wr[h]);
        un_cur[h] = src_u(zs, un_cur[h], s_u[h], s_um[h]);
        wn_cur[h] = src_w(zs, wn_cur[h], s_w[h], s_wr[h]);
        un_next[h] = src_u(zs + 1, un_next[h], s_u[h], s_um[h]);
      }
      su[j] = un_cur[h];
      su[kWin + j] = un_next[h];
      sw[j] = wn_cur[h];
      a2[h] = B.f[2][j];
      a3[h] = B.f[3][j];
      a4[h] = B.f[4][j];
      am[h] = B.mat[j];
    }
    if (tid == 0) {  // halo column c0: uu of rows zs and zs+1
      const bool hc = c0 == sp.y, ci = c0 >= 1 && c0 <= g.NX - 2;
      su[0] = src_u(zs, uu_at(B, A, 0, zs, ci), hc && (st == 2 || st == 3), hc && st == 2);
      su[kWin] = src_u(zs + 1, uu_at(Cc, B, 0, zs + 1, ci && in1), hc && (st == 2 || st == 3), hc && st == 2);
    }
    if (tid == NT - 1) {  // halo column c0+kCols+1: ww of row zs
      const int j = kCols + 1, xh = c0 + j;
      sw[j] = src_w(zs, ww_at(B, Cc, j, zs, xh >= 1 && xh <= g.NX - 2), xh == sp.y && st != 1 && st != 4,
                    xh == sp.y + 1 && st == 2);
    }
  }
  cta_sync<W>();  // prologue velocities published; row zs-1 no longer read
  stg.issue(ring_addr, zs - 1 + D, g);  // row zs+D-1 into row zs-1's slot
  cp_async_commit();

  // Row k sits in ring slot (u+1) % D, k+1 in (u+2) % D, k+2 in (u+3) % D; uu(k) in su[u % D],
  // ww(k) in sw[u & 1].
  for (int k0 = zs; k0 < ze; k0 += D)
#pragma unroll
  for (int u = 0; u < D; ++u) {
    const int k = k0 + u;
    if (k >= ze) break;
    cp_async_wait<D - 3>();  // row k+2 landed
    cta_sync<W>();           // ... and visible; velocities of rows <= k+1 published; row k's slot free
    stg.issue(ring_addr + ((u + 1) % D) * (unsigned)sizeof(R), k + D, g);
    cp_async_commit();
    const R& R1 = ring[(u + 2) % D];
    const R& R2 = ring[(u + 3) % D];
    const bool in1 = k + 1 <= g.NZ - 2, in2 = k + 2 <= g.NZ - 2;
    T* sw_n = sw + ((u + 1) & 1) * kWin;    // ww(k+1)
    T* su_n = su + ((u + 2) % D) * kWin;    // uu(k+2)
    const T* sw_c = sw + (u & 1) * kWin;    // ww(k)
    const T* su_c = su + (u % D) * kWin;    // uu(k)
    T wn_n[C], un_nn[C], b2[C], b3[C], b4[C];
    V4 bm[C];
    // velocities one row ahead: ww of row k+1, uu of row k+2
#pragma unroll
    for (int h = 0; h < C; ++h) {
      const int j = xl[h];
      wn_n[h] = ww_at(R1, R2, j, k + 1, xint[h] && in1);
      un_nn[h] = uu_at(R2, R1, j, k + 2, xint[h] && in2);
      if (src_any) {
        wn_n[h] = src_w(k + 1, wn_n[h], s_w[h], s_wr[h]);
        un_nn[h] = src_u(k + 2, un_nn[h], s_u[h], s_um[h]);
      }
      sw_n[j] = wn_n[h];
      su_n[j] = un_nn[h];
      b2[h] = R1.f[2][j];
      b3[h] = R1.f[3][j];
      b4[h] = R1.f[4][j];
      bm[h] = R1.mat[j];
    }
    if (tid == NT - 1) {  // halo column c0+kCols+1: ww of row k+1
      const int j = kCols + 1, xh = c0 + j;
      sw_n[j] = src_w(k + 1, ww_at(R1, R2, j, k + 1, xh >= 1 && xh <= g.NX - 2 && in1),
                      xh == sp.y && st != 1 && st != 4, xh == sp.y + 1 && st == 2);
    }
    if (tid == 0) {  // halo column c0: uu of row k+2
      const bool hc = c0 == sp.y;
      su_n[0] = src_u(k + 2, uu_at(R2, R1, 0, k + 2, c0 >= 1 && c0 <= g.NX - 2 && in2),
                      hc && (st == 2 || st == 3), hc && st == 2);
    }
    // stresses of row k from the published velocities (:302-306, :334-336, :340)
    const bool snap_row = SNAP && k >= z_img0 && k < z_img1;
#pragma unroll
    for (int h = 0; h < C; ++h) {
      const int j = xl[h];
      const T fux = un_cur[h] - su_c[j - 1];
      const T fuz = un_next[h] - un_cur[h];
      const T bwx = sw_c[j + 1] - wn_cur[h];
      const T bwz = wn_cur[h] - wn_prev[h];
      T xo = a2[h], zo = a3[h];
      if (src_any && s_xz[h] && k == sp.x) {
        if (st == 1) { xo = xo + sv; zo = zo + sv; }
        else { zo = zo + sv; }
      }
      const V4 m = am[h];
      const T te = m.x, ca = m.y, cl = m.z, cm1 = m.w;
      const T xxn = te * xo + (ca * fux + cl * bwz) * dtx;
      T zzn = te * zo + (ca * bwz + cl * fux) * dtx;
      const T xzn = te * a4[h] + (cm1 * (fuz + bwx)) * dtx;
      if (k == g.pad_top) zzn = T(0);
      if (xint[h]) {
        T* o = ob[h] + (size_t)k * g.pitch;
        o[0] = un_cur[h];
        o[F] = wn_cur[h];
        o[2 * F] = xxn;
        o[3 * F] = zzn;
        o[4 * F] = xzn;
      }
      if (rec_any && k == g.gz && recj[h] >= 0) {
        const size_t r = ((size_t)shot * g.nt + it) * g.ng + recj[h];
        a.seis_w[r] = wn_cur[h];
        if (a.seis_u) a.seis_u[r] = un_cur[h];
      }
      if (SNAP && snap_row && snapc[h]) {
        T* sp0 = snap_base + ((size_t)(k - z_img0) * g.nx + (x[h] - g.nbc));
        if (NF == 4) {
          sp0[0] = fux; sp0[plane] = fuz; sp0[2 * plane] = bwx; sp0[3 * plane] = bwz;
        } else {
          sp0[0] = fux; sp0[plane] = bwz; sp0[2 * plane] = fuz + bwx;
        }
      }
      wn_prev[h] = wn_cur[h];
      wn_cur[h] = wn_n[h];
      un_cur[h] = un_next[h];
      un_next[h] = un_nn[h];
      a2[h] = b2[h];
      a3[h] = b3[h];
      a4[h] = b4[h];
      am[h] = bm[h];
    }
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------- adjoint

template <typename T, int NF, int W, int C, int D, bool GB, bool IMG>
__global__ void __launch_bounds__(32 * W)
fd_adj_lead(AdjArgs<T> a, int it) {
  if (cta_cancelled(a.cancel)) return;  // every thread of the CTA reaches this first
  static_assert(D >= 4 && D % 2 == 0, "rows k+1, k+2 in use, rows in flight, even depth for static slots");
  constexpr int NT = 32 * W;
  using R = SRow<T, NT * C, GB>;
  constexpr int kCols = R::kCols, kWin = R::kWin;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* ring = reinterpret_cast<R*>(smem_raw);
  T* su = reinterpret_cast<T*>(ring + D);  // [D][kWin]
  T* sw = su + D * kWin;                    // [2][kWin]
  const unsigned ring_addr = (unsigned)__cvta_generic_to_shared(ring);
  const FdGeom& g = a.g;
  const int strip = blockIdx.x % g.n_strips;
  const int rest = blockIdx.x / g.n_strips;
  const int chunk = rest % g.n_chunks;
  const int shot = rest / g.n_chunks;
  const int tid = threadIdx.x;
  const int c0 = strip * kCols;
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const size_t F = g.field;
  const T* sbase = a.in + (size_t)shot * 5 * F;
  T* obase = a.out + (size_t)shot * 5 * F;
  const T dtx = a.dtx;
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  auto rec_of = [&](int xc) { return xc >= g.gx && (xc - g.gx) % g.dg == 0 && (xc - g.gx) / g.dg < g.ng; };
  const T* res_row = a.res + ((size_t)shot * g.nt + it) * g.ng;
  int xl[C], x[C];
  bool xint[C], ximg[C], rec[C];
  T inj[C];
#pragma unroll
  for (int h = 0; h < C; ++h) {
    xl[h] = tid + 1 + h * NT;
    x[h] = c0 + xl[h];
    xint[h] = x[h] >= 1 && x[h] <= g.NX - 2;
    ximg[h] = xint[h] && x[h] >= g.nbc && x[h] < g.nbc + g.nx;
    rec[h] = rec_of(x[h]);
    inj[h] = rec[h] ? a.dt * res_row[(x[h] - g.gx) / g.dg] : T(0);
  }
  const bool rec_h = tid == 0 && rec_of(c0);
  const T inj_h = rec_h ? a.dt * res_row[(c0 - g.gx) / g.dg] : T(0);
  const int xh = c0 + kCols + 1;
  const bool xhint = xh >= 1 && xh <= g.NX - 2;
  const bool c0int = c0 >= 1 && c0 <= g.NX - 2;
  Stager<T, kCols, GB, NT> stg;
  stg.init(sbase, F, a.mat, a.mb, c0, zs - 1, g);
  auto P1 = [](const R& S, int j) { return S.mat[j].y * S.f[2][j]; };
  auto P2 = [](const R& S, int j) { return S.mat[j].z * S.f[3][j]; };
  auto P3 = [](const R& S, int j) { return S.mat[j].w * S.f[4][j]; };
  auto Q1 = [](const R& S, int j) { return S.mat[j].z * S.f[2][j]; };
  auto Q2 = [](const R& S, int j) { return S.mat[j].y * S.f[3][j]; };
  // new ww at window column j of row z (rows Rz = z, Rd = z+1), with the injection
  auto vel_w_at = [&](const R& Rz, const R& Rd, int j, int z, bool inner, bool rc, T ij) -> T {
    const auto bb = bvals<T, GB>(Rz.mb, j, z, g, dtx);
    T r = adj_vel_w(inner, Rz.f[1][j], Q1(Rd, j), Q1(Rz, j), Q2(Rd, j), Q2(Rz, j), P3(Rz, j + 1), P3(Rz, j),
                    Rz.mat[j].x, bb.y);
    if (rc && z == g.gz) r = r + ij;
    return r;
  };
  // new uu at window column j of row z (rows Ru = z-1, Rz = z)
  auto vel_u_at = [&](const R& Ru, const R& Rz, int j, int z, bool inner) -> T {
    const auto bb = bvals<T, GB>(Rz.mb, j, z, g, dtx);
    return adj_vel_u(inner, Rz.f[0][j], P1(Rz, j), P1(Rz, j - 1), P2(Rz, j), P2(Rz, j - 1), P3(Rz, j), P3(Ru, j),
                     Rz.mat[j].x, bb.x);
  };
  const T* snap_b = IMG ? a.snap + ((size_t)shot * g.nrec + (it / g.nt_wf - a.rec0)) * NF * plane : nullptr;
  double* img_b = a.img + (size_t)shot * 3 * plane;
  float* img_f = a.img32 ? a.img32 + (size_t)shot * 3 * plane : nullptr;  // FP32 images, as the reference
  struct Img { T fx, bz, sg; double c0, c1, c2; };
  auto load_img = [&](Img& m, int h, int z) {
    if (IMG && ximg[h] && z >= z_img0 && z < z_img1) {
      const size_t cell = (size_t)(z - z_img0) * g.nx + (x[h] - g.nbc);
      const T* s0 = snap_b + cell;
      if (NF == 4) {
        m.fx = s0[0]; m.bz = s0[3 * plane]; m.sg = s0[plane] + s0[2 * plane];
      } else {
        m.fx = s0[0]; m.bz = s0[plane]; m.sg = s0[2 * plane];
      }
      if (img_f) {
        m.c0 = img_f[cell]; m.c1 = img_f[plane + cell]; m.c2 = img_f[2 * plane + cell];
      } else {
        m.c0 = img_b[cell]; m.c1 = img_b[plane + cell]; m.c2 = img_b[2 * plane + cell];
      }
    }
  };

#pragma unroll
  for (int r = 0; r < D; ++r) {
    stg.issue(ring_addr + r * (unsigned)sizeof(R), zs - 1 + r, g);
    cp_async_commit();
  }
  Img im_c[C], im_n[C];
#pragma unroll
  for (int h = 0; h < C; ++h) load_img(im_c[h], h, zs);
  cp_async_wait<D - 3>();
  cta_sync<W>();
  T wn_prev[C], wn_cur[C], un_cur[C], un_next[C];
  T a2[C], a3[C], a4[C], ate[C];  // old xx, zz, xz and temp of row k at the thread's column
  {
    const R& A = ring[0];
    const R& B = ring[1];
    const R& Cc = ring[2];
    const bool in1 = zs + 1 <= g.NZ - 2;
#pragma unroll
    for (int h = 0; h < C; ++h) {
      const int j = xl[h];
      wn_prev[h] = vel_w_at(A, B, j, zs - 1, xint[h] && zs - 1 >= 1, rec[h], inj[h]);
      un_cur[h] = vel_u_at(A, B, j, zs, xint[h]);
      wn_cur[h] = vel_w_at(B, Cc, j, zs, xint[h], rec[h], inj[h]);
      un_next[h] = vel_u_at(B, Cc, j, zs + 1, xint[h] && in1);
      su[j] = un_cur[h];
      su[kWin + j] = un_next[h];
      sw[j] = wn_cur[h];
      a2[h] = B.f[2][j];
      a3[h] = B.f[3][j];
      a4[h] = B.f[4][j];
      ate[h] = B.mat[j].x;
    }
    if (tid == NT - 1) {  // right halo: uu of rows zs and zs+1
      su[kCols + 1] = vel_u_at(A, B, kCols + 1, zs, xhint);
      su[kWin + kCols + 1] = vel_u_at(B, Cc, kCols + 1, zs + 1, xhint && in1);
    }
    if (tid == 0) sw[0] = vel_w_at(B, Cc, 0, zs, c0int, rec_h, inj_h);  // left halo: ww of row zs
  }
  cta_sync<W>();
  stg.issue(ring_addr, zs - 1 + D, g);
  cp_async_commit();

  for (int k0 = zs; k0 < ze; k0 += D)
#pragma unroll
  for (int u = 0; u < D; ++u) {
    const int k = k0 + u;
    if (k >= ze) break;
#pragma unroll
    for (int h = 0; h < C; ++h) load_img(im_n[h], h, k + 1);
    cp_async_wait<D - 3>();
    cta_sync<W>();
    stg.issue(ring_addr + ((u + 1) % D) * (unsigned)sizeof(R), k + D, g);
    cp_async_commit();
    const R& R1 = ring[(u + 2) % D];
    const R& R2 = ring[(u + 3) % D];
    const bool in1 = k + 1 <= g.NZ - 2, in2 = k + 2 <= g.NZ - 2;
    T* sw_n = sw + ((u + 1) & 1) * kWin;
    T* su_n = su + ((u + 2) % D) * kWin;
    const T* sw_c = sw + (u & 1) * kWin;
    const T* su_c = su + (u % D) * kWin;
    T wn_n[C], un_nn[C], b2[C], b3[C], b4[C], bte[C];
#pragma unroll
    for (int h = 0; h < C; ++h) {
      const int j = xl[h];
      wn_n[h] = vel_w_at(R1, R2, j, k + 1, xint[h] && in1, rec[h], inj[h]);
      un_nn[h] = vel_u_at(R1, R2, j, k + 2, xint[h] && in2);
      sw_n[j] = wn_n[h];
      su_n[j] = un_nn[h];
      b2[h] = R1.f[2][j];
      b3[h] = R1.f[3][j];
      b4[h] = R1.f[4][j];
      bte[h] = R1.mat[j].x;
    }
    if (tid == 0) sw_n[0] = vel_w_at(R1, R2, 0, k + 1, c0int && in1, rec_h, inj_h);
    if (tid == NT - 1) su_n[kCols + 1] = vel_u_at(R1, R2, kCols + 1, k + 2, xhint && in2);
#pragma unroll
    for (int h = 0; h < C; ++h) {
      const int j = xl[h];
      const T un_r = su_c[j + 1];
      const T wn_l = sw_c[j - 1];
      const T te = ate[h];
      const T xxn = te * a2[h] - dtx * (un_r - un_cur[h]);
      T zzn = te * a3[h] - dtx * (wn_cur[h] - wn_prev[h]);
      const T xzn = (te * a4[h] - dtx * (un_next[h] - un_cur[h])) - dtx * (wn_cur[h] - wn_l);
      if (k == g.pad_top) zzn = T(0);
      if (xint[h]) {
        T* o = obase + (size_t)k * g.pitch + x[h];
        o[0] = un_cur[h];
        o[F] = wn_cur[h];
        o[2 * F] = xxn;
        o[3 * F] = zzn;
        o[4 * F] = xzn;
        if (IMG && ximg[h] && k >= z_img0 && k < z_img1) {
          const size_t cell = (size_t)(k - z_img0) * g.nx + (x[h] - g.nbc);
          const T fx = im_c[h].fx, bz = im_c[h].bz, sg = im_c[h].sg;
          const T Fs = fx + bz;
          const T tcl = Fs * (xxn + zzn);
          const T tcm = T(2) * ((xxn * fx + zzn * bz) + T(0.5) * (xzn * sg));
          const T til = Fs * Fs;
          if (img_f) {  // accumulate in FP32 like the reference
            img_f[cell] = (float)((T)(im_c[h].c0) + tcl);
            img_f[plane + cell] = (float)((T)(im_c[h].c1) + tcm);
            img_f[2 * plane + cell] = (float)((T)(im_c[h].c2) + til);
          } else {
            img_b[cell] = im_c[h].c0 + (double)tcl;
            img_b[plane + cell] = im_c[h].c1 + (double)tcm;
            img_b[2 * plane + cell] = im_c[h].c2 + (double)til;
          }
        }
      }
      wn_prev[h] = wn_cur[h];
      wn_cur[h] = wn_n[h];
      un_cur[h] = un_next[h];
      un_next[h] = un_nn[h];
      im_c[h] = im_n[h];
      a2[h] = b2[h];
      a3[h] = b3[h];
      a4[h] = b4[h];
      ate[h] = bte[h];
    }
  }
  cp_async_wait<0>();
}

}  // namespace swd
