// Shared-memory-staged FD time steps (the production kernels).
//
// A CTA of NT = 32*W threads owns a strip of kCols = NT*C output columns (C
// columns per thread: t+1, t+1+NT, ...) over a chunk of rows of one shot, and
// streams down z.  Each padded row of the strip window [c0, c0 + kCols + 4) --
// the five state fields and the material vector -- is copied into a D-deep
// shared-memory ring with cp.async (16-byte copies, zero-filled outside the
// grid), issued D-2 rows ahead of use, so that many DRAM requests stay in
// flight.  Each thread's copy descriptors are computed once, so staging a row
// costs it a few instructions.  Neighbour values come from shared memory; the
// new velocities of a row are exchanged through two small shared arrays, with
// two barriers per row (warp barriers when the CTA is one warp).  The arithmetic
// is exactly that of the reference's Eigen expressions, in the same order
// (compile with -fmad=false), so FP32 results are bit-identical to the
// reference's single-precision MEX.
//
// Reference loops:  core/eigen_staggerfd_single.cpp:207-357 (forward),
//                   core/eigen_e2drtm_single.cpp:181-283 (adjoint + imaging).
#pragma once
#include <cstddef>

#include "fd_kernels.cuh"

namespace swd {

__device__ __forceinline__ void cp_async16(unsigned dst, const void* src, bool valid) {
  const int n = valid ? 16 : 0;  // 0 source bytes: the 16 destination bytes are zero-filled
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int W>
__device__ __forceinline__ void cta_sync() {
  if constexpr (W == 1) __syncwarp(); else __syncthreads();
}

// One padded row window in shared memory.
template <typename T, int NCOL, bool GB>
struct SRow {
  static constexpr int kCols = NCOL;
  static constexpr int kWin = NCOL + 4;
  using V4 = typename Vec4<T>::type;
  using V2 = typename Vec2<T>::type;
  T f[5][kWin];              // uu, ww, xx, zz, xz
  V4 mat[kWin];              // {temp, ca, cl, cm1}
  V2 mb[GB ? kWin : 1];      // {b, b1} (general-b path only)
};

// The 16-byte copies that stage one row window, divided among the CTA's NT threads.
// Each thread keeps, per copy, the source address of the next row to stage (rows
// are staged in increasing order), the bytes per row and the destination offset in
// a row slot, so staging a row is a cp.async and a pointer increment per copy.
// Copies of columns at or beyond the row pitch, and of rows at or beyond NZ, are
// skipped: no thread consumes those values.
template <typename T, int NCOL, bool GB, int NT>
struct Stager {
  using R = SRow<T, NCOL, GB>;
  using V4 = typename R::V4;
  using V2 = typename R::V2;
  static constexpr int EPC = 16 / (int)sizeof(T);
  static constexpr int CPF = R::kWin / EPC;                        // chunks per state field row
  static constexpr int NS = 5 * CPF;
  static constexpr int NM = R::kWin * (int)sizeof(V4) / 16;        // material chunks
  static constexpr int NB = GB ? R::kWin * (int)sizeof(V2) / 16 : 0;
  static constexpr int NC = NS + NM + NB;
  static constexpr int PER = (NC + NT - 1) / NT;
  const char* src[PER];
  unsigned rowb[PER];
  unsigned dst[PER];
  bool ok[PER];

  // descriptors for staging rows z0, z0+1, ...
  __device__ __forceinline__ void init(const T* sbase, size_t F, const V4* mat, const V2* mb, int c0, int z0,
                                       const FdGeom& g) {
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int i = threadIdx.x + j * NT;
      src[j] = reinterpret_cast<const char*>(sbase);
      rowb[j] = 0;
      dst[j] = 0;
      ok[j] = false;
      if (i < NS) {
        const int f = i / CPF, e = (i - f * CPF) * EPC, col = c0 + e;
        ok[j] = col < g.pitch;
        rowb[j] = (unsigned)(g.pitch * sizeof(T));
        src[j] = reinterpret_cast<const char*>(sbase + f * F + (size_t)z0 * g.pitch + (ok[j] ? col : 0));
        dst[j] = (unsigned)(offsetof(R, f) + (f * R::kWin + e) * sizeof(T));
      } else if (i < NS + NM) {
        const int m = i - NS, col = c0 + m * 16 / (int)sizeof(V4);
        ok[j] = col < g.pitch;
        rowb[j] = (unsigned)(g.pitch * sizeof(V4));
        src[j] = reinterpret_cast<const char*>(mat + (size_t)z0 * g.pitch + (ok[j] ? col : 0)) +
                 (ok[j] ? (m * 16) % (int)sizeof(V4) : 0);
        dst[j] = (unsigned)(offsetof(R, mat) + m * 16);
      } else if (i < NC) {
        const int m = i - NS - NM, col = c0 + m * 16 / (int)sizeof(V2);
        ok[j] = col < g.pitch;
        rowb[j] = (unsigned)(g.pitch * sizeof(V2));
        src[j] = reinterpret_cast<const char*>(mb + (size_t)z0 * g.pitch + (ok[j] ? col : 0));
        dst[j] = (unsigned)(offsetof(R, mb) + m * 16);
      }
    }
  }
  // stage the next row (z) into the slot at shared address slot_addr
  __device__ __forceinline__ void issue(unsigned slot_addr, int z, const FdGeom& g) {
    const bool zin = z < g.NZ;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      if (zin && ok[j]) cp_async16(slot_addr + dst[j], src[j], true);
      src[j] += rowb[j];
    }
  }
};

template <typename T, bool GB>
__device__ __forceinline__ typename Vec2<T>::type bvals(const typename Vec2<T>::type* mbrow, int xl, int z,
                                                         const FdGeom& g, T dtx) {
  if constexpr (GB) {
    return mbrow[xl];
  } else {
    typename Vec2<T>::type r;
    r.x = (z == g.pad_top) ? T(2) * dtx : dtx;
    r.y = r.x;
    return r;
  }
}

template <typename T, int W, int C, int D, bool GB>
constexpr size_t smem_bytes() {
  using R = SRow<T, 32 * W * C, GB>;
  return sizeof(R) * D + 3 * R::kWin * sizeof(T);
}

// ---------------------------------------------------------------- forward

// One tile (strip, row chunk, shot = `block` in that order) of a forward step.  SNAP: the step
// writes strain snapshots (it % nt_wf == 0); the other steps use the variant without the
// snapshot code.
template <typename T, int NF, int W, int C, int D, bool GB, bool SNAP>
__device__ __forceinline__ void fwd_smem_tile(const FwdArgs<T>& a, int it, int block) {
  if (cta_cancelled(a.cancel)) return;  // every thread of the CTA reaches this first
  static_assert(D >= 4 && D % 2 == 0, "rows k, k+1 in use, rows in flight, even depth for static slots");
  constexpr int NT = 32 * W;
  using R = SRow<T, NT * C, GB>;
  using V4 = typename Vec4<T>::type;
  constexpr int kCols = R::kCols, kWin = R::kWin;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* ring = reinterpret_cast<R*>(smem_raw);
  T* su = reinterpret_cast<T*>(ring + D);   // new uu of row k, parity (k - zs) & 1 [2][kWin]
  T* sw = su + 2 * kWin;                     // new ww of row k [kWin]
  const unsigned ring_addr = (unsigned)__cvta_generic_to_shared(ring);
  const FdGeom& g = a.g;
  const int strip = block % g.n_strips;
  const int rest = block / g.n_strips;
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
  // per-column, row-invariant predicates; the source and receiver flags are false for all
  // but a few threads, which alone take the (rare) source / receiver paths
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
    s_w[h] = sc && st != 1 && st != 4;     // ww(sz,sx) = s (type 5) or += s (types 2, 3)
    s_wr[h] = sr && st == 2;               // ww(sz,sx+1) += s
    s_u[h] = sc && (st == 2 || st == 3);   // uu(sz,sx) += s
    s_um[h] = sc && st == 2;               // uu(sz-1,sx) -= s
    s_xz[h] = sc && (st == 1 || st == 4);  // xx/zz sources before the stress update
    src_any = src_any || sc || sr;
    recj[h] = (a.seis_w != nullptr && xint[h] && x[h] >= g.gx && (x[h] - g.gx) % g.dg == 0 &&
               (x[h] - g.gx) / g.dg < g.ng) ? (x[h] - g.gx) / g.dg : -1;
    rec_any = rec_any || recj[h] >= 0;
    snapc[h] = SNAP && xint[h] && x[h] >= g.nbc && x[h] < g.nbc + g.nx;
    ob[h] = a.out + (size_t)shot * 5 * F + (xint[h] ? x[h] : 0);
  }
  Stager<T, kCols, GB, NT> stg;
  stg.init(sbase, F, a.mat, a.mb, c0, zs - 1, g);

  // velocity updates without the source (:224-228); the source is applied afterwards (:286-300)
  auto vel_w = [&](bool inner, T ww, T xz, T xzl, T zz, T zzd, T te, T b1) -> T {
    return inner ? te * ww + b1 * (((xz - xzl) + zzd) - zz) : ww;
  };
  auto vel_u = [&](bool inner, T uu, T xx, T xxr, T xz, T xzu, T te, T b) -> T {
    return inner ? te * uu + b * (((xxr - xx) + xz) - xzu) : uu;
  };
  auto src_w = [&](int z, T r, bool here, bool right) -> T {  // ww after the source, row z
    if (z == sp.x) {
      if (here) r = (st == 5) ? sv : r + sv;
      else if (right) r = r + sv;
    }
    return r;
  };
  auto src_u = [&](int z, T r, bool here, bool minus) -> T {  // uu after the source, row z
    if (here && z == sp.x) r = r + sv;
    if (minus && z == sp.x - 1) r = r - sv;
    return r;
  };

  // prologue: rows zs-1 .. zs+D-2 in flight; wait for zs-1 and zs
#pragma unroll
  for (int r = 0; r < D; ++r) {
    stg.issue(ring_addr + r * (unsigned)sizeof(R), zs - 1 + r, g);
    cp_async_commit();
  }
  cp_async_wait<D - 2>();
  cta_sync<W>();
  T wn_prev[C], un_cur[C];
  {
    const R& A = ring[0];  // row zs-1
    const R& B = ring[1];  // row zs
#pragma unroll
    for (int h = 0; h < C; ++h) {
      const int j = xl[h];
      const auto ba = bvals<T, GB>(A.mb, j, zs - 1, g, dtx);
      const auto bb = bvals<T, GB>(B.mb, j, zs, g, dtx);
      wn_prev[h] = vel_w(xint[h] && zs - 1 >= 1, A.f[1][j], A.f[4][j], A.f[4][j - 1], A.f[3][j], B.f[3][j],
                         A.mat[j].x, ba.y);
      un_cur[h] = vel_u(xint[h], B.f[0][j], B.f[2][j], B.f[2][j + 1], B.f[4][j], A.f[4][j], B.mat[j].x, bb.x);
      if (src_any) {
        wn_prev[h] = src_w(zs - 1, wn_prev[h], s_w[h], s_wr[h]);
        un_cur[h] = src_u(zs, un_cur[h], s_u[h], s_um[h]);
      }
      su[j] = un_cur[h];
    }
    if (tid == 0) {  // halo column c0 (needed for fux at c0+1)
      const auto b0 = bvals<T, GB>(B.mb, 0, zs, g, dtx);
      const bool hc = c0 == sp.y;
      su[0] = src_u(zs, vel_u(c0 >= 1 && c0 <= g.NX - 2, B.f[0][0], B.f[2][0], B.f[2][1], B.f[4][0], A.f[4][0],
                              B.mat[0].x, b0.x),
                    hc && (st == 2 || st == 3), hc && st == 2);
    }
  }

  // The row loop is unrolled by D: with k = k0 + u and k0 - zs a multiple of D, row k sits in
  // ring slot (u+1) % D, row k+1 in (u+2) % D, and the uu exchange parity of row k is u & 1.
  for (int k0 = zs; k0 < ze; k0 += D)
#pragma unroll
  for (int u = 0; u < D; ++u) {
    const int k = k0 + u;
    if (k >= ze) break;
    const int p0 = u & 1, p1 = (u + 1) & 1;
    cp_async_wait<D - 3>();
    cta_sync<W>();                                          // rows k, k+1 resident; row k-1 free
    stg.issue(ring_addr + (u % D) * (unsigned)sizeof(R), k - 1 + D, g);
    cp_async_commit();
    const R& R0 = ring[(u + 1) % D];
    const R& R1 = ring[(u + 2) % D];
    const bool inner1 = k + 1 <= g.NZ - 2;
    T wn[C], un_next[C];
    // velocities: ww at row k, uu at row k+1
#pragma unroll
    for (int h = 0; h < C; ++h) {
      const int j = xl[h];
      const auto b0 = bvals<T, GB>(R0.mb, j, k, g, dtx);
      const auto b1 = bvals<T, GB>(R1.mb, j, k + 1, g, dtx);
      wn[h] = vel_w(xint[h], R0.f[1][j], R0.f[4][j], R0.f[4][j - 1], R0.f[3][j], R1.f[3][j], R0.mat[j].x, b0.y);
      un_next[h] = vel_u(xint[h] && inner1, R1.f[0][j], R1.f[2][j], R1.f[2][j + 1], R1.f[4][j], R0.f[4][j],
                         R1.mat[j].x, b1.x);
      if (src_any) {
        wn[h] = src_w(k, wn[h], s_w[h], s_wr[h]);
        un_next[h] = src_u(k + 1, un_next[h], s_u[h], s_um[h]);
      }
      sw[j] = wn[h];
      su[p1 * kWin + j] = un_next[h];
    }
    if (tid == NT - 1) {  // halo column c0+kCols+1 (needed for bwx at c0+kCols)
      const int j = kCols + 1, xh = c0 + j;
      const auto bh = bvals<T, GB>(R0.mb, j, k, g, dtx);
      sw[j] = src_w(k, vel_w(xh >= 1 && xh <= g.NX - 2, R0.f[1][j], R0.f[4][j], R0.f[4][j - 1], R0.f[3][j],
                             R1.f[3][j], R0.mat[j].x, bh.y),
                    xh == sp.y && st != 1 && st != 4, xh == sp.y + 1 && st == 2);
    }
    if (tid == 0) {
      const bool hc = c0 == sp.y;
      const auto bh = bvals<T, GB>(R1.mb, 0, k + 1, g, dtx);
      su[p1 * kWin] = src_u(k + 1, vel_u(c0 >= 1 && c0 <= g.NX - 2 && inner1, R1.f[0][0], R1.f[2][0], R1.f[2][1],
                                         R1.f[4][0], R0.f[4][0], R1.mat[0].x, bh.x),
                            hc && (st == 2 || st == 3), hc && st == 2);
    }
    cta_sync<W>();                                          // new velocities of row k visible
    const bool snap_row = SNAP && k >= z_img0 && k < z_img1;
#pragma unroll
    for (int h = 0; h < C; ++h) {
      const int j = xl[h];
      // strains at row k (:302-306)
      const T fux = un_cur[h] - su[p0 * kWin + j - 1];
      const T fuz = un_next[h] - un_cur[h];
      const T bwx = sw[j + 1] - wn[h];
      const T bwz = wn[h] - wn_prev[h];
      // stresses at row k (:334-336), source types 1/4 first (:286-298), free surface (:340)
      T xo = R0.f[2][j], zo = R0.f[3][j];
      if (src_any && s_xz[h] && k == sp.x) {
        if (st == 1) { xo = xo + sv; zo = zo + sv; }
        else { zo = zo + sv; }
      }
      const V4 m = R0.mat[j];
      const T te = m.x, ca = m.y, cl = m.z, cm1 = m.w;
      const T xxn = te * xo + (ca * fux + cl * bwz) * dtx;
      T zzn = te * zo + (ca * bwz + cl * fux) * dtx;
      const T xzn = te * R0.f[4][j] + (cm1 * (fuz + bwx)) * dtx;
      if (k == g.pad_top) zzn = T(0);
      if (xint[h]) {
        T* o = ob[h] + (size_t)k * g.pitch;
        o[0] = un_cur[h];
        o[F] = wn[h];
        o[2 * F] = xxn;
        o[3 * F] = zzn;
        o[4 * F] = xzn;
      }
      if (rec_any && k == g.gz && recj[h] >= 0) {  // :342-345
        const size_t r = ((size_t)shot * g.nt + it) * g.ng + recj[h];
        a.seis_w[r] = wn[h];
        if (a.seis_u) a.seis_u[r] = un_cur[h];
      }
      if (SNAP && snap_row && snapc[h]) {  // :346-351
        T* sp0 = snap_base + ((size_t)(k - z_img0) * g.nx + (x[h] - g.nbc));
        if (NF == 4) {
          sp0[0] = fux; sp0[plane] = fuz; sp0[2 * plane] = bwx; sp0[3 * plane] = bwz;
        } else {  // the adjoint needs fux, bwz and fuz+bwx only
          sp0[0] = fux; sp0[plane] = bwz; sp0[2 * plane] = fuz + bwx;
        }
      }
      wn_prev[h] = wn[h];
      un_cur[h] = un_next[h];
    }
  }
  cp_async_wait<0>();  // no copy may still target this CTA's shared memory at exit
}

template <typename T, int NF, int W, int C, int D, bool GB, bool SNAP>
__global__ void __launch_bounds__(32 * W)
fd_fwd_smem(FwdArgs<T> a, int it) {
  fwd_smem_tile<T, NF, W, C, D, GB, SNAP>(a, it, blockIdx.x);
}

// The job that owns CTA b: the last j with cta0[j] <= b (binary search over the running tile counts,
// cta0[0] = 0 <= b < cta0[n_jobs]).
__device__ __forceinline__ int owning_job(const int* __restrict__ cta0, int n_jobs, int b) {
  int lo = 0, hi = n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cta0[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Several forward calls advanced by one launch per step, on grids of any sizes: CTA b runs tile
// b - cta0[j] of job j, where cta0 holds the running sums of the jobs' tile counts (cta0[0] = 0,
// cta0[n_jobs] = the grid); a job whose time steps are done leaves at once.  The jobs share the
// CTA shape, so one shared-memory size serves all of them; each reads its own geometry,
// materials, state, source, receivers and snapshot buffer from its FwdArgs, and takes the
// snapshot variant on its own snapshot steps (it % nt_wf == 0).
template <typename T, int NF, int W, int C, int D, bool GB>
__global__ void __launch_bounds__(32 * W)
fd_fwd_smem_multi(const FwdArgs<T>* __restrict__ jobs, const int* __restrict__ cta0, int n_jobs, int it) {
  const int j = owning_job(cta0, n_jobs, (int)blockIdx.x);
  const FwdArgs<T>& a = jobs[j];
  if (it >= a.g.nt) return;  // uniform over the CTA
  const int tile = (int)blockIdx.x - cta0[j];
  if (a.snap && it % a.g.nt_wf == 0) fwd_smem_tile<T, NF, W, C, D, GB, true>(a, it, tile);
  else fwd_smem_tile<T, NF, W, C, D, GB, false>(a, it, tile);
}

// ---------------------------------------------------------------- adjoint

// Adjoint velocities (:182-187) from material*stress products formed at each cell.
template <typename T>
__device__ __forceinline__ T adj_vel_u(bool inner, T uu, T P1, T P1l, T P2, T P2l, T P3, T P3u, T temp, T b) {
  if (inner) {
    const T du = ((P1 - P1l) + (P2 - P2l)) + (P3 - P3u);
    return temp * uu - b * du;
  }
  return uu;
}
template <typename T>
__device__ __forceinline__ T adj_vel_w(bool inner, T ww, T Q1d, T Q1, T Q2d, T Q2, T P3r, T P3, T temp, T b1) {
  if (inner) {
    const T dw = ((Q1d - Q1) + (Q2d - Q2)) + (P3r - P3);
    return temp * ww - b1 * dw;
  }
  return ww;
}

// One tile (strip, row chunk, shot = `block` in that order) of an adjoint step.  IMG: the step
// applies the imaging condition (it % nt_wf == 0).
template <typename T, int NF, int W, int C, int D, bool GB, bool IMG>
__device__ __forceinline__ void adj_smem_tile(const AdjArgs<T>& a, int it, int block) {
  if (cta_cancelled(a.cancel)) return;  // every thread of the CTA reaches this first
  static_assert(D >= 4 && D % 2 == 0, "rows k, k+1 in use, rows in flight, even depth for static slots");
  constexpr int NT = 32 * W;
  using R = SRow<T, NT * C, GB>;
  constexpr int kCols = R::kCols, kWin = R::kWin;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* ring = reinterpret_cast<R*>(smem_raw);
  T* su = reinterpret_cast<T*>(ring + D);   // new uu of row k, parity k&1 [2][kWin]
  T* sw = su + 2 * kWin;                     // new ww of row k [kWin]
  const unsigned ring_addr = (unsigned)__cvta_generic_to_shared(ring);
  const FdGeom& g = a.g;
  const int strip = block % g.n_strips;
  const int rest = block / g.n_strips;
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
  // dt*res at receiver columns (:238-242)
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
  const bool rec_h = tid == 0 && rec_of(c0);               // left halo column c0 (thread 0)
  const T inj_h = rec_h ? a.dt * res_row[(c0 - g.gx) / g.dg] : T(0);
  const int xh = c0 + kCols + 1;                           // right halo column (thread NT-1)
  const bool xhint = xh >= 1 && xh <= g.NX - 2;
  const bool c0int = c0 >= 1 && c0 <= g.NX - 2;
  Stager<T, kCols, GB, NT> stg;
  stg.init(sbase, F, a.mat, a.mb, c0, zs - 1, g);
  // material*stress products at window column j of row S
  auto P1 = [](const R& S, int j) { return S.mat[j].y * S.f[2][j]; };   // ca*xx
  auto P2 = [](const R& S, int j) { return S.mat[j].z * S.f[3][j]; };   // cl*zz
  auto P3 = [](const R& S, int j) { return S.mat[j].w * S.f[4][j]; };   // cm1*xz
  auto Q1 = [](const R& S, int j) { return S.mat[j].z * S.f[2][j]; };   // cl*xx
  auto Q2 = [](const R& S, int j) { return S.mat[j].y * S.f[3][j]; };   // ca*zz
  // new ww at window column j of row k (rows R0 = k, R1 = k+1), with the injection
  auto vel_w_at = [&](const R& R0, const R& R1, int j, int k, bool inner, bool rc, T ij) -> T {
    const auto bb = bvals<T, GB>(R0.mb, j, k, g, dtx);
    T r = adj_vel_w(inner, R0.f[1][j], Q1(R1, j), Q1(R0, j), Q2(R1, j), Q2(R0, j), P3(R0, j + 1), P3(R0, j),
                    R0.mat[j].x, bb.y);
    if (rc && k == g.gz) r = r + ij;
    return r;
  };
  // new uu at window column j of row k1 = k+1 (rows R0 = k, R1 = k+1)
  auto vel_u_at = [&](const R& R0, const R& R1, int j, int k1, bool inner) -> T {
    const auto bb = bvals<T, GB>(R1.mb, j, k1, g, dtx);
    return adj_vel_u(inner, R1.f[0][j], P1(R1, j), P1(R1, j - 1), P2(R1, j), P2(R1, j - 1), P3(R1, j), P3(R0, j),
                     R1.mat[j].x, bb.x);
  };

  // imaging operands (forward strains, FP64 accumulators) of this thread's cells in row z
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
  cp_async_wait<D - 2>();
  cta_sync<W>();
  T wn_prev[C], un_cur[C];
  {
    const R& A = ring[0];  // row zs-1
    const R& B = ring[1];  // row zs
#pragma unroll
    for (int h = 0; h < C; ++h) {
      wn_prev[h] = vel_w_at(A, B, xl[h], zs - 1, xint[h] && zs - 1 >= 1, rec[h], inj[h]);
      un_cur[h] = vel_u_at(A, B, xl[h], zs, xint[h]);
      su[0 * kWin + xl[h]] = un_cur[h];
    }
    if (tid == NT - 1) su[0 * kWin + kCols + 1] = vel_u_at(A, B, kCols + 1, zs, xhint);  // right halo
  }

  // unrolled by D as in the forward kernel: static ring slots and exchange parities
  for (int k0 = zs; k0 < ze; k0 += D)
#pragma unroll
  for (int u = 0; u < D; ++u) {
    const int k = k0 + u;
    if (k >= ze) break;
    const int p0 = u & 1, p1 = (u + 1) & 1;
#pragma unroll
    for (int h = 0; h < C; ++h) load_img(im_n[h], h, k + 1);
    cp_async_wait<D - 3>();
    cta_sync<W>();
    stg.issue(ring_addr + (u % D) * (unsigned)sizeof(R), k - 1 + D, g);
    cp_async_commit();
    const R& R0 = ring[(u + 1) % D];
    const R& R1 = ring[(u + 2) % D];
    const bool inner1 = k + 1 <= g.NZ - 2;
    T wn[C], un_next[C];
#pragma unroll
    for (int h = 0; h < C; ++h) {
      wn[h] = vel_w_at(R0, R1, xl[h], k, xint[h], rec[h], inj[h]);
      un_next[h] = vel_u_at(R0, R1, xl[h], k + 1, xint[h] && inner1);
      sw[xl[h]] = wn[h];
      su[p1 * kWin + xl[h]] = un_next[h];
    }
    if (tid == 0) sw[0] = vel_w_at(R0, R1, 0, k, c0int, rec_h, inj_h);                                   // left halo
    if (tid == NT - 1) su[p1 * kWin + kCols + 1] = vel_u_at(R0, R1, kCols + 1, k + 1, xhint && inner1);
    cta_sync<W>();
#pragma unroll
    for (int h = 0; h < C; ++h) {
      const int j = xl[h];
      // adjoint stresses at row k (:245-248), free surface (:270)
      const T un_r = su[p0 * kWin + j + 1];
      const T wn_l = sw[j - 1];
      const T te = R0.mat[j].x;
      const T xxn = te * R0.f[2][j] - dtx * (un_r - un_cur[h]);
      T zzn = te * R0.f[3][j] - dtx * (wn[h] - wn_prev[h]);
      const T xzn = (te * R0.f[4][j] - dtx * (un_next[h] - un_cur[h])) - dtx * (wn[h] - wn_l);
      if (k == g.pad_top) zzn = T(0);
      if (xint[h]) {
        T* o = obase + (size_t)k * g.pitch + x[h];
        o[0] = un_cur[h];
        o[F] = wn[h];
        o[2 * F] = xxn;
        o[3 * F] = zzn;
        o[4 * F] = xzn;
        if (IMG && ximg[h] && k >= z_img0 && k < z_img1) {  // imaging condition (:274-279)
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
      wn_prev[h] = wn[h];
      un_cur[h] = un_next[h];
      im_c[h] = im_n[h];
    }
  }
  cp_async_wait<0>();
}

template <typename T, int NF, int W, int C, int D, bool GB, bool IMG>
__global__ void __launch_bounds__(32 * W)
fd_adj_smem(AdjArgs<T> a, int it) {
  adj_smem_tile<T, NF, W, C, D, GB, IMG>(a, it, blockIdx.x);
}

// Several adjoint calls advanced by one launch per step, as fd_fwd_smem_multi: the jobs count
// their steps backwards from their own nt (step s of job j is it = nt_j - 2 - s, as
// core/eigen_e2drtm_single.cpp:181 counts), a job whose steps are done leaves at once, and each
// takes the imaging variant on its own it % nt_wf == 0 steps.
template <typename T, int NF, int W, int C, int D, bool GB>
__global__ void __launch_bounds__(32 * W)
fd_adj_smem_multi(const AdjArgs<T>* __restrict__ jobs, const int* __restrict__ cta0, int n_jobs, int step) {
  const int j = owning_job(cta0, n_jobs, (int)blockIdx.x);
  const AdjArgs<T>& a = jobs[j];
  const int it = a.g.nt - 2 - step;
  if (it < 0) return;  // uniform over the CTA
  const int tile = (int)blockIdx.x - cta0[j];
  if (it % a.g.nt_wf == 0) adj_smem_tile<T, NF, W, C, D, GB, true>(a, it, tile);
  else adj_smem_tile<T, NF, W, C, D, GB, false>(a, it, tile);
}

}  // namespace swd
