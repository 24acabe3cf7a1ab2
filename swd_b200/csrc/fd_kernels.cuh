// Shared definitions of the FD time-step kernels (fd_smem.cuh): grid geometry,
// launch arguments and the per-cell velocity updates.
//
// The velocity updates are written in exactly the order of the reference's Eigen
// expressions; the translation units that include this file are compiled with
// -fmad=false, so no multiply-add is contracted and the FP32 results are
// bit-identical to the reference's single-precision MEX.
//
// Reference loops:  core/eigen_staggerfd_single.cpp:207-357 (forward),
//                   core/eigen_e2drtm_single.cpp:181-283 (adjoint + imaging).
#pragma once
#include "swd_common.cuh"

namespace swd {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kCol2Pairs = 30;  // column pairs written per warp by the column-pair kernels (fd_col2.cuh)

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };
template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

// Geometry of one padded grid plus the warp decomposition of a launch.
struct FdGeom {
  int NZ, NX, pitch;         // padded grid (nzbc x nxbc), row pitch in elements
  int nz, nx, nbc;           // model interior: rows pad_top+1.., cols nbc..
  int pad_top;               // free-surface row (1 for fd_order 22)
  int nt, nt_wf, nrec;       // time steps, snapshot interval, snapshots per shot
  int ng, gz, gx, dg;        // receivers (0-based padded coordinates)
  int n_strips, n_chunks, chunk;
  int warps;                 // warps per CTA
  int cells;                 // output columns per thread; a CTA owns 32*warps*cells columns
  int ring_fwd, ring_adj;    // rows in the shared-memory ring of the forward / adjoint kernels (4, 6, 8)
  int sched;                 // 0: two barriers per row (fd_smem.cuh); 1: one, velocities a row ahead (fd_lead.cuh);
                             // 2: warp streaming (fd_warp.cuh; warps = warps per CTA); 3: warp streaming over
                             // column pairs, two steps per launch (fd_col2.cuh; pair-interleaved state)
  int pairs;                 // schedule 2: 1 = forward and adjoint advance two steps per launch; 2 = the same
                             // with two shots per warp in packed FP32 pairs (fd_warpx.cuh)
  size_t field;              // NZ * pitch
};

// Material rows: mat = {temp, ca, cl, cm1}; mb = {b, b1} when b/b1 are general arrays
// (the MEX interface).  Without mb, b = b1 = dtx with the free-surface row doubled,
// which is how core/staggerfd_eigen.m:103-105 builds them.
template <typename T>
struct FwdArgs {
  FdGeom g;
  const typename Vec4<T>::type* mat;  // [NZ][pitch]
  const typename Vec2<T>::type* mb;   // [NZ][pitch] or null
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
  const int* cancel;                  // engine's cancel word (null: never cancelled)
};

template <typename T>
struct AdjArgs {
  FdGeom g;
  const typename Vec4<T>::type* mat;
  const typename Vec2<T>::type* mb;
  const T* in;
  T* out;
  const T* res;                       // adjoint source [shot][nt][ng]
  const T* snap;                      // forward strain snapshots [shot][nrec][NF][nz][nx]
  double* img;                        // [shot][cl,cm,illum][nz][nx]
  float* img32;                       // when set: FP32 images (as the reference accumulates), img unused
  T dtx, dt;
  int rec0;                           // snapshot it/nt_wf is read from index it/nt_wf - rec0
  int n_shots;
  const int* cancel;                  // engine's cancel word (null: never cancelled)
};

// Cancellation of a call in flight: swd_engine_cancel sets a device word while the engine's time
// loops run, and every FD launch of the engine returns as soon as it finds it set, so the rest
// of a captured time loop drains as empty launches.  The decision is made once per warp (warp
// kernels, before their first wait) or once per CTA (kernels with barriers), never per thread.
__device__ __forceinline__ int cancel_word(const int* c) { return c ? *reinterpret_cast<const volatile int*>(c) : 0; }
__device__ __forceinline__ bool warp_cancelled(const int* c) { return __any_sync(kFull, cancel_word(c) != 0); }
__device__ __forceinline__ bool cta_cancelled(const int* c) { return __syncthreads_or(cancel_word(c) != 0) != 0; }

// ---------------------------------------------------------------- forward

// uu at (z,x) after the velocity update and the source (eigen_staggerfd_single.cpp:225-226, 286-300).
template <typename T>
__device__ __forceinline__ T fwd_vel_u(int z, int x, bool xint, const FdGeom& g, T uu, T xx, T xx_r, T xz, T xz_u,
                                       T temp, T b, int st, int2 sp, T sv) {
  T r = uu;
  if (xint && z >= 1 && z <= g.NZ - 2) r = temp * uu + b * (((xx_r - xx) + xz) - xz_u);
  if (x == sp.y) {
    if (z == sp.x && (st == 2 || st == 3)) r = r + sv;
    if (z == sp.x - 1 && st == 2) r = r - sv;
  }
  return r;
}

// ww at (z,x) after the velocity update and the source (:227-228, 286-300).
template <typename T>
__device__ __forceinline__ T fwd_vel_w(int z, int x, bool xint, const FdGeom& g, T ww, T xz, T xz_l, T zz, T zz_d,
                                       T temp, T b1, int st, int2 sp, T sv) {
  T r = ww;
  if (xint && z >= 1 && z <= g.NZ - 2) r = temp * ww + b1 * (((xz - xz_l) + zz_d) - zz);
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

}  // namespace swd
