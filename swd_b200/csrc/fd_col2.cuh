// Column-pair warp-streaming FD kernels (engine FD schedule 6).
//
// A warp owns 64 columns of one shot and streams down a chunk of rows, as the warp kernels of
// fd_warp.cuh do, but each lane holds TWO adjacent columns (2p, 2p+1).  The state and the
// materials of this schedule are stored pair-interleaved, so a lane's two values of a field sit
// next to each other in HBM, in shared memory and in one 64-bit register pair:
//
//   state of a shot   A: float4 {uu, uu', ww, ww'} [NZ][P]   (' = column 2p+1, P = pitch / 2)
//                     B: float4 {xx, xx', zz, zz'} [NZ][P]
//                     C: float2 {xz, xz'}          [NZ][P]   (the same 5 * NZ * pitch floats)
//   materials         float4 {temp, temp', ca, ca'}, float4 {cl, cl', cm1, cm1'} per pair
//
// Every add, subtract and multiply of the stencil is then one packed FP32x2 instruction over
// the lane's two columns (F2, fd_warpx.cuh: each half rounds as the scalar instruction does and
// products are never fused).  A horizontal difference f(x+1) - f(x) over the pair needs the
// neighbour lane's nearest column only: one shuffle and two scalar subtractions (dR / dL below).
// The row bookkeeping, staging and loop control are shared by two columns, and the warp's two
// edge lanes are the only halo (60 output columns of 64 for one or two steps).
//
// Border columns keep their state as in the two-step kernels of fd_warp.cuh: the material table
// holds temp = 1 there and the lane's time factor pair dl has 0 in a border half, so the update
// returns the state bit for bit (for finite neighbours).  Border rows (0, NZ-1) take the checked
// path and keep their state by a select.  Column pairs never straddle the interior boundary
// because the engine only runs this schedule when nbc and nx are even, so snapshot and image
// rows are read and written as aligned pairs.
//
// The arithmetic is that of fd_warp.cuh expression for expression (the file is compiled with
// -fmad=false), so the results are bit-identical to the other schedules and the oracle.
//
// Reference loops:  core/eigen_staggerfd_single.cpp:207-357 (forward),
//                   core/eigen_e2drtm_single.cpp:181-283 (adjoint + imaging).
#pragma once
#include "fd_warpx.cuh"  // F2 packed arithmetic, cp.async helpers, warp_tile, slow_rows

namespace swd {

constexpr int kCol2Out = 60;  // output columns per warp: 64 minus one halo lane (two columns) a side

// f(x+1) - f(x) and f(x) - f(x-1) over the lane's column pair: one shuffle of the neighbour
// lane's nearest column, two scalar subtractions in the order of the scalar kernels.
__device__ __forceinline__ F2 dR(const F2& f) {
  const float n = __shfl_down_sync(kFull, f.x, 1);
  return F2{f.y - f.x, n - f.y};
}
__device__ __forceinline__ F2 dL(const F2& f) {
  const float p = __shfl_up_sync(kFull, f.y, 1);
  return F2{f.x - p, f.y - f.x};
}

// Material pair of a row.
struct MP {
  F2 te, ca, cl, cm1;
};
// State pair of a row.
struct SP {
  F2 uu, ww, xx, zz, xz;
};

// One staging slot: one row of a warp's 32 column pairs.
struct C2Slot {
  float4 a[32];   // {uu, uu', ww, ww'}
  float4 b[32];   // {xx, xx', zz, zz'}
  float4 m0[32];  // {temp, temp', ca, ca'}
  float4 m1[32];  // {cl, cl', cm1, cm1'}
  float2 c[32];   // {xz, xz'}
};
// Imaging operands of one row of an adjoint step that images: forward strain pairs and the
// image sum pairs (FP64, or FP32 in the first half of each c row).
struct C2ImgSlot {
  float2 fx[32], bz[32], sg[32];
  double2 c[3][32];
};
template <int NW, int NS>
constexpr size_t col2_smem_bytes() { return (size_t)NW * NS * sizeof(C2Slot); }
template <int NW, int NS>
constexpr size_t col2_img_smem_bytes() { return (size_t)NW * NS * (sizeof(C2Slot) + sizeof(C2ImgSlot)); }

struct C2Stage {
  const float4* a;   // this lane's pair of plane A, row 0
  const float4* b;   // plane B
  const float2* c;   // plane C
  const float4* m;   // materials, row 0 (two float4 per pair)
  C2Slot* slots;     // this warp's NS slots
  int P, zmax, lane;
  // Stage row z into a slot as one copy group.  Rows outside 0..zmax are not needed; they are
  // clamped into the grid rather than skipped, so that the staging has no branch.
  __device__ __forceinline__ void issue(int slot, int z) const {
    const int o = min(max(z, 0), zmax) * P;  // 32-bit: the engine keeps 5 * NZ * pitch below 2^31
    C2Slot& s = slots[slot];
    wcp16(&s.a[lane], a + o);
    wcp16(&s.b[lane], b + o);
    wcp16(&s.m0[lane], m + 2 * o);
    wcp16(&s.m1[lane], m + 2 * o + 1);
    wcp8(&s.c[lane], c + o);
    wcp_commit();
  }
  __device__ __forceinline__ void read(SP& r, MP& mt, int slot) const {
    const C2Slot& s = slots[slot];
    const float4 va = s.a[lane], vb = s.b[lane], m0 = s.m0[lane], m1 = s.m1[lane];
    const float2 vc = s.c[lane];
    r.uu = F2{va.x, va.y};
    r.ww = F2{va.z, va.w};
    r.xx = F2{vb.x, vb.y};
    r.zz = F2{vb.z, vb.w};
    r.xz = F2{vc.x, vc.y};
    mt.te = F2{m0.x, m0.y};
    mt.ca = F2{m0.z, m0.w};
    mt.cl = F2{m1.x, m1.y};
    mt.cm1 = F2{m1.z, m1.w};
  }
};

// Per-lane geometry of the column-pair kernels.
struct C2Lane {
  int lane, pr, prc;  // lane, its column pair (may lie outside the grid), the pair it loads
  int x0;             // column of the first half
  bool own;           // writes its pair (lanes 1..30, pair inside the grid)
  F2 dl, dl2;         // time factor per half (0 on border columns), doubled for the free surface
};

__device__ __forceinline__ C2Lane col2_lane(const FdGeom& g, int strip, float dtx) {
  C2Lane L;
  L.lane = threadIdx.x & 31;
  L.pr = (kCol2Out / 2) * strip + L.lane - 1;
  const int NP = g.NX >> 1;
  L.prc = min(max(L.pr, 0), NP - 1);
  L.x0 = 2 * L.pr;
  L.own = L.lane >= 1 && L.lane <= kCol2Out / 2 && L.pr >= 0 && L.pr < NP;
  const bool i0 = L.x0 >= 1 && L.x0 <= g.NX - 2, i1 = L.x0 + 1 >= 1 && L.x0 + 1 <= g.NX - 2;
  L.dl = F2{i0 ? dtx : 0.f, i1 ? dtx : 0.f};
  const float d2 = 2.f * dtx;  // b = b1 = 2 * dtx on the free-surface row (core/staggerfd_eigen.m:103-105)
  L.dl2 = F2{i0 ? d2 : 0.f, i1 ? d2 : 0.f};
  return L;
}

// Receiver index of each half of the lane's pair (-1: none); receivers record own columns only.
__device__ __forceinline__ int2 col2_receivers(const FdGeom& g, const C2Lane& L, bool on) {
  int r[2] = {-1, -1};
  for (int h = 0; h < 2; ++h) {
    const int x = L.x0 + h;
    if (on && L.own && x >= 1 && x <= g.NX - 2 && x >= g.gx && (x - g.gx) % g.dg == 0 && (x - g.gx) / g.dg < g.ng)
      r[h] = (x - g.gx) / g.dg;
  }
  return make_int2(r[0], r[1]);
}

// Apply fn to one half (0: column 2p, 1: column 2p+1) of a pair; used on checked rows only.
template <class Fn>
__device__ __forceinline__ void on_half(F2& r, int h, Fn fn) {
  if (h) r.y = fn(r.y);
  else r.x = fn(r.x);
}

// ---------------------------------------------------------------- forward row step

// The forward update of one row k of one time step, over a lane's column pair, as the scalar
// `one` of fd_fwd_warp2 (fd_warp.cuh) and in its operation order.  SLOW rows are the checked
// ones: border rows, the free surface, sources; the others take the check-free path.
struct C2Fwd {
  FdGeom g;
  C2Lane L;
  int st;           // source type 1..5
  int sz;           // source row
  int s_pr, s_h;    // source column's pair and half
  int s_pr1, s_h1;  // column sx+1 (type 2 writes ww there too)

  __device__ __forceinline__ bool rowin(int z) const { return z >= 1 && z <= g.NZ - 2; }

  // new ww at row k from state rows R0 = k, R1 = k+1 (:227-228), sources (:286-300)
  template <bool SLOW>
  __device__ __forceinline__ F2 vel_w(const SP& R0, const MP& m0, const SP& R1, int k, float sv) const {
    const F2 b1 = (SLOW && k == g.pad_top) ? L.dl2 : L.dl;
    F2 w = m0.te * R0.ww + b1 * ((dL(R0.xz) + R1.zz) - R0.zz);
    if (SLOW) {
      if (!rowin(k)) w = R0.ww;
      if (k == sz) {
        if (L.pr == s_pr && st != 1 && st != 4) on_half(w, s_h, [&](float v) { return st == 5 ? sv : v + sv; });
        if (st == 2 && L.pr == s_pr1) on_half(w, s_h1, [&](float v) { return v + sv; });
      }
    }
    return w;
  }
  // new uu at row k from state rows R0 = k-1 (xz above), R1 = k (materials t = temp of row k) (:225-226)
  template <bool SLOW>
  __device__ __forceinline__ F2 vel_u(const SP& R0, const SP& R1, F2 t, int k, float sv) const {
    const F2 b = (SLOW && k == g.pad_top) ? L.dl2 : L.dl;
    F2 u = t * R1.uu + b * ((dR(R1.xx) + R1.xz) - R0.xz);
    if (SLOW) {
      if (!rowin(k)) u = R1.uu;
      if (L.pr == s_pr) {
        if (k == sz && (st == 2 || st == 3)) on_half(u, s_h, [&](float v) { return v + sv; });
        if (k == sz - 1 && st == 2) on_half(u, s_h, [&](float v) { return v - sv; });
      }
    }
    return u;
  }
  struct Strain {
    F2 fux, bwz, sg;  // sg = fuz + bwx, the third snapshot field
  };
  // One row k: R0 = state row k (materials m0), R1 = row k+1 (temp t1); wn_prev = new ww of
  // row k-1, un_cur = new uu of row k on entry, those of rows k and k+1 on exit.  Returns the
  // new state of row k and its strains.
  template <bool SLOW>
  __device__ __forceinline__ SP row(const SP& R0, const MP& m0, const SP& R1, F2 t1, int k, float sv, F2& wn_prev,
                                    F2& un_cur, Strain& sn) const {
    const F2 wn = vel_w<SLOW>(R0, m0, R1, k, sv);
    const F2 un_next = vel_u<SLOW>(R0, R1, t1, k + 1, sv);
    // strains at row k (:302-306)
    const F2 fux = dL(un_cur);
    const F2 fuz = un_next - un_cur;
    const F2 bwx = dR(wn);
    const F2 bwz = wn - wn_prev;
    F2 xo = R0.xx, zo = R0.zz;
    if (SLOW && k == sz && (st == 1 || st == 4) && L.pr == s_pr) {  // :286-298, before the stress update
      if (st == 1) on_half(xo, s_h, [&](float v) { return v + sv; });
      on_half(zo, s_h, [&](float v) { return v + sv; });
    }
    // stresses at row k (:334-336), free surface (:340)
    const F2 d = L.dl;
    const F2 sg = fuz + bwx;
    const F2 xxn = m0.te * xo + (m0.ca * fux + m0.cl * bwz) * d;
    F2 zzn = m0.te * zo + (m0.ca * bwz + m0.cl * fux) * d;
    const F2 xzn = m0.te * R0.xz + (m0.cm1 * sg) * d;
    if (SLOW && k == g.pad_top) zzn = F2{0.f, 0.f};
    SP r{un_cur, wn, xxn, zzn, xzn};
    if (SLOW && !rowin(k)) r = R0;  // border rows keep their state
    sn = Strain{fux, bwz, sg};
    wn_prev = wn;
    un_cur = un_next;
    return r;
  }
};

__device__ __forceinline__ C2Fwd col2_fwd(const FwdArgs<float>& a, const C2Lane& L, int shot) {
  const int2 sp = a.src[shot];
  C2Fwd f;
  f.g = a.g;
  f.L = L;
  f.st = a.src_type;
  f.sz = sp.x;
  f.s_pr = sp.y >> 1;
  f.s_h = sp.y & 1;
  f.s_pr1 = (sp.y + 1) >> 1;
  f.s_h1 = (sp.y + 1) & 1;
  return f;
}

// ---------------------------------------------------------------- forward kernels

// Output planes of one shot in the pair layout.
struct C2Out {
  float4* a;
  float4* b;
  float2* c;
  __device__ __forceinline__ void put(int o, const SP& r) const {
    a[o] = make_float4(r.uu.x, r.uu.y, r.ww.x, r.ww.y);
    b[o] = make_float4(r.xx.x, r.xx.y, r.zz.x, r.zz.y);
    c[o] = make_float2(r.xz.x, r.xz.y);
  }
};

__device__ __forceinline__ C2Stage col2_stage(const float* sb, const float4* mat, size_t F, const C2Lane& L, int NS,
                                              int P, int zmax) {
  extern __shared__ __align__(16) unsigned char wsmem[];
  return C2Stage{reinterpret_cast<const float4*>(sb) + L.prc, reinterpret_cast<const float4*>(sb + 2 * F) + L.prc,
                 reinterpret_cast<const float2*>(sb + 4 * F) + L.prc, mat + 2 * L.prc,
                 reinterpret_cast<C2Slot*>(wsmem) + (threadIdx.x >> 5) * NS, P, zmax, L.lane};
}
__device__ __forceinline__ C2Out col2_out(float* ob, size_t F, const C2Lane& L) {
  return C2Out{reinterpret_cast<float4*>(ob) + L.prc, reinterpret_cast<float4*>(ob + 2 * F) + L.prc,
               reinterpret_cast<float2*>(ob + 4 * F) + L.prc};
}

// Snapshot fields (fux, bwz, fuz+bwx) of one interior row, as a pair per field.
__device__ __forceinline__ void col2_put_snap(float* snap_base, size_t plane, const FdGeom& g, const C2Lane& L, int z,
                                              const C2Fwd::Strain& sn) {
  float* s0 = snap_base + ((size_t)(z - g.pad_top - 1) * g.nx + (L.x0 - g.nbc));
  *reinterpret_cast<float2*>(s0) = make_float2(sn.fux.x, sn.fux.y);
  *reinterpret_cast<float2*>(s0 + plane) = make_float2(sn.bwz.x, sn.bwz.y);
  *reinterpret_cast<float2*>(s0 + 2 * plane) = make_float2(sn.sg.x, sn.sg.y);
}

// seismo_w / seismo_u of one step at the receiver row (:342-345)
__device__ __forceinline__ void col2_record(const FwdArgs<float>& a, int shot, int step, int2 rj, const SP& r) {
  const size_t base = ((size_t)shot * a.g.nt + step) * a.g.ng;
  if (rj.x >= 0) {
    a.seis_w[base + rj.x] = r.ww.x;
    if (a.seis_u) a.seis_u[base + rj.x] = r.uu.x;
  }
  if (rj.y >= 0) {
    a.seis_w[base + rj.y] = r.ww.y;
    if (a.seis_u) a.seis_u[base + rj.y] = r.uu.y;
  }
}

// One forward time step over a chunk of rows (the odd step of a span; fd_fwd_col2 runs pairs).
template <int NW, int NS, bool SNAP>
__global__ void __launch_bounds__(32 * NW) fd_fwd_col1(FwdArgs<float> a, int it) {
  static_assert(NS >= 4 && NS % 2 == 0, "rows k, k+1 in use, at least two in flight; even for the unrolled rotation");
  const FdGeom& g = a.g;
  int strip, chunk, shot;
  if (!warp_tile(g, a.n_shots, NW, strip, chunk, shot)) return;
  const C2Lane L = col2_lane(g, strip, a.dtx);
  const C2Fwd op = col2_fwd(a, L, shot);
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const int P = g.pitch >> 1;
  const size_t F = g.field;
  const C2Stage ld = col2_stage(a.in + (size_t)shot * 5 * F, a.mat, F, L, NS, P, ze);
  const C2Out out = col2_out(a.out + (size_t)shot * 5 * F, F, L);
  const float sv = a.s[it];
  const int2 rj = col2_receivers(g, L, a.seis_w != nullptr);
  const size_t plane = (size_t)g.nz * g.nx;
  const bool snapc = SNAP && L.own && L.x0 >= g.nbc && L.x0 < g.nbc + g.nx;
  float* snap_base = SNAP ? a.snap + ((size_t)shot * g.nrec + (it / g.nt_wf - a.rec0)) * 3 * plane : nullptr;

  // row r is staged in slot (r - zs + 1) % NS and held in RR / MR[(r - zs + 1) & 1]
#pragma unroll
  for (int u = 0; u < NS; ++u) ld.issue(u, zs - 1 + u);
  if (warp_cancelled(a.cancel)) {  // the flag load overlaps the rows in flight
    wcp_wait<0>();
    return;
  }
  wcp_wait<NS - 2>();
  SP RR[2];
  MP MR[2];
  ld.read(RR[0], MR[0], 0);
  ld.read(RR[1], MR[1], 1);
  F2 wn_prev = op.vel_w<true>(RR[0], MR[0], RR[1], zs - 1, sv);   // new ww of row zs-1
  F2 un_cur = op.vel_u<true>(RR[0], RR[1], MR[1].te, zs, sv);     // new uu of row zs
  auto step = [&](auto slow_tag, int c0, int s1, int spf, int k) {
    constexpr bool SLOW = decltype(slow_tag)::value;
    ld.issue(spf, k + NS - 1);
    wcp_wait<NS - 2>();  // row k+1 has landed
    ld.read(RR[c0 ^ 1], MR[c0 ^ 1], s1);
    C2Fwd::Strain sn;
    const SP r = op.template row<SLOW>(RR[c0], MR[c0], RR[c0 ^ 1], MR[c0 ^ 1].te, k, sv, wn_prev, un_cur, sn);
    if (L.own) out.put(k * P, r);
    if (SLOW && k == g.gz) col2_record(a, shot, it, rj, r);
    if (SNAP && snapc && k >= g.pad_top + 1 && k < g.pad_top + 1 + g.nz) col2_put_snap(snap_base, plane, g, L, k, sn);
  };
  auto row = [&](int c0, int s1, int spf, int k) {
    if (k == g.pad_top || k == g.gz || k == g.NZ - 2 || (k >= op.sz - 2 && k <= op.sz))
      step(std::true_type{}, c0, s1, spf, k);
    else
      step(std::false_type{}, c0, s1, spf, k);
  };
  // row k = zs + u (mod NS): in RR[(u + 1) & 1]; row k+1 goes to RR[u & 1] from slot (u + 2) % NS
  int k = zs;
  for (; k + NS <= ze; k += NS) {
#pragma unroll
    for (int u = 0; u < NS; ++u) row((u + 1) & 1, (u + 2) % NS, u, k + u);
  }
#pragma unroll
  for (int u = 0; u < NS - 1; ++u)
    if (k + u < ze) row((u + 1) & 1, (u + 2) % NS, u, k + u);
  wcp_wait<0>();  // no copy may still target this warp's slots at exit
}

// Steps it and it+1 in one sweep, as fd_fwd_warp2: the state after step it (S1) is formed row
// by row and kept in registers, and step it+1 runs one row behind it on S1.  SNAPSUB: which of
// the two steps writes strain snapshots (-1 neither).
template <int NW, int NS, int SNAPSUB>
__global__ void __launch_bounds__(32 * NW) fd_fwd_col2(FwdArgs<float> a, int it) {
  static_assert(NS >= 4 && NS % 2 == 0, "rows k, k+1 in use, at least two in flight; even for the unrolled rotation");
  const FdGeom& g = a.g;
  int strip, chunk, shot;
  if (!warp_tile(g, a.n_shots, NW, strip, chunk, shot)) return;
  const C2Lane L = col2_lane(g, strip, a.dtx);
  const C2Fwd op = col2_fwd(a, L, shot);
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const int P = g.pitch >> 1;
  const size_t F = g.field;
  const C2Stage ld = col2_stage(a.in + (size_t)shot * 5 * F, a.mat, F, L, NS, P, min(ze + 1, g.NZ - 1));
  const C2Out out = col2_out(a.out + (size_t)shot * 5 * F, F, L);
  const float sv1 = a.s[it], sv2 = a.s[it + 1];
  const int2 rj = col2_receivers(g, L, a.seis_w != nullptr);
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  const bool snapc = SNAPSUB >= 0 && L.own && L.x0 >= g.nbc && L.x0 < g.nbc + g.nx;
  float* snap_base = SNAPSUB >= 0 ? a.snap + ((size_t)shot * g.nrec + ((it + (SNAPSUB > 0 ? 1 : 0)) / g.nt_wf -
                                                                       a.rec0)) * 3 * plane
                                  : nullptr;

  // State row r is staged in slot (r - zs + 2) % NS and held in RR / MR[(r - zs) & 1]; S1 row r
  // in T1 / MT[(r - zs + 1) & 1].
#pragma unroll
  for (int u = 0; u < NS; ++u) ld.issue(u, zs - 2 + u);
  if (warp_cancelled(a.cancel)) {  // the flag load overlaps the rows in flight
    wcp_wait<0>();
    return;
  }
  wcp_wait<NS - 2>();
  SP RR[2];
  MP MR[2];
  ld.read(RR[0], MR[0], 0);
  ld.read(RR[1], MR[1], 1);
  F2 wn1 = op.vel_w<true>(RR[0], MR[0], RR[1], zs - 2, sv1);  // first step: new ww of row k1-1
  F2 un1 = op.vel_u<true>(RR[0], RR[1], MR[1].te, zs - 1, sv1);  // and new uu of row k1
  SP T1[2];  // S1 rows k1-1 and k1 (alternating)
  MP MT[2];  // their materials
  F2 wn2, un2;  // second step: new ww of row k1-2, new uu of row k1-1
  // First-step row k1 from state rows RR[c0] (k1) and RR[c0^1] (k1+1, read from slot s1 after
  // staging row k1+NS-1 into slot spf, row k1-1's); its S1 row goes to T1[c1].
  auto first = [&](auto slow_tag, int c0, int s1, int spf, int c1, int k1) {
    constexpr bool SLOW = decltype(slow_tag)::value;
    ld.issue(spf, k1 + NS - 1);
    wcp_wait<NS - 2>();
    ld.read(RR[c0 ^ 1], MR[c0 ^ 1], s1);
    C2Fwd::Strain sn;
    T1[c1] = op.template row<SLOW>(RR[c0], MR[c0], RR[c0 ^ 1], MR[c0 ^ 1].te, k1, sv1, wn1, un1, sn);
    MT[c1] = MR[c0];
    if (SLOW && k1 == g.gz && k1 >= zs && k1 < ze) col2_record(a, shot, it, rj, T1[c1]);  // step it
    if (SNAPSUB == 0 && snapc && k1 >= z_img0 && k1 < z_img1 && k1 >= zs && k1 < ze)
      col2_put_snap(snap_base, plane, g, L, k1, sn);
  };
  // Second-step row j = k1-1 from S1 rows T1[c1^1] (j) and T1[c1] (k1); writes the new state.
  auto second = [&](auto slow_tag, int c1, int j) {
    constexpr bool SLOW = decltype(slow_tag)::value;
    C2Fwd::Strain sn;
    const SP r = op.template row<SLOW>(T1[c1 ^ 1], MT[c1 ^ 1], T1[c1], MT[c1].te, j, sv2, wn2, un2, sn);
    if (L.own) out.put(j * P, r);
    if (SLOW && j == g.gz) col2_record(a, shot, it + 1, rj, r);  // step it+1
    if (SNAPSUB == 1 && snapc && j >= z_img0 && j < z_img1) col2_put_snap(snap_base, plane, g, L, j, sn);
  };
  const int mb = zs - 2;
  const unsigned long long slowm = slow_rows(g.NZ, g.pad_top, g.gz, zs, op.sz);
  // peeled: S1 rows zs-1 and zs, then the second step's prologue (new ww of row zs-1, new uu of row zs)
  first(std::true_type{}, 1, 2 % NS, 0, 0, zs - 1);
  first(std::true_type{}, 0, 3 % NS, 1, 1, zs);
  wn2 = op.vel_w<true>(T1[0], MT[0], T1[1], zs - 1, sv2);
  un2 = op.vel_u<true>(T1[0], T1[1], MT[1].te, zs, sv2);
  // Rows k1 = zs+1 .. ze, u = k1 - zs - 1: state row k1 is RR[(u + 1) & 1], row k1+1 comes from
  // slot (u + 4) % NS, row k1-1's slot (u + 2) % NS is restaged, and S1 row k1 goes to T1[u & 1].
  auto both = [&](auto slow_tag, int u, int k1) {
    first(slow_tag, (u + 1) & 1, (u + 4) % NS, (u + 2) % NS, u & 1, k1);
    second(slow_tag, u & 1, k1 - 1);
  };
  int k1 = zs + 1;
  for (; k1 + NS <= ze + 1; k1 += NS) {
    const unsigned m = (unsigned)(slowm >> (k1 - 1 - mb));  // bit i: row k1-1+i has checks
#pragma unroll
    for (int u = 0; u < NS; ++u) {
      if (m & (3u << u)) both(std::true_type{}, u, k1 + u);  // row k1+u or k1+u-1
      else both(std::false_type{}, u, k1 + u);
    }
  }
#pragma unroll
  for (int u = 0; u < NS - 1; ++u)
    if (k1 + u <= ze) both(std::true_type{}, u, k1 + u);
  wcp_wait<0>();
}

// ---------------------------------------------------------------- adjoint row step

// The adjoint update of one row k of one step over a lane's column pair, as the scalar `one`
// of fd_adj_warp2 (fd_warp.cuh) and in its operation order.
struct C2Adj {
  FdGeom g;
  C2Lane L;
  int rec_h0, rec_h1;  // the halves that take the adjoint source at the receiver row (halo lanes too)

  struct Prod {
    F2 p1, p2, p3, q1, q2;  // ca*xx, cl*zz, cm1*xz, cl*xx, ca*zz
  };
  __device__ __forceinline__ static Prod prod(const SP& r, const MP& m) {
    return Prod{m.ca * r.xx, m.cl * r.zz, m.cm1 * r.xz, m.cl * r.xx, m.ca * r.zz};
  }
  __device__ __forceinline__ bool rowin(int z) const { return z >= 1 && z <= g.NZ - 2; }

  // new ww at row k (rows R0 = k, products Q0 / Q1 of rows k / k+1) (:184-187), injection (:238-242)
  template <bool SLOW>
  __device__ __forceinline__ F2 vel_w(const SP& R0, const MP& m0, const Prod& Q0, const Prod& Q1, int k,
                                      const F2& inj) const {
    const F2 b1 = (SLOW && k == g.pad_top) ? L.dl2 : L.dl;
    const F2 dw = ((Q1.q1 - Q0.q1) + (Q1.q2 - Q0.q2)) + dR(Q0.p3);
    F2 w = m0.te * R0.ww - b1 * dw;
    if (SLOW) {
      if (!rowin(k)) w = R0.ww;
      if (k == g.gz) {
        if (rec_h0) w.x = w.x + inj.x;
        if (rec_h1) w.y = w.y + inj.y;
      }
    }
    return w;
  }
  // new uu at row k1 (products Q0 of row k1-1, state R1 / products Q1 / temp t1 of row k1) (:182-183)
  template <bool SLOW>
  __device__ __forceinline__ F2 vel_u(const Prod& Q0, const SP& R1, const Prod& Q1, F2 t1, int k1) const {
    const F2 b = (SLOW && k1 == g.pad_top) ? L.dl2 : L.dl;
    const F2 du = (dL(Q1.p1) + dL(Q1.p2)) + (Q1.p3 - Q0.p3);
    F2 u = t1 * R1.uu - b * du;
    if (SLOW && !rowin(k1)) u = R1.uu;
    return u;
  }
  // One row k on rows R0 = k (materials m0, products Q0) and R1 = k+1 (temp t1, products Q1);
  // wn_prev = new ww of row k-1, un_cur = new uu of row k on entry, those of rows k, k+1 on
  // exit.  Returns the new state of row k (:245-248 stresses, :270 free surface).
  template <bool SLOW>
  __device__ __forceinline__ SP row(const SP& R0, const MP& m0, const Prod& Q0, const SP& R1, F2 t1, const Prod& Q1,
                                    int k, const F2& inj, F2& wn_prev, F2& un_cur) const {
    const F2 wn = vel_w<SLOW>(R0, m0, Q0, Q1, k, inj);
    const F2 un_next = vel_u<SLOW>(Q0, R1, Q1, t1, k + 1);
    const F2 d = L.dl;
    const F2 xxn = m0.te * R0.xx - d * dR(un_cur);
    F2 zzn = m0.te * R0.zz - d * (wn - wn_prev);
    const F2 xzn = (m0.te * R0.xz - d * (un_next - un_cur)) - d * dL(wn);
    if (SLOW && k == g.pad_top) zzn = F2{0.f, 0.f};
    SP r{un_cur, wn, xxn, zzn, xzn};
    if (SLOW && !rowin(k)) r = R0;  // border rows keep their state
    wn_prev = wn;
    un_cur = un_next;
    return r;
  }
};

__device__ __forceinline__ C2Adj col2_adj(const FdGeom& g, const C2Lane& L) {
  C2Adj o;
  o.g = g;
  o.L = L;
  int r[2];
  for (int h = 0; h < 2; ++h) {
    const int x = L.x0 + h;
    r[h] = x >= 0 && x < g.NX && x >= g.gx && (x - g.gx) % g.dg == 0 && (x - g.gx) / g.dg < g.ng;
  }
  o.rec_h0 = r[0];
  o.rec_h1 = r[1];
  return o;
}

// dt * res of one step at the lane's receiver columns (0 elsewhere)
__device__ __forceinline__ F2 col2_inj(const AdjArgs<float>& a, const C2Adj& op, int shot, int step) {
  const FdGeom& g = a.g;
  const size_t base = ((size_t)shot * g.nt + step) * g.ng;
  F2 v{0.f, 0.f};
  if (op.rec_h0) v.x = a.dt * a.res[base + (op.L.x0 - g.gx) / g.dg];
  if (op.rec_h1) v.y = a.dt * a.res[base + (op.L.x0 + 1 - g.gx) / g.dg];
  return v;
}

// Imaging operands of a row: strain pairs and the image sum pairs (as doubles; FP32 sums
// are converted exactly).
struct C2Img {
  F2 fx, bz, sg;
  double2 c0, c1, c2;
};

// Imaging condition (:274-279) at one interior row: FP32 sums as the reference accumulates them
// (img_f), else FP64.
__device__ __forceinline__ void col2_image(const C2Img& m, const SP& r, float* img_f, double* img_b, size_t cell,
                                           size_t plane) {
  const F2 Fs = m.fx + m.bz;
  const F2 tcl = Fs * (r.xx + r.zz);
  const F2 tcm = F2{2.f, 2.f} * ((r.xx * m.fx + r.zz * m.bz) + F2{0.5f, 0.5f} * (r.xz * m.sg));
  const F2 til = Fs * Fs;
  if (img_f) {
    const F2 a0 = F2{(float)m.c0.x, (float)m.c0.y} + tcl;
    const F2 a1 = F2{(float)m.c1.x, (float)m.c1.y} + tcm;
    const F2 a2 = F2{(float)m.c2.x, (float)m.c2.y} + til;
    *reinterpret_cast<float2*>(img_f + cell) = make_float2(a0.x, a0.y);
    *reinterpret_cast<float2*>(img_f + plane + cell) = make_float2(a1.x, a1.y);
    *reinterpret_cast<float2*>(img_f + 2 * plane + cell) = make_float2(a2.x, a2.y);
  } else {
    *reinterpret_cast<double2*>(img_b + cell) = make_double2(m.c0.x + (double)tcl.x, m.c0.y + (double)tcl.y);
    *reinterpret_cast<double2*>(img_b + plane + cell) = make_double2(m.c1.x + (double)tcm.x, m.c1.y + (double)tcm.y);
    *reinterpret_cast<double2*>(img_b + 2 * plane + cell) = make_double2(m.c2.x + (double)til.x, m.c2.y + (double)til.y);
  }
}

// ---------------------------------------------------------------- adjoint kernels

// One adjoint step over a chunk of rows (the odd step of a span; fd_adj_col2 runs pairs).  The
// imaging operands of the next row are loaded into registers one row ahead.
template <int NW, int NS, bool IMG>
__global__ void __launch_bounds__(32 * NW) fd_adj_col1(AdjArgs<float> a, int it) {
  static_assert(NS >= 4 && NS % 2 == 0, "rows k, k+1 in use, at least two in flight; even for the unrolled rotation");
  const FdGeom& g = a.g;
  int strip, chunk, shot;
  if (!warp_tile(g, a.n_shots, NW, strip, chunk, shot)) return;
  const C2Lane L = col2_lane(g, strip, a.dtx);
  const C2Adj op = col2_adj(g, L);
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const int P = g.pitch >> 1;
  const size_t F = g.field;
  const C2Stage ld = col2_stage(a.in + (size_t)shot * 5 * F, a.mat, F, L, NS, P, ze);
  const C2Out out = col2_out(a.out + (size_t)shot * 5 * F, F, L);
  const F2 inj = col2_inj(a, op, shot, it);
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  const bool ximg = IMG && L.own && L.x0 >= g.nbc && L.x0 < g.nbc + g.nx;
  const float* snap_b = IMG ? a.snap + ((size_t)shot * g.nrec + (it / g.nt_wf - a.rec0)) * 3 * plane : nullptr;
  double* img_b = a.img + (size_t)shot * 3 * plane;
  float* img_f = a.img32 ? a.img32 + (size_t)shot * 3 * plane : nullptr;
  auto cell_of = [&](int z) { return (size_t)(z - z_img0) * g.nx + (L.x0 - g.nbc); };
  auto img_row = [&](int z) { return IMG && ximg && z >= z_img0 && z < z_img1 && z < ze; };
  auto load_img = [&](C2Img& m, int z) {
    if (img_row(z)) {
      const size_t c = cell_of(z);
      const float2 f0 = *reinterpret_cast<const float2*>(snap_b + c);
      const float2 f1 = *reinterpret_cast<const float2*>(snap_b + plane + c);
      const float2 f2 = *reinterpret_cast<const float2*>(snap_b + 2 * plane + c);
      m.fx = F2{f0.x, f0.y};
      m.bz = F2{f1.x, f1.y};
      m.sg = F2{f2.x, f2.y};
      if (img_f) {
        const float2 c0 = *reinterpret_cast<const float2*>(img_f + c);
        const float2 c1 = *reinterpret_cast<const float2*>(img_f + plane + c);
        const float2 c2 = *reinterpret_cast<const float2*>(img_f + 2 * plane + c);
        m.c0 = make_double2(c0.x, c0.y);
        m.c1 = make_double2(c1.x, c1.y);
        m.c2 = make_double2(c2.x, c2.y);
      } else {
        m.c0 = *reinterpret_cast<const double2*>(img_b + c);
        m.c1 = *reinterpret_cast<const double2*>(img_b + plane + c);
        m.c2 = *reinterpret_cast<const double2*>(img_b + 2 * plane + c);
      }
    }
  };

#pragma unroll
  for (int u = 0; u < NS; ++u) ld.issue(u, zs - 1 + u);
  if (warp_cancelled(a.cancel)) {  // the flag load overlaps the rows in flight
    wcp_wait<0>();
    return;
  }
  wcp_wait<NS - 2>();
  SP RR[2];
  MP MR[2];
  ld.read(RR[0], MR[0], 0);
  ld.read(RR[1], MR[1], 1);
  C2Adj::Prod QP[2] = {C2Adj::prod(RR[0], MR[0]), C2Adj::prod(RR[1], MR[1])};
  C2Img IM[2] = {};
  load_img(IM[0], zs);
  F2 wn_prev = op.vel_w<true>(RR[0], MR[0], QP[0], QP[1], zs - 1, inj);  // new ww of row zs-1
  F2 un_cur = op.vel_u<true>(QP[0], RR[1], QP[1], MR[1].te, zs);         // new uu of row zs
  // row k: R0 = RR[c0] (products QP[c0], imaging IM[i0]); row k+1 comes from slot s1 into c0^1
  auto step = [&](auto slow_tag, int c0, int s1, int spf, int i0, int k) {
    constexpr bool SLOW = decltype(slow_tag)::value;
    ld.issue(spf, k + NS - 1);
    load_img(IM[i0 ^ 1], k + 1);
    wcp_wait<NS - 2>();  // row k+1 has landed
    ld.read(RR[c0 ^ 1], MR[c0 ^ 1], s1);
    QP[c0 ^ 1] = C2Adj::prod(RR[c0 ^ 1], MR[c0 ^ 1]);
    const SP r = op.template row<SLOW>(RR[c0], MR[c0], QP[c0], RR[c0 ^ 1], MR[c0 ^ 1].te, QP[c0 ^ 1], k, inj, wn_prev,
                                       un_cur);
    if (L.own) out.put(k * P, r);
    if (img_row(k)) col2_image(IM[i0], r, img_f, img_b, cell_of(k), plane);
  };
  auto row = [&](int c0, int s1, int spf, int i0, int k) {
    if (k == g.pad_top || k == g.gz || k == g.NZ - 2) step(std::true_type{}, c0, s1, spf, i0, k);
    else step(std::false_type{}, c0, s1, spf, i0, k);
  };
  // row k = zs + u: registers RR / QP[(u + 1) & 1], imaging IM[u & 1]
  int k = zs;
  for (; k + NS <= ze; k += NS) {
#pragma unroll
    for (int u = 0; u < NS; ++u) row((u + 1) & 1, (u + 2) % NS, u, u & 1, k + u);
  }
#pragma unroll
  for (int u = 0; u < NS - 1; ++u)
    if (k + u < ze) row((u + 1) & 1, (u + 2) % NS, u, u & 1, k + u);
  wcp_wait<0>();
}

// Adjoint steps it and it-1 in one sweep, as fd_adj_warp2: the state after step it (S1) is
// formed row by row in registers and step it-1 runs one row behind it.  IMGSUB: which of the two
// steps applies the imaging condition (0: step it, 1: step it-1, -1 neither); its operands are
// staged by cp.async beside the state rows.
template <int NW, int NS, int IMGSUB>
__global__ void __launch_bounds__(32 * NW) fd_adj_col2(AdjArgs<float> a, int it) {
  static_assert(NS >= 4 && NS % 2 == 0, "rows k, k+1 in use, at least two in flight; even for the unrolled rotation");
  const FdGeom& g = a.g;
  int strip, chunk, shot;
  if (!warp_tile(g, a.n_shots, NW, strip, chunk, shot)) return;
  const C2Lane L = col2_lane(g, strip, a.dtx);
  const C2Adj op = col2_adj(g, L);
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const int P = g.pitch >> 1;
  const size_t F = g.field;
  const C2Stage ld = col2_stage(a.in + (size_t)shot * 5 * F, a.mat, F, L, NS, P, min(ze + 1, g.NZ - 1));
  const C2Out out = col2_out(a.out + (size_t)shot * 5 * F, F, L);
  const F2 inj1 = col2_inj(a, op, shot, it), inj2 = col2_inj(a, op, shot, it - 1);
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  const bool ximg = IMGSUB >= 0 && L.own && L.x0 >= g.nbc && L.x0 < g.nbc + g.nx;
  const float* snap_b = IMGSUB >= 0 ? a.snap + ((size_t)shot * g.nrec + ((it - (IMGSUB > 0 ? 1 : 0)) / g.nt_wf -
                                                                         a.rec0)) * 3 * plane
                                    : nullptr;
  double* img_b = a.img + (size_t)shot * 3 * plane;
  float* img_f = a.img32 ? a.img32 + (size_t)shot * 3 * plane : nullptr;
  auto cell_of = [&](int z) { return (size_t)(z - z_img0) * g.nx + (L.x0 - g.nbc); };
  auto img_row = [&](int z) { return IMGSUB >= 0 && z >= z_img0 && z < z_img1 && z >= zs && z < ze; };
  extern __shared__ __align__(16) unsigned char wsmem[];
  C2ImgSlot* islots = reinterpret_cast<C2ImgSlot*>(wsmem + (size_t)NW * NS * sizeof(C2Slot)) + (threadIdx.x >> 5) * NS;
  const int lane = L.lane;
  auto issue_img = [&](int slot, int z) {
    if (IMGSUB >= 0 && ximg && img_row(z)) {
      const size_t c = cell_of(z);
      C2ImgSlot& s = islots[slot];
      wcp8(&s.fx[lane], snap_b + c);
      wcp8(&s.bz[lane], snap_b + plane + c);
      wcp8(&s.sg[lane], snap_b + 2 * plane + c);
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        if (img_f) wcp8(&s.c[i][lane], img_f + i * plane + c);  // a float pair in the first half
        else wcp16(&s.c[i][lane], img_b + i * plane + c);
      }
    }
  };
  auto read_img = [&](C2Img& m, int slot) {
    const C2ImgSlot& s = islots[slot];
    const float2 f0 = s.fx[lane], f1 = s.bz[lane], f2 = s.sg[lane];
    m.fx = F2{f0.x, f0.y};
    m.bz = F2{f1.x, f1.y};
    m.sg = F2{f2.x, f2.y};
    if (img_f) {
      const float2 c0 = *reinterpret_cast<const float2*>(&s.c[0][lane]);
      const float2 c1 = *reinterpret_cast<const float2*>(&s.c[1][lane]);
      const float2 c2 = *reinterpret_cast<const float2*>(&s.c[2][lane]);
      m.c0 = make_double2(c0.x, c0.y);
      m.c1 = make_double2(c1.x, c1.y);
      m.c2 = make_double2(c2.x, c2.y);
    } else {
      m.c0 = s.c[0][lane];
      m.c1 = s.c[1][lane];
      m.c2 = s.c[2][lane];
    }
  };
  auto image = [&](const C2Img& m, const SP& r, int z) {
    if (ximg && img_row(z)) col2_image(m, r, img_f, img_b, cell_of(z), plane);
  };

  // state rows staged from zs-2: row r in slot (r - zs + 2) % NS and RR / MR / QR[(r - zs) & 1]
#pragma unroll
  for (int u = 0; u < NS; ++u) {
    issue_img(u, zs - 2 + u);
    ld.issue(u, zs - 2 + u);  // commits the imaging copies too
  }
  if (warp_cancelled(a.cancel)) {  // the flag load overlaps the rows in flight
    wcp_wait<0>();
    return;
  }
  wcp_wait<NS - 2>();
  SP RR[2];
  MP MR[2];
  ld.read(RR[0], MR[0], 0);
  ld.read(RR[1], MR[1], 1);
  C2Adj::Prod QR[2] = {C2Adj::prod(RR[0], MR[0]), C2Adj::prod(RR[1], MR[1])};
  F2 wn1 = op.vel_w<true>(RR[0], MR[0], QR[0], QR[1], zs - 2, inj1);  // first step: new ww of row k1-1
  F2 un1 = op.vel_u<true>(QR[0], RR[1], QR[1], MR[1].te, zs - 1);     // and new uu of row k1
  SP T1[2];            // S1 rows, T1[(r - zs + 1) & 1]
  MP MT[2];            // their materials
  C2Adj::Prod QT[2];   // their products
  C2Img IMp{};         // imaging operands of the second step's row (read before its slot is restaged)
  F2 wn2, un2;         // second step: new ww of row k1-2, new uu of row k1-1
  // first-step row k1; s0: slot of state row k1 (its imaging operands when step it images)
  auto first = [&](auto slow_tag, int c0, int s0, int s1, int spf, int c1, int k1) {
    constexpr bool SLOW = decltype(slow_tag)::value;
    if (IMGSUB == 1) read_img(IMp, spf);  // row k1-1, which the second step images next
    issue_img(spf, k1 + NS - 1);
    ld.issue(spf, k1 + NS - 1);
    wcp_wait<NS - 2>();
    ld.read(RR[c0 ^ 1], MR[c0 ^ 1], s1);
    QR[c0 ^ 1] = C2Adj::prod(RR[c0 ^ 1], MR[c0 ^ 1]);
    T1[c1] = op.template row<SLOW>(RR[c0], MR[c0], QR[c0], RR[c0 ^ 1], MR[c0 ^ 1].te, QR[c0 ^ 1], k1, inj1, wn1,
                                   un1);
    MT[c1] = MR[c0];
    QT[c1] = C2Adj::prod(T1[c1], MR[c0]);
    if (IMGSUB == 0) {
      C2Img m;
      read_img(m, s0);
      image(m, T1[c1], k1);
    }
  };
  // second-step row j = k1-1 from S1 rows T1[c1^1] (j) and T1[c1] (k1); writes the new state
  auto second = [&](auto slow_tag, int c1, int j) {
    constexpr bool SLOW = decltype(slow_tag)::value;
    const SP r = op.template row<SLOW>(T1[c1 ^ 1], MT[c1 ^ 1], QT[c1 ^ 1], T1[c1], MT[c1].te, QT[c1], j, inj2, wn2,
                                       un2);
    if (L.own) out.put(j * P, r);
    if (IMGSUB == 1) image(IMp, r, j);
  };
  const int mb = zs - 2;
  const unsigned long long slowm = slow_rows(g.NZ, g.pad_top, g.gz, zs);
  first(std::true_type{}, 1, 1, 2 % NS, 0, 0, zs - 1);
  first(std::true_type{}, 0, 2 % NS, 3 % NS, 1, 1, zs);
  wn2 = op.vel_w<true>(T1[0], MT[0], QT[0], QT[1], zs - 1, inj2);
  un2 = op.vel_u<true>(QT[0], T1[1], QT[1], MT[1].te, zs);
  auto both = [&](auto slow_tag, int u, int k1) {
    first(slow_tag, (u + 1) & 1, (u + 3) % NS, (u + 4) % NS, (u + 2) % NS, u & 1, k1);
    second(slow_tag, u & 1, k1 - 1);
  };
  int k1 = zs + 1;
  for (; k1 + NS <= ze + 1; k1 += NS) {
    const unsigned m = (unsigned)(slowm >> (k1 - 1 - mb));  // bit i: row k1-1+i has checks
#pragma unroll
    for (int u = 0; u < NS; ++u) {
      if (m & (3u << u)) both(std::true_type{}, u, k1 + u);  // row k1+u or k1+u-1
      else both(std::false_type{}, u, k1 + u);
    }
  }
#pragma unroll
  for (int u = 0; u < NS - 1; ++u)
    if (k1 + u <= ze) both(std::true_type{}, u, k1 + u);
  wcp_wait<0>();
}

}  // namespace swd
