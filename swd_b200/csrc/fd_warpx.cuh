// Two shots per warp for the two-step warp-streaming kernels (engine FD schedule 5).
//
// fd_fwd_warp2x / fd_adj_warp2x are fd_fwd_warp2 / fd_adj_warp2 with each lane carrying the
// same column of two shots of the batch (shots 2p and 2p+1).  The two shots' values of a field
// sit in one 64-bit register pair, and every add, subtract and multiply of the stencil is one
// packed instruction, so a warp issues half the floating-point instructions per shot; the
// material row, the row bookkeeping and the loop control are shared by the two shots.  Each
// half of a packed instruction rounds to nearest as the scalar instruction does, so the results
// are bit-identical to the one-shot kernels (compiled with -fmad=false) as long as no multiply
// is fused into the add that consumes it (below).  The layout in HBM is that of the
// one-shot kernels (each shot cell-interleaved), so the one-step kernels still run the odd
// steps of a span.  With an odd number of shots the last warp carries its shot twice: both
// halves compute the same values and store them to the same places.
//
// Reference loops:  core/eigen_staggerfd_single.cpp:207-357 (forward),
//                   core/eigen_e2drtm_single.cpp:181-283 (adjoint + imaging).
#pragma once
#include "fd_smem.cuh"  // adj_vel_u / adj_vel_w
#include "fd_warp.cuh"

namespace swd {

// ------------------------------------------------------------ packed FP32 pairs

struct F2 {
  float x, y;  // shot 2p, shot 2p+1
};
union F2Bits {
  F2 f;
  unsigned long long u;
};
// The code generator fuses mul.rn.f32x2 into a following add.rn.f32x2 or sub.rn.f32x2 (the
// explicit rounding mode and -fmad=false do not stop it for the packed forms), which would
// round once where the scalar kernels round twice.  So a product is formed as
// fma.rn.f32x2(a, b, z) with z = (-0, -0) read from constant memory: a*b + (-0) rounds exactly
// as a*b does (signed zeros included), and since z is not a compile-time constant the fma is
// neither turned back into a multiply nor merged with the add.  On B200 this matched the
// scalar results bit for bit on 2^21 random operand pairs in a*b+c*d, a*b-c*d,
// ((a-b)+c)*d+a*c and (a*b+c*d)*a, subnormals and signed zeros included.
static __constant__ unsigned long long kF2NegZero = 0x8000000080000000ull;
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
  F2Bits r, p{a}, q{b};
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.u) : "l"(p.u), "l"(q.u));
  return r.f;
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  F2Bits r, p{a}, q{b};
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.u) : "l"(p.u), "l"(q.u));
  return r.f;
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
  F2Bits r, p{a}, q{b};
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.u) : "l"(p.u), "l"(q.u), "l"(kF2NegZero));
  return r.f;
}
__device__ __forceinline__ F2 bc(float s) { return F2{s, s}; }  // the same value for both shots
__device__ __forceinline__ float get(const F2& v, int h) { return h ? v.y : v.x; }
__device__ __forceinline__ float& at(F2& v, int h) { return h ? v.y : v.x; }
__device__ __forceinline__ F2 shfl_l(F2 v) { return F2{shfl_l(v.x), shfl_l(v.y)}; }
__device__ __forceinline__ F2 shfl_r(F2 v) { return F2{shfl_r(v.x), shfl_r(v.y)}; }

// ------------------------------------------------------------ staging

// A staging slot: one row of a warp's 32 columns, both shots; the material row once.
struct WSlotX {
  float4 q[2][32];  // {uu, ww, xx, zz} per shot
  float4 m[32];     // {temp, ca, cl, cm1}
  float xz[2][32];
};
// The imaging operands of one row, both shots: forward strains, image sums (FP64, or FP32 in
// the first half of each c row).
struct WImgSlotX {
  float fx[2][32], bz[2][32], sg[2][32];
  double c[2][3][32];
};
template <int NW, int NS>
constexpr size_t warpx_smem_bytes() { return (size_t)NW * NS * sizeof(WSlotX); }
template <int NW, int NS>
constexpr size_t warpx_img_smem_bytes() { return (size_t)NW * NS * (sizeof(WSlotX) + sizeof(WImgSlotX)); }

struct M2 {
  F2 te, ca, cl, cm1;  // {temp, ca, cl, cm1} for both shots
};
__device__ __forceinline__ M2 m2(const float4& m) { return M2{bc(m.x), bc(m.y), bc(m.z), bc(m.w)}; }
struct WRowX {
  F2 uu, ww, xx, zz, xz;
  M2 m;
};

struct WStageX {
  const float4* q0;   // shot 2p: this lane's column of {uu, ww, xx, zz}, row 0
  const float4* q1;   // shot 2p+1
  const float* xz0;
  const float* xz1;
  const float4* mat;  // this lane's column of the materials, row 0
  WSlotX* slots;      // this warp's NS slots
  int pitch, zmax, lane;
  // as WStage::issue: rows beyond zmax are not needed (an empty copy group keeps the count)
  __device__ __forceinline__ void issue(int slot, int z) const {
    if (z <= zmax) {
      const int o = max(z, 0) * pitch;  // 32-bit: the engine keeps 5 * NZ * pitch below 2^31
      WSlotX& s = slots[slot];
      wcp16(&s.q[0][lane], q0 + o);
      wcp16(&s.q[1][lane], q1 + o);
      wcp16(&s.m[lane], mat + o);
      wcp4(&s.xz[0][lane], xz0 + o);
      wcp4(&s.xz[1][lane], xz1 + o);
    }
    wcp_commit();
  }
  __device__ __forceinline__ void read(WRowX& r, int slot) const {
    const WSlotX& s = slots[slot];
    const float4 a = s.q[0][lane], b = s.q[1][lane];
    r.uu = F2{a.x, b.x};
    r.ww = F2{a.y, b.y};
    r.xx = F2{a.z, b.z};
    r.zz = F2{a.w, b.w};
    r.xz = F2{s.xz[0][lane], s.xz[1][lane]};
    r.m = m2(s.m[lane]);
  }
};

// ------------------------------------------------------------ forward

// Steps it and it+1 for shots 2p and 2p+1; the row schedule is that of fd_fwd_warp2.
template <int NW, int NS, int SNAPSUB>
__global__ void __launch_bounds__(32 * NW) fd_fwd_warp2x(FwdArgs<float> a, int it) {
  static_assert(NS >= 4 && NS % 2 == 0, "rows k, k+1 in use, at least two in flight; even for the unrolled rotation");
  using T = float;
  const FdGeom& g = a.g;
  int strip, chunk, pr;
  if (!warp_tile(g, (a.n_shots + 1) / 2, NW, strip, chunk, pr)) return;
  const int shot[2] = {2 * pr, min(2 * pr + 1, a.n_shots - 1)};
  const int lane = threadIdx.x & 31;
  const int x = kWarpOut2 * strip + lane - 1;
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const size_t F = g.field;
  const bool xint = x >= 1 && x <= g.NX - 2;
  const bool own = xint && lane >= 2 && lane <= kWarpOut2 + 1;
  const int xc = min(max(x, 0), g.NX - 1);
  const float* sb0 = a.in + (size_t)shot[0] * 5 * F;
  const float* sb1 = a.in + (size_t)shot[1] * 5 * F;
  extern __shared__ __align__(16) unsigned char wsmem[];
  const WStageX ld{reinterpret_cast<const float4*>(sb0) + xc, reinterpret_cast<const float4*>(sb1) + xc,
                   sb0 + 4 * F + xc, sb1 + 4 * F + xc, a.mat + xc,
                   reinterpret_cast<WSlotX*>(wsmem) + (threadIdx.x >> 5) * NS, g.pitch, min(ze + 1, g.NZ - 1), lane};
  float4* oq[2];
  float* oxz[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float* obs = a.out + (size_t)shot[h] * 5 * F;
    oq[h] = reinterpret_cast<float4*>(obs) + xc;
    oxz[h] = obs + 4 * F + xc;
  }
  const int st = a.src_type;
  const int2 sp[2] = {a.src[shot[0]], a.src[shot[1]]};
  const T sv1 = a.s[it], sv2 = a.s[it + 1];
  const T dtx = a.dtx;
  const F2 dtx2 = bc(dtx);
  const F2 dl2 = bc(xint ? dtx : T(0));  // time factor of the fast rows (0: border lane, state kept)
  bool s_w[2], s_wr[2], s_u[2], s_um[2], s_xz[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const bool sc = x == sp[h].y, sr = x == sp[h].y + 1;
    s_w[h] = sc && st != 1 && st != 4;
    s_wr[h] = sr && st == 2;
    s_u[h] = sc && (st == 2 || st == 3);
    s_um[h] = sc && st == 2;
    s_xz[h] = sc && (st == 1 || st == 4);
  }
  const int recj = (a.seis_w != nullptr && own && x >= g.gx && (x - g.gx) % g.dg == 0 && (x - g.gx) / g.dg < g.ng)
                       ? (x - g.gx) / g.dg : -1;
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  const bool snapc = SNAPSUB >= 0 && own && x >= g.nbc && x < g.nbc + g.nx;
  T* snap_base[2];
#pragma unroll
  for (int h = 0; h < 2; ++h)
    snap_base[h] = SNAPSUB >= 0 ? a.snap + ((size_t)shot[h] * g.nrec +
                                            ((it + (SNAPSUB > 0 ? 1 : 0)) / g.nt_wf - a.rec0)) * 3 * plane
                                : nullptr;
  auto bz = [&](int z) -> F2 { return bc(z == g.pad_top ? T(2) * dtx : dtx); };
  auto rowin = [&](int z) { return z >= 1 && z <= g.NZ - 2; };
  auto vel_w = [&](bool inner, F2 ww, F2 xz, F2 xzl, F2 zz, F2 zzd, F2 te, F2 b1) -> F2 {
    return inner ? te * ww + b1 * (((xz - xzl) + zzd) - zz) : ww;
  };
  auto vel_u = [&](bool inner, F2 uu, F2 xx, F2 xxr, F2 xz, F2 xzu, F2 te, F2 b) -> F2 {
    return inner ? te * uu + b * (((xxr - xx) + xz) - xzu) : uu;
  };
  auto src_w = [&](int z, F2 r, T sv) -> F2 {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      T& v = at(r, h);
      if (z == sp[h].x) {
        if (s_w[h]) v = (st == 5) ? sv : v + sv;
        else if (s_wr[h]) v = v + sv;
      }
    }
    return r;
  };
  auto src_u = [&](int z, F2 r, T sv) -> F2 {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      T& v = at(r, h);
      if (s_u[h] && z == sp[h].x) v = v + sv;
      if (s_um[h] && z == sp[h].x - 1) v = v - sv;
    }
    return r;
  };
  struct St { F2 uu, ww, xx, zz, xz; };
  struct Strain { F2 fux, bwz, sg; };
  // One row k of one step (as in fd_fwd_warp2), both shots.
  auto one = [&](auto slow_tag, const St& R0, const M2& m0, const St& R1, F2 t1, int k, T sv, F2& wn_prev,
                 F2& un_cur, Strain& sn) -> St {
    constexpr bool SLOW = decltype(slow_tag)::value;
    const bool in0 = !SLOW || rowin(k);
    const bool in1 = !SLOW || rowin(k + 1);
    const F2 d = SLOW ? dtx2 : dl2;  // fast rows: border lanes keep their state (as fd_fwd_warp2)
    const F2 xzl = shfl_l(R0.xz);
    F2 wn = vel_w(!SLOW || (xint && in0), R0.ww, R0.xz, xzl, R0.zz, R1.zz, m0.te, SLOW ? bz(k) : dl2);
    const F2 xxr = shfl_r(R1.xx);
    F2 un_next = vel_u(!SLOW || (xint && in1), R1.uu, R1.xx, xxr, R1.xz, R0.xz, t1, SLOW ? bz(k + 1) : dl2);
    if (SLOW) {
      wn = src_w(k, wn, sv);
      un_next = src_u(k + 1, un_next, sv);
    }
    const F2 ucl = shfl_l(un_cur);
    const F2 wnr = shfl_r(wn);
    const F2 fux = un_cur - ucl;
    const F2 fuz = un_next - un_cur;
    const F2 bwx = wnr - wn;
    const F2 bwz = wn - wn_prev;
    F2 xo = R0.xx, zo = R0.zz;
    if (SLOW) {
#pragma unroll
      for (int h = 0; h < 2; ++h)
        if (s_xz[h] && k == sp[h].x) {
          if (st == 1) { at(xo, h) = at(xo, h) + sv; at(zo, h) = at(zo, h) + sv; }
          else { at(zo, h) = at(zo, h) + sv; }
        }
    }
    const F2 xxn = m0.te * xo + (m0.ca * fux + m0.cl * bwz) * d;
    F2 zzn = m0.te * zo + (m0.ca * bwz + m0.cl * fux) * d;
    const F2 xzn = m0.te * R0.xz + (m0.cm1 * (fuz + bwx)) * d;
    if (SLOW && k == g.pad_top) zzn = bc(T(0));
    St r{un_cur, wn, xxn, zzn, xzn};
    if (SLOW && !(xint && in0)) r = R0;  // border cells keep their state
    sn = Strain{fux, bwz, fuz + bwx};
    wn_prev = wn;
    un_cur = un_next;
    return r;
  };
  auto as_st = [](const WRowX& w) { return St{w.uu, w.ww, w.xx, w.zz, w.xz}; };
  auto snap_write = [&](const Strain& sn, int z) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      T* s0 = snap_base[h] + ((z - z_img0) * g.nx + (x - g.nbc));
      s0[0] = get(sn.fux, h);
      s0[plane] = get(sn.bwz, h);
      s0[2 * plane] = get(sn.sg, h);
    }
  };
  auto seis_write = [&](const St& r, int step) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const size_t rr = ((size_t)shot[h] * g.nt + step) * g.ng + recj;
      a.seis_w[rr] = get(r.ww, h);
      if (a.seis_u) a.seis_u[rr] = get(r.uu, h);
    }
  };

  // slots and registers as in fd_fwd_warp2
#pragma unroll
  for (int u = 0; u < NS; ++u) ld.issue(u, zs - 2 + u);
  if (warp_cancelled(a.cancel)) {  // the flag load overlaps the rows in flight
    wcp_wait<0>();
    return;
  }
  wcp_wait<NS - 2>();
  WRowX RR[2];
  ld.read(RR[0], 0);
  ld.read(RR[1], 1);
  F2 wn1, un1;
  {
    const WRowX& A = RR[0];
    const WRowX& B = RR[1];
    wn1 = src_w(zs - 2, vel_w(xint && rowin(zs - 2), A.ww, A.xz, shfl_l(A.xz), A.zz, B.zz, A.m.te, bz(zs - 2)), sv1);
    un1 = src_u(zs - 1, vel_u(xint && rowin(zs - 1), B.uu, B.xx, shfl_r(B.xx), B.xz, A.xz, B.m.te, bz(zs - 1)), sv1);
  }
  St T1[2];
  M2 MT[2];
  F2 wn2, un2;
  auto first = [&](auto slow_tag, int c0, int s1, int spf, int c1, int k1) {
    ld.issue(spf, k1 + NS - 1);
    wcp_wait<NS - 2>();
    ld.read(RR[c0 ^ 1], s1);
    const WRowX& R0 = RR[c0];
    const WRowX& R1 = RR[c0 ^ 1];
    Strain sn;
    T1[c1] = one(slow_tag, as_st(R0), R0.m, as_st(R1), R1.m.te, k1, sv1, wn1, un1, sn);
    MT[c1] = R0.m;
    if (decltype(slow_tag)::value && recj >= 0 && k1 == g.gz && k1 >= zs && k1 < ze) seis_write(T1[c1], it);
    if (SNAPSUB == 0 && snapc && k1 >= z_img0 && k1 < z_img1 && k1 >= zs && k1 < ze) snap_write(sn, k1);
  };
  auto second = [&](auto slow_tag, int c1, int j) {
    Strain sn;
    const St r = one(slow_tag, T1[c1 ^ 1], MT[c1 ^ 1], T1[c1], MT[c1].te, j, sv2, wn2, un2, sn);
    if (own) {
      const int o = j * g.pitch;
      oq[0][o] = make_float4(r.uu.x, r.ww.x, r.xx.x, r.zz.x);
      oxz[0][o] = r.xz.x;
      oq[1][o] = make_float4(r.uu.y, r.ww.y, r.xx.y, r.zz.y);
      oxz[1][o] = r.xz.y;
    }
    if (decltype(slow_tag)::value && recj >= 0 && j == g.gz) seis_write(r, it + 1);
    if (SNAPSUB == 1 && snapc && j >= z_img0 && j < z_img1) snap_write(sn, j);
  };
  const int mb = zs - 2;  // rows with checks, as in fd_fwd_warp2, for both shots' sources
  const unsigned long long slowm = slow_rows(g.NZ, g.pad_top, g.gz, zs, sp[0].x, sp[1].x);
  first(std::true_type{}, 1, 2 % NS, 0, 0, zs - 1);
  first(std::true_type{}, 0, 3 % NS, 1, 1, zs);
  {
    const St& A = T1[0];
    const St& B = T1[1];
    wn2 = src_w(zs - 1, vel_w(xint && rowin(zs - 1), A.ww, A.xz, shfl_l(A.xz), A.zz, B.zz, MT[0].te, bz(zs - 1)), sv2);
    un2 = src_u(zs, vel_u(xint, B.uu, B.xx, shfl_r(B.xx), B.xz, A.xz, MT[1].te, bz(zs)), sv2);
  }
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

// ------------------------------------------------------------ adjoint

// Adjoint steps it and it-1 for shots 2p and 2p+1; the row schedule is that of fd_adj_warp2.
template <int NW, int NS, int IMGSUB>
__global__ void __launch_bounds__(32 * NW) fd_adj_warp2x(AdjArgs<float> a, int it) {
  static_assert(NS >= 4 && NS % 2 == 0, "rows k, k+1 in use, at least two in flight; even for the unrolled rotation");
  using T = float;
  const FdGeom& g = a.g;
  int strip, chunk, pr;
  if (!warp_tile(g, (a.n_shots + 1) / 2, NW, strip, chunk, pr)) return;
  const int shot[2] = {2 * pr, min(2 * pr + 1, a.n_shots - 1)};
  const int lane = threadIdx.x & 31;
  const int x = kWarpOut2 * strip + lane - 1;
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const size_t F = g.field;
  const bool xin = x >= 0 && x < g.NX;
  const bool xint = x >= 1 && x <= g.NX - 2;
  const bool own = xint && lane >= 2 && lane <= kWarpOut2 + 1;
  const int xc = min(max(x, 0), g.NX - 1);
  const float* sb0 = a.in + (size_t)shot[0] * 5 * F;
  const float* sb1 = a.in + (size_t)shot[1] * 5 * F;
  extern __shared__ __align__(16) unsigned char wsmem[];
  const WStageX ld{reinterpret_cast<const float4*>(sb0) + xc, reinterpret_cast<const float4*>(sb1) + xc,
                   sb0 + 4 * F + xc, sb1 + 4 * F + xc, a.mat + xc,
                   reinterpret_cast<WSlotX*>(wsmem) + (threadIdx.x >> 5) * NS, g.pitch, min(ze + 1, g.NZ - 1), lane};
  float4* oq[2];
  float* oxz[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float* obs = a.out + (size_t)shot[h] * 5 * F;
    oq[h] = reinterpret_cast<float4*>(obs) + xc;
    oxz[h] = obs + 4 * F + xc;
  }
  const T dtx = a.dtx;
  const F2 dtx2 = bc(dtx);
  const F2 dl2 = bc(xint ? dtx : T(0));  // time factor of the fast rows (0: border lane, state kept)
  // dt*res of steps it and it-1 at receiver columns (:238-242); halo lanes inject too
  const bool rec = xin && x >= g.gx && (x - g.gx) % g.dg == 0 && (x - g.gx) / g.dg < g.ng;
  F2 inj1 = bc(T(0)), inj2 = bc(T(0));
  if (rec) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const size_t rrow = ((size_t)shot[h] * g.nt + it) * g.ng + (x - g.gx) / g.dg;
      at(inj1, h) = a.dt * a.res[rrow];
      at(inj2, h) = a.dt * a.res[rrow - g.ng];
    }
  }
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  const bool ximg = IMGSUB >= 0 && own && x >= g.nbc && x < g.nbc + g.nx;
  const T* snap_b[2];
  double* img_b[2];
  float* img_f[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    snap_b[h] = IMGSUB >= 0 ? a.snap + ((size_t)shot[h] * g.nrec +
                                        ((it - (IMGSUB > 0 ? 1 : 0)) / g.nt_wf - a.rec0)) * 3 * plane
                            : nullptr;
    img_b[h] = a.img + (size_t)shot[h] * 3 * plane;
    img_f[h] = a.img32 ? a.img32 + (size_t)shot[h] * 3 * plane : nullptr;  // FP32 images, as the reference
  }
  const bool f32img = a.img32 != nullptr;
  auto bz = [&](int z) -> F2 { return bc(z == g.pad_top ? T(2) * dtx : dtx); };
  auto rowin = [&](int z) { return z >= 1 && z <= g.NZ - 2; };
  struct St { F2 uu, ww, xx, zz, xz; };
  struct Prod { F2 p1, p2, p3, q1, q2; };  // ca*xx, cl*zz, cm1*xz, cl*xx, ca*zz
  auto prod = [](const St& r, const M2& m) -> Prod {
    return Prod{m.ca * r.xx, m.cl * r.zz, m.cm1 * r.xz, m.cl * r.xx, m.ca * r.zz};
  };
  struct Img { F2 fx, bz, sg, f[3]; double d[2][3]; };  // f: FP32 image sums, d: FP64 image sums
  auto img_row = [&](int z) { return IMGSUB >= 0 && z >= z_img0 && z < z_img1 && z >= zs && z < ze; };
  WImgSlotX* islots = reinterpret_cast<WImgSlotX*>(wsmem + (size_t)NW * NS * sizeof(WSlotX)) + (threadIdx.x >> 5) * NS;
  auto issue_img = [&](int slot, int z) {
    if (IMGSUB >= 0 && ximg && img_row(z)) {
      const int cell = (z - z_img0) * g.nx + (x - g.nbc);
      WImgSlotX& s = islots[slot];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        wcp4(&s.fx[h][lane], snap_b[h] + cell);
        wcp4(&s.bz[h][lane], snap_b[h] + plane + cell);
        wcp4(&s.sg[h][lane], snap_b[h] + 2 * plane + cell);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          if (f32img) wcp4(reinterpret_cast<float*>(s.c[h][i]) + lane, img_f[h] + i * plane + cell);
          else wcp8(&s.c[h][i][lane], img_b[h] + i * plane + cell);
        }
      }
    }
  };
  auto read_img = [&](Img& m, int slot) {
    const WImgSlotX& s = islots[slot];
    m.fx = F2{s.fx[0][lane], s.fx[1][lane]};
    m.bz = F2{s.bz[0][lane], s.bz[1][lane]};
    m.sg = F2{s.sg[0][lane], s.sg[1][lane]};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (f32img) {
        m.f[i] = F2{reinterpret_cast<const float*>(s.c[0][i])[lane], reinterpret_cast<const float*>(s.c[1][i])[lane]};
      } else {
        m.d[0][i] = s.c[0][i][lane];
        m.d[1][i] = s.c[1][i][lane];
      }
    }
  };
  auto image = [&](const Img& m, const St& r, int z) {  // imaging condition (:274-279)
    if (ximg && img_row(z)) {
      const int cell = (z - z_img0) * g.nx + (x - g.nbc);
      const F2 Fs = m.fx + m.bz;
      const F2 tcl = Fs * (r.xx + r.zz);
      const F2 tcm = bc(T(2)) * ((r.xx * m.fx + r.zz * m.bz) + bc(T(0.5)) * (r.xz * m.sg));
      const F2 til = Fs * Fs;
      if (f32img) {  // accumulate in FP32 like the reference
        const F2 c0 = m.f[0] + tcl, c1 = m.f[1] + tcm, c2 = m.f[2] + til;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          img_f[h][cell] = get(c0, h);
          img_f[h][plane + cell] = get(c1, h);
          img_f[h][2 * plane + cell] = get(c2, h);
        }
      } else {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          img_b[h][cell] = m.d[h][0] + (double)get(tcl, h);
          img_b[h][plane + cell] = m.d[h][1] + (double)get(tcm, h);
          img_b[h][2 * plane + cell] = m.d[h][2] + (double)get(til, h);
        }
      }
    }
  };
  // One row k of one adjoint step (as in fd_adj_warp2), both shots.
  auto one = [&](auto slow_tag, const St& R0, const M2& m0, const Prod& Q0, const St& R1, F2 t1, const Prod& Q1,
                 int k, F2 inj, F2& wn_prev, F2& un_cur) -> St {
    constexpr bool SLOW = decltype(slow_tag)::value;
    const bool in0 = !SLOW || rowin(k);
    const bool in1 = !SLOW || rowin(k + 1);
    const F2 d = SLOW ? dtx2 : dl2;  // fast rows: border lanes keep their state (as fd_adj_warp2)
    F2 wn = adj_vel_w(!SLOW || (xint && in0), R0.ww, Q1.q1, Q0.q1, Q1.q2, Q0.q2, shfl_r(Q0.p3), Q0.p3, m0.te,
                      SLOW ? bz(k) : dl2);
    if (SLOW && rec && k == g.gz) wn = wn + inj;
    const F2 p1l = shfl_l(Q1.p1), p2l = shfl_l(Q1.p2);
    const F2 un_next = adj_vel_u(!SLOW || (xint && in1), R1.uu, Q1.p1, p1l, Q1.p2, p2l, Q1.p3, Q0.p3, t1,
                                 SLOW ? bz(k + 1) : dl2);
    const F2 un_r = shfl_r(un_cur);
    const F2 wn_l = shfl_l(wn);
    const F2 te = m0.te;
    const F2 xxn = te * R0.xx - d * (un_r - un_cur);
    F2 zzn = te * R0.zz - d * (wn - wn_prev);
    const F2 xzn = (te * R0.xz - d * (un_next - un_cur)) - d * (wn - wn_l);
    if (SLOW && k == g.pad_top) zzn = bc(T(0));
    St r{un_cur, wn, xxn, zzn, xzn};
    if (SLOW && !(xint && in0)) r = R0;  // border cells keep their state
    wn_prev = wn;
    un_cur = un_next;
    return r;
  };
  auto as_st = [](const WRowX& w) { return St{w.uu, w.ww, w.xx, w.zz, w.xz}; };

#pragma unroll
  for (int u = 0; u < NS; ++u) {
    issue_img(u, zs - 2 + u);
    ld.issue(u, zs - 2 + u);
  }
  if (warp_cancelled(a.cancel)) {  // the flag load overlaps the rows in flight
    wcp_wait<0>();
    return;
  }
  wcp_wait<NS - 2>();
  WRowX RR[2];
  ld.read(RR[0], 0);
  ld.read(RR[1], 1);
  Prod QR[2] = {prod(as_st(RR[0]), RR[0].m), prod(as_st(RR[1]), RR[1].m)};
  F2 wn1, un1;
  {
    const St B = as_st(RR[1]);
    const int k = zs - 2;
    F2 w = adj_vel_w(xint && rowin(k), RR[0].ww, QR[1].q1, QR[0].q1, QR[1].q2, QR[0].q2, shfl_r(QR[0].p3), QR[0].p3,
                     RR[0].m.te, bz(k));
    if (rec && k == g.gz) w = w + inj1;
    wn1 = w;
    const F2 p1l = shfl_l(QR[1].p1), p2l = shfl_l(QR[1].p2);
    un1 = adj_vel_u(xint && rowin(k + 1), B.uu, QR[1].p1, p1l, QR[1].p2, p2l, QR[1].p3, QR[0].p3, RR[1].m.te,
                    bz(k + 1));
  }
  St T1[2];
  M2 MT[2];
  Prod QT[2];
  Img IMp{};
  F2 wn2, un2;
  auto first = [&](auto slow_tag, int c0, int s0, int s1, int spf, int c1, int k1) {
    if (IMGSUB == 1) read_img(IMp, spf);  // row k1-1, which the second step images next
    issue_img(spf, k1 + NS - 1);
    ld.issue(spf, k1 + NS - 1);
    wcp_wait<NS - 2>();
    ld.read(RR[c0 ^ 1], s1);
    QR[c0 ^ 1] = prod(as_st(RR[c0 ^ 1]), RR[c0 ^ 1].m);
    const WRowX& R0 = RR[c0];
    const WRowX& R1 = RR[c0 ^ 1];
    T1[c1] = one(slow_tag, as_st(R0), R0.m, QR[c0], as_st(R1), R1.m.te, QR[c0 ^ 1], k1, inj1, wn1, un1);
    MT[c1] = R0.m;
    QT[c1] = prod(T1[c1], R0.m);
    if (IMGSUB == 0) {
      Img m;
      read_img(m, s0);
      image(m, T1[c1], k1);
    }
  };
  auto second = [&](auto slow_tag, int c1, int j) {
    const St r = one(slow_tag, T1[c1 ^ 1], MT[c1 ^ 1], QT[c1 ^ 1], T1[c1], MT[c1].te, QT[c1], j, inj2, wn2, un2);
    if (own) {
      const int o = j * g.pitch;
      oq[0][o] = make_float4(r.uu.x, r.ww.x, r.xx.x, r.zz.x);
      oxz[0][o] = r.xz.x;
      oq[1][o] = make_float4(r.uu.y, r.ww.y, r.xx.y, r.zz.y);
      oxz[1][o] = r.xz.y;
    }
    if (IMGSUB == 1) image(IMp, r, j);
  };
  const int mb = zs - 2;  // rows with checks, as in fd_adj_warp2
  const unsigned long long slowm = slow_rows(g.NZ, g.pad_top, g.gz, zs);
  first(std::true_type{}, 1, 1, 2 % NS, 0, 0, zs - 1);
  first(std::true_type{}, 0, 2 % NS, 3 % NS, 1, 1, zs);
  {
    const St& A = T1[0];
    const St& B = T1[1];
    const int k = zs - 1;
    F2 w = adj_vel_w(xint && rowin(k), A.ww, QT[1].q1, QT[0].q1, QT[1].q2, QT[0].q2, shfl_r(QT[0].p3), QT[0].p3,
                     MT[0].te, bz(k));
    if (rec && k == g.gz) w = w + inj2;
    wn2 = w;
    const F2 p1l = shfl_l(QT[1].p1), p2l = shfl_l(QT[1].p2);
    un2 = adj_vel_u(xint, B.uu, QT[1].p1, p1l, QT[1].p2, p2l, QT[1].p3, QT[0].p3, MT[1].te, bz(zs));
  }
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
