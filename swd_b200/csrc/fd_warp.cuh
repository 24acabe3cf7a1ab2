// Warp-streaming FD time steps (engine path: FP32, b/b1 from the row index, 3 snapshot fields).
//
// Each warp owns a strip of 32 columns x = xs-1 .. xs+30 of one shot and streams down a
// chunk of rows, one column per lane.  Horizontal neighbours come from the adjacent lanes
// through warp shuffles.  The step at a column depends on the columns next to it only, so
// lanes 1..30 produce the strip's 30 outputs and lanes 0 and 31 are halo lanes that compute
// values for their neighbours and write nothing.  Vertical neighbours stay in registers:
// rows k and k+1 are held by each lane.  The rows ahead are staged by cp.async into NS
// shared-memory slots per warp, each lane copying and later reading only its own column, so
// no barrier of any kind is needed and the rows in flight cost no registers: rows k+2 ..
// k+NS-1 are outstanding while row k is computed.  The state of a shot is stored
// cell-interleaved for this schedule: float4 {uu, ww, xx, zz} [NZ][pitch] followed by
// xz [NZ][pitch] (the same 5*NZ*pitch floats as the other schedules), so a row costs a lane
// three 16/4-byte copies and two stores.  The arithmetic is that of fd_smem.cuh, expression
// for expression (the file is compiled with -fmad=false), so the results are bit-identical.
//
// Reference loops:  core/eigen_staggerfd_single.cpp:207-357 (forward),
//                   core/eigen_e2drtm_single.cpp:181-283 (adjoint + imaging).
#pragma once
#include <type_traits>

#include "fd_kernels.cuh"

namespace swd {

constexpr int kWarpOut = 30;  // output columns per warp (32 lanes minus two halo lanes)

__device__ __forceinline__ float shfl_l(float v) { return __shfl_up_sync(kFull, v, 1); }   // value at x-1
__device__ __forceinline__ float shfl_r(float v) { return __shfl_down_sync(kFull, v, 1); } // value at x+1

// One padded row of a lane's column: the five state fields and {temp, ca, cl, cm1}.
struct WRow {
  float uu, ww, xx, zz, xz;
  float4 m;
};

// A staging slot: one row of a warp's 32 columns.
struct WSlot {
  float4 q[32];   // {uu, ww, xx, zz}
  float4 m[32];   // {temp, ca, cl, cm1}
  float xz[32];
};

// The imaging operands of one row of a warp's 32 columns: the forward strains (fux, bwz,
// fuz+bwx) and the three image sums (FP64, or FP32 in the first half of each c row).
struct WImgSlot {
  float fx[32], bz[32], sg[32];
  double c[3][32];
};

template <int NW, int NS>
constexpr size_t warp_smem_bytes() { return (size_t)NW * NS * sizeof(WSlot); }
// two-step adjoint launches that image stage the imaging operands beside the rows
template <int NW, int NS>
constexpr size_t warp_img_smem_bytes() { return (size_t)NW * NS * (sizeof(WSlot) + sizeof(WImgSlot)); }

__device__ __forceinline__ void wcp16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src) : "memory");
}
__device__ __forceinline__ void wcp4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src) : "memory");
}
__device__ __forceinline__ void wcp8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src) : "memory");
}
__device__ __forceinline__ void wcp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void wcp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

struct WStage {
  const float4* q;    // this lane's column of {uu, ww, xx, zz}, row 0
  const float* xz;    // this lane's column of xz, row 0
  const float4* mat;  // this lane's column of the materials, row 0
  WSlot* slots;       // this warp's NS slots
  int pitch, zmax, lane;
  // Stage row z into a slot (rows beyond zmax are not needed: an empty copy group keeps the
  // group count).  Lanes past the last column copy the last column instead: their values only
  // reach border columns, which are never updated or written.
  __device__ __forceinline__ void issue(int slot, int z) const {
    if (z <= zmax) {
      const int o = max(z, 0) * pitch;  // 32-bit: the engine keeps 5 * NZ * pitch below 2^31
      WSlot& s = slots[slot];
      wcp16(&s.q[lane], q + o);
      wcp16(&s.m[lane], mat + o);
      wcp4(&s.xz[lane], xz + o);
    }
    wcp_commit();
  }
  __device__ __forceinline__ void read(WRow& r, int slot) const {
    const WSlot& s = slots[slot];
    const float4 v = s.q[lane];
    r.uu = v.x;
    r.ww = v.y;
    r.xx = v.z;
    r.zz = v.w;
    r.xz = s.xz[lane];
    r.m = s.m[lane];
  }
};

// Map a warp of the launch to (strip, chunk, shot); false for the padding warps of the last CTA.
__device__ __forceinline__ bool warp_tile(const FdGeom& g, int n_shots, int NW, int& strip, int& chunk, int& shot) {
  const long wid = (long)blockIdx.x * NW + (threadIdx.x >> 5);
  if (wid >= (long)g.n_strips * g.n_chunks * n_shots) return false;
  strip = (int)(wid % g.n_strips);
  const long rest = wid / g.n_strips;
  chunk = (int)(rest % g.n_chunks);
  shot = (int)(rest / g.n_chunks);
  return true;
}

// ---------------------------------------------------------------- forward

template <int NW, int NS, bool SNAP>
__global__ void __launch_bounds__(32 * NW) fd_fwd_warp(FwdArgs<float> a, int it) {
  static_assert(NS >= 4 && NS % 2 == 0, "rows k, k+1 in use, at least two in flight; even for the unrolled rotation");
  using T = float;
  const FdGeom& g = a.g;
  int strip, chunk, shot;
  if (!warp_tile(g, a.n_shots, NW, strip, chunk, shot)) return;  // whole warps only
  const int lane = threadIdx.x & 31;
  const int x = kWarpOut * strip + lane;
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const size_t F = g.field;
  const bool xin = x < g.NX;
  const bool xint = x >= 1 && x <= g.NX - 2;
  const bool own = xint && lane >= 1 && lane <= kWarpOut;
  const int xc = xin ? x : g.NX - 1;
  const float* sb = a.in + (size_t)shot * 5 * F;
  extern __shared__ __align__(16) unsigned char wsmem[];
  const WStage ld{reinterpret_cast<const float4*>(sb) + xc, sb + 4 * F + xc, a.mat + xc,
                  reinterpret_cast<WSlot*>(wsmem) + (threadIdx.x >> 5) * NS, g.pitch, ze, lane};
  float* obs = a.out + (size_t)shot * 5 * F;
  float4* oq = reinterpret_cast<float4*>(obs) + xc;
  float* oxz = obs + 4 * F + xc;
  const int st = a.src_type;
  const int2 sp = a.src[shot];
  const T sv = a.s[it];
  const T dtx = a.dtx;
  const bool sc = x == sp.y, sr = x == sp.y + 1;
  const bool s_w = sc && st != 1 && st != 4;    // ww(sz,sx) = s (type 5) or += s (types 2, 3)
  const bool s_wr = sr && st == 2;              // ww(sz,sx+1) += s
  const bool s_u = sc && (st == 2 || st == 3);  // uu(sz,sx) += s
  const bool s_um = sc && st == 2;              // uu(sz-1,sx) -= s
  const bool s_xz = sc && (st == 1 || st == 4); // xx/zz sources before the stress update
  const int recj = (a.seis_w != nullptr && own && x >= g.gx && (x - g.gx) % g.dg == 0 && (x - g.gx) / g.dg < g.ng)
                       ? (x - g.gx) / g.dg : -1;
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  const bool snapc = SNAP && own && x >= g.nbc && x < g.nbc + g.nx;
  T* snap_base = SNAP ? a.snap + ((size_t)shot * g.nrec + (it / g.nt_wf - a.rec0)) * 3 * plane : nullptr;
  auto bz = [&](int z) -> T { return z == g.pad_top ? T(2) * dtx : dtx; };  // b = b1 = dtx, doubled at the surface
  auto vel_w = [&](bool inner, T ww, T xz, T xzl, T zz, T zzd, T te, T b1) -> T {
    return inner ? te * ww + b1 * (((xz - xzl) + zzd) - zz) : ww;
  };
  auto vel_u = [&](bool inner, T uu, T xx, T xxr, T xz, T xzu, T te, T b) -> T {
    return inner ? te * uu + b * (((xxr - xx) + xz) - xzu) : uu;
  };
  auto src_w = [&](int z, T r) -> T {
    if (z == sp.x) {
      if (s_w) r = (st == 5) ? sv : r + sv;
      else if (s_wr) r = r + sv;
    }
    return r;
  };
  auto src_u = [&](int z, T r) -> T {
    if (s_u && z == sp.x) r = r + sv;
    if (s_um && z == sp.x - 1) r = r - sv;
    return r;
  };

  // Row r is staged in slot (r - zs + 1) % NS; rows k and k+1 are held in the registers RR[0] /
  // RR[1], alternating; the row loop is unrolled by NS so that slots and registers rotate
  // without moves.
#pragma unroll
  for (int u = 0; u < NS; ++u) ld.issue(u, zs - 1 + u);
  if (warp_cancelled(a.cancel)) {  // the flag load overlaps the rows in flight
    wcp_wait<0>();
    return;
  }
  wcp_wait<NS - 2>();
  WRow RR[2];
  ld.read(RR[0], 0);
  ld.read(RR[1], 1);
  // prologue: new ww at row zs-1 and new uu at row zs
  T wn_prev, un_cur;
  {
    const WRow& A = RR[0];
    const WRow& B = RR[1];
    const T xzl = shfl_l(A.xz);
    wn_prev = src_w(zs - 1, vel_w(xint && zs - 1 >= 1, A.ww, A.xz, xzl, A.zz, B.zz, A.m.x, bz(zs - 1)));
    const T xxr = shfl_r(B.xx);
    un_cur = src_u(zs, vel_u(xint, B.uu, B.xx, xxr, B.xz, A.xz, B.m.x, bz(zs)));
  }
  // One row k: R0 = row k (registers), R1 receives row k+1 from slot s1, row k+NS-1 is staged
  // into slot sp (row k-1's).  SLOW rows are those where a source, the receivers, the free
  // surface or the bottom row need their checks; every other row takes the check-free path.
  auto step = [&](auto slow_tag, const WRow& R0, WRow& R1, int s1, int spf, int k) {
    constexpr bool SLOW = decltype(slow_tag)::value;
    ld.issue(spf, k + NS - 1);
    wcp_wait<NS - 2>();  // row k+1 has landed
    ld.read(R1, s1);
    const bool inner1 = !SLOW || k + 1 <= g.NZ - 2;
    // velocities: ww at row k, uu at row k+1 (:224-228, source :286-300)
    const T xzl = shfl_l(R0.xz);
    T wn = vel_w(xint, R0.ww, R0.xz, xzl, R0.zz, R1.zz, R0.m.x, SLOW ? bz(k) : dtx);
    const T xxr = shfl_r(R1.xx);
    T un_next = vel_u(xint && inner1, R1.uu, R1.xx, xxr, R1.xz, R0.xz, R1.m.x, SLOW ? bz(k + 1) : dtx);
    if (SLOW) {
      wn = src_w(k, wn);
      un_next = src_u(k + 1, un_next);
    }
    // strains at row k (:302-306)
    const T ucl = shfl_l(un_cur);
    const T wnr = shfl_r(wn);
    const T fux = un_cur - ucl;
    const T fuz = un_next - un_cur;
    const T bwx = wnr - wn;
    const T bwz = wn - wn_prev;
    // stresses at row k (:334-336), source types 1/4 first (:286-298), free surface (:340)
    T xo = R0.xx, zo = R0.zz;
    if (SLOW && s_xz && k == sp.x) {
      if (st == 1) { xo = xo + sv; zo = zo + sv; }
      else { zo = zo + sv; }
    }
    const T te = R0.m.x, ca = R0.m.y, cl = R0.m.z, cm1 = R0.m.w;
    const T xxn = te * xo + (ca * fux + cl * bwz) * dtx;
    T zzn = te * zo + (ca * bwz + cl * fux) * dtx;
    const T xzn = te * R0.xz + (cm1 * (fuz + bwx)) * dtx;
    if (SLOW && k == g.pad_top) zzn = T(0);
    if (own) {
      const int o = k * g.pitch;
      oq[o] = make_float4(un_cur, wn, xxn, zzn);
      oxz[o] = xzn;
    }
    if (SLOW && recj >= 0 && k == g.gz) {  // :342-345
      const size_t r = ((size_t)shot * g.nt + it) * g.ng + recj;
      a.seis_w[r] = wn;
      if (a.seis_u) a.seis_u[r] = un_cur;
    }
    if (SNAP && snapc && k >= z_img0 && k < z_img1) {  // :346-351 (the adjoint needs fux, bwz, fuz+bwx)
      T* s0 = snap_base + ((k - z_img0) * g.nx + (x - g.nbc));
      s0[0] = fux;
      s0[plane] = bwz;
      s0[2 * plane] = fuz + bwx;
    }
    wn_prev = wn;
    un_cur = un_next;
  };
  auto row = [&](const WRow& R0, WRow& R1, int s1, int spf, int k) {
    if (k == g.pad_top || k == g.gz || k == g.NZ - 2 || (k >= sp.x - 2 && k <= sp.x))
      step(std::true_type{}, R0, R1, s1, spf, k);
    else
      step(std::false_type{}, R0, R1, s1, spf, k);
  };
  // row k = zs + u (mod NS): in RR[(u + 1) & 1], row k+1 goes to RR[u & 1] from slot (u + 2) % NS
  int k = zs;
  for (; k + NS <= ze; k += NS) {
#pragma unroll
    for (int u = 0; u < NS; ++u) row(RR[(u + 1) & 1], RR[u & 1], (u + 2) % NS, u, k + u);
  }
#pragma unroll
  for (int u = 0; u < NS - 1; ++u)
    if (k + u < ze) row(RR[(u + 1) & 1], RR[u & 1], (u + 2) % NS, u, k + u);
  wcp_wait<0>();  // no copy may still target this warp's slots at exit
}

// ---------------------------------------------------------------- forward, two steps per launch

constexpr int kWarpOut2 = 28;  // output columns per warp of the two-step kernels (two halo lanes a side)
constexpr int kWarpChunkMax = 60;  // rows per chunk of the warp kernels (the two-step row masks below)

// The two-step kernels mark the rows that take the checked path (sources, receivers, free
// surface, top and bottom rows) as bits of a 64-bit mask over rows base .. base+63, base = zs-2,
// so that a row's test is one bit test instead of a chain of compares.  row_span sets the bits
// of rows lo..hi.  A chunk of at most kWarpChunkMax rows tests rows up to zs+60, inside the mask.
__host__ __device__ __forceinline__ unsigned long long row_span(int base, int lo, int hi) {
  lo = max(lo, base);
  hi = min(hi, base + 63);
  return lo > hi ? 0ull : (~0ull >> (63 - (hi - lo))) << (lo - base);
}

// The checked rows of a two-step chunk that starts at row zs, as a mask over rows zs-2 ..
// zs+61: rows <= 1 and >= NZ-2, the free surface, the receiver row and the rows sx-2 .. sx
// above and at each source row sx in {src0, src1} (kNoSourceRow: none; the adjoint has none,
// the two-shots-per-warp forward kernels have two).
constexpr int kNoSourceRow = -1000000;
__host__ __device__ __forceinline__ unsigned long long slow_rows(int NZ, int pad_top, int gz, int zs,
                                                                int src0 = kNoSourceRow, int src1 = kNoSourceRow) {
  const int mb = zs - 2;
  return row_span(mb, mb, 1) | row_span(mb, NZ - 2, mb + 63) | row_span(mb, pad_top, pad_top) |
         row_span(mb, gz, gz) | row_span(mb, src0 - 2, src0) | row_span(mb, src1 - 2, src1);
}

// Steps it and it+1 in one sweep: the state after step it (S1) is formed row by row as in
// fd_fwd_warp and kept in registers, and step it+1 runs one row behind it on S1, so S1 never
// goes to memory and a launch moves the state once for two steps.  Lanes x = 28*strip-1 ..
// 28*strip+30: S1 is valid on lanes 1..30, the new state on lanes 2..29, which write.  Border
// cells keep their state, as the one-step kernels leave them unwritten: on the checked rows by
// a select, on the others because the engine's material table holds temp = 1 on the border
// columns and border lanes use a time factor of 0, so their update returns the state exactly
// (x*1 + 0*y = x for the finite values of a wavefield).  SNAPSUB: which of
// the two steps writes strain snapshots (-1 neither).
template <int NW, int NS, int SNAPSUB>
__global__ void __launch_bounds__(32 * NW) fd_fwd_warp2(FwdArgs<float> a, int it) {
  static_assert(NS >= 4 && NS % 2 == 0, "rows k, k+1 in use, at least two in flight; even for the unrolled rotation");
  using T = float;
  const FdGeom& g = a.g;
  int strip, chunk, shot;
  if (!warp_tile(g, a.n_shots, NW, strip, chunk, shot)) return;
  const int lane = threadIdx.x & 31;
  const int x = kWarpOut2 * strip + lane - 1;
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const size_t F = g.field;
  const bool xint = x >= 1 && x <= g.NX - 2;
  const bool own = xint && lane >= 2 && lane <= kWarpOut2 + 1;
  const int xc = min(max(x, 0), g.NX - 1);
  const float* sb = a.in + (size_t)shot * 5 * F;
  extern __shared__ __align__(16) unsigned char wsmem[];
  const WStage ld{reinterpret_cast<const float4*>(sb) + xc, sb + 4 * F + xc, a.mat + xc,
                  reinterpret_cast<WSlot*>(wsmem) + (threadIdx.x >> 5) * NS, g.pitch, min(ze + 1, g.NZ - 1), lane};
  float* obs = a.out + (size_t)shot * 5 * F;
  float4* oq = reinterpret_cast<float4*>(obs) + xc;
  float* oxz = obs + 4 * F + xc;
  const int st = a.src_type;
  const int2 sp = a.src[shot];
  const T sv1 = a.s[it], sv2 = a.s[it + 1];
  const T dtx = a.dtx;
  const T dl = xint ? dtx : T(0);  // time factor of the fast rows (0: border lane, state kept)
  const bool sc = x == sp.y, sr = x == sp.y + 1;
  const bool s_w = sc && st != 1 && st != 4;
  const bool s_wr = sr && st == 2;
  const bool s_u = sc && (st == 2 || st == 3);
  const bool s_um = sc && st == 2;
  const bool s_xz = sc && (st == 1 || st == 4);
  const int recj = (a.seis_w != nullptr && own && x >= g.gx && (x - g.gx) % g.dg == 0 && (x - g.gx) / g.dg < g.ng)
                       ? (x - g.gx) / g.dg : -1;
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  const bool snapc = SNAPSUB >= 0 && own && x >= g.nbc && x < g.nbc + g.nx;
  T* snap_base = SNAPSUB >= 0 ? a.snap + ((size_t)shot * g.nrec + ((it + (SNAPSUB > 0 ? 1 : 0)) / g.nt_wf - a.rec0)) *
                                            3 * plane : nullptr;
  auto bz = [&](int z) -> T { return z == g.pad_top ? T(2) * dtx : dtx; };
  auto rowin = [&](int z) { return z >= 1 && z <= g.NZ - 2; };
  auto vel_w = [&](bool inner, T ww, T xz, T xzl, T zz, T zzd, T te, T b1) -> T {
    return inner ? te * ww + b1 * (((xz - xzl) + zzd) - zz) : ww;
  };
  auto vel_u = [&](bool inner, T uu, T xx, T xxr, T xz, T xzu, T te, T b) -> T {
    return inner ? te * uu + b * (((xxr - xx) + xz) - xzu) : uu;
  };
  auto src_w = [&](int z, T r, T sv) -> T {
    if (z == sp.x) {
      if (s_w) r = (st == 5) ? sv : r + sv;
      else if (s_wr) r = r + sv;
    }
    return r;
  };
  auto src_u = [&](int z, T r, T sv) -> T {
    if (s_u && z == sp.x) r = r + sv;
    if (s_um && z == sp.x - 1) r = r - sv;
    return r;
  };
  // One row k of one step, on rows R0 = k and R1 = k+1 of the state before it (materials m0 of
  // row k, temp t1 of row k+1); wn_prev = new ww of row k-1, un_cur = new uu of row k on entry,
  // those of rows k and k+1 on exit.  Returns the new state of row k and its strains.
  struct St { T uu, ww, xx, zz, xz; };
  struct Strain { T fux, bwz, sg; };
  auto one = [&](auto slow_tag, const St& R0, const float4& m0, const St& R1, T t1, int k, T sv, T& wn_prev,
                 T& un_cur, Strain& sn) -> St {
    constexpr bool SLOW = decltype(slow_tag)::value;
    const bool in0 = !SLOW || rowin(k);
    const bool in1 = !SLOW || rowin(k + 1);
    // Fast rows skip the border test: a border lane updates with its time factor dl = 0 and the
    // engine's temp = 1 on border columns, which returns its state bit for bit.
    const T d = SLOW ? dtx : dl;
    const T xzl = shfl_l(R0.xz);
    T wn = vel_w(!SLOW || (xint && in0), R0.ww, R0.xz, xzl, R0.zz, R1.zz, m0.x, SLOW ? bz(k) : dl);
    const T xxr = shfl_r(R1.xx);
    T un_next = vel_u(!SLOW || (xint && in1), R1.uu, R1.xx, xxr, R1.xz, R0.xz, t1, SLOW ? bz(k + 1) : dl);
    if (SLOW) {
      wn = src_w(k, wn, sv);
      un_next = src_u(k + 1, un_next, sv);
    }
    const T ucl = shfl_l(un_cur);
    const T wnr = shfl_r(wn);
    const T fux = un_cur - ucl;
    const T fuz = un_next - un_cur;
    const T bwx = wnr - wn;
    const T bwz = wn - wn_prev;
    T xo = R0.xx, zo = R0.zz;
    if (SLOW && s_xz && k == sp.x) {
      if (st == 1) { xo = xo + sv; zo = zo + sv; }
      else { zo = zo + sv; }
    }
    const T xxn = m0.x * xo + (m0.y * fux + m0.z * bwz) * d;
    T zzn = m0.x * zo + (m0.y * bwz + m0.z * fux) * d;
    const T xzn = m0.x * R0.xz + (m0.w * (fuz + bwx)) * d;
    if (SLOW && k == g.pad_top) zzn = T(0);
    St r{un_cur, wn, xxn, zzn, xzn};
    if (SLOW && !(xint && in0)) r = R0;  // border cells keep their state
    sn = Strain{fux, bwz, fuz + bwx};
    wn_prev = wn;
    un_cur = un_next;
    return r;
  };
  auto as_st = [](const WRow& w) { return St{w.uu, w.ww, w.xx, w.zz, w.xz}; };

  // State row r is staged in slot (r - zs + 2) % NS and held in RR[(r - zs) & 1]; S1 row r in
  // T1[(r - zs + 1) & 1].
#pragma unroll
  for (int u = 0; u < NS; ++u) ld.issue(u, zs - 2 + u);
  if (warp_cancelled(a.cancel)) {  // the flag load overlaps the rows in flight
    wcp_wait<0>();
    return;
  }
  wcp_wait<NS - 2>();
  WRow RR[2];
  ld.read(RR[0], 0);
  ld.read(RR[1], 1);
  T wn1, un1;  // first step: new ww of row k1-1, new uu of row k1
  {
    const WRow& A = RR[0];
    const WRow& B = RR[1];
    wn1 = src_w(zs - 2, vel_w(xint && rowin(zs - 2), A.ww, A.xz, shfl_l(A.xz), A.zz, B.zz, A.m.x, bz(zs - 2)), sv1);
    un1 = src_u(zs - 1, vel_u(xint && rowin(zs - 1), B.uu, B.xx, shfl_r(B.xx), B.xz, A.xz, B.m.x, bz(zs - 1)), sv1);
  }
  St T1[2];      // S1 rows k1-1 and k1 (alternating)
  float4 MT[2];  // their materials
  T wn2, un2;    // second step: new ww of row k1-2, new uu of row k1-1
  // First-step row k1 from state rows RR[c0] (k1) and RR[c0^1] (k1+1, read from slot s1 after
  // staging row k1+NS-1 into slot spf, row k1-1's); its S1 row goes to T1[c1].
  auto first = [&](auto slow_tag, int c0, int s1, int spf, int c1, int k1) {
    ld.issue(spf, k1 + NS - 1);
    wcp_wait<NS - 2>();
    ld.read(RR[c0 ^ 1], s1);
    const WRow& R0 = RR[c0];
    const WRow& R1 = RR[c0 ^ 1];
    Strain sn;
    T1[c1] = one(slow_tag, as_st(R0), R0.m, as_st(R1), R1.m.x, k1, sv1, wn1, un1, sn);
    MT[c1] = R0.m;
    if (decltype(slow_tag)::value && recj >= 0 && k1 == g.gz && k1 >= zs && k1 < ze) {  // :342-345, step it
      const size_t r = ((size_t)shot * g.nt + it) * g.ng + recj;
      a.seis_w[r] = T1[c1].ww;
      if (a.seis_u) a.seis_u[r] = T1[c1].uu;
    }
    if (SNAPSUB == 0 && snapc && k1 >= z_img0 && k1 < z_img1 && k1 >= zs && k1 < ze) {
      T* s0 = snap_base + ((k1 - z_img0) * g.nx + (x - g.nbc));
      s0[0] = sn.fux;
      s0[plane] = sn.bwz;
      s0[2 * plane] = sn.sg;
    }
  };
  // Second-step row j = k1-1 from S1 rows T1[c1^1] (j) and T1[c1] (k1); writes the new state.
  auto second = [&](auto slow_tag, int c1, int j) {
    Strain sn;
    const St r = one(slow_tag, T1[c1 ^ 1], MT[c1 ^ 1], T1[c1], MT[c1].x, j, sv2, wn2, un2, sn);
    if (own) {
      const int o = j * g.pitch;
      oq[o] = make_float4(r.uu, r.ww, r.xx, r.zz);
      oxz[o] = r.xz;
    }
    if (decltype(slow_tag)::value && recj >= 0 && j == g.gz) {  // step it+1
      const size_t rr = ((size_t)shot * g.nt + it + 1) * g.ng + recj;
      a.seis_w[rr] = r.ww;
      if (a.seis_u) a.seis_u[rr] = r.uu;
    }
    if (SNAPSUB == 1 && snapc && j >= z_img0 && j < z_img1) {
      T* s0 = snap_base + ((j - z_img0) * g.nx + (x - g.nbc));
      s0[0] = sn.fux;
      s0[plane] = sn.bwz;
      s0[2 * plane] = sn.sg;
    }
  };
  // rows with checks: k <= 1, k >= NZ-2, the free surface, the receiver row, the source rows
  const int mb = zs - 2;
  const unsigned long long slowm = slow_rows(g.NZ, g.pad_top, g.gz, zs, sp.x);
  // peeled: S1 rows zs-1 and zs, then the second step's prologue (new ww of row zs-1, new uu of row zs)
  first(std::true_type{}, 1, 2 % NS, 0, 0, zs - 1);
  first(std::true_type{}, 0, 3 % NS, 1, 1, zs);
  {
    const St& A = T1[0];
    const St& B = T1[1];
    wn2 = src_w(zs - 1, vel_w(xint && rowin(zs - 1), A.ww, A.xz, shfl_l(A.xz), A.zz, B.zz, MT[0].x, bz(zs - 1)), sv2);
    un2 = src_u(zs, vel_u(xint, B.uu, B.xx, shfl_r(B.xx), B.xz, A.xz, MT[1].x, bz(zs)), sv2);
  }
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

// ---------------------------------------------------------------- adjoint

template <int NW, int NS, bool IMG>
__global__ void __launch_bounds__(32 * NW) fd_adj_warp(AdjArgs<float> a, int it) {
  static_assert(NS >= 4 && NS % 2 == 0, "rows k, k+1 in use, at least two in flight; even for the unrolled rotation");
  using T = float;
  const FdGeom& g = a.g;
  int strip, chunk, shot;
  if (!warp_tile(g, a.n_shots, NW, strip, chunk, shot)) return;
  const int lane = threadIdx.x & 31;
  const int x = kWarpOut * strip + lane;
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const size_t F = g.field;
  const bool xin = x < g.NX;
  const bool xint = x >= 1 && x <= g.NX - 2;
  const bool own = xint && lane >= 1 && lane <= kWarpOut;
  const int xc = xin ? x : g.NX - 1;
  const float* sb = a.in + (size_t)shot * 5 * F;
  extern __shared__ __align__(16) unsigned char wsmem[];
  const WStage ld{reinterpret_cast<const float4*>(sb) + xc, sb + 4 * F + xc, a.mat + xc,
                  reinterpret_cast<WSlot*>(wsmem) + (threadIdx.x >> 5) * NS, g.pitch, ze, lane};
  float* obs = a.out + (size_t)shot * 5 * F;
  float4* oq = reinterpret_cast<float4*>(obs) + xc;
  float* oxz = obs + 4 * F + xc;
  const T dtx = a.dtx;
  // dt*res at receiver columns (:238-242); halo lanes inject too, their ww feeds the neighbours
  const bool rec = xin && x >= g.gx && (x - g.gx) % g.dg == 0 && (x - g.gx) / g.dg < g.ng;
  const T inj = rec ? a.dt * a.res[((size_t)shot * g.nt + it) * g.ng + (x - g.gx) / g.dg] : T(0);
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  const bool ximg = own && x >= g.nbc && x < g.nbc + g.nx;
  const T* snap_b = IMG ? a.snap + ((size_t)shot * g.nrec + (it / g.nt_wf - a.rec0)) * 3 * plane : nullptr;
  double* img_b = a.img + (size_t)shot * 3 * plane;
  float* img_f = a.img32 ? a.img32 + (size_t)shot * 3 * plane : nullptr;  // FP32 images, as the reference
  auto bz = [&](int z) -> T { return z == g.pad_top ? T(2) * dtx : dtx; };
  // material*stress products of a row: ca*xx, cl*zz, cm1*xz, cl*xx, ca*zz
  struct Prod { T p1, p2, p3, q1, q2; };
  auto prod = [](const WRow& r) -> Prod {
    return Prod{r.m.y * r.xx, r.m.z * r.zz, r.m.w * r.xz, r.m.z * r.xx, r.m.y * r.zz};
  };
  struct Img { T fx, bz, sg; double c0, c1, c2; };
  auto load_img = [&](Img& m, int z) {
    if (IMG && ximg && z >= z_img0 && z < z_img1 && z < ze) {
      const int cell = (z - z_img0) * g.nx + (x - g.nbc);
      const T* s0 = snap_b + cell;
      m.fx = s0[0]; m.bz = s0[plane]; m.sg = s0[2 * plane];
      if (img_f) {
        m.c0 = img_f[cell]; m.c1 = img_f[plane + cell]; m.c2 = img_f[2 * plane + cell];
      } else {
        m.c0 = img_b[cell]; m.c1 = img_b[plane + cell]; m.c2 = img_b[2 * plane + cell];
      }
    }
  };
  // new ww at row k (rows r0 = k, r1 = k+1, products q0 / q1, p3 of row k at x+1)
  auto vel_w = [&](bool inner, const WRow& r0, const Prod& q0, const Prod& q1, T p3r, int k) -> T {
    T r = adj_vel_w(inner, r0.ww, q1.q1, q0.q1, q1.q2, q0.q2, p3r, q0.p3, r0.m.x, bz(k));
    if (rec && k == g.gz) r = r + inj;
    return r;
  };

#pragma unroll
  for (int u = 0; u < NS; ++u) ld.issue(u, zs - 1 + u);
  if (warp_cancelled(a.cancel)) {  // the flag load overlaps the rows in flight
    wcp_wait<0>();
    return;
  }
  wcp_wait<NS - 2>();
  WRow RR[2];
  ld.read(RR[0], 0);
  ld.read(RR[1], 1);
  Prod QP[2] = {prod(RR[0]), prod(RR[1])};  // products of rows k and k+1
  Img IM[2] = {};                           // imaging operands of rows k and k+1
  load_img(IM[0], zs);
  T wn_prev, un_cur;
  {
    const WRow& A = RR[0];
    const WRow& B = RR[1];
    wn_prev = vel_w(xint && zs - 1 >= 1, A, QP[0], QP[1], shfl_r(QP[0].p3), zs - 1);
    const T p1l = shfl_l(QP[1].p1), p2l = shfl_l(QP[1].p2);
    un_cur = adj_vel_u(xint, B.uu, QP[1].p1, p1l, QP[1].p2, p2l, QP[1].p3, QP[0].p3, B.m.x, bz(zs));
  }
  // One row k: R0 = row k with products Q0, R1 receives row k+1 from slot s1 and its products
  // go to Q1, row k+NS-1 is staged into slot spf; im_c holds row k's imaging operands, im_n
  // receives row k+1's.
  auto step = [&](auto slow_tag, const WRow& R0, WRow& R1, int s1, int spf, const Prod& Q0, Prod& Q1,
                  const Img& im_c, Img& im_n, int k) {
    constexpr bool SLOW = decltype(slow_tag)::value;
    ld.issue(spf, k + NS - 1);
    load_img(im_n, k + 1);
    wcp_wait<NS - 2>();  // row k+1 has landed
    ld.read(R1, s1);
    const bool inner1 = !SLOW || k + 1 <= g.NZ - 2;
    Q1 = prod(R1);
    // velocities: ww at row k, uu at row k+1 (:182-187), injection (:238-242)
    T wn = adj_vel_w(xint, R0.ww, Q1.q1, Q0.q1, Q1.q2, Q0.q2, shfl_r(Q0.p3), Q0.p3, R0.m.x, SLOW ? bz(k) : dtx);
    if (SLOW && rec && k == g.gz) wn = wn + inj;
    const T p1l = shfl_l(Q1.p1), p2l = shfl_l(Q1.p2);
    const T un_next = adj_vel_u(xint && inner1, R1.uu, Q1.p1, p1l, Q1.p2, p2l, Q1.p3, Q0.p3, R1.m.x,
                                SLOW ? bz(k + 1) : dtx);
    // adjoint stresses at row k (:245-248), free surface (:270)
    const T un_r = shfl_r(un_cur);
    const T wn_l = shfl_l(wn);
    const T te = R0.m.x;
    const T xxn = te * R0.xx - dtx * (un_r - un_cur);
    T zzn = te * R0.zz - dtx * (wn - wn_prev);
    const T xzn = (te * R0.xz - dtx * (un_next - un_cur)) - dtx * (wn - wn_l);
    if (SLOW && k == g.pad_top) zzn = T(0);
    if (own) {
      const int o = k * g.pitch;
      oq[o] = make_float4(un_cur, wn, xxn, zzn);
      oxz[o] = xzn;
      if (IMG && ximg && k >= z_img0 && k < z_img1) {  // imaging condition (:274-279)
        const int cell = (k - z_img0) * g.nx + (x - g.nbc);
        const T fx = im_c.fx, bzv = im_c.bz, sg = im_c.sg;
        const T Fs = fx + bzv;
        const T tcl = Fs * (xxn + zzn);
        const T tcm = T(2) * ((xxn * fx + zzn * bzv) + T(0.5) * (xzn * sg));
        const T til = Fs * Fs;
        if (img_f) {  // accumulate in FP32 like the reference
          img_f[cell] = (float)((T)(im_c.c0) + tcl);
          img_f[plane + cell] = (float)((T)(im_c.c1) + tcm);
          img_f[2 * plane + cell] = (float)((T)(im_c.c2) + til);
        } else {
          img_b[cell] = im_c.c0 + (double)tcl;
          img_b[plane + cell] = im_c.c1 + (double)tcm;
          img_b[2 * plane + cell] = im_c.c2 + (double)til;
        }
      }
    }
    wn_prev = wn;
    un_cur = un_next;
  };
  auto row = [&](const WRow& R0, WRow& R1, int s1, int spf, const Prod& Q0, Prod& Q1, const Img& im_c, Img& im_n,
                 int k) {
    if (k == g.pad_top || k == g.gz || k == g.NZ - 2)
      step(std::true_type{}, R0, R1, s1, spf, Q0, Q1, im_c, im_n, k);
    else
      step(std::false_type{}, R0, R1, s1, spf, Q0, Q1, im_c, im_n, k);
  };
  // unrolled by NS: slots rotate with period NS; rows, products and imaging operands with period 2
  // (row k = zs + u: registers RR[(u + 1) & 1], products QP[(u + 1) & 1], imaging IM[u & 1])
  int k = zs;
  for (; k + NS <= ze; k += NS) {
#pragma unroll
    for (int u = 0; u < NS; ++u)
      row(RR[(u + 1) & 1], RR[u & 1], (u + 2) % NS, u, QP[(u + 1) & 1], QP[u & 1], IM[u & 1], IM[(u + 1) & 1],
          k + u);
  }
#pragma unroll
  for (int u = 0; u < NS - 1; ++u)
    if (k + u < ze)
      row(RR[(u + 1) & 1], RR[u & 1], (u + 2) % NS, u, QP[(u + 1) & 1], QP[u & 1], IM[u & 1], IM[(u + 1) & 1],
          k + u);
  wcp_wait<0>();
}

// ---------------------------------------------------------------- adjoint, two steps per launch

// Adjoint steps it and it-1 in one sweep, built as fd_fwd_warp2: the state after step it (S1)
// is formed row by row in registers and step it-1 runs one row behind it.  IMGSUB: which of
// the two steps applies the imaging condition (0: step it, 1: step it-1, -1 neither).
template <int NW, int NS, int IMGSUB>
__global__ void __launch_bounds__(32 * NW) fd_adj_warp2(AdjArgs<float> a, int it) {
  static_assert(NS >= 4 && NS % 2 == 0, "rows k, k+1 in use, at least two in flight; even for the unrolled rotation");
  using T = float;
  const FdGeom& g = a.g;
  int strip, chunk, shot;
  if (!warp_tile(g, a.n_shots, NW, strip, chunk, shot)) return;
  const int lane = threadIdx.x & 31;
  const int x = kWarpOut2 * strip + lane - 1;
  const int zs = 1 + chunk * g.chunk;
  const int ze = min(zs + g.chunk, g.NZ - 1);
  const size_t F = g.field;
  const bool xin = x >= 0 && x < g.NX;
  const bool xint = x >= 1 && x <= g.NX - 2;
  const bool own = xint && lane >= 2 && lane <= kWarpOut2 + 1;
  const int xc = min(max(x, 0), g.NX - 1);
  const float* sb = a.in + (size_t)shot * 5 * F;
  extern __shared__ __align__(16) unsigned char wsmem[];
  const WStage ld{reinterpret_cast<const float4*>(sb) + xc, sb + 4 * F + xc, a.mat + xc,
                  reinterpret_cast<WSlot*>(wsmem) + (threadIdx.x >> 5) * NS, g.pitch, min(ze + 1, g.NZ - 1), lane};
  float* obs = a.out + (size_t)shot * 5 * F;
  float4* oq = reinterpret_cast<float4*>(obs) + xc;
  float* oxz = obs + 4 * F + xc;
  const T dtx = a.dtx;
  const T dl = xint ? dtx : T(0);  // time factor of the fast rows (0: border lane, state kept)
  // dt*res of steps it and it-1 at receiver columns (:238-242); halo lanes inject too
  const bool rec = xin && x >= g.gx && (x - g.gx) % g.dg == 0 && (x - g.gx) / g.dg < g.ng;
  const size_t rrow = ((size_t)shot * g.nt + it) * g.ng + (rec ? (x - g.gx) / g.dg : 0);
  const T inj1 = rec ? a.dt * a.res[rrow] : T(0);
  const T inj2 = rec ? a.dt * a.res[rrow - g.ng] : T(0);
  const int z_img0 = g.pad_top + 1, z_img1 = g.pad_top + 1 + g.nz;
  const size_t plane = (size_t)g.nz * g.nx;
  const bool ximg = IMGSUB >= 0 && own && x >= g.nbc && x < g.nbc + g.nx;
  const T* snap_b = IMGSUB >= 0 ? a.snap + ((size_t)shot * g.nrec + ((it - (IMGSUB > 0 ? 1 : 0)) / g.nt_wf - a.rec0)) *
                                               3 * plane : nullptr;
  double* img_b = a.img + (size_t)shot * 3 * plane;
  float* img_f = a.img32 ? a.img32 + (size_t)shot * 3 * plane : nullptr;  // FP32 images, as the reference
  auto bz = [&](int z) -> T { return z == g.pad_top ? T(2) * dtx : dtx; };
  auto rowin = [&](int z) { return z >= 1 && z <= g.NZ - 2; };
  struct St { T uu, ww, xx, zz, xz; };
  struct Prod { T p1, p2, p3, q1, q2; };  // ca*xx, cl*zz, cm1*xz, cl*xx, ca*zz
  auto prod = [](const St& r, const float4& m) -> Prod {
    return Prod{m.y * r.xx, m.z * r.zz, m.w * r.xz, m.z * r.xx, m.y * r.zz};
  };
  struct Img { T fx, bz, sg; double c0, c1, c2; };
  auto img_row = [&](int z) { return IMGSUB >= 0 && z >= z_img0 && z < z_img1 && z >= zs && z < ze; };
  // Imaging operands are staged by cp.async beside the state rows (same slot, same copy group),
  // so their DRAM latency hides behind the rows in flight instead of costing registers.
  WImgSlot* islots = reinterpret_cast<WImgSlot*>(wsmem + (size_t)NW * NS * sizeof(WSlot)) + (threadIdx.x >> 5) * NS;
  auto issue_img = [&](int slot, int z) {
    if (IMGSUB >= 0 && ximg && img_row(z)) {
      const int cell = (z - z_img0) * g.nx + (x - g.nbc);
      WImgSlot& s = islots[slot];
      wcp4(&s.fx[lane], snap_b + cell);
      wcp4(&s.bz[lane], snap_b + plane + cell);
      wcp4(&s.sg[lane], snap_b + 2 * plane + cell);
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        if (img_f) wcp4(reinterpret_cast<float*>(s.c[i]) + lane, img_f + i * plane + cell);
        else wcp8(&s.c[i][lane], img_b + i * plane + cell);
      }
    }
  };
  auto read_img = [&](Img& m, int slot) {
    const WImgSlot& s = islots[slot];
    m.fx = s.fx[lane];
    m.bz = s.bz[lane];
    m.sg = s.sg[lane];
    if (img_f) {
      m.c0 = reinterpret_cast<const float*>(s.c[0])[lane];
      m.c1 = reinterpret_cast<const float*>(s.c[1])[lane];
      m.c2 = reinterpret_cast<const float*>(s.c[2])[lane];
    } else {
      m.c0 = s.c[0][lane];
      m.c1 = s.c[1][lane];
      m.c2 = s.c[2][lane];
    }
  };
  auto image = [&](const Img& m, const St& r, int z) {  // imaging condition (:274-279)
    if (ximg && img_row(z)) {
      const int cell = (z - z_img0) * g.nx + (x - g.nbc);
      const T Fs = m.fx + m.bz;
      const T tcl = Fs * (r.xx + r.zz);
      const T tcm = T(2) * ((r.xx * m.fx + r.zz * m.bz) + T(0.5) * (r.xz * m.sg));
      const T til = Fs * Fs;
      if (img_f) {  // accumulate in FP32 like the reference
        img_f[cell] = (float)((T)(m.c0) + tcl);
        img_f[plane + cell] = (float)((T)(m.c1) + tcm);
        img_f[2 * plane + cell] = (float)((T)(m.c2) + til);
      } else {
        img_b[cell] = m.c0 + (double)tcl;
        img_b[plane + cell] = m.c1 + (double)tcm;
        img_b[2 * plane + cell] = m.c2 + (double)til;
      }
    }
  };
  // One row k of one adjoint step on rows R0 = k (materials m0, products Q0) and R1 = k+1
  // (temp t1, products Q1); wn_prev / un_cur as in fd_adj_warp.  Returns the new state of row k.
  auto one = [&](auto slow_tag, const St& R0, const float4& m0, const Prod& Q0, const St& R1, T t1, const Prod& Q1,
                 int k, T inj, T& wn_prev, T& un_cur) -> St {
    constexpr bool SLOW = decltype(slow_tag)::value;
    const bool in0 = !SLOW || rowin(k);
    const bool in1 = !SLOW || rowin(k + 1);
    const T d = SLOW ? dtx : dl;  // fast rows: border lanes keep their state through dl = 0, temp = 1
    T wn = adj_vel_w(!SLOW || (xint && in0), R0.ww, Q1.q1, Q0.q1, Q1.q2, Q0.q2, shfl_r(Q0.p3), Q0.p3, m0.x,
                     SLOW ? bz(k) : dl);
    if (SLOW && rec && k == g.gz) wn = wn + inj;
    const T p1l = shfl_l(Q1.p1), p2l = shfl_l(Q1.p2);
    const T un_next = adj_vel_u(!SLOW || (xint && in1), R1.uu, Q1.p1, p1l, Q1.p2, p2l, Q1.p3, Q0.p3, t1,
                                SLOW ? bz(k + 1) : dl);
    const T un_r = shfl_r(un_cur);
    const T wn_l = shfl_l(wn);
    const T te = m0.x;
    const T xxn = te * R0.xx - d * (un_r - un_cur);
    T zzn = te * R0.zz - d * (wn - wn_prev);
    const T xzn = (te * R0.xz - d * (un_next - un_cur)) - d * (wn - wn_l);
    if (SLOW && k == g.pad_top) zzn = T(0);
    St r{un_cur, wn, xxn, zzn, xzn};
    if (SLOW && !(xint && in0)) r = R0;  // border cells keep their state
    wn_prev = wn;
    un_cur = un_next;
    return r;
  };
  auto as_st = [](const WRow& w) { return St{w.uu, w.ww, w.xx, w.zz, w.xz}; };

  // state rows staged from zs-2: row r in slot (r - zs + 2) % NS and RR[(r - zs) & 1]
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
  WRow RR[2];
  ld.read(RR[0], 0);
  ld.read(RR[1], 1);
  Prod QR[2] = {prod(as_st(RR[0]), RR[0].m), prod(as_st(RR[1]), RR[1].m)};  // products of the state rows
  T wn1, un1;  // first step: new ww of row k1-1, new uu of row k1
  {
    const St B = as_st(RR[1]);
    const int k = zs - 2;
    T w = adj_vel_w(xint && rowin(k), RR[0].ww, QR[1].q1, QR[0].q1, QR[1].q2, QR[0].q2, shfl_r(QR[0].p3), QR[0].p3,
                    RR[0].m.x, bz(k));
    if (rec && k == g.gz) w = w + inj1;
    wn1 = w;
    const T p1l = shfl_l(QR[1].p1), p2l = shfl_l(QR[1].p2);
    un1 = adj_vel_u(xint && rowin(k + 1), B.uu, QR[1].p1, p1l, QR[1].p2, p2l, QR[1].p3, QR[0].p3, RR[1].m.x,
                    bz(k + 1));
  }
  St T1[2];      // S1 rows, T1[(r - zs + 1) & 1]
  float4 MT[2];  // their materials
  Prod QT[2];    // their products
  Img IMp{};  // imaging operands of the second step's row (read before its slot is restaged)
  T wn2, un2;    // second step: new ww of row k1-2, new uu of row k1-1
  // first-step row k1 (slot and register bookkeeping as in fd_fwd_warp2)
  // s0: slot of state row k1 (its imaging operands when step it images)
  auto first = [&](auto slow_tag, int c0, int s0, int s1, int spf, int c1, int k1) {
    if (IMGSUB == 1) read_img(IMp, spf);  // row k1-1, which the second step images next
    issue_img(spf, k1 + NS - 1);
    ld.issue(spf, k1 + NS - 1);
    wcp_wait<NS - 2>();
    ld.read(RR[c0 ^ 1], s1);
    QR[c0 ^ 1] = prod(as_st(RR[c0 ^ 1]), RR[c0 ^ 1].m);
    const WRow& R0 = RR[c0];
    const WRow& R1 = RR[c0 ^ 1];
    T1[c1] = one(slow_tag, as_st(R0), R0.m, QR[c0], as_st(R1), R1.m.x, QR[c0 ^ 1], k1, inj1, wn1, un1);
    MT[c1] = R0.m;
    QT[c1] = prod(T1[c1], R0.m);
    if (IMGSUB == 0) {
      Img m;
      read_img(m, s0);
      image(m, T1[c1], k1);
    }
  };
  // second-step row j = k1-1 from S1 rows T1[c1^1] (j) and T1[c1] (k1); writes the new state
  auto second = [&](auto slow_tag, int c1, int j) {
    const St r = one(slow_tag, T1[c1 ^ 1], MT[c1 ^ 1], QT[c1 ^ 1], T1[c1], MT[c1].x, QT[c1], j, inj2, wn2, un2);
    if (own) {
      const int o = j * g.pitch;
      oq[o] = make_float4(r.uu, r.ww, r.xx, r.zz);
      oxz[o] = r.xz;
    }
    if (IMGSUB == 1) image(IMp, r, j);
  };
  // rows with checks: k <= 1, k >= NZ-2, the free surface, the receiver row
  const int mb = zs - 2;
  const unsigned long long slowm = slow_rows(g.NZ, g.pad_top, g.gz, zs);
  first(std::true_type{}, 1, 1, 2 % NS, 0, 0, zs - 1);
  first(std::true_type{}, 0, 2 % NS, 3 % NS, 1, 1, zs);
  {
    const St& A = T1[0];
    const St& B = T1[1];
    const int k = zs - 1;
    T w = adj_vel_w(xint && rowin(k), A.ww, QT[1].q1, QT[0].q1, QT[1].q2, QT[0].q2, shfl_r(QT[0].p3), QT[0].p3,
                    MT[0].x, bz(k));
    if (rec && k == g.gz) w = w + inj2;
    wn2 = w;
    const T p1l = shfl_l(QT[1].p1), p2l = shfl_l(QT[1].p2);
    un2 = adj_vel_u(xint, B.uu, QT[1].p1, p1l, QT[1].p2, p2l, QT[1].p3, QT[0].p3, MT[1].x, bz(zs));
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
