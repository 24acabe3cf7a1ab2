// Host side of the FD kernels: geometry planning, launchers, MATLAB-layout
// conversion and the MEX-convention C entry points (swd_staggerfd_*, swd_e2drtm_*).
// Compiled with -fmad=false (see fd_kernels.cuh).
#include <cstdarg>
#include <cstring>
#include <atomic>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "fd_host.cuh"
#include "fd_kernels.cuh"
#include "fd_lead.cuh"
#include "fd_warp.cuh"

namespace swd {

static thread_local char g_err[1024] = "";
static std::atomic<uint64_t> g_launches{0};

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
void clear_error() { g_err[0] = 0; }
void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ------------------------------------------------------------ layout kernels

// out[bo*ob + c*R + r] = in[bi*ib + r*C + c]: batched transpose of R x C planes.
template <typename Ti, typename To>
__global__ void transpose_kernel(const Ti* __restrict__ in, size_t ib, To* __restrict__ out, size_t ob, int R, int C) {
  __shared__ Ti tile[32][33];
  const int b = blockIdx.z;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const Ti* src = in + (size_t)b * ib;
  To* dst = out + (size_t)b * ob;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int r = r0 + i, c = c0 + threadIdx.x;
    if (r < R && c < C) tile[i][threadIdx.x] = src[(size_t)r * C + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int c = c0 + i, r = r0 + threadIdx.x;
    if (r < R && c < C) dst[(size_t)c * R + r] = (To)tile[threadIdx.x][i];
  }
}

template <typename Ti, typename To>
int transpose(const Ti* in, size_t ib, To* out, size_t ob, int B, int R, int C, cudaStream_t st) {
  if (B <= 0 || R <= 0 || C <= 0) return SWD_OK;
  dim3 grid((C + 31) / 32, (R + 31) / 32, B), block(32, 8);
  transpose_kernel<Ti, To><<<grid, block, 0, st>>>(in, ib, out, ob, R, C);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}
template int transpose<float, float>(const float*, size_t, float*, size_t, int, int, int, cudaStream_t);
template int transpose<double, double>(const double*, size_t, double*, size_t, int, int, int, cudaStream_t);
template int transpose<double, float>(const double*, size_t, float*, size_t, int, int, int, cudaStream_t);
template int transpose<float, double>(const float*, size_t, double*, size_t, int, int, int, cudaStream_t);

// Pack the MATLAB column-major material fields (nzbc x nxbc) into the row-major
// vector layout the step kernels read: mat = {temp, ca, cl, cm1}, mb = {b, b1}.
template <typename T>
__global__ void pack_materials_cm(const T* __restrict__ temp, const T* __restrict__ b, const T* __restrict__ b1,
                                  const T* __restrict__ ca, const T* __restrict__ cl, const T* __restrict__ cm1,
                                  typename Vec4<T>::type* mat, typename Vec2<T>::type* mb, int NZ, int NX,
                                  int pitch) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x;  // z fastest: coalesced reads
  const int x = blockIdx.y;
  if (z >= NZ || x >= NX) return;
  const size_t c = (size_t)x * NZ + z;
  typename Vec4<T>::type u;
  typename Vec2<T>::type v;
  u.x = temp[c]; u.y = ca[c]; u.z = cl[c]; u.w = cm1[c];
  v.x = b[c]; v.y = b1[c];
  mat[(size_t)z * pitch + x] = u;
  mb[(size_t)z * pitch + x] = v;
}

template <typename T>
int pack_materials(const T* temp, const T* b, const T* b1, const T* ca, const T* cl, const T* cm1,
                   typename Vec4<T>::type* mat, typename Vec2<T>::type* mb, int NZ, int NX, int pitch,
                   cudaStream_t st) {
  dim3 grid((NZ + 127) / 128, NX), block(128);
  pack_materials_cm<T><<<grid, block, 0, st>>>(temp, b, b1, ca, cl, cm1, mat, mb, NZ, NX, pitch);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}
template int pack_materials<float>(const float*, const float*, const float*, const float*, const float*,
                                   const float*, float4*, float2*, int, int, int, cudaStream_t);
template int pack_materials<double>(const double*, const double*, const double*, const double*,
                                    const double*, const double*, double4*, double2*, int, int, int,
                                    cudaStream_t);

// ------------------------------------------------------------ planning

// (warps, cells, ring depth) variants built for the engine path.  The kernels unroll the row
// loop by the ring depth, so it is even; depth 4 is the fastest on the 100 x 600 survey.
#define SWD_SHAPES(X) \
  X(1, 2, 4) X(1, 2, 6) X(1, 2, 8) X(1, 3, 4) X(1, 3, 6) X(2, 1, 4) X(2, 1, 6) X(2, 1, 8) X(3, 1, 4) X(3, 1, 6) \
  X(3, 1, 8) X(4, 1, 4) X(4, 1, 6) X(4, 1, 8)

// Variants of the one-barrier-per-row schedule (fd_lead.cuh).
#define SWD_LEAD_SHAPES(X) X(2, 1, 4) X(3, 1, 4) X(3, 1, 6) X(4, 1, 4)

bool fd_variant_built(int w, int c, int d) {
#define X(W, C, D) if (w == W && c == C && d == D) return true;
  SWD_SHAPES(X)
#undef X
  return false;
}

bool fd_lead_built(int w, int c, int d) {
#define X(W, C, D) if (w == W && c == C && d == D) return true;
  SWD_LEAD_SHAPES(X)
#undef X
  return false;
}

void plan_decomposition(FdGeom& g, int n_shots, int chunk_rows) {
  const int rows = g.NZ - 2;
  if (g.sched == 3) {  // column pairs (fd_col2.cuh): 60 output columns per warp, 2, 4 or 8 warps per CTA
    if (g.warps != 2 && g.warps != 8) g.warps = 4;
    g.cells = 2;
    if (!fd_col2_built(g.warps, g.ring_fwd)) g.ring_fwd = 4;
    if (!fd_col2_built(g.warps, g.ring_adj)) g.ring_adj = 4;
    g.pairs = 0;
    g.n_strips = (g.NX / 2 + kCol2Pairs - 1) / kCol2Pairs;
    if (chunk_rows <= 0) {
      // about 2.5 waves of warps (148 SMs x ~16 resident): 96 shots of 132 x 660 -> 22 rows
      const long target = 148L * 16 * 5 / 2;
      const long per = (long)g.n_strips * n_shots;
      int nch = (int)((target + per - 1) / per);
      nch = std::max(1, std::min(nch, std::max(1, rows / 8)));
      chunk_rows = (rows + nch - 1) / nch;
    }
    g.chunk = std::max(1, std::min({chunk_rows, rows, kWarpChunkMax}));
    g.n_chunks = (rows + g.chunk - 1) / g.chunk;
    return;
  }
  if (g.sched == 2) {  // warp streaming (fd_warp.cuh): 30 output columns per warp, warps per CTA 2, 4 or 8,
                       // 4, 6 or 8 register row slots (ring_fwd / ring_adj)
    if (g.warps != 2 && g.warps != 8) g.warps = 4;
    g.cells = 1;
    if (g.ring_fwd != 6 && !(g.ring_fwd == 8 && g.warps != 8)) g.ring_fwd = 4;
    if (g.ring_adj != 6 && !(g.ring_adj == 8 && g.warps != 8)) g.ring_adj = 4;
    if (g.pairs == 2) {  // two shots per warp: 2 or 4 warps per CTA, 4 or 6 slots
      if (g.warps != 2) g.warps = 4;
      if (g.ring_fwd != 6) g.ring_fwd = 4;
      if (g.ring_adj != 6) g.ring_adj = 4;
    }
    g.n_strips = (g.NX - 2 + kWarpOut - 1) / kWarpOut;
    if (chunk_rows <= 0) {
      // about 5 waves of warps (148 SMs x 28 resident warps): short chunks keep more rows in
      // flight and every SM busy through the tail of a step; 96 shots of 132 x 660 -> 13 rows.
      // Two-step launches recompute rows at each chunk edge and take half as many waves (26 rows);
      // two-shot warps hold twice the registers (12 resident per SM) and count shot pairs.
      const long target = g.pairs == 2 ? 148L * 12 * 5 / 2 : g.pairs ? 148L * 28 * 5 / 2 : 148L * 28 * 5;
      const long per = (long)g.n_strips * (g.pairs == 2 ? (n_shots + 1) / 2 : n_shots);
      int nch = (int)((target + per - 1) / per);
      nch = std::max(1, std::min(nch, std::max(1, rows / 8)));
      chunk_rows = (rows + nch - 1) / nch;
    }
    g.chunk = std::max(1, std::min({chunk_rows, rows, kWarpChunkMax}));
    g.n_chunks = (rows + g.chunk - 1) / g.chunk;
    return;
  }
  if (!fd_variant_built(g.warps, g.cells, 4)) { g.warps = 3; g.cells = 1; }
  if (!fd_variant_built(g.warps, g.cells, g.ring_fwd)) g.ring_fwd = 4;
  if (!fd_variant_built(g.warps, g.cells, g.ring_adj)) g.ring_adj = 4;
  if (g.sched == 1 && !(fd_lead_built(g.warps, g.cells, g.ring_fwd) && fd_lead_built(g.warps, g.cells, g.ring_adj)))
    g.sched = 0;
  const int cols = 32 * g.warps * g.cells;
  g.n_strips = (g.NX - 2 + cols - 1) / cols;
  if (chunk_rows <= 0) {
    // about 2.5 waves of CTAs (148 SMs x ~(30 / warps) resident CTAs at 64 registers): short
    // chunks keep every SM busy through the tail of a step; 96 shots of 132 x 660 -> 22 rows
    const long target = 148L * (30 / g.warps) * 5 / 2;
    const long per = (long)g.n_strips * n_shots;
    int nch = (int)((target + per - 1) / per);
    nch = std::max(1, std::min(nch, std::max(1, rows / 8)));
    chunk_rows = (rows + nch - 1) / nch;
  }
  g.chunk = std::max(1, std::min(chunk_rows, rows));
  g.n_chunks = (rows + g.chunk - 1) / g.chunk;
}

template <typename K>
static int set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) SWD_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return SWD_OK;
}

template <typename T, int NF, int W, int C, int D, bool GB, bool SNAP>
static int fwd_launch(const FwdArgs<T>& a, int it, cudaStream_t st) {
  constexpr size_t smem = smem_bytes<T, W, C, D, GB>();
  static int ready = set_smem(fd_fwd_smem<T, NF, W, C, D, GB, SNAP>, smem);
  if (ready != SWD_OK) return ready;
  const long blocks = (long)a.g.n_strips * a.g.n_chunks * a.n_shots;
  fd_fwd_smem<T, NF, W, C, D, GB, SNAP><<<(unsigned)blocks, 32 * W, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
// strain snapshots are written every nt_wf steps: a separate variant keeps the code off the other steps
template <typename T, int NF, int W, int C, int D, bool GB>
static int fwd_impl(const FwdArgs<T>& a, int it, cudaStream_t st) {
  if (a.snap && it % a.g.nt_wf == 0) return fwd_launch<T, NF, W, C, D, GB, true>(a, it, st);
  return fwd_launch<T, NF, W, C, D, GB, false>(a, it, st);
}

template <typename T, int NF, int W, int C, int D, bool GB, bool SNAP>
static int fwd_lead_launch(const FwdArgs<T>& a, int it, cudaStream_t st) {
  constexpr size_t smem = lead_smem_bytes<T, W, C, D, GB>();
  static int ready = set_smem(fd_fwd_lead<T, NF, W, C, D, GB, SNAP>, smem);
  if (ready != SWD_OK) return ready;
  const long blocks = (long)a.g.n_strips * a.g.n_chunks * a.n_shots;
  fd_fwd_lead<T, NF, W, C, D, GB, SNAP><<<(unsigned)blocks, 32 * W, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <typename T, int NF, int W, int C, int D, bool GB>
static int fwd_lead_impl(const FwdArgs<T>& a, int it, cudaStream_t st) {
  if (a.snap && it % a.g.nt_wf == 0) return fwd_lead_launch<T, NF, W, C, D, GB, true>(a, it, st);
  return fwd_lead_launch<T, NF, W, C, D, GB, false>(a, it, st);
}
template <typename T, int NF, int W, int C, int D, bool GB, bool IMG>
static int adj_lead_impl(const AdjArgs<T>& a, int it, cudaStream_t st) {
  constexpr size_t smem = lead_smem_bytes<T, W, C, D, GB>();
  static int ready = set_smem(fd_adj_lead<T, NF, W, C, D, GB, IMG>, smem);
  if (ready != SWD_OK) return ready;
  const long blocks = (long)a.g.n_strips * a.g.n_chunks * a.n_shots;
  fd_adj_lead<T, NF, W, C, D, GB, IMG><<<(unsigned)blocks, 32 * W, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}

template <int NW, int NS, bool SNAP>
static int fwd_warp_launch(const FwdArgs<float>& a, int it, cudaStream_t st) {
  constexpr size_t smem = warp_smem_bytes<NW, NS>();
  static int ready = set_smem(fd_fwd_warp<NW, NS, SNAP>, smem);
  if (ready != SWD_OK) return ready;
  const long warps = (long)a.g.n_strips * a.g.n_chunks * a.n_shots;
  fd_fwd_warp<NW, NS, SNAP><<<(unsigned)((warps + NW - 1) / NW), 32 * NW, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <int NW, int NS>
static int fwd_warp_impl(const FwdArgs<float>& a, int it, cudaStream_t st) {
  if (a.snap && it % a.g.nt_wf == 0) return fwd_warp_launch<NW, NS, true>(a, it, st);
  return fwd_warp_launch<NW, NS, false>(a, it, st);
}
template <int NW, int NS, bool IMG>
static int adj_warp_impl(const AdjArgs<float>& a, int it, cudaStream_t st) {
  constexpr size_t smem = warp_smem_bytes<NW, NS>();
  static int ready = set_smem(fd_adj_warp<NW, NS, IMG>, smem);
  if (ready != SWD_OK) return ready;
  const long warps = (long)a.g.n_strips * a.g.n_chunks * a.n_shots;
  fd_adj_warp<NW, NS, IMG><<<(unsigned)((warps + NW - 1) / NW), 32 * NW, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <int NW, int NS, int SS>
static int fwd_warp2_launch(const FwdArgs<float>& a0, int it, cudaStream_t st) {
  constexpr size_t smem = warp_smem_bytes<NW, NS>();
  static int ready = set_smem(fd_fwd_warp2<NW, NS, SS>, smem);
  if (ready != SWD_OK) return ready;
  SWD_CHECK(a0.g.chunk <= kWarpChunkMax, "internal: two-step chunk of %d rows (at most %d)", a0.g.chunk, kWarpChunkMax);
  FwdArgs<float> a = a0;
  a.g.n_strips = (a.g.NX - 2 + kWarpOut2 - 1) / kWarpOut2;  // 28-column strips
  const long warps = (long)a.g.n_strips * a.g.n_chunks * a.n_shots;
  fd_fwd_warp2<NW, NS, SS><<<(unsigned)((warps + NW - 1) / NW), 32 * NW, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <int NW, int NS>
static int fwd_warp2_impl(const FwdArgs<float>& a, int it, cudaStream_t st) {
  if (a.snap && it % a.g.nt_wf == 0) return fwd_warp2_launch<NW, NS, 0>(a, it, st);
  if (a.snap && (it + 1) % a.g.nt_wf == 0) return fwd_warp2_launch<NW, NS, 1>(a, it, st);
  return fwd_warp2_launch<NW, NS, -1>(a, it, st);
}
template <int NW, int NS, int IS>
static int adj_warp2_launch(const AdjArgs<float>& a0, int it, cudaStream_t st) {
  constexpr size_t smem = IS >= 0 ? warp_img_smem_bytes<NW, NS>() : warp_smem_bytes<NW, NS>();
  static int ready = set_smem(fd_adj_warp2<NW, NS, IS>, smem);
  if (ready != SWD_OK) return ready;
  SWD_CHECK(a0.g.chunk <= kWarpChunkMax, "internal: two-step chunk of %d rows (at most %d)", a0.g.chunk, kWarpChunkMax);
  AdjArgs<float> a = a0;
  a.g.n_strips = (a.g.NX - 2 + kWarpOut2 - 1) / kWarpOut2;
  const long warps = (long)a.g.n_strips * a.g.n_chunks * a.n_shots;
  fd_adj_warp2<NW, NS, IS><<<(unsigned)((warps + NW - 1) / NW), 32 * NW, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <int NW, int NS>
static int adj_warp2_impl(const AdjArgs<float>& a, int it, cudaStream_t st) {
  if (it % a.g.nt_wf == 0) return adj_warp2_launch<NW, NS, 0>(a, it, st);
  if ((it - 1) % a.g.nt_wf == 0) return adj_warp2_launch<NW, NS, 1>(a, it, st);
  return adj_warp2_launch<NW, NS, -1>(a, it, st);
}
// (warps per CTA, row slots) of the warp-streaming kernels
#define SWD_WARP_SHAPES(X) X(2, 4) X(4, 4) X(8, 4) X(2, 6) X(4, 6) X(8, 6) X(4, 8) X(2, 8)

template <typename T, int NF, int W, int C, int D, bool GB, bool IMG>
static int adj_impl(const AdjArgs<T>& a, int it, cudaStream_t st) {
  constexpr size_t smem = smem_bytes<T, W, C, D, GB>();
  static int ready = set_smem(fd_adj_smem<T, NF, W, C, D, GB, IMG>, smem);
  if (ready != SWD_OK) return ready;
  const long blocks = (long)a.g.n_strips * a.g.n_chunks * a.n_shots;
  fd_adj_smem<T, NF, W, C, D, GB, IMG><<<(unsigned)blocks, 32 * W, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}

// Engine path (FP32, 3 snapshot fields, b/b1 from the row index): CTA shape and ring depth are
// runtime choices.  MEX path (general b/b1 arrays, 4 snapshot fields, FP32 or FP64): 4 warps x 1.
template <typename T, int NF>
int launch_fwd_step(const FwdArgs<T>& a, int it, cudaStream_t st) {
  if (a.mb) return fwd_impl<T, NF, 4, 1, 4, true>(a, it, st);
  if constexpr (NF == 3 && sizeof(T) == 4) {
    if (a.g.sched == 3) return launch_fwd_step_c2(a, it, st);
    if (a.g.sched == 2) {
      switch (a.g.warps * 10 + a.g.ring_fwd) {
#define X(w, s) case w * 10 + s: return fwd_warp_impl<w, s>(a, it, st);
        SWD_WARP_SHAPES(X)
#undef X
        default: break;
      }
      set_error("internal: unsupported FD kernel variant");
      return SWD_ERR_INVALID;
    }
    const int key = a.g.warps * 100 + a.g.cells * 10 + a.g.ring_fwd;
    if (a.g.sched == 1) {
      switch (key) {
#define X(w, c, d) case w * 100 + c * 10 + d: return fwd_lead_impl<T, NF, w, c, d, false>(a, it, st);
        SWD_LEAD_SHAPES(X)
#undef X
        default: break;
      }
      set_error("internal: unsupported FD kernel variant");
      return SWD_ERR_INVALID;
    }
    switch (key) {
#define X(w, c, d) case w * 100 + c * 10 + d: return fwd_impl<T, NF, w, c, d, false>(a, it, st);
      SWD_SHAPES(X)
#undef X
      default: break;
    }
  }
  set_error("internal: unsupported FD kernel variant");
  return SWD_ERR_INVALID;
}

template <typename T, int NF, bool IMG>
static int adj_dispatch(const AdjArgs<T>& a, int it, cudaStream_t st) {
  if (a.mb) return adj_impl<T, NF, 4, 1, 4, true, IMG>(a, it, st);
  if constexpr (NF == 3 && sizeof(T) == 4) {
    if (a.g.sched == 3) return launch_adj_step_c2(a, it, st);
    if (a.g.sched == 2) {
      switch (a.g.warps * 10 + a.g.ring_adj) {
#define X(w, s) case w * 10 + s: return adj_warp_impl<w, s, IMG>(a, it, st);
        SWD_WARP_SHAPES(X)
#undef X
        default: break;
      }
      set_error("internal: unsupported FD kernel variant");
      return SWD_ERR_INVALID;
    }
    const int key = a.g.warps * 100 + a.g.cells * 10 + a.g.ring_adj;
    if (a.g.sched == 1) {
      switch (key) {
#define X(w, c, d) case w * 100 + c * 10 + d: return adj_lead_impl<T, NF, w, c, d, false, IMG>(a, it, st);
        SWD_LEAD_SHAPES(X)
#undef X
        default: break;
      }
      set_error("internal: unsupported FD kernel variant");
      return SWD_ERR_INVALID;
    }
    switch (key) {
#define X(w, c, d) case w * 100 + c * 10 + d: return adj_impl<T, NF, w, c, d, false, IMG>(a, it, st);
      SWD_SHAPES(X)
#undef X
      default: break;
    }
  }
  set_error("internal: unsupported FD kernel variant");
  return SWD_ERR_INVALID;
}

template <typename T, int NF>
int launch_adj_step(const AdjArgs<T>& a, int it, cudaStream_t st) {
  // the imaging condition only runs every nt_wf steps: a separate variant keeps the
  // other steps free of its registers
  if (it % a.g.nt_wf == 0) return adj_dispatch<T, NF, true>(a, it, st);
  return adj_dispatch<T, NF, false>(a, it, st);
}
int launch_fwd_pair(const FwdArgs<float>& a, int it, cudaStream_t st) {
  if (a.g.sched == 3) return launch_fwd_pair_c2(a, it, st);
  if (!fd_pairs(a.g) || a.mb || it + 1 >= a.g.nt) {
    set_error("internal: two-step forward launch outside the warp-streaming schedule");
    return SWD_ERR_INVALID;
  }
  if (a.g.pairs == 2) return launch_fwd_pair_x(a, it, st);
  switch (a.g.warps * 10 + a.g.ring_fwd) {
#define X(w, s) case w * 10 + s: return fwd_warp2_impl<w, s>(a, it, st);
    SWD_WARP_SHAPES(X)
#undef X
    default: break;
  }
  set_error("internal: unsupported FD kernel variant");
  return SWD_ERR_INVALID;
}

int launch_adj_pair(const AdjArgs<float>& a, int it, cudaStream_t st) {
  if (a.g.sched == 3) return launch_adj_pair_c2(a, it, st);
  if (!fd_pairs(a.g) || a.mb || it < 1) {
    set_error("internal: two-step adjoint launch outside the warp-streaming schedule");
    return SWD_ERR_INVALID;
  }
  if (a.g.pairs == 2) return launch_adj_pair_x(a, it, st);
  switch (a.g.warps * 10 + a.g.ring_adj) {
#define X(w, s) case w * 10 + s: return adj_warp2_impl<w, s>(a, it, st);
    SWD_WARP_SHAPES(X)
#undef X
    default: break;
  }
  set_error("internal: unsupported FD kernel variant");
  return SWD_ERR_INVALID;
}

template int launch_fwd_step<float, 3>(const FwdArgs<float>&, int, cudaStream_t);
template int launch_fwd_step<float, 4>(const FwdArgs<float>&, int, cudaStream_t);
template int launch_fwd_step<double, 4>(const FwdArgs<double>&, int, cudaStream_t);
template int launch_adj_step<float, 3>(const AdjArgs<float>&, int, cudaStream_t);
template int launch_adj_step<float, 4>(const AdjArgs<float>&, int, cudaStream_t);
template int launch_adj_step<double, 4>(const AdjArgs<double>&, int, cudaStream_t);

// ------------------------------------------------------------ MEX-convention entry points

namespace {

struct FwdIv {
  int nt, nzbc, nxbc, ng, sz, sx, gz, gx, dg, src_type, fd_order, nt_wf, nz, nx, fmt;
  double dtx;
};

template <typename T>
int parse_fwd_iv(const T* iv, int n_iv, FwdIv& p) {
  SWD_CHECK(iv != nullptr && n_iv >= 16, "input_vector needs 16 entries (got %d)", n_iv);
  // core/eigen_staggerfd_single.cpp:98-115 reads the entries by truncation, 1-based positions
  p.nt = (int)iv[0]; p.nzbc = (int)iv[1]; p.nxbc = (int)iv[2]; p.dtx = (double)iv[3];
  p.ng = (int)iv[4]; p.sz = (int)iv[5] - 1; p.sx = (int)iv[6] - 1; p.gz = (int)iv[7] - 1;
  p.gx = (int)iv[8] - 1; p.dg = (int)iv[9]; p.src_type = (int)iv[10]; p.fd_order = (int)iv[11];
  p.nt_wf = (int)iv[12]; p.nz = (int)iv[13]; p.nx = (int)iv[14]; p.fmt = (int)iv[15];
  return SWD_OK;
}

int validate_geom(int nt, int NZ, int NX, int nz, int nx, int nbc, int nt_wf, int fd_order, int ng, int gz,
                  int gx, int dg) {
  if (fd_order == 24 || fd_order == 26 || fd_order == 28) {
    set_error("fd_order %d is accepted by the reference MEX but only fd_order 22 (the one SWD.m uses) is built",
              fd_order);
    return SWD_ERR_UNSUPPORTED;
  }
  SWD_CHECK(fd_order == 22, "fd_order must be 22 (got %d)", fd_order);
  SWD_CHECK(nt >= 2, "nt must be >= 2 (got %d)", nt);
  SWD_CHECK(nt_wf >= 1 && nt % nt_wf == 0, "nt (%d) must be a multiple of nt_wf (%d)", nt, nt_wf);
  SWD_CHECK(NZ >= 3 && NX >= 3, "padded grid %d x %d too small", NZ, NX);
  SWD_CHECK(nz >= 1 && nx >= 1 && nbc >= 1 && NX == nx + 2 * nbc && NZ >= nz + 3,
            "interior %d x %d (nbc %d) does not fit the padded grid %d x %d", nz, nx, nbc, NZ, NX);
  SWD_CHECK(ng >= 1 && dg >= 1, "need ng >= 1 and dg >= 1 (ng %d, dg %d)", ng, dg);
  SWD_CHECK(gz >= 1 && gz <= NZ - 2 && gx >= 1 && gx + (long)(ng - 1) * dg <= NX - 2,
            "receivers (row %d, cols %d..%ld) must lie inside rows/cols 1..n-2 of the padded grid", gz + 1,
            gx + 1, gx + 1 + (long)(ng - 1) * dg);
  return SWD_OK;
}

int validate_source(int st, int sz, int sx, int NZ, int NX) {
  SWD_CHECK(st >= 1 && st <= 5, "source_type must be 1..5 (got %d)", st);
  const int zlo = (st == 2) ? 2 : 1, xhi = (st == 2) ? NX - 3 : NX - 2;
  SWD_CHECK(sz >= zlo && sz <= NZ - 2 && sx >= 1 && sx <= xhi,
            "source (%d,%d) and its stencil taps must lie inside rows/cols 1..n-2", sz + 1, sx + 1);
  return SWD_OK;
}

template <typename T>
int fill_geom(FdGeom& g, int NZ, int NX, int nz, int nx, int nbc, int nt, int nt_wf, int ng, int gz, int gx,
              int dg) {
  g.NZ = NZ; g.NX = NX;
  g.pitch = round_up(NX, 128 / (int)sizeof(T));
  g.nz = nz; g.nx = nx; g.nbc = nbc; g.pad_top = 1;
  g.nt = nt; g.nt_wf = nt_wf; g.nrec = nt / nt_wf;
  g.ng = ng; g.gz = gz; g.gx = gx; g.dg = dg;
  g.field = (size_t)NZ * g.pitch;
  g.warps = 4;
  g.cells = 1;
  g.ring_fwd = 4;
  g.ring_adj = 4;
  return SWD_OK;
}

// The device side of one MEX-convention forward call: its buffers, arguments and host outputs.
template <typename T>
struct FwdJob {
  FwdIv p{};
  FdGeom g{};
  DevBuf slab;  // one allocation holding every buffer below
  DevView d_in, d_m1, d_m2, d_state, d_seis, d_seis_t, d_snap, d_snap_t, d_src;
  FwdArgs<T> a{};
  T* bufs[2] = {nullptr, nullptr};
  T* out[6] = {};  // host: seis_u, seis_w, fux, fuz, bwx, bwz
};

// Validates the call, allocates and fills the job's device buffers on st (materials packed,
// state and seismograms cleared); the time loop then sets a.in / a.out from bufs.
// keep_wf records the strain snapshots on the device even when fux..bwz are NULL.
template <typename T>
int fwd_job_setup(FwdJob<T>& J, const T* iv, int n_iv, const T* temp, const T* ca, const T* cl, const T* cm1,
                  const T* b, const T* b1, const T* s, T* seis_u, T* seis_w, T* fux, T* fuz, T* bwx, T* bwz,
                  cudaStream_t st, bool keep_wf = false) {
  FwdIv& p = J.p;
  SWD_TRY(parse_fwd_iv(iv, n_iv, p));
  const int nbc = (p.nxbc - p.nx) / 2;  // core/eigen_staggerfd_single.cpp:116
  SWD_TRY(validate_geom(p.nt, p.nzbc, p.nxbc, p.nz, p.nx, nbc, p.nt_wf, p.fd_order, p.ng, p.gz, p.gx, p.dg));
  SWD_TRY(validate_source(p.src_type, p.sz, p.sx, p.nzbc, p.nxbc));
  SWD_CHECK(temp && ca && cl && cm1 && b && b1 && s && seis_w, "null input/output pointer");
  const bool host_wf = fux || fuz || bwx || bwz;
  SWD_CHECK(!host_wf || (fux && fuz && bwx && bwz), "fux/fuz/bwx/bwz must all be given or all be NULL");
  const bool want_wf = host_wf || keep_wf;
  FdGeom& g = J.g;
  fill_geom<T>(g, p.nzbc, p.nxbc, p.nz, p.nx, nbc, p.nt, p.nt_wf, p.ng, p.gz, p.gx, p.dg);
  plan_decomposition(g, 1, 0);
  using V = typename Vec4<T>::type;
  using V2 = typename Vec2<T>::type;
  const size_t NN = (size_t)p.nzbc * p.nxbc, plane = (size_t)p.nz * p.nx;
  const size_t n_in = 6 * NN * sizeof(T) + p.nt * sizeof(T), n_m1 = g.field * sizeof(V), n_m2 = g.field * sizeof(V2);
  const size_t n_state = 2 * 5 * g.field * sizeof(T), n_seis = 2 * (size_t)p.nt * p.ng * sizeof(T);
  const size_t n_snap = want_wf ? (size_t)g.nrec * 4 * plane * sizeof(T) : 0;
  const size_t n_snap_t = host_wf ? (size_t)g.nrec * plane * sizeof(T) : 0;
  SlabPlan sl;
  const size_t o_in = sl.add(n_in), o_m1 = sl.add(n_m1), o_m2 = sl.add(n_m2), o_state = sl.add(n_state);
  const size_t o_seis = sl.add(n_seis), o_seis_t = sl.add(n_seis), o_src = sl.add(sizeof(int2));
  const size_t o_snap = sl.add(n_snap), o_snap_t = sl.add(n_snap_t);
  SWD_TRY(J.slab.alloc(sl.bytes));
  J.d_in = DevView(J.slab, o_in, n_in);
  J.d_m1 = DevView(J.slab, o_m1, n_m1);
  J.d_m2 = DevView(J.slab, o_m2, n_m2);
  J.d_state = DevView(J.slab, o_state, n_state);
  J.d_seis = DevView(J.slab, o_seis, n_seis);
  J.d_seis_t = DevView(J.slab, o_seis_t, n_seis);
  J.d_src = DevView(J.slab, o_src, sizeof(int2));
  J.d_snap = DevView(J.slab, o_snap, n_snap);
  J.d_snap_t = DevView(J.slab, o_snap_t, n_snap_t);
  T* din = J.d_in.template as<T>();
  const T* hsrc[6] = {temp, b, b1, ca, cl, cm1};
  for (int i = 0; i < 6; ++i) SWD_CUDA(cudaMemcpyAsync(din + i * NN, hsrc[i], NN * sizeof(T), cudaMemcpyHostToDevice, st));
  T* d_s = din + 6 * NN;
  SWD_CUDA(cudaMemcpyAsync(d_s, s, p.nt * sizeof(T), cudaMemcpyHostToDevice, st));
  const int2 sp = make_int2(p.sz, p.sx);
  SWD_CUDA(cudaMemcpyAsync(J.d_src.p, &sp, sizeof(int2), cudaMemcpyHostToDevice, st));
  SWD_TRY(pack_materials<T>(din, din + NN, din + 2 * NN, din + 3 * NN, din + 4 * NN, din + 5 * NN, J.d_m1.template as<V>(),
                            J.d_m2.template as<V2>(), p.nzbc, p.nxbc, g.pitch, st));
  SWD_CUDA(cudaMemsetAsync(J.d_state.p, 0, J.d_state.bytes, st));
  SWD_CUDA(cudaMemsetAsync(J.d_seis.p, 0, J.d_seis.bytes, st));
  FwdArgs<T>& a = J.a;
  a.g = g; a.mat = J.d_m1.template as<V>(); a.mb = J.d_m2.template as<V2>();
  a.src = J.d_src.template as<int2>(); a.src_type = p.src_type; a.s = d_s; a.dtx = (T)p.dtx;
  a.seis_w = J.d_seis.template as<T>(); a.seis_u = a.seis_w + (size_t)p.nt * p.ng;
  a.snap = want_wf ? J.d_snap.template as<T>() : nullptr;
  a.n_shots = 1;
  J.bufs[0] = J.d_state.template as<T>();
  J.bufs[1] = J.d_state.template as<T>() + 5 * g.field;
  T* const outs[6] = {seis_u, seis_w, fux, fuz, bwx, bwz};
  for (int i = 0; i < 6; ++i) J.out[i] = outs[i];
  return SWD_OK;
}

// Enqueues the job's outputs on st: seismograms [2][nt][ng] -> MATLAB nt x ng (column-major)
// each; snapshots [nrec][f][nz][nx] -> nz x nx x nrec per field.
template <typename T>
int fwd_job_finish(FwdJob<T>& J, cudaStream_t st) {
  const FwdIv& p = J.p;
  const size_t plane = (size_t)p.nz * p.nx, nn = (size_t)p.nt * p.ng;
  SWD_TRY(transpose<T, T>(J.d_seis.template as<T>(), nn, J.d_seis_t.template as<T>(), nn, 2, p.nt, p.ng, st));
  SWD_CUDA(cudaMemcpyAsync(J.out[1], J.d_seis_t.template as<T>(), nn * sizeof(T), cudaMemcpyDeviceToHost, st));
  if (J.out[0]) SWD_CUDA(cudaMemcpyAsync(J.out[0], J.d_seis_t.template as<T>() + nn, nn * sizeof(T), cudaMemcpyDeviceToHost, st));
  if (J.a.snap && J.out[2]) {
    for (int f = 0; f < 4; ++f) {
      SWD_TRY(transpose<T, T>(J.d_snap.template as<T>() + f * plane, 4 * plane, J.d_snap_t.template as<T>(), plane, J.g.nrec, p.nz,
                              p.nx, st));
      SWD_CUDA(cudaMemcpyAsync(J.out[2 + f], J.d_snap_t.p, (size_t)J.g.nrec * plane * sizeof(T),
                               cudaMemcpyDeviceToHost, st));
    }
  }
  return SWD_OK;
}

template <typename T>
int staggerfd_mex(const T* iv, int n_iv, const T* temp, const T* ca, const T* cl, const T* cm, const T* cm1,
                  const T* b, const T* b1, const T* s, T* seis_u, T* seis_w, T* fux, T* fuz, T* bwx, T* bwz) {
  clear_error();
  (void)cm;  // passed by the reference, unused by its kernel (cm1 carries mu)
  cudaStream_t st = 0;
  FwdJob<T> J;
  SWD_TRY(fwd_job_setup(J, iv, n_iv, temp, ca, cl, cm1, b, b1, s, seis_u, seis_w, fux, fuz, bwx, bwz, st));
  for (int it = 0; it < J.p.nt; ++it) {
    J.a.in = J.bufs[it & 1];
    J.a.out = J.bufs[(it + 1) & 1];
    SWD_TRY(launch_fwd_step<T, 4>(J.a, it, st));  // a dispatch or geometry error ends the call
  }
  SWD_CUDA(cudaGetLastError());
  SWD_TRY(fwd_job_finish(J, st));
  SWD_CUDA(cudaStreamSynchronize(st));
  return SWD_OK;
}

// The device side of one MEX-convention adjoint call: its buffers, arguments and host outputs.
template <typename T, typename TO>
struct AdjJob {
  int nt = 0;
  size_t plane = 0;
  FdGeom g{};
  DevBuf slab;  // one allocation holding every buffer below
  DevView d_in, d_m1, d_m2, d_state, d_res, d_snap, d_img, d_out;
  AdjArgs<T> a{};
  T* bufs[2] = {nullptr, nullptr};
  TO* out[3] = {};  // host: cl_img, cm_img, illum
  // single in, single out: the images accumulate in FP32, as the reference's single MEX
  // accumulates them (core/eigen_e2drtm_single.cpp:274-279); otherwise in FP64
  static constexpr bool f32img = std::is_same<T, float>::value && std::is_same<TO, float>::value;
};

// Validates the call, allocates and fills the job's device buffers on st: materials packed, the
// residual [nt][ng] and the snapshots [nrec][f][nz][nx] transposed from MATLAB's layout, state
// and images cleared; the time loop then sets a.in / a.out from bufs.
// d_snap, when given, is a forward job's device snapshots in this layout, read in place of
// fux..bwz (which are then ignored).
template <typename T, typename TO>
int adj_job_setup(AdjJob<T, TO>& J, const T* iv, int n_iv, const T* temp, const T* ca, const T* cl, const T* cm1,
                  const T* b, const T* b1, const T* res, const T* fux, const T* fuz, const T* bwx, const T* bwz,
                  TO* cl_img, TO* cm_img, TO* illum, cudaStream_t st, const T* d_snap = nullptr) {
  SWD_CHECK(iv != nullptr && n_iv >= 14, "input_vector needs 14 entries (got %d)", n_iv);
  // core/eigen_e2drtm_single.cpp:69-84
  const int nt = (int)iv[0], NZ = (int)iv[1], NX = (int)iv[2], ng = (int)iv[4], nbc = (int)iv[5];
  const int gz = (int)iv[6] - 1, gx = (int)iv[7] - 1, dg = (int)iv[8], fd_order = (int)iv[9];
  const int nt_wf = (int)iv[10], nz = (int)iv[11], nx = (int)iv[12];
  const T dtx = iv[3], dt = iv[13];
  SWD_TRY(validate_geom(nt, NZ, NX, nz, nx, nbc, nt_wf, fd_order, ng, gz, gx, dg));
  SWD_CHECK(temp && ca && cl && cm1 && b && b1 && res && (d_snap || (fux && fuz && bwx && bwz)) && cl_img &&
                cm_img && illum,
            "null input/output pointer");
  FdGeom& g = J.g;
  fill_geom<T>(g, NZ, NX, nz, nx, nbc, nt, nt_wf, ng, gz, gx, dg);
  plan_decomposition(g, 1, 0);
  using V = typename Vec4<T>::type;
  using V2 = typename Vec2<T>::type;
  const size_t NN = (size_t)NZ * NX, plane = (size_t)nz * nx, nsnap = (size_t)g.nrec * plane;
  J.nt = nt;
  J.plane = plane;
  const size_t n_stage = d_snap ? 6 * NN : std::max(6 * NN, nsnap);
  const size_t n_in = n_stage * sizeof(T) + (size_t)nt * ng * sizeof(T);
  const size_t n_m1 = g.field * sizeof(V), n_m2 = g.field * sizeof(V2), n_state = 2 * 5 * g.field * sizeof(T);
  const size_t n_res = (size_t)nt * ng * sizeof(T), n_snap = d_snap ? 0 : 4 * nsnap * sizeof(T);
  const size_t n_img = 3 * plane * sizeof(double), n_out = 3 * plane * sizeof(TO);
  SlabPlan sl;
  const size_t o_in = sl.add(n_in), o_m1 = sl.add(n_m1), o_m2 = sl.add(n_m2), o_state = sl.add(n_state);
  const size_t o_res = sl.add(n_res), o_snap = sl.add(n_snap), o_img = sl.add(n_img), o_out = sl.add(n_out);
  SWD_TRY(J.slab.alloc(sl.bytes));
  J.d_in = DevView(J.slab, o_in, n_in);
  J.d_m1 = DevView(J.slab, o_m1, n_m1);
  J.d_m2 = DevView(J.slab, o_m2, n_m2);
  J.d_state = DevView(J.slab, o_state, n_state);
  J.d_res = DevView(J.slab, o_res, n_res);
  J.d_snap = DevView(J.slab, o_snap, n_snap);
  J.d_img = DevView(J.slab, o_img, n_img);
  J.d_out = DevView(J.slab, o_out, n_out);
  T* din = J.d_in.template as<T>();
  T* dstage = din + n_stage;
  const T* hsrc[6] = {temp, b, b1, ca, cl, cm1};
  for (int i = 0; i < 6; ++i) SWD_CUDA(cudaMemcpyAsync(din + i * NN, hsrc[i], NN * sizeof(T), cudaMemcpyHostToDevice, st));
  SWD_TRY(pack_materials<T>(din, din + NN, din + 2 * NN, din + 3 * NN, din + 4 * NN, din + 5 * NN,
                            J.d_m1.template as<V>(), J.d_m2.template as<V2>(), NZ, NX, g.pitch, st));
  // residual: MATLAB nt x ng -> [nt][ng]
  SWD_CUDA(cudaMemcpyAsync(dstage, res, (size_t)nt * ng * sizeof(T), cudaMemcpyHostToDevice, st));
  SWD_TRY(transpose<T, T>(dstage, 0, J.d_res.template as<T>(), 0, 1, ng, nt, st));
  // snapshots: MATLAB nz x nx x nrec per field -> [nrec][f][nz][nx]
  const T* wf[4] = {fux, fuz, bwx, bwz};
  for (int f = 0; f < 4 && !d_snap; ++f) {
    SWD_CUDA(cudaMemcpyAsync(din, wf[f], nsnap * sizeof(T), cudaMemcpyHostToDevice, st));
    SWD_TRY(transpose<T, T>(din, plane, J.d_snap.template as<T>() + f * plane, 4 * plane, g.nrec, nx, nz, st));
  }
  SWD_CUDA(cudaMemsetAsync(J.d_state.p, 0, J.d_state.bytes, st));
  SWD_CUDA(cudaMemsetAsync(J.d_img.p, 0, J.d_img.bytes, st));
  AdjArgs<T>& a = J.a;
  a.g = g; a.mat = J.d_m1.template as<V>(); a.mb = J.d_m2.template as<V2>();
  a.res = J.d_res.template as<T>(); a.snap = d_snap ? d_snap : J.d_snap.template as<T>();
  a.img = J.d_img.template as<double>();
  if (AdjJob<T, TO>::f32img) a.img32 = J.d_img.template as<float>();
  a.dtx = dtx; a.dt = dt; a.n_shots = 1;
  J.bufs[0] = J.d_state.template as<T>();
  J.bufs[1] = J.d_state.template as<T>() + 5 * g.field;
  J.out[0] = cl_img; J.out[1] = cm_img; J.out[2] = illum;
  return SWD_OK;
}

// Enqueues the job's images on st: [3][nz][nx] -> MATLAB nz x nx each, in the output type.
template <typename T, typename TO>
int adj_job_finish(AdjJob<T, TO>& J, cudaStream_t st) {
  const size_t plane = J.plane;
  if constexpr (AdjJob<T, TO>::f32img)
    SWD_TRY(transpose<float, float>(J.d_img.template as<float>(), plane, J.d_out.template as<float>(), plane, 3,
                                    J.g.nz, J.g.nx, st));
  else
    SWD_TRY(transpose<double, TO>(J.d_img.template as<double>(), plane, J.d_out.template as<TO>(), plane, 3, J.g.nz,
                                  J.g.nx, st));
  for (int i = 0; i < 3; ++i)
    SWD_CUDA(cudaMemcpyAsync(J.out[i], J.d_out.template as<TO>() + i * plane, plane * sizeof(TO),
                             cudaMemcpyDeviceToHost, st));
  return SWD_OK;
}

template <typename T, typename TO>
int e2drtm_mex(const T* iv, int n_iv, const T* temp, const T* ca, const T* cl, const T* cm, const T* cm1,
               const T* b, const T* b1, const T* res, const T* fux, const T* fuz, const T* bwx, const T* bwz,
               TO* cl_img, TO* cm_img, TO* illum) {
  clear_error();
  (void)cm;
  cudaStream_t st = 0;
  AdjJob<T, TO> J;
  SWD_TRY(adj_job_setup(J, iv, n_iv, temp, ca, cl, cm1, b, b1, res, fux, fuz, bwx, bwz, cl_img, cm_img, illum, st));
  int cur = 0;
  for (int it = J.nt - 2; it >= 0; --it) {  // core/eigen_e2drtm_single.cpp:181
    J.a.in = J.bufs[cur];
    J.a.out = J.bufs[cur ^ 1];
    SWD_TRY(launch_adj_step<T, 4>(J.a, it, st));
    cur ^= 1;
  }
  SWD_CUDA(cudaGetLastError());
  SWD_TRY(adj_job_finish(J, st));
  SWD_CUDA(cudaStreamSynchronize(st));
  return SWD_OK;
}

}  // namespace
}  // namespace swd

using namespace swd;

// The forward jobs of a batch whose strain snapshots stay on the device for an adjoint batch.
struct swd_fd_batch {
  std::vector<std::unique_ptr<swd::FwdJob<float>>> jobs;
};

namespace swd {
namespace {

const float* kept_snap(const swd_fd_batch* kept, int j) { return kept->jobs[j]->a.snap; }

// The forward batch; keep_wf records every job's snapshots on the device for a later adjoint batch.
int fwd_batch(int n_jobs, const swd_staggerfd_job* jobs, std::vector<std::unique_ptr<FwdJob<float>>>& J,
              bool keep_wf) {
  SWD_CHECK(jobs && n_jobs >= 1, "a batch needs at least one job (got %d)", n_jobs);
  cudaStream_t st = 0;
  J.clear();
  std::vector<int> cta0(n_jobs + 1, 0);
  int nt_max = 0;
  for (int j = 0; j < n_jobs; ++j) {
    const swd_staggerfd_job& q = jobs[j];
    J.push_back(std::make_unique<FwdJob<float>>());
    FwdJob<float>& w = *J.back();
    const int rc = fwd_job_setup(w, q.iv, q.n_iv, q.temp, q.ca, q.cl, q.cm1, q.b, q.b1, q.s, q.seismo_u, q.seismo_w,
                                 q.fux, q.fuz, q.bwx, q.bwz, st, keep_wf);
    if (rc != SWD_OK) {
      set_error("job %d: %s", j, std::string(swd_last_error()).c_str());
      return rc;
    }
    // the one kernel shape of the MEX-convention forward (launch_fwd_step with b, b1 arrays)
    SWD_CHECK(w.g.sched == 0 && w.g.warps == 4 && w.g.cells == 1 && w.g.ring_fwd == 4,
              "internal: batch job %d planned for another FD kernel", j);
    const long blocks = (long)w.g.n_strips * w.g.n_chunks;
    SWD_CHECK(cta0[j] + blocks < (1L << 31), "batch too large for one launch");
    cta0[j + 1] = cta0[j] + (int)blocks;
    nt_max = std::max(nt_max, w.p.nt);
  }
  // the jobs' arguments for even and odd steps (state buffers swapped) and their first tiles
  std::vector<FwdArgs<float>> args(2 * (size_t)n_jobs);
  for (int j = 0; j < n_jobs; ++j) {
    args[j] = J[j]->a;
    args[j].in = J[j]->bufs[0];
    args[j].out = J[j]->bufs[1];
    args[n_jobs + j] = J[j]->a;
    args[n_jobs + j].in = J[j]->bufs[1];
    args[n_jobs + j].out = J[j]->bufs[0];
  }
  DevBuf d_args, d_cta;
  SWD_TRY(d_args.alloc(args.size() * sizeof(FwdArgs<float>)));
  SWD_TRY(d_cta.alloc(cta0.size() * sizeof(int)));
  SWD_CUDA(cudaMemcpyAsync(d_args.p, args.data(), args.size() * sizeof(FwdArgs<float>), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(d_cta.p, cta0.data(), cta0.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  auto kernel = fd_fwd_smem_multi<float, 4, 4, 1, 4, true>;
  constexpr size_t smem = smem_bytes<float, 4, 1, 4, true>();
  static int ready = set_smem(kernel, smem);
  SWD_TRY(ready);
  const FwdArgs<float>* da = d_args.as<FwdArgs<float>>();
  for (int it = 0; it < nt_max; ++it) {  // one launch per step for every job's tiles
    kernel<<<(unsigned)cta0[n_jobs], 32 * 4, smem, st>>>(it & 1 ? da + n_jobs : da, d_cta.as<int>(), n_jobs, it);
    count_launch(1);
  }
  SWD_CUDA(cudaGetLastError());
  for (int j = 0; j < n_jobs; ++j) SWD_TRY(fwd_job_finish(*J[j], st));
  SWD_CUDA(cudaStreamSynchronize(st));
  return SWD_OK;
}
// The adjoint batch; with kept, job j reads forward job j's device snapshots in place of fux..bwz.
int adj_batch(int n_jobs, const swd_e2drtm_job* jobs, const swd_fd_batch* kept) {
  SWD_CHECK(jobs && n_jobs >= 1, "a batch needs at least one job (got %d)", n_jobs);
  cudaStream_t st = 0;
  std::vector<std::unique_ptr<AdjJob<float, float>>> J;
  std::vector<int> cta0(n_jobs + 1, 0);
  int steps = 0;
  for (int j = 0; j < n_jobs; ++j) {
    const swd_e2drtm_job& q = jobs[j];
    J.push_back(std::make_unique<AdjJob<float, float>>());
    AdjJob<float, float>& w = *J.back();
    const int rc = adj_job_setup(w, q.iv, q.n_iv, q.temp, q.ca, q.cl, q.cm1, q.b, q.b1, q.seismo_w, q.fux, q.fuz, q.bwx,
                                 q.bwz, q.cl_img, q.cm_img, q.illum_div, st, kept ? kept_snap(kept, j) : nullptr);
    if (rc != SWD_OK) {
      set_error("job %d: %s", j, std::string(swd_last_error()).c_str());
      return rc;
    }
    if (kept) {  // the forward job's snapshots must have this job's shape
      const FdGeom& fg = kept->jobs[j]->g;
      SWD_CHECK(fg.nrec == w.g.nrec && fg.nz == w.g.nz && fg.nx == w.g.nx,
                "job %d: the kept forward job has %d snapshots of %d x %d, this job needs %d of %d x %d", j, fg.nrec,
                fg.nz, fg.nx, w.g.nrec, w.g.nz, w.g.nx);
    }
    // the one kernel shape of the MEX-convention adjoint (launch_adj_step with b, b1 arrays)
    SWD_CHECK(w.g.sched == 0 && w.g.warps == 4 && w.g.cells == 1 && w.g.ring_adj == 4,
              "internal: batch job %d planned for another FD kernel", j);
    const long blocks = (long)w.g.n_strips * w.g.n_chunks;
    SWD_CHECK(cta0[j] + blocks < (1L << 31), "batch too large for one launch");
    cta0[j + 1] = cta0[j] + (int)blocks;
    steps = std::max(steps, w.nt - 1);  // it = nt-2 .. 0
  }
  // the jobs' arguments for even and odd steps (state buffers swapped) and their first tiles
  std::vector<AdjArgs<float>> args(2 * (size_t)n_jobs);
  for (int j = 0; j < n_jobs; ++j) {
    args[j] = J[j]->a;
    args[j].in = J[j]->bufs[0];
    args[j].out = J[j]->bufs[1];
    args[n_jobs + j] = J[j]->a;
    args[n_jobs + j].in = J[j]->bufs[1];
    args[n_jobs + j].out = J[j]->bufs[0];
  }
  DevBuf d_args, d_cta;
  SWD_TRY(d_args.alloc(args.size() * sizeof(AdjArgs<float>)));
  SWD_TRY(d_cta.alloc(cta0.size() * sizeof(int)));
  SWD_CUDA(cudaMemcpyAsync(d_args.p, args.data(), args.size() * sizeof(AdjArgs<float>), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(d_cta.p, cta0.data(), cta0.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  auto kernel = fd_adj_smem_multi<float, 4, 4, 1, 4, true>;
  constexpr size_t smem = smem_bytes<float, 4, 1, 4, true>();
  static int ready = set_smem(kernel, smem);
  SWD_TRY(ready);
  const AdjArgs<float>* da = d_args.as<AdjArgs<float>>();
  for (int step = 0; step < steps; ++step) {  // one launch per step for every job's tiles
    kernel<<<(unsigned)cta0[n_jobs], 32 * 4, smem, st>>>(step & 1 ? da + n_jobs : da, d_cta.as<int>(), n_jobs, step);
    count_launch(1);
  }
  SWD_CUDA(cudaGetLastError());
  for (int j = 0; j < n_jobs; ++j) SWD_TRY(adj_job_finish(*J[j], st));
  SWD_CUDA(cudaStreamSynchronize(st));
  return SWD_OK;
}
}  // namespace
}  // namespace swd

extern "C" {

const char* swd_last_error(void) { return g_err; }
int swd_version(void) { return 100; }
uint64_t swd_kernel_launches(void) { return g_launches.load(); }

int swd_staggerfd_single(const float* iv, int n_iv, const float* temp, const float* ca, const float* cl,
                         const float* cm, const float* cm1, const float* b, const float* b1, const float* s,
                         float* seismo_u, float* seismo_w, float* fux, float* fuz, float* bwx, float* bwz) {
  return staggerfd_mex<float>(iv, n_iv, temp, ca, cl, cm, cm1, b, b1, s, seismo_u, seismo_w, fux, fuz, bwx, bwz);
}
int swd_staggerfd_single_batch(int n_jobs, const swd_staggerfd_job* jobs) {
  clear_error();
  std::vector<std::unique_ptr<FwdJob<float>>> J;
  return fwd_batch(n_jobs, jobs, J, false);
}
int swd_staggerfd_single_batch_keep(int n_jobs, const swd_staggerfd_job* jobs, swd_fd_batch** kept) {
  clear_error();
  SWD_CHECK(kept != nullptr, "kept must point to a swd_fd_batch* to fill");
  *kept = nullptr;
  std::unique_ptr<swd_fd_batch> b(new swd_fd_batch);
  SWD_TRY(fwd_batch(n_jobs, jobs, b->jobs, true));
  *kept = b.release();
  return SWD_OK;
}
int swd_e2drtm_single_batch(int n_jobs, const swd_e2drtm_job* jobs) {
  clear_error();
  return adj_batch(n_jobs, jobs, nullptr);
}
int swd_e2drtm_single_batch_kept(int n_jobs, const swd_e2drtm_job* jobs, const swd_fd_batch* kept) {
  clear_error();
  SWD_CHECK(kept != nullptr && (int)kept->jobs.size() == n_jobs,
            "the kept forward batch has %d jobs, this adjoint batch %d", kept ? (int)kept->jobs.size() : 0, n_jobs);
  return adj_batch(n_jobs, jobs, kept);
}
void swd_fd_batch_free(swd_fd_batch* kept) { delete kept; }
int swd_staggerfd_double(const double* iv, int n_iv, const double* temp, const double* ca, const double* cl,
                         const double* cm, const double* cm1, const double* b, const double* b1, const double* s,
                         double* seismo_u, double* seismo_w, double* fux, double* fuz, double* bwx,
                         double* bwz) {
  return staggerfd_mex<double>(iv, n_iv, temp, ca, cl, cm, cm1, b, b1, s, seismo_u, seismo_w, fux, fuz, bwx, bwz);
}
int swd_e2drtm_single(const float* iv, int n_iv, const float* temp, const float* ca, const float* cl,
                      const float* cm, const float* cm1, const float* b, const float* b1, const float* seismo_w,
                      const float* fux, const float* fuz, const float* bwx, const float* bwz, float* cl_img,
                      float* cm_img, float* illum_div) {
  return e2drtm_mex<float, float>(iv, n_iv, temp, ca, cl, cm, cm1, b, b1, seismo_w, fux, fuz, bwx, bwz, cl_img,
                                  cm_img, illum_div);
}
int swd_e2drtm_single_f64out(const float* iv, int n_iv, const float* temp, const float* ca, const float* cl,
                             const float* cm, const float* cm1, const float* b, const float* b1,
                             const float* seismo_w, const float* fux, const float* fuz, const float* bwx,
                             const float* bwz, double* cl_img, double* cm_img, double* illum_div) {
  return e2drtm_mex<float, double>(iv, n_iv, temp, ca, cl, cm, cm1, b, b1, seismo_w, fux, fuz, bwx, bwz, cl_img,
                                   cm_img, illum_div);
}
int swd_e2drtm_double(const double* iv, int n_iv, const double* temp, const double* ca, const double* cl,
                      const double* cm, const double* cm1, const double* b, const double* b1,
                      const double* seismo_w, const double* fux, const double* fuz, const double* bwx,
                      const double* bwz, double* cl_img, double* cm_img, double* illum_div) {
  return e2drtm_mex<double, double>(iv, n_iv, temp, ca, cl, cm, cm1, b, b1, seismo_w, fux, fuz, bwx, bwz, cl_img,
                                    cm_img, illum_div);
}

}  // extern "C"
