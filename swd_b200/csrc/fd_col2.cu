// Launchers of the column-pair FD kernels (fd_col2.cuh) and the pair-interleaved material
// table they read.  Compiled with -fmad=false like the other FD translation units.
#include "fd_col2.cuh"
#include "fd_host.cuh"

namespace swd {

// (warps per CTA, row slots) of the column-pair kernels
#define SWD_COL2_SHAPES(X) X(2, 4) X(4, 4) X(2, 6) X(4, 6) X(8, 4)

bool fd_col2_built(int w, int s) {
#define X(W, S) if (w == W && s == S) return true;
  SWD_COL2_SHAPES(X)
#undef X
  return false;
}

bool fd_col2_fits(const FdGeom& g) {
  // column pairs must not straddle the interior boundary (snapshot and image pairs), and the
  // padded width must hold whole pairs
  return (g.nbc % 2 == 0) && (g.nx % 2 == 0) && (g.NX % 2 == 0) && (g.pitch % 32 == 0);
}

// {temp, ca, cl, cm1}[NZ][pitch] -> per column pair {temp, temp', ca, ca'}, {cl, cl', cm1, cm1'}
__global__ void mat_pairs_kernel(const float4* __restrict__ mat, float4* __restrict__ mp, int NZ, int pitch) {
  const int P = pitch >> 1;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)NZ * P) return;
  const int z = (int)(i / P), p = (int)(i % P);
  const float4 l = mat[(size_t)z * pitch + 2 * p], r = mat[(size_t)z * pitch + 2 * p + 1];
  mp[2 * i] = make_float4(l.x, r.x, l.y, r.y);
  mp[2 * i + 1] = make_float4(l.z, r.z, l.w, r.w);
}

int col2_material_pairs(const float4* mat, float4* mp, int NZ, int pitch, cudaStream_t st) {
  const long n = (long)NZ * (pitch >> 1);
  mat_pairs_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(mat, mp, NZ, pitch);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}

namespace {

template <typename K>
int set_smem_c2(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) SWD_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return SWD_OK;
}

inline long col2_warps(const FdGeom& g, int n_shots) { return (long)g.n_strips * g.n_chunks * n_shots; }

int col2_check(const FdGeom& g) {
  SWD_CHECK(fd_col2_fits(g), "internal: column-pair FD kernels on a grid with odd nbc, nx or width");
  SWD_CHECK(g.chunk <= kWarpChunkMax, "internal: column-pair chunk of %d rows (at most %d)", g.chunk, kWarpChunkMax);
  SWD_CHECK(g.n_strips == (g.NX / 2 + kCol2Out / 2 - 1) / (kCol2Out / 2), "internal: column-pair strips not planned");
  return SWD_OK;
}

template <int NW, int NS, int SS>
int fwd2_launch(const FwdArgs<float>& a, int it, cudaStream_t st) {
  constexpr size_t smem = col2_smem_bytes<NW, NS>();
  static int ready = set_smem_c2(fd_fwd_col2<NW, NS, SS>, smem);
  if (ready != SWD_OK) return ready;
  SWD_TRY(col2_check(a.g));
  const long warps = col2_warps(a.g, a.n_shots);
  fd_fwd_col2<NW, NS, SS><<<(unsigned)((warps + NW - 1) / NW), 32 * NW, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <int NW, int NS>
int fwd2_impl(const FwdArgs<float>& a, int it, cudaStream_t st) {
  if (a.snap && it % a.g.nt_wf == 0) return fwd2_launch<NW, NS, 0>(a, it, st);
  if (a.snap && (it + 1) % a.g.nt_wf == 0) return fwd2_launch<NW, NS, 1>(a, it, st);
  return fwd2_launch<NW, NS, -1>(a, it, st);
}
template <int NW, int NS, bool SNAP>
int fwd1_launch(const FwdArgs<float>& a, int it, cudaStream_t st) {
  constexpr size_t smem = col2_smem_bytes<NW, NS>();
  static int ready = set_smem_c2(fd_fwd_col1<NW, NS, SNAP>, smem);
  if (ready != SWD_OK) return ready;
  SWD_TRY(col2_check(a.g));
  const long warps = col2_warps(a.g, a.n_shots);
  fd_fwd_col1<NW, NS, SNAP><<<(unsigned)((warps + NW - 1) / NW), 32 * NW, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <int NW, int NS>
int fwd1_impl(const FwdArgs<float>& a, int it, cudaStream_t st) {
  if (a.snap && it % a.g.nt_wf == 0) return fwd1_launch<NW, NS, true>(a, it, st);
  return fwd1_launch<NW, NS, false>(a, it, st);
}
template <int NW, int NS, int IS>
int adj2_launch(const AdjArgs<float>& a, int it, cudaStream_t st) {
  constexpr size_t smem = IS >= 0 ? col2_img_smem_bytes<NW, NS>() : col2_smem_bytes<NW, NS>();
  static int ready = set_smem_c2(fd_adj_col2<NW, NS, IS>, smem);
  if (ready != SWD_OK) return ready;
  SWD_TRY(col2_check(a.g));
  const long warps = col2_warps(a.g, a.n_shots);
  fd_adj_col2<NW, NS, IS><<<(unsigned)((warps + NW - 1) / NW), 32 * NW, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <int NW, int NS>
int adj2_impl(const AdjArgs<float>& a, int it, cudaStream_t st) {
  if (it % a.g.nt_wf == 0) return adj2_launch<NW, NS, 0>(a, it, st);
  if ((it - 1) % a.g.nt_wf == 0) return adj2_launch<NW, NS, 1>(a, it, st);
  return adj2_launch<NW, NS, -1>(a, it, st);
}
template <int NW, int NS, bool IMG>
int adj1_launch(const AdjArgs<float>& a, int it, cudaStream_t st) {
  constexpr size_t smem = col2_smem_bytes<NW, NS>();
  static int ready = set_smem_c2(fd_adj_col1<NW, NS, IMG>, smem);
  if (ready != SWD_OK) return ready;
  SWD_TRY(col2_check(a.g));
  const long warps = col2_warps(a.g, a.n_shots);
  fd_adj_col1<NW, NS, IMG><<<(unsigned)((warps + NW - 1) / NW), 32 * NW, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <int NW, int NS>
int adj1_impl(const AdjArgs<float>& a, int it, cudaStream_t st) {
  if (it % a.g.nt_wf == 0) return adj1_launch<NW, NS, true>(a, it, st);
  return adj1_launch<NW, NS, false>(a, it, st);
}

}  // namespace

#define SWD_COL2_DISPATCH(FN, RING)                    \
  switch (a.g.warps * 10 + a.g.RING) {                 \
    SWD_COL2_SHAPES(X)                                 \
    default: break;                                    \
  }                                                    \
  set_error("internal: unsupported column-pair FD kernel variant"); \
  return SWD_ERR_INVALID;

int launch_fwd_pair_c2(const FwdArgs<float>& a, int it, cudaStream_t st) {
  if (a.g.sched != 3 || a.mb || it + 1 >= a.g.nt) {
    set_error("internal: two-step column-pair forward launch outside its schedule");
    return SWD_ERR_INVALID;
  }
#define X(w, s) case w * 10 + s: return fwd2_impl<w, s>(a, it, st);
  SWD_COL2_DISPATCH(fwd2_impl, ring_fwd)
#undef X
}
int launch_fwd_step_c2(const FwdArgs<float>& a, int it, cudaStream_t st) {
  if (a.g.sched != 3 || a.mb) {
    set_error("internal: column-pair forward launch outside its schedule");
    return SWD_ERR_INVALID;
  }
#define X(w, s) case w * 10 + s: return fwd1_impl<w, s>(a, it, st);
  SWD_COL2_DISPATCH(fwd1_impl, ring_fwd)
#undef X
}
int launch_adj_pair_c2(const AdjArgs<float>& a, int it, cudaStream_t st) {
  if (a.g.sched != 3 || a.mb || it < 1) {
    set_error("internal: two-step column-pair adjoint launch outside its schedule");
    return SWD_ERR_INVALID;
  }
#define X(w, s) case w * 10 + s: return adj2_impl<w, s>(a, it, st);
  SWD_COL2_DISPATCH(adj2_impl, ring_adj)
#undef X
}
int launch_adj_step_c2(const AdjArgs<float>& a, int it, cudaStream_t st) {
  if (a.g.sched != 3 || a.mb) {
    set_error("internal: column-pair adjoint launch outside its schedule");
    return SWD_ERR_INVALID;
  }
#define X(w, s) case w * 10 + s: return adj1_impl<w, s>(a, it, st);
  SWD_COL2_DISPATCH(adj1_impl, ring_adj)
#undef X
}

}  // namespace swd
