// Launchers of the two-shot two-step FD kernels (fd_warpx.cuh).  Compiled with -fmad=false
// like the other FD translation units.
#include "fd_host.cuh"
#include "fd_warpx.cuh"

namespace swd {

// (warps per CTA, row slots) of the two-shot kernels
#define SWD_WARPX_SHAPES(X) X(2, 4) X(4, 4) X(2, 6) X(4, 6)

bool fd_warpx_built(int w, int s) {
#define X(W, S) if (w == W && s == S) return true;
  SWD_WARPX_SHAPES(X)
#undef X
  return false;
}

namespace {

template <typename K>
int set_smem_x(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) SWD_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return SWD_OK;
}

// warps of a launch: 28-column strips x chunks x shot pairs
inline long pair_warps(const FdGeom& g, int n_shots) { return (long)g.n_strips * g.n_chunks * ((n_shots + 1) / 2); }

template <int NW, int NS, int SS>
int fwd_launch(const FwdArgs<float>& a0, int it, cudaStream_t st) {
  constexpr size_t smem = warpx_smem_bytes<NW, NS>();
  static int ready = set_smem_x(fd_fwd_warp2x<NW, NS, SS>, smem);
  if (ready != SWD_OK) return ready;
  SWD_CHECK(a0.g.chunk <= kWarpChunkMax, "internal: two-step chunk of %d rows (at most %d)", a0.g.chunk, kWarpChunkMax);
  FwdArgs<float> a = a0;
  a.g.n_strips = (a.g.NX - 2 + kWarpOut2 - 1) / kWarpOut2;
  const long warps = pair_warps(a.g, a.n_shots);
  fd_fwd_warp2x<NW, NS, SS><<<(unsigned)((warps + NW - 1) / NW), 32 * NW, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <int NW, int NS>
int fwd_impl(const FwdArgs<float>& a, int it, cudaStream_t st) {
  if (a.snap && it % a.g.nt_wf == 0) return fwd_launch<NW, NS, 0>(a, it, st);
  if (a.snap && (it + 1) % a.g.nt_wf == 0) return fwd_launch<NW, NS, 1>(a, it, st);
  return fwd_launch<NW, NS, -1>(a, it, st);
}
template <int NW, int NS, int IS>
int adj_launch(const AdjArgs<float>& a0, int it, cudaStream_t st) {
  constexpr size_t smem = IS >= 0 ? warpx_img_smem_bytes<NW, NS>() : warpx_smem_bytes<NW, NS>();
  static int ready = set_smem_x(fd_adj_warp2x<NW, NS, IS>, smem);
  if (ready != SWD_OK) return ready;
  SWD_CHECK(a0.g.chunk <= kWarpChunkMax, "internal: two-step chunk of %d rows (at most %d)", a0.g.chunk, kWarpChunkMax);
  AdjArgs<float> a = a0;
  a.g.n_strips = (a.g.NX - 2 + kWarpOut2 - 1) / kWarpOut2;
  const long warps = pair_warps(a.g, a.n_shots);
  fd_adj_warp2x<NW, NS, IS><<<(unsigned)((warps + NW - 1) / NW), 32 * NW, smem, st>>>(a, it);
  count_launch(1);
  return SWD_OK;
}
template <int NW, int NS>
int adj_impl(const AdjArgs<float>& a, int it, cudaStream_t st) {
  if (it % a.g.nt_wf == 0) return adj_launch<NW, NS, 0>(a, it, st);
  if ((it - 1) % a.g.nt_wf == 0) return adj_launch<NW, NS, 1>(a, it, st);
  return adj_launch<NW, NS, -1>(a, it, st);
}

}  // namespace

int launch_fwd_pair_x(const FwdArgs<float>& a, int it, cudaStream_t st) {
  if (!fd_pairs(a.g) || a.g.pairs != 2 || a.mb || it + 1 >= a.g.nt) {
    set_error("internal: two-shot forward launch outside its schedule");
    return SWD_ERR_INVALID;
  }
  switch (a.g.warps * 10 + a.g.ring_fwd) {
#define X(w, s) case w * 10 + s: return fwd_impl<w, s>(a, it, st);
    SWD_WARPX_SHAPES(X)
#undef X
    default: break;
  }
  set_error("internal: unsupported two-shot FD kernel variant");
  return SWD_ERR_INVALID;
}

int launch_adj_pair_x(const AdjArgs<float>& a, int it, cudaStream_t st) {
  if (!fd_pairs(a.g) || a.g.pairs != 2 || a.mb || it < 1) {
    set_error("internal: two-shot adjoint launch outside its schedule");
    return SWD_ERR_INVALID;
  }
  switch (a.g.warps * 10 + a.g.ring_adj) {
#define X(w, s) case w * 10 + s: return adj_impl<w, s>(a, it, st);
    SWD_WARPX_SHAPES(X)
#undef X
    default: break;
  }
  set_error("internal: unsupported two-shot FD kernel variant");
  return SWD_ERR_INVALID;
}

}  // namespace swd
