// Host-side helpers shared by the FD, Radon and batched-engine translation units.
#pragma once
#include <algorithm>

#include "swd_common.cuh"
#include "fd_kernels.cuh"

namespace swd {

void clear_error();
void count_launch(uint64_t n);

// Batched transpose: out[b*ob + c*R + r] = in[b*ib + r*C + c] for B planes of R x C.
template <typename Ti, typename To>
int transpose(const Ti* in, size_t ib, To* out, size_t ob, int B, int R, int C, cudaStream_t st);

// MATLAB column-major materials -> packed row-major mat {temp,ca,cl,cm1} and mb {b,b1}.
template <typename T>
int pack_materials(const T* temp, const T* b, const T* b1, const T* ca, const T* cl, const T* cm1,
                   typename Vec4<T>::type* mat, typename Vec2<T>::type* mb, int NZ, int NX, int pitch,
                   cudaStream_t st);

// Choose strips/chunks for a launch over n_shots shots (chunk_rows <= 0: heuristic).
void plan_decomposition(FdGeom& g, int n_shots, int chunk_rows);
// true when the engine-path FD kernels are built for (warps, cells, ring depth)
bool fd_variant_built(int w, int c, int d);
// true when the one-barrier-per-row (lead) schedule is built for (warps, cells, ring depth)
bool fd_lead_built(int w, int c, int d);

template <typename T, int NF>
int launch_fwd_step(const FwdArgs<T>& a, int it, cudaStream_t st);
template <typename T, int NF>
int launch_adj_step(const AdjArgs<T>& a, int it, cudaStream_t st);
// true when the forward and the adjoint advance two steps per launch under g (warp-streaming
// schedule with pairs; needs nt_wf >= 2 so that at most one step of a pair is a snapshot step)
inline bool fd_pairs(const FdGeom& g) { return ((g.sched == 2 && g.pairs) || g.sched == 3) && g.nt_wf >= 2; }
// true when the two-shot two-step kernels (fd_warpx.cuh) are built for (warps per CTA, row slots)
bool fd_warpx_built(int w, int s);
// the two-shot forms of launch_fwd_pair / launch_adj_pair (g.pairs == 2)
int launch_fwd_pair_x(const FwdArgs<float>& a, int it, cudaStream_t st);
int launch_adj_pair_x(const AdjArgs<float>& a, int it, cudaStream_t st);
// Column-pair schedule (fd_col2.cuh, g.sched == 3): built shapes, whether a grid suits it
// (even nbc and nx), the pair-interleaved material table, and its one- and two-step launches.
bool fd_col2_built(int w, int s);
bool fd_col2_fits(const FdGeom& g);
int col2_material_pairs(const float4* mat, float4* mp, int NZ, int pitch, cudaStream_t st);
int launch_fwd_pair_c2(const FwdArgs<float>& a, int it, cudaStream_t st);
int launch_fwd_step_c2(const FwdArgs<float>& a, int it, cudaStream_t st);
int launch_adj_pair_c2(const AdjArgs<float>& a, int it, cudaStream_t st);
int launch_adj_step_c2(const AdjArgs<float>& a, int it, cudaStream_t st);
// Forward steps it and it+1 in one launch (it+1 < nt), from a.in to a.out.
int launch_fwd_pair(const FwdArgs<float>& a, int it, cudaStream_t st);
// Adjoint steps it and it-1 in one launch (it >= 1), from a.in to a.out.
int launch_adj_pair(const AdjArgs<float>& a, int it, cudaStream_t st);

}  // namespace swd
