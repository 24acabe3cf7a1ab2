// Batched SWD gradient engine: every shot of an iteration on the GPU at once.
//
// One gradient call does, for each batch of shots (SWD.m:171-194, all shots in
// one batch when memory allows):
//   forward FD of every shot, one launch per time step, strain snapshots kept
//   in HBM (or state checkpoints every K steps, recomputed segment by segment)
//   -> Radon spectra of both sides of every shot -> guided picks and misfits
//   -> SoftMax gradient, adjoint Radon, inverse DFT into the adjoint sources
//   -> adjoint FD with FP64 imaging -> shot sum in FP64 (fixed shot order),
// then illumination normalisation, Vs gradient and smoothing (SWD.m:196-201).
// Time loops are captured once into CUDA graphs and replayed on later calls.
// Compiled with -fmad=false like the FD kernels.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <memory>
#include <vector>

#include "fd_host.cuh"
#include "model_prep.cuh"
#include "radon.cuh"
#include "wd.cuh"

namespace swd {

// ------------------------------------------------------------------ small kernels

// gsum[c][cell] += sum_b img[b][c][cell], shots in batch order (deterministic FP64 sum).
template <typename I>
__global__ void shot_sum_kernel(const I* __restrict__ img, int nb, size_t plane, double* gsum) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * plane) return;
  double acc = gsum[i];
  for (int b = 0; b < nb; ++b) acc = acc + (double)img[(size_t)b * 3 * plane + i];
  gsum[i] = acc;
}

// dk = -4*vs.*(g_cl./g_illum) + 2*vs.*(g_cm./g_illum) (SWD.m:199-200); vs is MATLAB column-major.
__global__ void assemble_kernel(int nz, int nx, const double* __restrict__ vs, const double* __restrict__ gsum,
                                double* dk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nz * nx) return;
  const int z = i / nx, x = i % nx;
  const size_t plane = (size_t)nz * nx;
  const double gcl = gsum[i] / gsum[2 * plane + i];
  const double gcm = gsum[plane + i] / gsum[2 * plane + i];
  const double v = vs[(size_t)x * nz + z];
  dk[i] = -4 * v * gcl + 2 * v * gcm;
}

// smooth2a(A, Nr, Nc) (core/smooth2a.m:52-76): box mean over the window clipped to the
// grid; NaNs are excluded from sums and counts and stay NaN.  in/out row-major [z][x].
__global__ void smooth2a_kernel(int nz, int nx, int Nr, int Nc, const double* __restrict__ in, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nz * nx) return;
  const int z = i / nx, x = i % nx;
  if (isnan(in[i])) { out[i] = in[i]; return; }
  double s = 0.0, n = 0.0;
  for (int xx = max(0, x - Nc); xx <= min(nx - 1, x + Nc); ++xx) {
    double cs = 0.0, cn = 0.0;
    for (int zz = max(0, z - Nr); zz <= min(nz - 1, z + Nr); ++zz) {
      const double v = in[(size_t)zz * nx + xx];
      if (!isnan(v)) { cs += v; cn += 1.0; }
    }
    s += cs;
    n += cn;
  }
  out[i] = s / n;
}

}  // namespace swd

using namespace swd;

// ====================================================================== engine

struct swd_engine {
  swd_survey sv{};
  swd_engine_opts opt{};
  std::vector<int> sx, sz;
  std::vector<int> shot_no;  // 1-based shot number `is` of each shot in the whole survey
  int ns_total = 0;          // shots in the whole survey
  FdGeom g{};          // store mode geometry (nrec = nt/nt_wf)
  FdGeom gseg{};       // checkpoint mode segment geometry (nrec = ckpt/nt_wf)
  PrepParams pp{};
  RadonGeom rg{};
  int ns = 0, B = 0, nbatch = 0, mode = 1, ckpt = 0, nseg = 0;
  size_t plane = 0, bytes = 0;
  cudaStream_t st = nullptr;
  int device = 0;
  // device memory
  DevBuf model;        // vp, vs (nz*nx each) + vmin
  DevBuf mat;          // packed materials {temp, ca, cl, cm1}
  DevBuf mat2;         // the same per column pair, for the column-pair FD kernels (fd_col2.cuh)
  DevBuf fstate;       // forward state ping-pong [2][B][5][field]
  DevBuf astate;       // adjoint state ping-pong (checkpoint mode)
  DevBuf ckbuf;        // checkpoints [nseg][B][5][field]
  DevBuf snap;         // snapshots [B][nrec][3][plane]
  DevBuf src, wav;     // int2 [ns], float [nt]
  DevBuf seis, res;    // [B][nt][ng] float
  DevBuf img, gsum, dk, dk2;
  DevBuf W, K, gath, D, MM, mlraw, ml, Gx;
  DevBuf cr0, crp, dc, gres, status;
  DevBuf outbuf;       // staging for host outputs
  // WD adjoint source (adjoint_weight 2): geometry, gathers, bin table, pick frequencies, DFT scratch
  WdGeom wg{};
  DevBuf wgath, Ww, wfre, Xw;
  bool have_source = false, have_observed = false;
  double tuned_fwd_us = 0, tuned_adj_us = 0;  // autotune: chosen variants' step times
  swd_contract* tc = nullptr;                  // split-BF16 forward contraction (radon_precision)
  DevBuf cflag, ccount;                        // split-BF16 picks: gathers to recompute in FP64, their count
  std::vector<int> valid_gathers;              // per batch: gathers with a window (picked)
  uint64_t radon_gathers = 0;                  // gathers picked on split-BF16 spectra so far
  std::map<long, cudaGraphExec_t> graphs;
  std::vector<double> h_gres, h_crp;
  // optional per-phase timing of the last call (events on the engine stream)
  bool timing = false;
  std::vector<cudaEvent_t> ev;  // 4 per batch: before forward, after forward, after spectra, after adjoint
  double phase_ms[3] = {0, 0, 0};
  // cancellation of a call in flight: swd_engine_cancel (any host thread) raises cancel_req and
  // copies 1 into the device word cancelw on its own stream, which the FD kernels read
  DevBuf cancelw;
  std::atomic<int> cancel_req{0};
  std::mutex cancel_mu;
  cudaStream_t cst = nullptr;
  int* h_one = nullptr;  // pinned 1, the source of that copy
  ~swd_engine() {
    if (tc) swd_contract_destroy(tc);
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    for (auto x : ev) cudaEventDestroy(x);
    if (cst) cudaStreamSynchronize(cst), cudaStreamDestroy(cst);
    if (h_one) cudaFreeHost(h_one);
    if (st) cudaStreamDestroy(st);
  }
};

namespace swd {

static int plan(swd_engine* e) {
  const FdGeom& g = e->g;
  const size_t field = g.field * sizeof(float);
  const size_t plane = e->plane;
  const RadonGeom& rg = e->rg;
  const size_t tables = (size_t)rg.npair * rg.ntd * 16 + (size_t)rg.npair * rg.offset * rg.np * 16;
  size_t fixed = 2 * e->g.field * sizeof(float4) + 2 * (size_t)e->sv.nz * e->sv.nx * 8 + tables +
                       5 * plane * 8 + (size_t)2 * e->ns * rg.npair * 8 * 3 + (64 << 20);
  const size_t gather = (size_t)rg.npair * rg.offset * 16 * 2 + (size_t)rg.npair * rg.np * (16 + 8 + 8);
  const bool wd = e->opt.adjoint_weight == 2;
  const size_t wd_fixed = wd ? (size_t)e->wg.win * g.nt * 16 + (size_t)e->wg.nfre * 8 + (size_t)2 * e->ns * 32 : 0;
  fixed += wd_fixed;
  const size_t per_common = 2 * 5 * field + 2 * (size_t)g.nt * g.ng * 4 + 3 * plane * 8 + 2 * gather +
                            (wd ? (size_t)2 * e->wg.win * rg.offset * 16 : 0);
  const size_t per_store = per_common + (size_t)g.nrec * 3 * plane * 4;
  size_t budget = e->opt.hbm_budget;
  if (budget == 0) {
    size_t fr = 0, tot = 0;
    SWD_CUDA(cudaMemGetInfo(&fr, &tot));
    budget = (size_t)(fr * 0.92);
  }
  SWD_CHECK(budget > fixed, "HBM budget %zu bytes below the fixed tables (%zu)", budget, fixed);
  const size_t avail = budget - fixed;
  int ck = e->opt.ckpt_interval;
  if (ck <= 0) {
    // memory-optimal interval: a shot holds nt/ck checkpoints of 5 fields and ck/nt_wf
    // snapshot records of 3 planes; their sum is smallest at ck = sqrt(nt * 5 field * nt_wf / (3 plane))
    const double c = std::sqrt((double)g.nt * 5.0 * (double)field * g.nt_wf / (3.0 * (double)plane * 4.0));
    ck = std::max(g.nt_wf, std::min(g.nt, (int)std::lround(c / g.nt_wf) * g.nt_wf));
  }
  ck = std::max(g.nt_wf, ck / g.nt_wf * g.nt_wf);
  const int nseg = (g.nt + ck - 1) / ck;
  const size_t per_ckpt = per_common + 2 * 5 * field + (size_t)nseg * 5 * field + (size_t)(ck / g.nt_wf) * 3 * plane * 4;
  int maxb = e->opt.max_batch > 0 ? std::min(e->opt.max_batch, e->ns) : e->ns;
  const int b_store = (int)std::min<size_t>(maxb, avail / per_store);
  const int b_ckpt = (int)std::min<size_t>(maxb, avail / per_ckpt);
  int mode = e->opt.snapshot_mode;
  if (mode == 0) {
    // store every snapshot when a batch keeps the GPU full; otherwise checkpoint
    const long cells = (long)g.NZ * g.NX;
    const int full = (int)std::max<long>(1, std::min<long>(maxb, (2L << 20) / std::max(1L, cells) + 1));
    mode = (b_store >= std::min(full, maxb)) ? 1 : 2;
  }
  const int b = mode == 1 ? b_store : b_ckpt;
  if (b < 1) {
    set_error("HBM budget too small: %zu bytes available, a shot needs %zu (store) / %zu (checkpoint)", avail,
              per_store, per_ckpt);
    return SWD_ERR_OOM;
  }
  e->mode = mode;
  e->ckpt = ck;
  e->nseg = nseg;
  e->nbatch = (e->ns + b - 1) / b;
  e->B = (e->ns + e->nbatch - 1) / e->nbatch;  // balance the batches
  e->bytes = fixed + (size_t)e->B * (mode == 1 ? per_store : per_ckpt);
  return SWD_OK;
}

static int alloc_all(swd_engine* e) {
  const FdGeom& g = e->g;
  const RadonGeom& rg = e->rg;
  const size_t n = (size_t)e->sv.nz * e->sv.nx, B = e->B, plane = e->plane;
  const size_t fieldB = (size_t)B * 5 * g.field;
  SWD_TRY(e->model.alloc((2 * n + 1) * sizeof(double)));
  SWD_TRY(e->mat.alloc(g.field * sizeof(float4)));
  if (fd_col2_fits(g)) SWD_TRY(e->mat2.alloc(g.field * sizeof(float4)));
  SWD_TRY(e->fstate.alloc(2 * fieldB * sizeof(float)));
  if (e->mode == 2) {
    SWD_TRY(e->astate.alloc(2 * fieldB * sizeof(float)));
    SWD_TRY(e->ckbuf.alloc((size_t)e->nseg * fieldB * sizeof(float)));
    SWD_TRY(e->snap.alloc(B * (size_t)(e->ckpt / g.nt_wf) * 3 * plane * sizeof(float)));
  } else {
    SWD_TRY(e->snap.alloc(B * (size_t)g.nrec * 3 * plane * sizeof(float)));
  }
  SWD_TRY(e->src.alloc(e->ns * sizeof(int2)));
  SWD_TRY(e->wav.alloc(g.nt * sizeof(float)));
  SWD_TRY(e->seis.alloc(B * (size_t)g.nt * g.ng * sizeof(float)));
  SWD_TRY(e->res.alloc(B * (size_t)g.nt * g.ng * sizeof(float)));
  SWD_TRY(e->img.alloc(B * 3 * plane * sizeof(double)));
  SWD_TRY(e->gsum.alloc(3 * plane * sizeof(double)));
  SWD_TRY(e->dk.alloc(plane * sizeof(double)));
  SWD_TRY(e->dk2.alloc(plane * sizeof(double)));
  SWD_TRY(e->outbuf.alloc(4 * plane * sizeof(double)));
  SWD_TRY(e->W.alloc((size_t)rg.npair * rg.ntd * sizeof(double2)));
  SWD_TRY(e->K.alloc((size_t)rg.npair * rg.offset * rg.np * sizeof(double2)));
  // per-gather outputs cover every batch slot, padding gathers of a short last batch included
  const size_t G2 = 2 * B, GA = (size_t)e->nbatch * G2;
  SWD_TRY(e->gath.alloc((size_t)e->nbatch * G2 * sizeof(Gather)));
  SWD_TRY(e->D.alloc(G2 * rg.npair * rg.offset * sizeof(double2)));
  SWD_TRY(e->Gx.alloc(G2 * rg.npair * rg.offset * sizeof(double2)));
  SWD_TRY(e->MM.alloc(G2 * rg.npair * rg.np * sizeof(double2)));
  SWD_TRY(e->mlraw.alloc(G2 * rg.npair * rg.np * sizeof(double)));
  SWD_TRY(e->ml.alloc(G2 * rg.npair * rg.np * sizeof(double)));
  SWD_TRY(e->cr0.alloc(GA * rg.npair * sizeof(double)));
  SWD_TRY(e->crp.alloc(GA * rg.npair * sizeof(double)));
  SWD_TRY(e->dc.alloc(GA * rg.npair * sizeof(double)));
  SWD_TRY(e->gres.alloc(GA * sizeof(double)));
  SWD_TRY(e->status.alloc(GA * sizeof(int)));
  if (e->opt.adjoint_weight == 2) {
    SWD_TRY(e->wgath.alloc((size_t)e->nbatch * G2 * sizeof(Gather)));
    SWD_TRY(e->Ww.alloc((size_t)e->wg.win * g.nt * sizeof(double2)));
    SWD_TRY(e->wfre.alloc((size_t)e->wg.nfre * sizeof(double)));
    SWD_TRY(e->Xw.alloc(G2 * e->wg.win * rg.offset * sizeof(double2)));
  }
  return SWD_OK;
}

// Run (or capture once and replay) a sequence of launches identified by key.
template <typename F>
static int run_seq(swd_engine* e, long key, uint64_t nkernels, F&& body) {
  if (!e->opt.use_graphs) return body();
  auto it = e->graphs.find(key);
  if (it == e->graphs.end()) {
    cudaGraph_t gr;
    SWD_CUDA(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
    const int rc = body();
    const cudaError_t ce = cudaStreamEndCapture(e->st, &gr);
    if (rc != SWD_OK) { if (ce == cudaSuccess) cudaGraphDestroy(gr); return rc; }
    SWD_CUDA(ce);
    cudaGraphExec_t ex;
    const cudaError_t ie = cudaGraphInstantiate(&ex, gr, 0);
    cudaGraphDestroy(gr);
    SWD_CUDA(ie);
    it = e->graphs.emplace(key, ex).first;
  } else {
    count_launch(nkernels);  // the kernels a replay launches
  }
  SWD_CUDA(cudaGraphLaunch(it->second, e->st));
  return SWD_OK;
}

static FwdArgs<float> fwd_args(swd_engine* e, const FdGeom& g, int s0, int nb) {
  FwdArgs<float> a{};
  a.g = g;
  a.mat = g.sched == 3 ? e->mat2.as<float4>() : e->mat.as<float4>();  // pair-interleaved for schedule 3
  a.mb = nullptr;
  a.src = e->src.as<int2>() + s0;
  a.src_type = e->sv.source_type;
  a.s = e->wav.as<float>();
  a.dtx = (float)(e->sv.dt / e->sv.dx);
  a.n_shots = nb;
  a.cancel = e->cancelw.as<int>();
  return a;
}

static AdjArgs<float> adj_args(swd_engine* e, const FdGeom& g, int nb) {
  AdjArgs<float> a{};
  a.g = g;
  a.mat = g.sched == 3 ? e->mat2.as<float4>() : e->mat.as<float4>();
  a.mb = nullptr;
  a.res = e->res.as<float>();
  a.img = e->img.as<double>();
  a.img32 = e->opt.image_precision == 0 ? e->img.as<float>() : nullptr;  // same buffer, half used
  a.dtx = (float)(e->sv.dt / e->sv.dx);
  a.dt = (float)e->sv.dt;
  a.n_shots = nb;
  a.cancel = e->cancelw.as<int>();
  return a;
}

// Steps advanced by the forward launch at step it of [.., t1): two when the schedule pairs
// steps, the pair ends inside the range and does not step over a checkpoint (ckev > 0: the
// state at multiples of ckev is saved).
static int fwd_span(const FdGeom& g, int it, int t1, int ckev) {
  return (fd_pairs(g) && it + 1 < t1 && !(ckev > 0 && (it + 1) % ckev == 0)) ? 2 : 1;
}
static uint64_t fwd_launches(const FdGeom& g, int t0, int t1, int ckev) {
  uint64_t n = 0;
  for (int it = t0; it < t1; it += fwd_span(g, it, t1, ckev)) ++n;
  return n;
}
// Adjoint steps it, it-1, .. down to t0: two per launch when the schedule pairs them.
static int adj_span(const FdGeom& g, int it, int t0) { return (fd_pairs(g) && it - 1 >= t0) ? 2 : 1; }
static uint64_t adj_launches(const FdGeom& g, int hi, int t0) {
  uint64_t n = 0;
  for (int it = hi; it >= t0; it -= adj_span(g, it, t0)) ++n;
  return n;
}

// Forward of one batch: seismograms always; snapshots (store mode) or checkpoints (mode 2).
static int forward_batch(swd_engine* e, int bi, int s0, int nb, bool keep_wavefield) {
  const FdGeom& g = e->g;
  const size_t fieldB = (size_t)e->B * 5 * g.field;
  float* S[2] = {e->fstate.as<float>(), e->fstate.as<float>() + fieldB};
  SWD_CUDA(cudaMemsetAsync(e->fstate.p, 0, 2 * fieldB * sizeof(float), e->st));
  const bool store = keep_wavefield && e->mode == 1;
  const bool ck = keep_wavefield && e->mode == 2;
  const long key = ((long)bi << 8) | (store ? 1 : ck ? 2 : 3);
  const int ckev = ck ? e->ckpt : 0;
  return run_seq(e, key, fwd_launches(g, 0, g.nt, ckev), [&]() -> int {
    FwdArgs<float> a = fwd_args(e, g, s0, nb);
    a.seis_w = e->seis.as<float>();
    a.snap = store ? e->snap.as<float>() : nullptr;
    int c = 0;
    for (int it = 0; it < g.nt;) {
      if (ck && it % e->ckpt == 0)
        SWD_CUDA(cudaMemcpyAsync(e->ckbuf.as<float>() + (size_t)(it / e->ckpt) * fieldB, S[c],
                                 (size_t)nb * 5 * g.field * sizeof(float), cudaMemcpyDeviceToDevice, e->st));
      a.in = S[c];
      a.out = S[c ^ 1];
      const int n = fwd_span(g, it, g.nt, ckev);
      SWD_TRY(n == 2 ? launch_fwd_pair(a, it, e->st) : launch_fwd_step<float, 3>(a, it, e->st));
      c ^= 1;
      it += n;
    }
    SWD_CUDA(cudaGetLastError());
    return SWD_OK;
  });
}

static int adjoint_batch(swd_engine* e, int bi, int s0, int nb) {
  const FdGeom& g = e->g;
  const size_t fieldB = (size_t)e->B * 5 * g.field;
  DevBuf& ab = e->mode == 1 ? e->fstate : e->astate;
  float* A[2] = {ab.as<float>(), ab.as<float>() + fieldB};
  SWD_CUDA(cudaMemsetAsync(ab.p, 0, 2 * fieldB * sizeof(float), e->st));
  SWD_CUDA(cudaMemsetAsync(e->img.p, 0, (size_t)e->B * 3 * e->plane * sizeof(double), e->st));
  int cur = 0;
  if (e->mode == 1) {
    return run_seq(e, ((long)bi << 8) | 4, adj_launches(g, g.nt - 2, 0), [&]() -> int {
      AdjArgs<float> a = adj_args(e, g, nb);
      a.snap = e->snap.as<float>();
      int c = 0;
      for (int it = g.nt - 2; it >= 0;) {
        a.in = A[c];
        a.out = A[c ^ 1];
        const int n = adj_span(g, it, 0);
        SWD_TRY(n == 2 ? launch_adj_pair(a, it, e->st) : launch_adj_step<float, 3>(a, it, e->st));
        c ^= 1;
        it -= n;
      }
      SWD_CUDA(cudaGetLastError());
      return SWD_OK;
    });
  }
  // checkpoint mode: segments last to first; recompute the forward of a segment, then its adjoint
  float* F[2] = {e->fstate.as<float>(), e->fstate.as<float>() + fieldB};
  for (int k = e->nseg - 1; k >= 0; --k) {
    const int t0 = k * e->ckpt, t1 = std::min(t0 + e->ckpt, g.nt);
    const int a_hi = std::min(t1 - 1, g.nt - 2);
    const int nal = a_hi >= t0 ? (int)adj_launches(e->gseg, a_hi, t0) : 0;
    const int cur_in = cur;
    const long key = ((long)bi << 20) | ((long)k << 8) | 5;
    SWD_TRY(run_seq(e, key, fwd_launches(e->gseg, t0, t1, 0) + nal, [&]() -> int {
      SWD_CUDA(cudaMemcpyAsync(F[0], e->ckbuf.as<float>() + (size_t)k * fieldB, (size_t)nb * 5 * g.field * sizeof(float),
                               cudaMemcpyDeviceToDevice, e->st));
      FwdArgs<float> f = fwd_args(e, e->gseg, s0, nb);
      f.snap = e->snap.as<float>();
      f.rec0 = t0 / g.nt_wf;
      int cf = 0;
      for (int it = t0; it < t1;) {
        f.in = F[cf];
        f.out = F[cf ^ 1];
        const int n = fwd_span(e->gseg, it, t1, 0);
        SWD_TRY(n == 2 ? launch_fwd_pair(f, it, e->st) : launch_fwd_step<float, 3>(f, it, e->st));
        cf ^= 1;
        it += n;
      }
      AdjArgs<float> a = adj_args(e, e->gseg, nb);
      a.snap = e->snap.as<float>();
      a.rec0 = t0 / g.nt_wf;
      int c = cur_in;
      for (int it = a_hi; it >= t0;) {
        a.in = A[c];
        a.out = A[c ^ 1];
        const int n = adj_span(e->gseg, it, t0);
        SWD_TRY(n == 2 ? launch_adj_pair(a, it, e->st) : launch_adj_step<float, 3>(a, it, e->st));
        c ^= 1;
        it -= n;
      }
      SWD_CUDA(cudaGetLastError());
      return SWD_OK;
    }));
    cur ^= (nal & 1);
  }
  return SWD_OK;
}

// Autotuner: times the forward and adjoint step kernels of every built CTA shape, ring depth
// and chunk height (the planner's, 2/3 and 3/2 of it) on this engine's own buffers, a batch of
// B shots, and keeps the fastest forward + adjoint pair.  Runs once at create, before any
// graph is captured; the buffers it touches are all overwritten by the first real call.
static int autotune(swd_engine* e) {
  static const int shapes[][2] = {{3, 1}, {2, 1}, {4, 1}, {1, 2}};
  static const int rings[] = {4, 6};
  static const int scheds[] = {0, 1};
  const FdGeom base = e->g;
  FdGeom h = base;
  h.warps = 3; h.cells = 1; h.ring_fwd = h.ring_adj = 4;
  plan_decomposition(h, e->B, 0);
  const int rows = base.NZ - 2;
  std::vector<int> chunks = {h.chunk, std::max(8, h.chunk * 2 / 3), std::min(rows, h.chunk * 3 / 2)};
  std::sort(chunks.begin(), chunks.end());
  chunks.erase(std::unique(chunks.begin(), chunks.end()), chunks.end());
  const int span = (e->mode == 2 ? e->ckpt : base.nt) - 1;  // adjoint steps must index stored snapshots
  const int n = std::max(1, std::min(16, span));
  const int snap_nrec = e->mode == 2 ? e->gseg.nrec : base.nrec;
  const size_t fieldB = (size_t)e->B * 5 * base.field;
  float* S[2] = {e->fstate.as<float>(), e->fstate.as<float>() + fieldB};
  cudaEvent_t t0, t1;
  SWD_CUDA(cudaEventCreate(&t0));
  SWD_CUDA(cudaEventCreate(&t1));
  auto time_steps = [&](const FdGeom& gc, bool fwd, float* ms) -> int {
    FwdArgs<float> f = fwd_args(e, gc, 0, e->B);
    f.seis_w = e->seis.as<float>();
    AdjArgs<float> a = adj_args(e, gc, e->B);
    a.snap = e->snap.as<float>();
    const bool two = fd_pairs(gc) && n >= 2;
    const int n2 = two ? n & ~1 : n;  // steps timed
    for (int i = -2, c = 0; i < n2; i += two ? 2 : 1, c ^= 1) {  // two untimed warm-up launches
      if (i == 0) SWD_CUDA(cudaEventRecord(t0, e->st));
      const int it = std::max(i, 0);
      if (fwd) {
        f.in = S[c];
        f.out = S[c ^ 1];
        SWD_TRY(two ? launch_fwd_pair(f, it, e->st) : launch_fwd_step<float, 3>(f, it, e->st));
      } else {
        a.in = S[c];
        a.out = S[c ^ 1];
        // adjoint pairs run steps it+1 and it (both index stored snapshots: it + 1 <= n <= span)
        SWD_TRY(two ? launch_adj_pair(a, it + 1, e->st) : launch_adj_step<float, 3>(a, it, e->st));
      }
    }
    SWD_CUDA(cudaEventRecord(t1, e->st));
    SWD_CUDA(cudaEventSynchronize(t1));
    SWD_CUDA(cudaEventElapsedTime(ms, t0, t1));
    *ms = *ms * (float)n / (float)n2;  // per n steps, as the other variants
    return SWD_OK;
  };
  double best = 1e30;
  FdGeom pick = base;
  int rc = SWD_OK;
  for (int sc : scheds)
  if (rc == SWD_OK)
  for (const auto& sh : shapes) {
    for (int ch : chunks) {
      double bf = 1e30, ba = 1e30;
      int rf = 4, ra = 4;
      for (int d : rings) {
        if (!fd_variant_built(sh[0], sh[1], d) || (sc == 1 && !fd_lead_built(sh[0], sh[1], d))) continue;
        FdGeom gc = base;
        gc.nrec = snap_nrec;  // records per shot in the snapshot buffer (one segment in checkpoint mode)
        gc.warps = sh[0]; gc.cells = sh[1]; gc.ring_fwd = gc.ring_adj = d; gc.sched = sc;
        plan_decomposition(gc, e->B, ch);
        float mf = 0, ma = 0;
        if ((rc = time_steps(gc, true, &mf)) != SWD_OK) break;
        if ((rc = time_steps(gc, false, &ma)) != SWD_OK) break;
        if (mf < bf) { bf = mf; rf = d; }
        if (ma < ba) { ba = ma; ra = d; }
      }
      if (rc != SWD_OK) break;
      if (bf + ba < best) {
        best = bf + ba;
        pick = base;
        pick.warps = sh[0]; pick.cells = sh[1]; pick.ring_fwd = rf; pick.ring_adj = ra; pick.sched = sc;
        plan_decomposition(pick, e->B, ch);
        e->tuned_fwd_us = bf * 1e3 / n;
        e->tuned_adj_us = ba * 1e3 / n;
      }
    }
    if (rc != SWD_OK) break;
  }
  // warp-streaming schedule (no shared memory): warps per CTA and chunk height
  if (rc == SWD_OK) {
    FdGeom hw = base;
    hw.sched = 2;
    hw.warps = 4;
    plan_decomposition(hw, e->B, 0);
    // two-step launches recompute two rows per chunk, so they also get chunks twice as long
    std::vector<int> wch = {hw.chunk, std::max(8, hw.chunk * 2 / 3), std::min(rows, hw.chunk * 3 / 2),
                            std::min(rows, hw.chunk * 2)};
    std::sort(wch.begin(), wch.end());
    wch.erase(std::unique(wch.begin(), wch.end()), wch.end());
    for (int nw : {4, 2, 8}) {
      for (int ch : wch) {
        double bf = 1e30, ba = 1e30;
        int rf = 4, ra = 4, pf = 0;
        // one or two steps per launch, forward and adjoint alike; 2: two steps, two shots per warp
        for (int pairs : {0, 1, 2}) {
          double pbf = 1e30, pba = 1e30;
          int prf = 4, pra = 4;
          for (int slots : {4, 6, 8}) {
            if (slots == 8 && nw == 8) continue;
            if (pairs == 2 && !fd_warpx_built(nw, slots)) continue;
            FdGeom gc = base;
            gc.nrec = snap_nrec;
            gc.sched = 2;
            gc.pairs = pairs;
            gc.warps = nw;
            gc.ring_fwd = gc.ring_adj = slots;
            plan_decomposition(gc, e->B, ch);
            float mf = 0, ma = 0;
            if ((rc = time_steps(gc, true, &mf)) != SWD_OK) break;
            if ((rc = time_steps(gc, false, &ma)) != SWD_OK) break;
            if (mf < pbf) { pbf = mf; prf = slots; }
            if (ma < pba) { pba = ma; pra = slots; }
          }
          if (rc != SWD_OK) break;
          if (pbf + pba < bf + ba) { bf = pbf; ba = pba; rf = prf; ra = pra; pf = pairs; }
        }
        if (rc != SWD_OK) break;
        if (bf + ba < best) {
          best = bf + ba;
          pick = base;
          pick.sched = 2;
          pick.pairs = pf;
          pick.warps = nw;
          pick.ring_fwd = rf;
          pick.ring_adj = ra;
          plan_decomposition(pick, e->B, ch);
          e->tuned_fwd_us = bf * 1e3 / n;
          e->tuned_adj_us = ba * 1e3 / n;
        }
      }
      if (rc != SWD_OK) break;
    }
  }
  // column pairs (two steps per launch): warps per CTA, row slots and chunk height
  if (rc == SWD_OK && fd_col2_fits(base) && e->mat2.p) {
    FdGeom hc = base;
    hc.sched = 3;
    hc.warps = 4;
    plan_decomposition(hc, e->B, 0);
    std::vector<int> cch = {hc.chunk, std::max(8, hc.chunk * 2 / 3), std::min(rows, hc.chunk * 3 / 2),
                            std::min(rows, hc.chunk * 2)};
    std::sort(cch.begin(), cch.end());
    cch.erase(std::unique(cch.begin(), cch.end()), cch.end());
    for (int nw : {4, 2, 8}) {
      for (int ch : cch) {
        double bf = 1e30, ba = 1e30;
        int rf = 4, ra = 4;
        for (int slots : {4, 6}) {
          if (!fd_col2_built(nw, slots)) continue;
          FdGeom gc = base;
          gc.nrec = snap_nrec;
          gc.sched = 3;
          gc.warps = nw;
          gc.ring_fwd = gc.ring_adj = slots;
          plan_decomposition(gc, e->B, ch);
          float mf = 0, ma = 0;
          if ((rc = time_steps(gc, true, &mf)) != SWD_OK) break;
          if ((rc = time_steps(gc, false, &ma)) != SWD_OK) break;
          if (mf < bf) { bf = mf; rf = slots; }
          if (ma < ba) { ba = ma; ra = slots; }
        }
        if (rc != SWD_OK) break;
        if (bf + ba < best) {
          best = bf + ba;
          pick = base;
          pick.sched = 3;
          pick.warps = nw;
          pick.ring_fwd = rf;
          pick.ring_adj = ra;
          plan_decomposition(pick, e->B, ch);
          e->tuned_fwd_us = bf * 1e3 / n;
          e->tuned_adj_us = ba * 1e3 / n;
        }
      }
      if (rc != SWD_OK) break;
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (rc != SWD_OK) return rc;
  e->g = pick;
  const int nrec = e->gseg.nrec;
  e->gseg = pick;
  e->gseg.nrec = nrec;
  return SWD_OK;
}

// Spectra, picks, misfits (+ adjoint sources when `grad`) for the gathers of one batch.
// A split-BF16 spectrum column (normalised to 1) is within ~1e-5 of the FP64 one (measured:
// 3.4e-6 relative L2 over the 100 x 600 survey's spectra); a pick decision whose two compared
// values differ by more than ten times that cannot flip, so only gathers with a closer decision
// are recomputed in FP64.
constexpr double kBf16PickMargin = 1e-4;

static int spectrum_batch(swd_engine* e, int bi, int s0, int nb, bool grad) {
  const RadonGeom& rg = e->rg;
  const int G = 2 * e->B;
  const Gather* gs = e->gath.as<Gather>() + (size_t)bi * G;
  const size_t sstride = (size_t)e->g.nt * e->g.ng;
  if (e->tc) {  // offsets beyond a gather's window must be zero for the padded tensor-core tiles
    SWD_CUDA(cudaMemsetAsync(e->D.p, 0, (size_t)G * rg.npair * rg.offset * sizeof(double2), e->st));
  }
  SWD_TRY(radon_dft<float>(rg, gs, G, e->seis.as<float>(), sstride, e->W.as<double2>(), e->D.as<double2>(), e->st));
  const size_t go = (size_t)2 * s0;
  auto pick = [&](PickSeed ps) {
    return pick_batch(rg.np, rg.npair, G, e->sv.ini, e->sv.pick_method, e->sv.vmin, gs, e->ml.as<double>(),
                      e->cr0.as<double>() + go * rg.npair, e->crp.as<double>() + go * rg.npair,
                      e->dc.as<double>() + go * rg.npair, e->gres.as<double>() + go, e->status.as<int>() + go, e->st,
                      ps);
  };
  if (e->tc) {
    // split-BF16 spectra on the tensor cores; the picker certifies each gather's decisions and
    // the gathers with a decision inside kBf16PickMargin are recomputed in FP64 and picked again,
    // so that the picks are the FP64 picks
    SWD_TRY(swd_contract_run(e->tc, e->D.as<double>(), e->MM.as<double>(), e->st));
    SWD_TRY(radon_amplitudes(rg, gs, G, e->MM.as<double2>(), e->mlraw.as<double>(), e->ml.as<double>(), e->st));
    SWD_CUDA(cudaMemsetAsync(e->cflag.p, 0, G * sizeof(int), e->st));
    PickSeed cert;
    cert.cert = e->cflag.as<int>();
    cert.delta = kBf16PickMargin;
    cert.cert_count = e->ccount.as<unsigned long long>();
    SWD_TRY(pick(cert));
    SWD_TRY(radon_contract(rg, gs, G, e->K.as<double2>(), e->D.as<double2>(), e->MM.as<double2>(),
                           e->mlraw.as<double>(), e->ml.as<double>(), e->st, e->cflag.as<int>()));
    PickSeed again;
    again.only = e->cflag.as<int>();
    SWD_TRY(pick(again));
    e->radon_gathers += (uint64_t)e->valid_gathers[bi];
  } else {
    SWD_TRY(radon_contract(rg, gs, G, e->K.as<double2>(), e->D.as<double2>(), e->MM.as<double2>(),
                           e->mlraw.as<double>(), e->ml.as<double>(), e->st));
    SWD_TRY(pick(PickSeed{}));
  }
  if (!grad) return SWD_OK;
  if (e->opt.adjoint_weight == 2) {  // WD residual of the predicted data (SWD.m:188, F1 = 0)
    SWD_CUDA(cudaMemsetAsync(e->res.p, 0, (size_t)e->B * sstride * sizeof(float), e->st));
    const Gather* wgs = e->wgath.as<Gather>() + (size_t)bi * G;
    return wd_adjoint<float, float>(e->wg, wgs, G, e->seis.as<float>(), sstride, e->Ww.as<double2>(),
                                    e->wfre.as<double>(), e->cr0.as<double>() + go * rg.npair,
                                    e->crp.as<double>() + go * rg.npair, e->Xw.as<double2>(), e->res.as<float>(),
                                    sstride, e->st);
  }
  const bool gauss = e->opt.adjoint_weight == 1;  // ADWDgrad_norm: Gaussian around the picks
  SWD_TRY(softmax_adjoint(rg, gs, G, e->mlraw.as<double>(), e->MM.as<double2>(), e->dc.as<double>() + go * rg.npair,
                          nullptr, e->sv.soft_arg_norm, e->K.as<double2>(), e->Gx.as<double2>(), e->st,
                          gauss ? e->crp.as<double>() + go * rg.npair : nullptr, e->sv.vmin));
  SWD_CUDA(cudaMemsetAsync(e->res.p, 0, (size_t)e->B * sstride * sizeof(float), e->st));
  SWD_TRY(radon_idft_scatter<float>(rg, gs, G, e->Gx.as<double2>(), e->W.as<double2>(), e->res.as<float>(), sstride,
                                    e->st));
  return SWD_OK;
}

static int load_model(swd_engine* e, const double* vp, const double* vs, bool device_ptrs) {
  const size_t n = (size_t)e->sv.nz * e->sv.nx;
  double* d = e->model.as<double>();
  const cudaMemcpyKind kind = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  SWD_CUDA(cudaMemcpyAsync(d, vp, n * sizeof(double), kind, e->st));
  SWD_CUDA(cudaMemcpyAsync(d + n, vs, n * sizeof(double), kind, e->st));
  SWD_TRY(vmin_device(d, d + n, n, d + 2 * n, e->st));
  SWD_TRY(prep_packed<float>(e->pp, d, d + n, d + 2 * n, e->mat.as<float4>(), e->g.pitch, e->st));
  if (e->mat2.p) SWD_TRY(col2_material_pairs(e->mat.as<float4>(), e->mat2.as<float4>(), e->g.NZ, e->g.pitch, e->st));
  return SWD_OK;
}

// A cancel raised during (or before) this call: wait for its copy, clear the device word for the
// next call, and report the call as cancelled (its results are partial and are not returned).
static int take_cancel(swd_engine* e) {
  if (!e->cancel_req.load()) return SWD_OK;
  std::lock_guard<std::mutex> lk(e->cancel_mu);
  SWD_CUDA(cudaStreamSynchronize(e->cst));
  SWD_CUDA(cudaMemsetAsync(e->cancelw.p, 0, sizeof(int), e->st));
  SWD_CUDA(cudaStreamSynchronize(e->st));
  e->cancel_req.store(0);
  set_error("the call was cancelled (swd_engine_cancel)");
  return SWD_ERR_CANCELLED;
}

static int check_status(swd_engine* e) {
  SWD_TRY(take_cancel(e));  // a cancelled call's picks are meaningless: report the cancel first
  std::vector<int> stv(2 * e->ns);
  SWD_CUDA(cudaMemcpyAsync(stv.data(), e->status.p, stv.size() * sizeof(int), cudaMemcpyDeviceToHost, e->st));
  SWD_CUDA(cudaStreamSynchronize(e->st));
  for (size_t i = 0; i < stv.size(); ++i)
    if (stv[i]) {
      set_error("shot %d %s side: %s", e->shot_no[i / 2], (i & 1) ? "left" : "right",
                stv[i] == 1 ? "NaN in the dispersion spectrum" : "interp1 needs at least two retained picks");
      return SWD_ERR_NUMERIC;
    }
  return SWD_OK;
}

static int assemble(swd_engine* e, const double* d_gsum) {
  const int nn = e->sv.nz * e->sv.nx;
  const double* d_vs = e->model.as<double>() + nn;
  assemble_kernel<<<(nn + 255) / 256, 256, 0, e->st>>>(e->sv.nz, e->sv.nx, d_vs, d_gsum, e->dk.as<double>());
  smooth2a_kernel<<<(nn + 255) / 256, 256, 0, e->st>>>(e->sv.nz, e->sv.nx, e->sv.smooth_z, e->sv.smooth_x,
                                                       e->dk.as<double>(), e->dk2.as<double>());
  count_launch(2);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}

static int mark(swd_engine* e, int bi, int k) {
  if (e->timing) SWD_CUDA(cudaEventRecord(e->ev[4 * bi + k], e->st));
  return SWD_OK;
}

// Forward (+ adjoint and shot sums when grad) of every batch; grad && finish also assembles dk_vs.
static int run(swd_engine* e, const double* vp, const double* vs, bool device_ptrs, bool grad, bool finish = true) {
  SWD_CHECK(e->have_source, "swd_engine_set_source was not called");
  SWD_CUDA(cudaSetDevice(e->device));
  SWD_TRY(load_model(e, vp, vs, device_ptrs));
  if (grad) SWD_CUDA(cudaMemsetAsync(e->gsum.p, 0, 3 * e->plane * sizeof(double), e->st));
  for (int bi = 0; bi < e->nbatch; ++bi) {
    const int s0 = bi * e->B, nb = std::min(e->B, e->ns - s0);
    SWD_TRY(mark(e, bi, 0));
    SWD_TRY(forward_batch(e, bi, s0, nb, grad));
    SWD_TRY(mark(e, bi, 1));
    SWD_TRY(spectrum_batch(e, bi, s0, nb, grad));
    SWD_TRY(mark(e, bi, 2));
    if (!grad) { SWD_TRY(mark(e, bi, 3)); continue; }
    SWD_TRY(adjoint_batch(e, bi, s0, nb));
    const size_t n3 = 3 * e->plane;
    if (e->opt.image_precision == 0)
      shot_sum_kernel<float><<<(unsigned)((n3 + 255) / 256), 256, 0, e->st>>>(e->img.as<float>(), nb, e->plane,
                                                                              e->gsum.as<double>());
    else
      shot_sum_kernel<double><<<(unsigned)((n3 + 255) / 256), 256, 0, e->st>>>(e->img.as<double>(), nb, e->plane,
                                                                               e->gsum.as<double>());
    count_launch(1);
    SWD_CUDA(cudaGetLastError());
    SWD_TRY(mark(e, bi, 3));
  }
  if (grad && finish) SWD_TRY(assemble(e, e->gsum.as<double>()));
  SWD_TRY(check_status(e));
  if (e->timing) {
    for (double& x : e->phase_ms) x = 0;
    for (int bi = 0; bi < e->nbatch; ++bi)
      for (int k = 0; k < 3; ++k) {
        float ms = 0;
        SWD_CUDA(cudaEventElapsedTime(&ms, e->ev[4 * bi + k], e->ev[4 * bi + k + 1]));
        e->phase_ms[k] += ms;
      }
  }
  return SWD_OK;
}

// per-shot outputs from the per-gather device arrays (MATLAB npair x ns layouts)
static int copy_picks(swd_engine* e, double* res_r, double* res_l, double* crp_r, double* crp_l, double* residual) {
  const int GA = 2 * e->ns, np2 = e->rg.npair;
  e->h_gres.resize(GA);
  e->h_crp.resize((size_t)GA * np2);
  SWD_CUDA(cudaMemcpyAsync(e->h_gres.data(), e->gres.p, GA * sizeof(double), cudaMemcpyDeviceToHost, e->st));
  SWD_CUDA(cudaMemcpyAsync(e->h_crp.data(), e->crp.p, (size_t)GA * np2 * sizeof(double), cudaMemcpyDeviceToHost, e->st));
  SWD_CUDA(cudaStreamSynchronize(e->st));
  double sum = 0.0;
  int cnt = 0;
  for (int s = 0; s < e->ns; ++s) {
    const bool r_on = side_active(e->shot_no[s], 0, e->ns_total, e->sv.m, e->sv.M, e->sv.w);
    const bool l_on = side_active(e->shot_no[s], 1, e->ns_total, e->sv.m, e->sv.M, e->sv.w);
    if (res_r) res_r[s] = r_on ? e->h_gres[2 * s] : NAN;
    if (res_l) res_l[s] = l_on ? e->h_gres[2 * s + 1] : NAN;
    for (int f = 0; f < np2; ++f) {  // cr_pre defaults to 1 where a side is skipped (SWD.m:164-165)
      if (crp_r) crp_r[(size_t)s * np2 + f] = r_on ? e->h_crp[(size_t)(2 * s) * np2 + f] : 1.0;
      if (crp_l) crp_l[(size_t)s * np2 + f] = l_on ? e->h_crp[(size_t)(2 * s + 1) * np2 + f] : 1.0;
    }
    if (r_on) { sum += e->h_gres[2 * s]; ++cnt; }
  }
  if (residual) *residual = cnt ? sum / cnt : NAN;  // SWD.m:196 mean(res_r)
  return SWD_OK;
}

static int copy_plane(swd_engine* e, const double* d_rowmajor, double* h_colmajor) {
  if (!h_colmajor) return SWD_OK;
  double* t = e->outbuf.as<double>();
  SWD_TRY(transpose<double, double>(d_rowmajor, 0, t, 0, 1, e->sv.nz, e->sv.nx, e->st));
  SWD_CUDA(cudaMemcpyAsync(h_colmajor, t, e->plane * sizeof(double), cudaMemcpyDeviceToHost, e->st));
  SWD_CUDA(cudaStreamSynchronize(e->st));
  return SWD_OK;
}

// Validation, geometry and the memory plan of an engine (no device allocation).
static int engine_setup(const swd_survey* s, const swd_engine_opts* o, swd_engine* e) {
  SWD_CHECK(s->ns >= 1 && s->sx && s->sz, "need ns >= 1 shots with sx/sz");
  SWD_CHECK(s->ng >= 2 && s->dgx >= 1, "need ng >= 2 receivers with spacing dgx >= 1");
  SWD_CHECK(s->source_type >= 1 && s->source_type <= 5, "source_type must be 1..5");
  e->sv = *s;
  if (o) e->opt = *o; else e->opt.use_graphs = 1;
  e->ns = s->ns;
  e->sx.assign(s->sx, s->sx + s->ns);
  e->sz.assign(s->sz, s->sz + s->ns);
  e->ns_total = s->ns_total > 0 ? s->ns_total : s->ns;
  SWD_CHECK(e->ns_total >= e->ns, "ns_total (%d) below ns (%d)", e->ns_total, e->ns);
  e->shot_no.resize(e->ns);
  for (int i = 0; i < e->ns; ++i) {
    e->shot_no[i] = s->shot_no ? s->shot_no[i] : i + 1;
    SWD_CHECK(e->shot_no[i] >= 1 && e->shot_no[i] <= e->ns_total, "shot_no[%d] = %d outside 1..%d", i,
              e->shot_no[i], e->ns_total);
  }
  e->sv.sx = nullptr;
  e->sv.sz = nullptr;
  e->sv.shot_no = nullptr;
  // option ranges: checked before the first CUDA call, so that they are reported on any host
  SWD_CHECK(e->opt.fd_schedule >= 0 && e->opt.fd_schedule <= 6, "fd_schedule must lie in 0..6 (got %d)",
            e->opt.fd_schedule);
  SWD_CHECK(e->opt.image_precision == 0 || e->opt.image_precision == 1, "image_precision must be 0 (FP32) or 1 (FP64)");
  SWD_CHECK(e->opt.adjoint_weight >= 0 && e->opt.adjoint_weight <= 2,
            "adjoint_weight must be 0 (ADWDgrad_1), 1 (ADWDgrad_norm) or 2 (weight_data_muti3)");
  e->device = e->opt.device;
  SWD_CUDA(cudaSetDevice(e->device));
  // model prep / FD geometry
  PrepParams& pp = e->pp;
  pp.nz = s->nz; pp.nx = s->nx; pp.nbc = s->nbc; pp.isfs = s->isfs; pp.fd_order = s->fd_order;
  pp.dx = s->dx; pp.dt = s->dt; pp.dtx = s->dt / s->dx;
  SWD_TRY(prep_check(pp));
  prep_fill(pp);
  SWD_CHECK(s->nt >= 2 && s->nt_wf >= 1 && s->nt % s->nt_wf == 0, "nt (%d) must be a multiple of nt_wf (%d)", s->nt,
            s->nt_wf);
  FdGeom& g = e->g;
  g.NZ = pp.NZ; g.NX = pp.NX; g.pitch = round_up(pp.NX, 32);
  g.nz = s->nz; g.nx = s->nx; g.nbc = s->nbc; g.pad_top = 1;
  g.nt = s->nt; g.nt_wf = s->nt_wf; g.nrec = s->nt / s->nt_wf;
  g.ng = s->ng; g.gz = s->gz + pp.pad_top - 1; g.gx = s->gx0 + s->nbc - 1; g.dg = s->dgx;
  g.field = (size_t)g.NZ * g.pitch;
  SWD_CHECK(g.gz >= 1 && g.gz <= g.NZ - 2 && g.gx >= 1 && g.gx + (long)(g.ng - 1) * g.dg <= g.NX - 2,
            "receivers must lie inside the padded grid's rows/cols 1..n-2");
  for (int i = 0; i < e->ns; ++i) {
    const int z = e->sz[i] + pp.pad_top - 1, x = e->sx[i] + s->nbc - 1;
    const int zlo = s->source_type == 2 ? 2 : 1, xhi = s->source_type == 2 ? g.NX - 3 : g.NX - 2;
    SWD_CHECK(z >= zlo && z <= g.NZ - 2 && x >= 1 && x <= xhi, "shot %d source (%d,%d) outside the grid interior",
              i + 1, e->sz[i], e->sx[i]);
  }
  e->plane = (size_t)g.nz * g.nx;
  // the warp-streaming kernels index a shot's fields and images with 32-bit offsets
  SWD_CHECK(5.0 * (double)g.field < 2147483647.0 && 3.0 * (double)e->plane < 2147483647.0,
            "grid too large: 5 * nzbc * pitch and 3 * nz * nx must stay below 2^31");
  g.warps = e->opt.warps;
  g.cells = e->opt.cells;
  g.ring_fwd = e->opt.ring_fwd;
  g.ring_adj = e->opt.ring_adj;
  // fd_schedule: 0 (default) and 3 warp streaming with two steps per launch, 1 one barrier per
  // row, 2 warp streaming one step per launch, 4 two barriers per row, 5 as 3 with two shots
  // per warp in packed FP32 pairs, 6 as 3 with two columns per lane in packed FP32 pairs
  const int fs = e->opt.fd_schedule;
  g.sched = fs == 1 ? 1 : fs == 4 ? 0 : fs == 6 ? 3 : 2;
  g.pairs = (fs == 0 || fs == 3) ? 1 : fs == 5 ? 2 : 0;
  SWD_CHECK(fs != 6 || fd_col2_fits(g), "fd_schedule 6 (column pairs) needs even nbc and nx (got nbc %d, nx %d)",
            g.nbc, g.nx);
  plan_decomposition(g, std::max(1, std::min(e->opt.max_batch > 0 ? e->opt.max_batch : e->ns, e->ns)),
                     e->opt.chunk_rows);
  // Radon geometry
  swd_radon_params rp{};
  rp.df = s->df; rp.dt = s->dt; rp.fmin = s->fmin; rp.fmax = s->fmax; rp.vmin = s->vmin; rp.vmax = s->vmax;
  rp.dv = s->dv > 0 ? s->dv : 1.0; rp.ds = s->dgx * s->dx; rp.nt = s->nt; rp.ng = s->ng;
  rp.offset = s->offset; rp.m = s->m; rp.M = s->M;
  SWD_TRY(radon_geom(&rp, e->rg));
  SWD_CHECK(e->rg.ccn >= s->nt, "ADWDgrad_1 needs ccn = fix(1/df/dt) (%d) >= nt (%d)", e->rg.ccn, s->nt);
  SWD_CHECK(s->ini >= 1 && s->ini <= e->rg.npair, "ini (%d) must lie in 1..npair (%d)", s->ini, e->rg.npair);
  if (e->opt.adjoint_weight == 2) {
    // SWD.m:124-127: ind = fmin/df+1, npair = length(fmin:df:fmax), win = npair+2*ind
    const double ind = s->fmin / s->df + 1;
    SWD_CHECK(ind == std::floor(ind) && ind >= 1 && ind < 1e7, "the WD residual needs fmin/df+1 (%g) to be an integer",
              ind);
    const int win = e->rg.npair + 2 * (int)ind;
    SWD_TRY(wd_geom(s->nt, s->ng, s->dt, s->df, s->offset, s->m, win, (int)ind, s->fmin, s->fmax, s->dgx * s->dx, 0,
                    e->wg));
    SWD_CHECK(e->wg.nfre == e->rg.npair, "linspace(fmin,fmax,(fmax-fmin)/df+1) has %d points, the picks %d",
              e->wg.nfre, e->rg.npair);
    e->wg.npair = e->rg.npair;
  }
  SWD_TRY(plan(e));
  plan_decomposition(g, e->B, e->opt.chunk_rows);
  e->gseg = g;
  e->gseg.nrec = e->ckpt / g.nt_wf;
  return SWD_OK;
}

static int engine_create(const swd_survey* s, const swd_engine_opts* o, swd_engine** out) {
  clear_error();
  SWD_CHECK(s && out, "null argument");
  *out = nullptr;
  auto e = new swd_engine();
  std::unique_ptr<swd_engine> guard(e);
  SWD_TRY(engine_setup(s, o, e));
  std::vector<int2> hsrc(e->ns);
  for (int i = 0; i < e->ns; ++i)
    hsrc[i] = make_int2(e->sz[i] + e->pp.pad_top - 1, e->sx[i] + s->nbc - 1);
  SWD_CUDA(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
  SWD_CUDA(cudaStreamCreateWithFlags(&e->cst, cudaStreamNonBlocking));
  SWD_CUDA(cudaHostAlloc((void**)&e->h_one, sizeof(int), cudaHostAllocDefault));
  *e->h_one = 1;
  SWD_TRY(alloc_all(e));
  SWD_TRY(e->cancelw.alloc(sizeof(int)));
  SWD_CUDA(cudaMemsetAsync(e->cancelw.p, 0, sizeof(int), e->st));
  SWD_CUDA(cudaMemcpyAsync(e->src.p, hsrc.data(), e->ns * sizeof(int2), cudaMemcpyHostToDevice, e->st));
  // gathers per batch (local shot index), validated against the reference's window rules
  std::vector<Gather> hg((size_t)e->nbatch * 2 * e->B);
  for (int bi = 0; bi < e->nbatch; ++bi)
    for (int b = 0; b < e->B; ++b) {
      const int sidx = bi * e->B + b;
      for (int side = 0; side < 2; ++side) {
        Gather gg{};
        if (sidx < e->ns) {
          gg = make_gather(e->rg, e->shot_no[sidx], side, b, e->ns_total, s->w);
          SWD_CHECK(gg.valid >= 0, "shot %d: the %s window is empty or leaves the receiver line",
                    e->shot_no[sidx], side ? "left" : "right");
        }
        hg[((size_t)bi * e->B + b) * 2 + side] = gg;
      }
    }
  SWD_CUDA(cudaMemcpyAsync(e->gath.p, hg.data(), hg.size() * sizeof(Gather), cudaMemcpyHostToDevice, e->st));
  e->valid_gathers.assign(e->nbatch, 0);
  for (size_t i = 0; i < hg.size(); ++i) e->valid_gathers[i / (2 * (size_t)e->B)] += hg[i].valid > 0 ? 1 : 0;
  SWD_TRY(radon_tables(e->rg, e->W.as<double2>(), e->K.as<double2>(), e->st));
  std::vector<Gather> hw;
  std::vector<double> hfre;
  if (e->opt.adjoint_weight == 2) {  // WD gathers: refsx = floor(sx/dg)+1 (SWD.m:96)
    hw.resize(hg.size());
    for (int bi = 0; bi < e->nbatch; ++bi)
      for (int b = 0; b < e->B; ++b) {
        const int sidx = bi * e->B + b;
        for (int side = 0; side < 2; ++side) {
          Gather gg{};
          if (sidx < e->ns) {
            const int refsx = (int)std::floor((double)e->sx[sidx] / s->dgx) + 1;
            gg = make_wd_gather(e->wg, e->shot_no[sidx], side, b, e->ns_total, s->w, (double)s->M, refsx);
            SWD_CHECK(gg.valid >= 0, "shot %d: the %s WD window is empty or leaves the receiver line",
                      e->shot_no[sidx], side ? "left" : "right");
          }
          hw[((size_t)bi * e->B + b) * 2 + side] = gg;
        }
      }
    hfre.resize(e->wg.nfre);
    wd_fre(s->fmin, s->fmax, e->wg.nfre, hfre.data());
    SWD_CUDA(cudaMemcpyAsync(e->wgath.p, hw.data(), hw.size() * sizeof(Gather), cudaMemcpyHostToDevice, e->st));
    SWD_CUDA(cudaMemcpyAsync(e->wfre.p, hfre.data(), hfre.size() * sizeof(double), cudaMemcpyHostToDevice, e->st));
    SWD_TRY(radon_tables(e->wg.dft, e->Ww.as<double2>(), nullptr, e->st));
  }
  if (e->opt.autotune) SWD_TRY(autotune(e));
  if (e->opt.radon_precision == SWD_PREC_BF16X2 || e->opt.radon_precision == SWD_PREC_BF16X3) {
    // the engine's axes: kept bins lf..nf, velocities vmin + dv*p, offsets (m + x)*ds (RTrAD.m:11,18-21)
    const RadonGeom& rg = e->rg;
    std::vector<double> fr(rg.npair), vel(rg.np), off(rg.offset);
    for (int f = 0; f < rg.npair; ++f) fr[f] = rg.df * (rg.lf - 1 + f);
    for (int p = 0; p < rg.np; ++p) vel[p] = rg.vmin + rg.dv * p;
    for (int x = 0; x < rg.offset; ++x) off[x] = (rg.m + x) * rg.ds;
    SWD_TRY(swd_contract_create(rg.npair, fr.data(), rg.np, vel.data(), rg.offset, off.data(), 2 * e->B,
                                e->opt.radon_precision, e->device, &e->tc));
    SWD_TRY(e->cflag.alloc(2 * (size_t)e->B * sizeof(int)));
    SWD_TRY(e->ccount.alloc(sizeof(unsigned long long)));
    SWD_CUDA(cudaMemsetAsync(e->ccount.p, 0, sizeof(unsigned long long), e->st));
  } else {
    SWD_CHECK(e->opt.radon_precision == SWD_PREC_FP64, "radon_precision must be SWD_PREC_FP64, _BF16X2 or _BF16X3");
  }
  // default observed curves: ones (SWD.m:153-154)
  std::vector<double> ones((size_t)e->nbatch * 2 * e->B * e->rg.npair, 1.0);
  SWD_CUDA(cudaMemcpyAsync(e->cr0.p, ones.data(), ones.size() * sizeof(double), cudaMemcpyHostToDevice, e->st));
  SWD_CUDA(cudaStreamSynchronize(e->st));
  *out = guard.release();
  return SWD_OK;
}

}  // namespace swd

extern "C" {

int swd_engine_create(const swd_survey* s, const swd_engine_opts* o, swd_engine** out) {
  return engine_create(s, o, out);
}

int swd_engine_destroy(swd_engine* e) {
  delete e;
  return SWD_OK;
}

static void fill_info(const swd_engine* e, swd_engine_info_t* info) {
  info->batch = e->B;
  info->nbatch = e->nbatch;
  info->mode = e->mode;
  info->ckpt_interval = e->ckpt;
  info->bytes = e->bytes;
  info->npair = e->rg.npair;
  info->np = e->rg.np;
  info->ccn = e->rg.ccn;
  info->nzbc = e->g.NZ;
  info->nxbc = e->g.NX;
  info->chunk_rows = e->g.chunk;
  info->warps = e->g.warps;
  info->cells = e->g.cells;
  info->ring_fwd = e->g.ring_fwd;
  info->ring_adj = e->g.ring_adj;
  info->tuned_fwd_us = e->tuned_fwd_us;
  info->tuned_adj_us = e->tuned_adj_us;
  info->fd_schedule = e->g.sched == 3 ? 6 : fd_pairs(e->g) ? (e->g.pairs == 2 ? 5 : 3) : e->g.sched == 0 ? 4 : e->g.sched;
}

int swd_engine_info(const swd_engine* e, swd_engine_info_t* info) {
  clear_error();
  SWD_CHECK(e && info, "null argument");
  fill_info(e, info);
  return SWD_OK;
}

int swd_engine_plan(const swd_survey* s, const swd_engine_opts* o, swd_engine_info_t* info) {
  clear_error();
  SWD_CHECK(s && info, "null argument");
  swd_engine e;
  SWD_TRY(engine_setup(s, o, &e));
  fill_info(&e, info);
  return SWD_OK;
}

int swd_engine_set_source(swd_engine* e, const double* s) {
  clear_error();
  SWD_CHECK(e && s, "null argument");
  std::vector<float> h(e->g.nt);
  for (int i = 0; i < e->g.nt; ++i) h[i] = (float)s[i];  // single(s) (SWD_single.m:92)
  SWD_CUDA(cudaMemcpyAsync(e->wav.p, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, e->st));
  SWD_CUDA(cudaStreamSynchronize(e->st));
  e->have_source = true;
  return SWD_OK;
}

int swd_engine_set_observed(swd_engine* e, const double* cr0_r, const double* cr0_l) {
  clear_error();
  SWD_CHECK(e && cr0_r && cr0_l, "null argument");
  const int np2 = e->rg.npair;
  std::vector<double> h((size_t)2 * e->ns * np2);
  for (int s = 0; s < e->ns; ++s)
    for (int f = 0; f < np2; ++f) {
      h[(size_t)(2 * s) * np2 + f] = cr0_r[(size_t)s * np2 + f];
      h[(size_t)(2 * s + 1) * np2 + f] = cr0_l[(size_t)s * np2 + f];
    }
  SWD_CUDA(cudaMemcpyAsync(e->cr0.p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, e->st));
  SWD_CUDA(cudaStreamSynchronize(e->st));
  e->have_observed = true;
  return SWD_OK;
}

int swd_engine_misfit(swd_engine* e, const double* vp, const double* vs, double* res_r, double* res_l,
                      double* cr_pre_r, double* cr_pre_l, double* residual) {
  clear_error();
  SWD_CHECK(e && vp && vs, "null argument");
  SWD_TRY(run(e, vp, vs, false, false));
  return copy_picks(e, res_r, res_l, cr_pre_r, cr_pre_l, residual);
}

int swd_engine_observed_curves(swd_engine* e, const double* vp, const double* vs, double* cr0_r, double* cr0_l) {
  clear_error();
  SWD_CHECK(e && vp && vs && cr0_r && cr0_l, "null argument");
  SWD_TRY(run(e, vp, vs, false, false));
  SWD_TRY(copy_picks(e, nullptr, nullptr, cr0_r, cr0_l, nullptr));
  return SWD_OK;
}

int swd_engine_gradient(swd_engine* e, const double* vp, const double* vs, swd_gradient_out* out) {
  clear_error();
  SWD_CHECK(e && vp && vs && out, "null argument");
  SWD_TRY(run(e, vp, vs, false, true));
  const size_t P = e->plane;
  SWD_TRY(copy_plane(e, e->gsum.as<double>(), out->g_cl));
  SWD_TRY(copy_plane(e, e->gsum.as<double>() + P, out->g_cm));
  SWD_TRY(copy_plane(e, e->gsum.as<double>() + 2 * P, out->g_illum));
  SWD_TRY(copy_plane(e, e->dk2.as<double>(), out->dk_vs));
  return copy_picks(e, out->res_r, out->res_l, out->cr_pre_r, out->cr_pre_l, &out->residual);
}

int swd_engine_gradient_device(swd_engine* e, const double* d_vp, const double* d_vs, double* d_dk_vs,
                               double* residual) {
  clear_error();
  SWD_CHECK(e && d_vp && d_vs, "null argument");
  SWD_TRY(run(e, d_vp, d_vs, true, true));
  if (d_dk_vs) {
    SWD_TRY(transpose<double, double>(e->dk2.as<double>(), 0, d_dk_vs, 0, 1, e->sv.nz, e->sv.nx, e->st));
    SWD_CUDA(cudaStreamSynchronize(e->st));
  }
  if (residual) SWD_TRY(copy_picks(e, nullptr, nullptr, nullptr, nullptr, residual));
  return SWD_OK;
}

int swd_engine_cancel(swd_engine* e) {
  clear_error();
  SWD_CHECK(e, "null engine");
  std::lock_guard<std::mutex> lk(e->cancel_mu);
  SWD_CUDA(cudaSetDevice(e->device));
  e->cancel_req.store(1);
  SWD_CUDA(cudaMemcpyAsync(e->cancelw.p, e->h_one, sizeof(int), cudaMemcpyHostToDevice, e->cst));
  return SWD_OK;
}

int swd_engine_cancel_clear(swd_engine* e) {
  clear_error();
  SWD_CHECK(e, "null engine");
  if (!e->cancel_req.load()) return SWD_OK;
  SWD_CUDA(cudaSetDevice(e->device));
  std::lock_guard<std::mutex> lk(e->cancel_mu);
  SWD_CUDA(cudaStreamSynchronize(e->cst));
  SWD_CUDA(cudaMemsetAsync(e->cancelw.p, 0, sizeof(int), e->st));
  SWD_CUDA(cudaStreamSynchronize(e->st));
  e->cancel_req.store(0);
  return SWD_OK;
}

int swd_engine_radon_stats(swd_engine* e, uint64_t* gathers, uint64_t* recomputed) {
  clear_error();
  SWD_CHECK(e && gathers && recomputed, "null argument");
  *gathers = e->radon_gathers;
  unsigned long long c = 0;
  if (e->ccount.p) {
    SWD_CUDA(cudaMemcpyAsync(&c, e->ccount.p, sizeof(c), cudaMemcpyDeviceToHost, e->st));
    SWD_CUDA(cudaStreamSynchronize(e->st));
  }
  *recomputed = c;
  return SWD_OK;
}

int swd_engine_stream(const swd_engine* e, void** stream) {
  clear_error();
  SWD_CHECK(e && stream, "null argument");
  *stream = (void*)e->st;
  return SWD_OK;
}

int swd_engine_shot_sums_device(swd_engine* e, const double* d_vp, const double* d_vs, double* d_gsum,
                                double* res_sum, int* res_count) {
  clear_error();
  SWD_CHECK(e && d_vp && d_vs && d_gsum, "null argument");
  SWD_TRY(run(e, d_vp, d_vs, true, true, false));
  SWD_CUDA(cudaMemcpyAsync(d_gsum, e->gsum.p, 3 * e->plane * sizeof(double), cudaMemcpyDeviceToDevice, e->st));
  double r = 0;
  SWD_TRY(copy_picks(e, nullptr, nullptr, nullptr, nullptr, &r));
  int cnt = 0;
  for (int s = 0; s < e->ns; ++s)
    cnt += side_active(e->shot_no[s], 0, e->ns_total, e->sv.m, e->sv.M, e->sv.w) ? 1 : 0;
  if (res_sum) *res_sum = cnt ? r * cnt : 0.0;
  if (res_count) *res_count = cnt;
  return SWD_OK;
}

int swd_engine_assemble_device(swd_engine* e, const double* d_gsum, double* d_dk_vs) {
  clear_error();
  SWD_CHECK(e && d_gsum && d_dk_vs, "null argument");
  SWD_TRY(assemble(e, d_gsum));
  SWD_TRY(transpose<double, double>(e->dk2.as<double>(), 0, d_dk_vs, 0, 1, e->sv.nz, e->sv.nx, e->st));
  SWD_CUDA(cudaStreamSynchronize(e->st));
  return SWD_OK;
}

int swd_engine_set_timing(swd_engine* e, int on) {
  clear_error();
  SWD_CHECK(e, "null engine");
  if (on && e->ev.empty()) {
    e->ev.resize(4 * e->nbatch);
    for (auto& x : e->ev) SWD_CUDA(cudaEventCreate(&x));
  }
  e->timing = on != 0;
  return SWD_OK;
}

int swd_engine_phase_times(const swd_engine* e, double* fwd_ms, double* spec_ms, double* adj_ms) {
  clear_error();
  SWD_CHECK(e, "null engine");
  if (fwd_ms) *fwd_ms = e->phase_ms[0];
  if (spec_ms) *spec_ms = e->phase_ms[1];
  if (adj_ms) *adj_ms = e->phase_ms[2];
  return SWD_OK;
}

}  // extern "C"
