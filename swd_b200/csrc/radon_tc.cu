// Batched Radon contraction with general frequency, velocity and offset axes:
//
//   mm[s][f][p] = sum_x exp(i*2*pi*freq[f]*off[x]/vel[p]) * spec[s][f][x]
//
// which is the per-frequency slant stack of core/RTrAD.m:20-26 (l = exp(ll0*(j-1)),
// mm(:,j) = l*d(:,j)) over many shots at once.  For every frequency it is a complex
// GEMM: (velocities x offsets) times (offsets x shots).
//
// Four precisions:
//   SWD_PREC_FP64   CUDA cores, double (the reference computes this in MATLAB double)
//   SWD_PREC_FP32   CUDA cores, float operands and accumulation
//   SWD_PREC_BF16X2 tcgen05 tensor cores: each FP32 operand split into bf16 hi + lo, the
//                   products hi*hi + hi*lo + lo*hi accumulated in FP32 in TMEM
//   SWD_PREC_BF16X3 the same with hi + mid + lo and the six products of order <= 2
//
// The kernel table K is built once per axis set (in FP64, then rounded or split) and kept
// in HBM, pre-tiled in the tensor cores' shared-memory operand layout so that a tile is
// one contiguous block.
#include <cuda_bf16.h>

#include <cmath>
#include <memory>
#include <vector>

#include "fd_host.cuh"

namespace swd {
namespace tc {

constexpr int BM = 128;  // velocities per tile = TMEM lanes
constexpr int BN = 96;   // shots per tile (MMA N)
constexpr int BK = 32;   // offsets per pipeline stage (two MMA K-steps of 16)
constexpr int kThreads = 128;

// Operand tile of R rows x BK bf16 in the canonical K-major layout without swizzle:
// 8-row x 16-byte core matrices, [R/8][BK/8][8 rows][8 elements].  Leading byte offset
// (next 8 elements along K) = 128 B, stride byte offset (next 8 rows) = BK/8 * 128 B.
constexpr uint32_t kLBO = 128;
constexpr uint32_t kSBO = (BK / 8) * 128;

__host__ __device__ inline size_t tile_offset(int r, int k) {  // element offset inside a tile
  return ((size_t)(r >> 3) * (BK / 8) + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

// SM100 shared-memory matrix descriptor: start, LBO, SBO (16-byte units), version 1,
// base offset 0, no swizzle.
__device__ inline uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((kLBO >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((kSBO >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, bf16 A and B, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool neg_a) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ inline uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ inline void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ inline void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}
__device__ inline void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
// Bounded wait for phase `parity` of an mbarrier (non-blocking tests with a short sleep
// between them, about half a second at most); false if it did not complete.
__device__ inline bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 22); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (it > 64) __nanosleep(100);
  }
  return false;
}
__device__ inline void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ inline void cp16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ inline void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ inline void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// 32 lanes x 32 consecutive FP32 columns of TMEM into registers (this warp's lane quarter).
__device__ inline void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%"
      "19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// v rounded to FP32, then split into ns bf16 terms: hi = bf16(v), next = bf16(v - hi), ...
__device__ inline void split_value(double v, int ns, __nv_bfloat16* out) {
  float r = (float)v;
  for (int i = 0; i < ns; ++i) {
    const __nv_bfloat16 h = __float2bfloat16_rn(r);
    out[i] = h;
    r = r - __bfloat162float(h);
  }
}

struct TcArgs {
  int nf, np, nx, ns;             // axes
  int mtiles, ntiles, ktiles;     // tiles along velocities, shots, offsets
  const __nv_bfloat16* A;         // [f][mt][kt][2*NS parts][tile BM]
  const __nv_bfloat16* B;         // [f][nt][kt][2*NS parts][tile BN]
  double2* mm;                    // [s][f][p]
  int* status;                    // set to 1 when a wait timed out
};

// One CTA: frequency f, a BM-velocity tile and a BN-shot tile; all offsets through a
// STAGES-deep cp.async pipeline.  Thread 0 issues the MMAs; TMEM holds the real part in
// columns [0, BN) and the imaginary part in [BN, 2 BN).
template <int NS, int STAGES>
__global__ void __launch_bounds__(kThreads) tc_contract_kernel(TcArgs a) {
  constexpr int P = 2 * NS;  // parts per operand tile set
  constexpr size_t A_STAGE = (size_t)P * BM * BK * 2, B_STAGE = (size_t)P * BN * BK * 2;
  constexpr size_t STAGE = A_STAGE + B_STAGE;
  constexpr uint32_t kCols = 256;  // >= 2*BN, power of two
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t mbar[STAGES];
  __shared__ uint32_t tmem_slot;
  __shared__ int failed;

  const int mt = blockIdx.x, nt = blockIdx.y, f = blockIdx.z;
  const int tid = threadIdx.x, warp = tid >> 5;
  const size_t a_blk = (size_t)P * BM * BK, b_blk = (size_t)P * BN * BK;
  const __nv_bfloat16* Ag = a.A + (((size_t)f * a.mtiles + mt) * a.ktiles) * a_blk;
  const __nv_bfloat16* Bg = a.B + (((size_t)f * a.ntiles + nt) * a.ktiles) * b_blk;

  if (tid == 0) {
    failed = 0;
    for (int s = 0; s < STAGES; ++s) mbar_init(smem_u32(&mbar[s]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;

  auto load_stage = [&](int kt) {
    const int slot = kt % STAGES;
    const uint32_t sa = smem_u32(smem + slot * STAGE);
    const uint8_t* ga = (const uint8_t*)(Ag + (size_t)kt * a_blk);
    const uint8_t* gb = (const uint8_t*)(Bg + (size_t)kt * b_blk);
    for (int i = tid; i < (int)(A_STAGE / 16); i += kThreads) cp16(sa + i * 16, ga + (size_t)i * 16);
    for (int i = tid; i < (int)(B_STAGE / 16); i += kThreads) cp16(sa + A_STAGE + i * 16, gb + (size_t)i * 16);
  };

  const int nk = a.ktiles;
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load_stage(s);
    cp_commit();
  }
  // A wait that times out sets `failed`.  Every write to it comes before the barrier at the top of
  // the next stage, so all threads read the same value there and leave the loop together: no
  // further copies into slots that MMAs may still read, and no further MMAs.
  int kt = 0;
  for (; kt < nk; ++kt) {
    cp_wait<STAGES - 2>();  // this thread's copies of stage kt have landed
    fence_proxy_async();
    __syncthreads();
    if (failed) break;
    const int slot = kt % STAGES;
    if (tid == 0) {
      fence_after_sync();
      const uint32_t sa = smem_u32(smem + slot * STAGE), sb = sa + (uint32_t)A_STAGE;
      constexpr uint32_t a_part = BM * BK * 2, b_part = BN * BK * 2;
      const uint32_t id_pos = idesc_bf16(BM, BN, false), id_neg = idesc_bf16(BM, BN, true);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint32_t ko = kk * 2 * kLBO;  // two core matrices of K per MMA
#pragma unroll
        for (int i = 0; i < NS; ++i)
#pragma unroll
          for (int j = 0; j < NS; ++j) {
            if (i + j >= NS) continue;  // keep products of order < NS (hi*hi, hi*lo, lo*hi, ...)
            const uint64_t ar = smem_desc(sa + i * a_part + ko), ai = smem_desc(sa + (NS + i) * a_part + ko);
            const uint64_t br = smem_desc(sb + j * b_part + ko), bi = smem_desc(sb + (NS + j) * b_part + ko);
            const uint32_t acc = (kt | kk | i | j) ? 1u : 0u;
            mma_bf16(tmem, ar, br, id_pos, acc);            // re += Kr Dr
            mma_bf16(tmem, ai, bi, id_neg, 1u);             // re -= Ki Di
            mma_bf16(tmem + BN, ar, bi, id_pos, acc);       // im += Kr Di
            mma_bf16(tmem + BN, ai, br, id_pos, 1u);        // im += Ki Dr
          }
      }
      mma_commit(smem_u32(&mbar[slot]));
    }
    // refill the slot consumed by the previous stage once its MMAs are done; a thread whose
    // wait gave up copies nothing into it
    const int kn = kt + STAGES - 1;
    if (kn < nk) {
      bool free_slot = true;
      if (kn >= STAGES) {
        const int ps = kn % STAGES;  // == (kt - 1) % STAGES
        free_slot = mbar_wait(smem_u32(&mbar[ps]), (uint32_t)((kn / STAGES - 1) & 1));
        if (!free_slot) failed = 1;
      }
      if (free_slot) load_stage(kn);
    }
    cp_commit();
  }
  cp_wait<0>();  // this thread's copies in flight
  // the MMAs: the last commit (stage kt-1) covers every earlier tcgen05 operation of thread 0;
  // after a failure this one more wait is bounded too, and TMEM is released either way
  if (kt > 0) {
    const int last = kt - 1;
    if (!mbar_wait(smem_u32(&mbar[last % STAGES]), (uint32_t)((last / STAGES) & 1))) failed = 1;
  }
  fence_after_sync();
  __syncthreads();

  if (!failed) {
    const int p = mt * BM + warp * 32 + (tid & 31);
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      float re[32], im[32];
      tmem_ld32(tmem + lane_base + c0, re);
      tmem_ld32(tmem + lane_base + BN + c0, im);
      if (p < a.np) {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const int s = nt * BN + c0 + c;
          if (s < a.ns) a.mm[((size_t)s * a.nf + f) * a.np + p] = make_double2(re[c], im[c]);
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(a.status, 1);
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

template <int NS>
constexpr size_t tc_smem_bytes(int stages) {
  return (size_t)stages * (2 * NS) * (BM + BN) * BK * 2;
}

// K table, split and pre-tiled: A[f][mt][kt][part][tile] with parts re_0..re_{NS-1}, im_0..
__global__ void tc_ktable_kernel(int nf, int np, int nx, int mtiles, int ktiles, int ns_split,
                                 const double* freq, const double* vel, const double* off, __nv_bfloat16* A) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int x = blockIdx.y, f = blockIdx.z;
  if (p >= mtiles * BM) return;
  double c = 0.0, s = 0.0;
  if (p < np && x < nx) {
    // theta / (2 pi) = f x / v; sincospi of twice its fractional part keeps the argument small
    const double cyc = freq[f] * off[x] / vel[p];
    const double fr = cyc - floor(cyc);
    sincospi(2.0 * fr, &s, &c);
  }
  const int mt = p / BM, r = p % BM, kt = x / BK, k = x % BK;
  const size_t blk = (size_t)2 * ns_split * BM * BK;
  __nv_bfloat16* base = A + (((size_t)f * mtiles + mt) * ktiles + kt) * blk;
  __nv_bfloat16 h[3];
  split_value(c, ns_split, h);
  for (int i = 0; i < ns_split; ++i) base[(size_t)i * BM * BK + tile_offset(r, k)] = h[i];
  split_value(s, ns_split, h);
  for (int i = 0; i < ns_split; ++i) base[(size_t)(ns_split + i) * BM * BK + tile_offset(r, k)] = h[i];
}

// Spectra [s][f][x] (complex double) split and pre-tiled: B[f][nt][kt][part][tile].
__global__ void tc_split_spec_kernel(int nf, int nx, int nsh, int ntiles, int ktiles, int ns_split,
                                     const double2* spec, __nv_bfloat16* B) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y, f = blockIdx.z;
  if (x >= ktiles * BK) return;
  double2 v = make_double2(0.0, 0.0);
  if (s < nsh && x < nx) v = spec[((size_t)s * nf + f) * nx + x];
  const int nt = s / BN, r = s % BN, kt = x / BK, k = x % BK;
  const size_t blk = (size_t)2 * ns_split * BN * BK;
  __nv_bfloat16* base = B + (((size_t)f * ntiles + nt) * ktiles + kt) * blk;
  __nv_bfloat16 h[3];
  split_value(v.x, ns_split, h);
  for (int i = 0; i < ns_split; ++i) base[(size_t)i * BN * BK + tile_offset(r, k)] = h[i];
  split_value(v.y, ns_split, h);
  for (int i = 0; i < ns_split; ++i) base[(size_t)(ns_split + i) * BN * BK + tile_offset(r, k)] = h[i];
}

}  // namespace tc

// ------------------------------------------------------------------ CUDA-core paths

template <typename T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };

template <typename T>
__global__ void cc_ktable_kernel(int nf, int np, int nx, const double* freq, const double* vel, const double* off,
                                 typename Cplx<T>::type* K) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y, f = blockIdx.z;
  if (p >= np) return;
  const double cyc = freq[f] * off[x] / vel[p];
  double s, c;
  sincospi(2.0 * (cyc - floor(cyc)), &s, &c);
  typename Cplx<T>::type v;
  v.x = (T)c;
  v.y = (T)s;
  K[((size_t)f * nx + x) * np + p] = v;
}

// C[s][f][p] = sum_x K[f][x][p] * D[s][f][x]: a 64-velocity x 32-shot tile per block,
// 16 x 16 threads with 4 x 2 complex outputs each, offsets in chunks of 16 through shared memory.
template <typename T>
__global__ void __launch_bounds__(256) cc_contract_kernel(int nf, int np, int nx, int nsh,
                                                         const typename Cplx<T>::type* __restrict__ K,
                                                         const double2* __restrict__ spec, double2* mm) {
  using C = typename Cplx<T>::type;
  __shared__ C Ks[16][64];
  __shared__ C Ds[16][32];
  const int f = blockIdx.z, p0 = blockIdx.x * 64, s0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T ar[4][2] = {}, ai[4][2] = {};
  for (int x0 = 0; x0 < nx; x0 += 16) {
    for (int i = threadIdx.x; i < 16 * 64; i += 256) {
      const int xx = i / 64, pp = i % 64;
      C v;
      v.x = 0;
      v.y = 0;
      if (x0 + xx < nx && p0 + pp < np) v = K[((size_t)f * nx + x0 + xx) * np + p0 + pp];
      Ks[xx][pp] = v;
    }
    for (int i = threadIdx.x; i < 16 * 32; i += 256) {
      const int xx = i / 32, ss = i % 32;
      C v;
      v.x = 0;
      v.y = 0;
      if (x0 + xx < nx && s0 + ss < nsh) {
        const double2 d = spec[((size_t)(s0 + ss) * nf + f) * nx + x0 + xx];
        v.x = (T)d.x;
        v.y = (T)d.y;
      }
      Ds[xx][ss] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int xx = 0; xx < 16; ++xx) {
      C k[4], d[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) k[i] = Ks[xx][tx * 4 + i];
#pragma unroll
      for (int j = 0; j < 2; ++j) d[j] = Ds[xx][ty * 2 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          ar[i][j] += k[i].x * d[j].x - k[i].y * d[j].y;
          ai[i][j] += k[i].x * d[j].y + k[i].y * d[j].x;
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int p = p0 + tx * 4 + i, s = s0 + ty * 2 + j;
      if (p < np && s < nsh) mm[((size_t)s * nf + f) * np + p] = make_double2((double)ar[i][j], (double)ai[i][j]);
    }
}

}  // namespace swd

using namespace swd;

struct swd_contract {
  int nf = 0, np = 0, nx = 0, ns = 0, precision = 0, device = 0;
  int mtiles = 0, ntiles = 0, ktiles = 0, nsplit = 0;
  DevBuf axes;    // freq, vel, off
  DevBuf table;   // K (CUDA cores) or split pre-tiled A (tensor cores)
  DevBuf bsplit;  // split pre-tiled spectra
  DevBuf status;
};

extern "C" {

int swd_contract_create(int nf, const double* freq, int np, const double* vel, int nx, const double* offset,
                        int ns, int precision, int device, swd_contract** out) {
  clear_error();
  SWD_CHECK(out && freq && vel && offset, "null argument");
  SWD_CHECK(nf >= 1 && np >= 1 && nx >= 1 && ns >= 1, "axes must be non-empty (nf %d np %d nx %d ns %d)", nf, np,
            nx, ns);
  SWD_CHECK(precision >= SWD_PREC_FP64 && precision <= SWD_PREC_BF16X3, "unknown precision %d", precision);
  for (int p = 0; p < np; ++p) SWD_CHECK(vel[p] > 0, "velocities must be positive");
  *out = nullptr;
  auto c = std::make_unique<swd_contract>();
  c->nf = nf; c->np = np; c->nx = nx; c->ns = ns; c->precision = precision; c->device = device;
  SWD_CUDA(cudaSetDevice(device));
  SWD_TRY(c->axes.alloc((size_t)(nf + np + nx) * sizeof(double)));
  double* d_ax = c->axes.as<double>();
  SWD_CUDA(cudaMemcpy(d_ax, freq, nf * sizeof(double), cudaMemcpyHostToDevice));
  SWD_CUDA(cudaMemcpy(d_ax + nf, vel, np * sizeof(double), cudaMemcpyHostToDevice));
  SWD_CUDA(cudaMemcpy(d_ax + nf + np, offset, nx * sizeof(double), cudaMemcpyHostToDevice));
  SWD_TRY(c->status.alloc(sizeof(int)));
  SWD_CUDA(cudaMemset(c->status.p, 0, sizeof(int)));
  if (precision == SWD_PREC_FP64 || precision == SWD_PREC_FP32) {
    const size_t esz = precision == SWD_PREC_FP64 ? sizeof(double2) : sizeof(float2);
    SWD_TRY(c->table.alloc((size_t)nf * nx * np * esz));
    dim3 grid((np + 127) / 128, nx, nf);
    if (precision == SWD_PREC_FP64)
      cc_ktable_kernel<double><<<grid, 128>>>(nf, np, nx, d_ax, d_ax + nf, d_ax + nf + np, c->table.as<double2>());
    else
      cc_ktable_kernel<float><<<grid, 128>>>(nf, np, nx, d_ax, d_ax + nf, d_ax + nf + np, c->table.as<float2>());
    count_launch(1);
  } else {
    c->nsplit = precision == SWD_PREC_BF16X2 ? 2 : 3;
    c->mtiles = (np + tc::BM - 1) / tc::BM;
    c->ntiles = (ns + tc::BN - 1) / tc::BN;
    c->ktiles = (nx + tc::BK - 1) / tc::BK;
    const size_t parts = 2 * (size_t)c->nsplit;
    SWD_TRY(c->table.alloc((size_t)nf * c->mtiles * c->ktiles * parts * tc::BM * tc::BK * 2));
    SWD_TRY(c->bsplit.alloc((size_t)nf * c->ntiles * c->ktiles * parts * tc::BN * tc::BK * 2));
    dim3 grid((c->mtiles * tc::BM + 127) / 128, c->ktiles * tc::BK, nf);
    tc::tc_ktable_kernel<<<grid, 128>>>(nf, np, nx, c->mtiles, c->ktiles, c->nsplit, d_ax, d_ax + nf,
                                        d_ax + nf + np, c->table.as<__nv_bfloat16>());
    count_launch(1);
    const size_t smem = c->nsplit == 2 ? tc::tc_smem_bytes<2>(3) : tc::tc_smem_bytes<3>(2);
    if (c->nsplit == 2)
      SWD_CUDA(cudaFuncSetAttribute(tc::tc_contract_kernel<2, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
    else
      SWD_CUDA(cudaFuncSetAttribute(tc::tc_contract_kernel<3, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
  }
  SWD_CUDA(cudaGetLastError());
  SWD_CUDA(cudaDeviceSynchronize());
  *out = c.release();
  return SWD_OK;
}

int swd_contract_run(swd_contract* c, const double* d_spec, double* d_mm, void* stream) {
  clear_error();
  SWD_CHECK(c && d_spec && d_mm, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double2* spec = reinterpret_cast<const double2*>(d_spec);
  double2* mm = reinterpret_cast<double2*>(d_mm);
  if (c->precision == SWD_PREC_FP64 || c->precision == SWD_PREC_FP32) {
    dim3 grid((c->np + 63) / 64, (c->ns + 31) / 32, c->nf);
    if (c->precision == SWD_PREC_FP64)
      cc_contract_kernel<double><<<grid, 256, 0, st>>>(c->nf, c->np, c->nx, c->ns, c->table.as<double2>(), spec, mm);
    else
      cc_contract_kernel<float><<<grid, 256, 0, st>>>(c->nf, c->np, c->nx, c->ns, c->table.as<float2>(), spec, mm);
    count_launch(1);
    SWD_CUDA(cudaGetLastError());
    return SWD_OK;
  }
  {
    dim3 grid((c->ktiles * tc::BK + 127) / 128, c->ntiles * tc::BN, c->nf);
    tc::tc_split_spec_kernel<<<grid, 128, 0, st>>>(c->nf, c->nx, c->ns, c->ntiles, c->ktiles, c->nsplit, spec,
                                                   c->bsplit.as<__nv_bfloat16>());
  }
  tc::TcArgs a{c->nf, c->np, c->nx, c->ns, c->mtiles, c->ntiles, c->ktiles, c->table.as<__nv_bfloat16>(),
               c->bsplit.as<__nv_bfloat16>(), mm, c->status.as<int>()};
  dim3 grid(c->mtiles, c->ntiles, c->nf);
  if (c->nsplit == 2)
    tc::tc_contract_kernel<2, 3><<<grid, tc::kThreads, tc::tc_smem_bytes<2>(3), st>>>(a);
  else
    tc::tc_contract_kernel<3, 2><<<grid, tc::kThreads, tc::tc_smem_bytes<3>(2), st>>>(a);
  count_launch(2);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}

int swd_contract_status(swd_contract* c, int* timed_out) {
  clear_error();
  SWD_CHECK(c && timed_out, "null argument");
  SWD_CUDA(cudaMemcpy(timed_out, c->status.p, sizeof(int), cudaMemcpyDeviceToHost));
  return SWD_OK;
}

int swd_contract_flops(const swd_contract* c, double* useful, double* issued) {
  clear_error();
  SWD_CHECK(c, "null argument");
  const double u = 8.0 * c->nf * (double)c->np * c->nx * c->ns;
  if (useful) *useful = u;
  if (issued) {
    if (c->nsplit == 0) *issued = u;
    else {  // padded tiles, products per real GEMM: 3 (X2) or 6 (X3)
      const double terms = c->nsplit == 2 ? 3.0 : 6.0;
      *issued = 8.0 * terms * c->nf * (double)(c->mtiles * tc::BM) * (c->ktiles * tc::BK) * (c->ntiles * tc::BN);
    }
  }
  return SWD_OK;
}

int swd_contract_destroy(swd_contract* c) {
  clear_error();
  delete c;
  return SWD_OK;
}

}  // extern "C"
