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
// pipeline slots: BF16X2 2 x 56 KB (two CTAs per SM), BF16X3 2 x 84 KB (one CTA per SM)
constexpr int kStagesX2 = 2;
constexpr int kStagesX3 = 2;

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
// Bounded wait for phase `parity` of an mbarrier: try_wait suspends the warp in hardware until
// the phase completes or a short time limit passes, so a waiting warp takes no issue slots from
// the others; the loop gives up after about half a second of SM clock (or 2^26 tries),
// returning false.
constexpr long long kWaitCycles = 1LL << 30;
__device__ inline bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  for (uint32_t it = 0; it < (1u << 26); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > kWaitCycles) break;
  }
  return false;
}
__device__ inline void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

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

// 1-D bulk copy (the TMA engine, no tensor map, no multicast) of `bytes` from global memory into
// this CTA's shared memory; completion is counted on `mbar` as transaction bytes.  Both
// addresses 16-byte aligned, bytes a multiple of 16.
__device__ inline void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
__device__ inline void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// The MMAs of one stage: two K-steps of 16 offsets, the split products of order < NS
// (hi*hi, hi*lo, lo*hi, ...), real and imaginary accumulators.  Operand parts in the slot:
// A re_0..re_{NS-1}, im_0..; then B likewise.  The descriptors of a slot differ only in their
// start-address field (bits 0-13, 16-byte units; shared memory ends below 2^18 bytes, so no
// carry leaves the field): one base per operand, compile-time offsets per MMA.  Only the first
// MMA into each accumulator of the first stage overwrites it.
template <int NS>
__device__ inline void stage_mmas(uint32_t tmem, uint32_t sa, uint32_t sb, bool first) {
  constexpr uint64_t a_part = (BM * BK * 2) >> 4, b_part = (BN * BK * 2) >> 4, k_step = (2 * kLBO) >> 4;
  const uint64_t da = smem_desc(sa), db = smem_desc(sb);
  const uint32_t id_pos = idesc_bf16(BM, BN, false), id_neg = idesc_bf16(BM, BN, true);
  const uint32_t acc0 = first ? 0u : 1u;
#pragma unroll
  for (int kk = 0; kk < BK / 16; ++kk)
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
      for (int j = 0; j < NS; ++j) {
        if (i + j >= NS) continue;
        const uint64_t ar = da + (i * a_part + kk * k_step), ai = da + ((NS + i) * a_part + kk * k_step);
        const uint64_t br = db + (j * b_part + kk * k_step), bi = db + ((NS + j) * b_part + kk * k_step);
        const uint32_t acc = (kk | i | j) ? 1u : acc0;
        mma_bf16(tmem, ar, br, id_pos, acc);       // re += Kr Dr
        mma_bf16(tmem, ai, bi, id_neg, 1u);        // re -= Ki Di
        mma_bf16(tmem + BN, ar, bi, id_pos, acc);  // im += Kr Di
        mma_bf16(tmem + BN, ai, br, id_pos, 1u);   // im += Ki Dr
      }
}

// The tile's accumulators to mm in FP64: warp w (0..3) reads TMEM lanes 32w..32w+31, one
// velocity per thread, the real part from columns [0, BN) and the imaginary from [BN, 2 BN).
__device__ inline void store_tile(const TcArgs& a, uint32_t tmem, int mt, int nt, int f, int warp, int lane) {
  const int p = mt * BM + warp * 32 + lane;
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
}

// One CTA: frequency f, a BM-velocity tile and a BN-shot tile; all offsets through a STAGES-deep pipeline of shared-memory slots, warp-specialised:
//   warp 0, lane 0   producer: one bulk copy of the stage's pre-tiled kernel block and one of
//                    its spectra block into a free slot (slot `full` barrier: transaction bytes);
//   warp 1, lane 0   MMA issuer: waits for a full slot, issues its tcgen05.mma and commits to the
//                    slot's `empty` barrier, which frees the slot for the producer;
//   all 4 warps      epilogue (store_tile).
// With two stages a CTA takes 112 KB of shared memory and 256 TMEM columns, so two CTAs share
// an SM and one's epilogue overlaps the other's main loop.
//
// Every wait is bounded (mbar_wait).  A producer or MMA wait that gives up sets `failed` and
// stops that role issuing; the producer then waits for the copies it issued, the MMA issuer
// commits once more so that `done` covers every MMA it issued, all threads wait for `done`, and
// TMEM is released either way; the launch reports through `status`.
template <int NS, int STAGES>
__global__ void __launch_bounds__(kThreads) tc_contract_kernel(TcArgs a) {
  constexpr int P = 2 * NS;  // parts per operand tile set
  constexpr uint32_t A_STAGE = (uint32_t)P * BM * BK * 2, B_STAGE = (uint32_t)P * BN * BK * 2;
  constexpr uint32_t STAGE = A_STAGE + B_STAGE;
  constexpr uint32_t kCols = 256;  // >= 2*BN, power of two
  extern __shared__ __align__(128) uint8_t smem[];  // no-swizzle operand tiles need 16-byte alignment
  __shared__ __align__(8) uint64_t full[STAGES];
  __shared__ __align__(8) uint64_t empty[STAGES];
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t tmem_slot;
  __shared__ int failed;

  const int mt = blockIdx.x, nt = blockIdx.y, f = blockIdx.z;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint8_t* Ag = reinterpret_cast<const uint8_t*>(a.A) + ((size_t)f * a.mtiles + mt) * a.ktiles * A_STAGE;
  const uint8_t* Bg = reinterpret_cast<const uint8_t*>(a.B) + ((size_t)f * a.ntiles + nt) * a.ktiles * B_STAGE;

  if (tid == 0) {
    failed = 0;
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(smem_u32(&full[s]), 1);   // the producer's arrive (with the expected bytes)
      mbar_init(smem_u32(&empty[s]), 1);  // the MMA issuer's commit
    }
    mbar_init(smem_u32(&done), 1);
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
  const uint32_t s0 = smem_u32(smem);
  const int nk = a.ktiles;

  if (warp == 0) {
    if (lane == 0) {
      int kt = 0;
      for (; kt < nk; ++kt) {
        const int slot = kt % STAGES;
        if (kt >= STAGES && !mbar_wait(smem_u32(&empty[slot]), (uint32_t)((kt / STAGES - 1) & 1))) {
          failed = 1;
          break;
        }
        const uint32_t fb = smem_u32(&full[slot]), sa = s0 + slot * STAGE;
        mbar_expect_tx(fb, STAGE);
        bulk_g2s(sa, Ag + (size_t)kt * A_STAGE, A_STAGE, fb);
        bulk_g2s(sa + A_STAGE, Bg + (size_t)kt * B_STAGE, B_STAGE, fb);
      }
      // the copies issued last into each slot have landed before the CTA may leave (already so
      // when the MMA issuer consumed them)
      for (int j = kt > STAGES ? kt - STAGES : 0; j < kt; ++j)
        if (!mbar_wait(smem_u32(&full[j % STAGES]), (uint32_t)((j / STAGES) & 1))) failed = 1;
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      for (int kt = 0; kt < nk; ++kt) {
        const int slot = kt % STAGES;
        if (!mbar_wait(smem_u32(&full[slot]), (uint32_t)((kt / STAGES) & 1))) {
          failed = 1;
          break;
        }
        fence_after_sync();
        const uint32_t sa = s0 + slot * STAGE;
        stage_mmas<NS>(tmem, sa, sa + A_STAGE, kt == 0);
        mma_commit(smem_u32(&empty[slot]));
      }
      mma_commit(smem_u32(&done));  // arrives once every MMA issued above has completed
    }
    __syncwarp();
  }
  if (!mbar_wait(smem_u32(&done), 0u)) failed = 1;
  fence_after_sync();
  __syncthreads();

  if (!failed) store_tile(a, tmem, mt, nt, f, warp, lane);
  else if (tid == 0) atomicExch(a.status, 1);
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

// Spectra [s][f][x] (complex double) split and pre-tiled: B[f][nt][kt][part][tile].  One warp
// per (frequency, 8 shots, 32 offsets): lane = row (shot) r & 7 + 8 * (offset group of 8), so
// each lane reads 8 consecutive offsets of one shot (128 contiguous bytes) and the warp writes
// each part's 8 rows x 32 offsets as one contiguous 512-byte run of the tile layout.
__global__ void __launch_bounds__(256) tc_split_spec_kernel(int nf, int nx, int nsh, int ntiles, int ktiles,
                                                            int ns_split, const double2* __restrict__ spec,
                                                            __nv_bfloat16* __restrict__ B) {
  const int lane = threadIdx.x & 31;
  const int rg = blockIdx.y * 8 + (threadIdx.x >> 5);  // group of 8 shot rows
  const int kt = blockIdx.x, f = blockIdx.z;
  if (rg * 8 >= ntiles * BN) return;
  const int s = rg * 8 + (lane & 7), g = lane >> 3;  // shot, offset group within the tile
  const int x0 = kt * BK + g * 8;
  float re[8], im[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    double2 v = make_double2(0.0, 0.0);
    if (s < nsh && x0 + e < nx) v = spec[((size_t)s * nf + f) * nx + x0 + e];
    re[e] = (float)v.x;
    im[e] = (float)v.y;
  }
  const int nt = s / BN, r = s % BN;
  const size_t blk = (size_t)2 * ns_split * BN * BK;
  __nv_bfloat16* base = B + (((size_t)f * ntiles + nt) * ktiles + kt) * blk + tile_offset(r, g * 8);
  for (int part = 0; part < ns_split; ++part) {
    uint32_t wr[4], wi[4];
#pragma unroll
    for (int e = 0; e < 8; e += 2) {
      const __nv_bfloat16 r0 = __float2bfloat16_rn(re[e]), r1 = __float2bfloat16_rn(re[e + 1]);
      const __nv_bfloat16 i0 = __float2bfloat16_rn(im[e]), i1 = __float2bfloat16_rn(im[e + 1]);
      re[e] -= __bfloat162float(r0);
      re[e + 1] -= __bfloat162float(r1);
      im[e] -= __bfloat162float(i0);
      im[e + 1] -= __bfloat162float(i1);
      wr[e / 2] = (uint32_t)__bfloat16_as_ushort(r0) | ((uint32_t)__bfloat16_as_ushort(r1) << 16);
      wi[e / 2] = (uint32_t)__bfloat16_as_ushort(i0) | ((uint32_t)__bfloat16_as_ushort(i1) << 16);
    }
    *reinterpret_cast<uint4*>(base + (size_t)part * BN * BK) = make_uint4(wr[0], wr[1], wr[2], wr[3]);
    *reinterpret_cast<uint4*>(base + (size_t)(ns_split + part) * BN * BK) = make_uint4(wi[0], wi[1], wi[2], wi[3]);
  }
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
  DevBuf table;   // K (CUDA cores) or split pre-tiled A (tensor cores, offsets not uniform)
  DevBuf bsplit;  // split pre-tiled spectra
  DevBuf status;
};

namespace {
template <typename K>
int smem_attrs(K kernel, size_t bytes) {
  SWD_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  // two CTAs per SM (BF16X2) need the largest shared-memory carveout
  SWD_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  return SWD_OK;
}
}  // namespace

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
    if (c->nsplit == 2)
      SWD_TRY(smem_attrs(tc::tc_contract_kernel<2, tc::kStagesX2>, tc::tc_smem_bytes<2>(tc::kStagesX2)));
    else
      SWD_TRY(smem_attrs(tc::tc_contract_kernel<3, tc::kStagesX3>, tc::tc_smem_bytes<3>(tc::kStagesX3)));
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
    const int row_groups = c->ntiles * tc::BN / 8;  // 8 shot rows per warp, 8 warps per block
    dim3 grid(c->ktiles, (row_groups + 7) / 8, c->nf);
    tc::tc_split_spec_kernel<<<grid, 256, 0, st>>>(c->nf, c->nx, c->ns, c->ntiles, c->ktiles, c->nsplit, spec,
                                                   c->bsplit.as<__nv_bfloat16>());
  }
  tc::TcArgs a{c->nf, c->np, c->nx, c->ns, c->mtiles, c->ntiles, c->ktiles, c->table.as<__nv_bfloat16>(),
               c->bsplit.as<__nv_bfloat16>(), mm, c->status.as<int>()};
  dim3 grid(c->mtiles, c->ntiles, c->nf);
  if (c->nsplit == 2)
    tc::tc_contract_kernel<2, tc::kStagesX2><<<grid, tc::kThreads, tc::tc_smem_bytes<2>(tc::kStagesX2), st>>>(a);
  else
    tc::tc_contract_kernel<3, tc::kStagesX3><<<grid, tc::kThreads, tc::tc_smem_bytes<3>(tc::kStagesX3), st>>>(a);
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
