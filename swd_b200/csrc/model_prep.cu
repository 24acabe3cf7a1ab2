// Device-side model preparation: the FD inputs that the reference's .m wrappers
// build before calling the MEX (core/staggerfd_eigen.m:37-107,
// core/e2drtm_eigen.m:44-101 with core/calparam.m, core/pad.m, core/damp_circle.m),
// computed per padded cell on the GPU.  Compiled with -fmad=false so that every
// double/float operation rounds exactly as written.
#include "fd_host.cuh"
#include "model_prep.cuh"

namespace swd {

// min(min(vp(:),vs(:))) (core/staggerfd_eigen.m:89); exact in any order.
__global__ void vmin_kernel(const double* __restrict__ vp, const double* __restrict__ vs, size_t n, double* out) {
  __shared__ double sm[32];
  double v = 1.0 / 0.0;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) v = fmin(v, fmin(vp[i], vs[i]));
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 1.0 / 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) *out = v;
  }
}

// damp_circle value at 0-based padded cell (z, x) (core/damp_circle.m:22-81).
__device__ double damp_at(const PrepParams& p, double kappa, int z, int x) {
  const int nbc = p.nbc, top = p.pad_top, nzbc = p.NZ, nz = p.nz, nx = p.nx;
  const int iz = z + 1, ix = x + 1;  // the reference's 1-based indices
  const double a = (nbc - 1) * p.dx;
  auto d1 = [&](int i) {  // damp1d(i+1), 0-based i
    const double r = (i * p.dx) / a;
    return kappa * (r * r);
  };
  auto circ = [&](int di, int dj) {
    const double d = sqrt((double)(di * di + dj * dj));
    const double q = d / nbc;
    return kappa * (q * q);
  };
  const bool left = ix <= nbc, right = ix >= nx + nbc + 1;
  if (iz >= top + 1 && iz <= nz + top) {  // left/right bands (:36-39)
    if (left) return d1(nbc - ix);
    if (right) return d1(ix - nx - nbc - 1);
    return 0.0;
  }
  if (!left && !right) {                  // top/bottom bands (:41-48)
    if (iz <= top) return p.isfs ? 0.0 : d1(nbc - iz);
    if (iz >= nzbc - nbc + 1) return d1(iz - (nzbc - nbc) - 1);
    return 0.0;
  }
  if (iz <= top) {                        // upper corners (:52-66)
    if (p.isfs) return 0.0;
    return left ? circ(ix - nbc - 1, iz - top - 1) : circ(ix - nx - nbc, iz - top - 1);
  }
  // lower corners (:69-81)
  return left ? circ(ix - nbc - 1, iz - nz - top) : circ(ix - nbc - nx, iz - nz - top);
}

template <typename T>
__device__ void prep_cell(const PrepParams& p, double kappa, const double* vp, const double* vs, int z, int x,
                          T& temp, T& ca, T& cl, T& cm, T& b) {
  const int top = p.pad_top;
  int mz = z - top, mx = x - p.nbc;                 // edge replication (core/pad.m:3-8)
  mz = mz < 0 ? 0 : (mz > p.nz - 1 ? p.nz - 1 : mz);
  mx = mx < 0 ? 0 : (mx > p.nx - 1 ? p.nx - 1 : mx);
  const double vpv = vp[(size_t)mx * p.nz + mz], vsv = vs[(size_t)mx * p.nz + mz];
  ca = (T)(vpv * vpv);                              // calparam with den = 1 (core/calparam.m:3-5)
  cm = (T)(vsv * vsv);
  cl = ca - (T)2 * cm;
  b = (T)p.dtx;                                     // dtx./den
  if (z == top - 1) {                               // free-surface row (core/staggerfd_eigen.m:98-107)
    ca = (T)2 * cm;
    cl = (T)0;
    b = (T)2 * b;
  }
  temp = (T)(1.0 - damp_at(p, kappa, z, x) * p.dt); // core/staggerfd_eigen.m:91
}

__device__ __forceinline__ double kappa_of(const PrepParams& p, double vmin) {
  const double a = (p.nbc - 1) * p.dx;
  return 3.0 * vmin * p.log1e7 / (2.0 * a);
}

// MATLAB column-major outputs (nzbc x nxbc): temp, ca, cl, cm, cm1(=cm), b, b1(=b).
template <typename T>
__global__ void prep_cm_kernel(PrepParams p, const double* vp, const double* vs, const double* vmin, T* temp, T* ca,
                               T* cl, T* cm, T* cm1, T* b, T* b1) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y;
  if (z >= p.NZ) return;
  const double kappa = kappa_of(p, *vmin);
  T t, a_, l, m, bb;
  prep_cell<T>(p, kappa, vp, vs, z, x, t, a_, l, m, bb);
  const size_t c = (size_t)x * p.NZ + z;
  temp[c] = t; ca[c] = a_; cl[c] = l; cm[c] = m; cm1[c] = m; b[c] = bb; b1[c] = bb;
}

// Packed row-major {temp, ca, cl, cm1} read by the step kernels (b = b1 = dtx, doubled on the
// free-surface row, is formed in the kernels from the row index).
template <typename T>
__global__ void prep_packed_kernel(PrepParams p, const double* vp, const double* vs, const double* vmin,
                                   typename Vec4<T>::type* mat, int pitch) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y;
  if (x >= p.NX) return;
  const double kappa = kappa_of(p, *vmin);
  T t, a_, l, m, bb;
  prep_cell<T>(p, kappa, vp, vs, z, x, t, a_, l, m, bb);
  typename Vec4<T>::type u;
  // Border columns are never updated.  Their temp is used for nothing but their own update,
  // so it is set to 1: the two-step warp kernels then keep those cells with a zero time factor
  // instead of a select per row (fd_warp.cuh).
  u.x = (x == 0 || x == p.NX - 1) ? (T)1 : t;
  u.y = a_; u.z = l; u.w = m;
  mat[(size_t)z * pitch + x] = u;
}

int prep_check(const PrepParams& p) {
  SWD_CHECK(p.nz >= 1 && p.nx >= 1 && p.nbc >= 2, "model %d x %d with nbc %d: need nbc >= 2", p.nz, p.nx, p.nbc);
  SWD_CHECK(p.isfs == 1, "isfs=0 leaves b1/cm1 undefined in the reference wrappers (core/staggerfd_eigen.m:98-107)");
  SWD_CHECK(p.fd_order == 22, "fd_order must be 22");
  SWD_CHECK(p.dx > 0 && p.dt > 0, "dx and dt must be positive");
  return SWD_OK;
}

void prep_fill(PrepParams& p) {
  p.pad_top = (p.fd_order - 20) / 2 + 1;  // core/staggerfd_eigen.m:51
  p.NZ = p.nz + p.pad_top + p.nbc;
  p.NX = p.nx + 2 * p.nbc;
  p.log1e7 = log(10000000.0);
}

int vmin_device(const double* d_vp, const double* d_vs, size_t n, double* d_out, cudaStream_t st) {
  vmin_kernel<<<1, 1024, 0, st>>>(d_vp, d_vs, n, d_out);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}

template <typename T>
int prep_packed(const PrepParams& p, const double* d_vp, const double* d_vs, const double* d_vmin,
                typename Vec4<T>::type* mat, int pitch, cudaStream_t st) {
  dim3 grid((p.NX + 127) / 128, p.NZ), block(128);
  prep_packed_kernel<T><<<grid, block, 0, st>>>(p, d_vp, d_vs, d_vmin, mat, pitch);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  return SWD_OK;
}
template int prep_packed<float>(const PrepParams&, const double*, const double*, const double*, float4*, int,
                                cudaStream_t);
template int prep_packed<double>(const PrepParams&, const double*, const double*, const double*, double4*, int,
                                 cudaStream_t);

template <typename T>
int prep_host(int nz, int nx, int nbc, int isfs, int fd_order, double dx, double dt, double dtx, const double* vp,
              const double* vs, T* temp, T* ca, T* cl, T* cm, T* cm1, T* b, T* b1) {
  clear_error();
  PrepParams p{};
  p.nz = nz; p.nx = nx; p.nbc = nbc; p.isfs = isfs; p.fd_order = fd_order; p.dx = dx; p.dt = dt; p.dtx = dtx;
  SWD_TRY(prep_check(p));
  SWD_CHECK(vp && vs && temp && ca && cl && cm && cm1 && b && b1, "null pointer");
  prep_fill(p);
  const size_t n = (size_t)nz * nx, NN = (size_t)p.NZ * p.NX;
  DevBuf d_v, d_o;
  SWD_TRY(d_v.alloc((2 * n + 1) * sizeof(double)));
  SWD_TRY(d_o.alloc(7 * NN * sizeof(T)));
  cudaStream_t st = 0;
  double* dv = d_v.as<double>();
  SWD_CUDA(cudaMemcpyAsync(dv, vp, n * sizeof(double), cudaMemcpyHostToDevice, st));
  SWD_CUDA(cudaMemcpyAsync(dv + n, vs, n * sizeof(double), cudaMemcpyHostToDevice, st));
  SWD_TRY(vmin_device(dv, dv + n, n, dv + 2 * n, st));
  T* o = d_o.as<T>();
  dim3 grid((p.NZ + 127) / 128, p.NX), block(128);
  prep_cm_kernel<T><<<grid, block, 0, st>>>(p, dv, dv + n, dv + 2 * n, o, o + NN, o + 2 * NN, o + 3 * NN, o + 4 * NN,
                                            o + 5 * NN, o + 6 * NN);
  count_launch(1);
  SWD_CUDA(cudaGetLastError());
  T* outs[7] = {temp, ca, cl, cm, cm1, b, b1};
  for (int i = 0; i < 7; ++i)
    SWD_CUDA(cudaMemcpyAsync(outs[i], o + i * NN, NN * sizeof(T), cudaMemcpyDeviceToHost, st));
  SWD_CUDA(cudaStreamSynchronize(st));
  return SWD_OK;
}

}  // namespace swd

extern "C" {

int swd_prep_model_single(int nz, int nx, int nbc, int isfs, int fd_order, double dx, double dt, double dtx,
                          const double* vp, const double* vs, float* temp, float* ca, float* cl, float* cm,
                          float* cm1, float* b, float* b1) {
  return swd::prep_host<float>(nz, nx, nbc, isfs, fd_order, dx, dt, dtx, vp, vs, temp, ca, cl, cm, cm1, b, b1);
}
int swd_prep_model_double(int nz, int nx, int nbc, int isfs, int fd_order, double dx, double dt, double dtx,
                          const double* vp, const double* vs, double* temp, double* ca, double* cl, double* cm,
                          double* cm1, double* b, double* b1) {
  return swd::prep_host<double>(nz, nx, nbc, isfs, fd_order, dx, dt, dtx, vp, vs, temp, ca, cl, cm, cm1, b, b1);
}

}  // extern "C"
