// Device-side construction of the padded FD material fields from (vp, vs).
#pragma once
#include "fd_host.cuh"

namespace swd {

struct PrepParams {
  int nz, nx, nbc, isfs, fd_order;
  double dx, dt, dtx;
  // derived by prep_fill()
  int pad_top;      // rows added on top (the .m wrappers' pad_top, 1-based free-surface row)
  int NZ, NX;       // nzbc, nxbc
  double log1e7;    // log(10000000.0), evaluated on the host (core/damp_circle.m:26)
};

int prep_check(const PrepParams& p);
void prep_fill(PrepParams& p);
int vmin_device(const double* d_vp, const double* d_vs, size_t n, double* d_out, cudaStream_t st);
template <typename T>
int prep_packed(const PrepParams& p, const double* d_vp, const double* d_vs, const double* d_vmin,
                typename Vec4<T>::type* mat, int pitch, cudaStream_t st);

}  // namespace swd
