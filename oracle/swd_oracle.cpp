// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the SWD finite-difference path.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
// this library; nothing in the product (swd_b200/) links or calls it.
//
// Parity status: PINNED for the FP32 instantiation.  The reference (zhangchang271/SWD)
// ships no tests, golden vectors or stored outputs, and MATLAB, Eigen and the MEX headers
// are absent here; instead its two MEX sources are compiled unmodified into oracle/_ref/
// (oracle/ref_entry.cpp, oracle/ref_shim/, `make -C oracle ref`) and tests/ checks this
// file against them bit for bit (seismograms, snapshots, FP32 images) on the tiny,
// 30x120, 100x600 and 400x3000 grids.  This file is a from-source restatement of
//   core/eigen_staggerfd_single.cpp:98-357   (forward time loop)
//   core/eigen_e2drtm_single.cpp:69-283      (adjoint time loop + imaging)
// as explicit loops in the same IEEE operation order as the Eigen expressions
// (no FMA contraction: build with -ffp-contract=off), templated on the scalar
// so that T=float is the single-precision MEX and T=double stands in for the
// binary-only eigen_*_double MEX (that instantiation has no source to pin it to; the
// double wrappers differ from the single ones only in class, staggerfd_eigend.m:38,70,91).
// It is also cross-checked bit-for-bit against an independent numpy restatement
// (oracle/swd_oracle.py) in tests/.
//
// Arrays are MATLAB column-major: A(z,x) = A[z + x*nzbc].
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

template <typename T>
struct Fwd {
  int nt, nzbc, nxbc, ng, sz, sx, gz, gx, dg, src_type, fd_order, nt_wf, nz, nx, fmt;
  T dtx;
};

// input_vector of staggerfd_eigen.m:138, read as core/eigen_staggerfd_single.cpp:98-118
template <typename T>
int parse_fwd(const T* iv, int n_iv, Fwd<T>& p) {
  if (n_iv < 16) return 1;
  p.nt = (int)iv[0]; p.nzbc = (int)iv[1]; p.nxbc = (int)iv[2]; p.dtx = iv[3];
  p.ng = (int)iv[4]; p.sz = (int)iv[5] - 1; p.sx = (int)iv[6] - 1;
  p.gz = (int)iv[7] - 1; p.gx = (int)iv[8] - 1; p.dg = (int)iv[9];
  p.src_type = (int)iv[10]; p.fd_order = (int)iv[11]; p.nt_wf = (int)iv[12];
  p.nz = (int)iv[13]; p.nx = (int)iv[14]; p.fmt = (int)iv[15];
  if (p.fd_order != 22) return 2;
  if (p.nt < 1 || p.nzbc < 3 || p.nxbc < 3 || p.nt_wf < 1 || p.nt % p.nt_wf) return 1;
  return 0;
}

template <typename T>
int staggerfd(const T* iv, int n_iv, const T* temp, const T* ca, const T* cl, const T* /*cm*/,
              const T* cm1, const T* b, const T* b1, const T* s, T* seis_u, T* seis_w,
              T* wf_fux, T* wf_fuz, T* wf_bwx, T* wf_bwz) {
  Fwd<T> p;
  int rc = parse_fwd(iv, n_iv, p);
  if (rc) return rc;
  const int NZ = p.nzbc, NX = p.nxbc;
  const size_t N = (size_t)NZ * NX;
  std::vector<T> uu(N, T(0)), ww(N, T(0)), xx(N, T(0)), xz(N, T(0)), zz(N, T(0));
  std::vector<T> fux(N, T(0)), fuz(N, T(0)), bwx(N, T(0)), bwz(N, T(0));
  const int pad_top = 1;                 // eigen_staggerfd_single.cpp:194-195 (fd_order 22)
  const int nbc = (p.nxbc - p.nx) / 2;   // :116
  const T dtx = p.dtx;
  auto I = [NZ](int z, int x) { return (size_t)z + (size_t)x * NZ; };
  for (int it = 0; it < p.nt; ++it) {
    // (1) velocity update on rows/cols 1..n-2 (:224-228)
    for (int x = 1; x <= NX - 2; ++x)
      for (int z = 1; z <= NZ - 2; ++z) {
        size_t c = I(z, x);
        uu[c] = temp[c] * uu[c] + b[c] * (((xx[I(z, x + 1)] - xx[c]) + xz[c]) - xz[I(z - 1, x)]);
        ww[c] = temp[c] * ww[c] + b1[c] * (((xz[c] - xz[I(z, x - 1)]) + zz[I(z + 1, x)]) - zz[c]);
      }
    // (2) source (:286-300)
    const T sv = s[it];
    const size_t cs = I(p.sz, p.sx);
    switch (p.src_type) {
      case 1: xx[cs] = xx[cs] + sv; zz[cs] = zz[cs] + sv; break;
      case 2:
        uu[cs] = uu[cs] + sv; uu[I(p.sz - 1, p.sx)] = uu[I(p.sz - 1, p.sx)] - sv;
        ww[cs] = ww[cs] + sv; ww[I(p.sz, p.sx + 1)] = ww[I(p.sz, p.sx + 1)] + sv; break;
      case 3: uu[cs] = uu[cs] + sv; ww[cs] = ww[cs] + sv; break;
      case 4: zz[cs] = zz[cs] + sv; break;
      case 5: ww[cs] = sv; break;
      default: break;
    }
    // (3) strains on rows/cols 1..n-2 (:302-306); the border stays 0
    for (int x = 1; x <= NX - 2; ++x)
      for (int z = 1; z <= NZ - 2; ++z) {
        size_t c = I(z, x);
        fux[c] = uu[c] - uu[I(z, x - 1)];
        fuz[c] = uu[I(z + 1, x)] - uu[c];
        bwx[c] = ww[I(z, x + 1)] - ww[c];
        bwz[c] = ww[c] - ww[I(z - 1, x)];
      }
    // (4) stress update over the whole array (:334-336)
    for (size_t c = 0; c < N; ++c) {
      xx[c] = temp[c] * xx[c] + (ca[c] * fux[c] + cl[c] * bwz[c]) * dtx;
      zz[c] = temp[c] * zz[c] + (ca[c] * bwz[c] + cl[c] * fux[c]) * dtx;
      xz[c] = temp[c] * xz[c] + (cm1[c] * (fuz[c] + bwx[c])) * dtx;
    }
    // (5) free surface (:340)
    for (int x = 0; x < NX; ++x) zz[I(pad_top, x)] = T(0);
    // (6) receivers (:342-345): the first ng entries of seq(gx, gx+ng*dg, dg)
    for (int j = 0; j < p.ng; ++j) {
      size_t c = I(p.gz, p.gx + j * p.dg);
      seis_w[(size_t)it + (size_t)j * p.nt] = ww[c];
      seis_u[(size_t)it + (size_t)j * p.nt] = uu[c];
    }
    // (7) strain snapshots of the interior every nt_wf steps (:346-351)
    if (it % p.nt_wf == 0 && wf_fux) {
      const size_t k = (size_t)(it / p.nt_wf);
      const size_t off = k * (size_t)p.nz * p.nx;
      for (int x = 0; x < p.nx; ++x)
        for (int z = 0; z < p.nz; ++z) {
          size_t c = I(pad_top + 1 + z, nbc + x);
          size_t o = off + (size_t)z + (size_t)x * p.nz;
          wf_fux[o] = fux[c]; wf_fuz[o] = fuz[c]; wf_bwx[o] = bwx[c]; wf_bwz[o] = bwz[c];
        }
    }
  }
  return 0;
}

template <typename T>
struct Adj {
  int nt, nzbc, nxbc, ng, nbc, gz, gx, dg, fd_order, nt_wf, nz, nx;
  T dtx, dt;
};

// input_vector of e2drtm_eigen.m:121, read as core/eigen_e2drtm_single.cpp:69-84
template <typename T>
int parse_adj(const T* iv, int n_iv, Adj<T>& p) {
  if (n_iv < 14) return 1;
  p.nt = (int)iv[0]; p.nzbc = (int)iv[1]; p.nxbc = (int)iv[2]; p.dtx = iv[3];
  p.ng = (int)iv[4]; p.nbc = (int)iv[5]; p.gz = (int)iv[6] - 1; p.gx = (int)iv[7] - 1;
  p.dg = (int)iv[8]; p.fd_order = (int)iv[9]; p.nt_wf = (int)iv[10]; p.nz = (int)iv[11];
  p.nx = (int)iv[12]; p.dt = iv[13];
  if (p.fd_order != 22) return 2;
  if (p.nt < 2 || p.nzbc < 3 || p.nxbc < 3 || p.nt_wf < 1 || p.nt % p.nt_wf) return 1;
  return 0;
}

// accum_fp64 = 0: images accumulate in T like the reference (:275-279);
// accum_fp64 = 1: each step's image term is formed in T and added to an FP64 sum.
template <typename T>
int e2drtm(const T* iv, int n_iv, const T* temp, const T* ca, const T* cl, const T* /*cm*/,
           const T* cm1, const T* b, const T* b1, const T* res, const T* wf_fux,
           const T* wf_fuz, const T* wf_bwx, const T* wf_bwz, int accum_fp64,
           double* cl_img, double* cm_img, double* illum) {
  Adj<T> p;
  int rc = parse_adj(iv, n_iv, p);
  if (rc) return rc;
  const int NZ = p.nzbc, NX = p.nxbc;
  const size_t N = (size_t)NZ * NX;
  std::vector<T> uu(N, T(0)), ww(N, T(0)), xx(N, T(0)), xz(N, T(0)), zz(N, T(0));
  const size_t NI = (size_t)p.nz * p.nx;
  std::vector<T> acl(NI, T(0)), acm(NI, T(0)), ail(NI, T(0));
  std::vector<double> dcl(NI, 0.0), dcm(NI, 0.0), dil(NI, 0.0);
  const int pad_top = 1;  // eigen_e2drtm_single.cpp:166-167
  const int nbc = p.nbc;
  const T dtx = p.dtx, dt = p.dt;
  auto I = [NZ](int z, int x) { return (size_t)z + (size_t)x * NZ; };
  for (int it = p.nt - 2; it > -1; --it) {
    // (1) adjoint velocity, material inside the derivative (:182-187)
    for (int x = 1; x <= NX - 2; ++x)
      for (int z = 1; z <= NZ - 2; ++z) {
        size_t c = I(z, x), cl_ = I(z, x - 1), cu = I(z - 1, x), cd = I(z + 1, x), cr = I(z, x + 1);
        T du = ((ca[c] * xx[c] - ca[cl_] * xx[cl_]) + (cl[c] * zz[c] - cl[cl_] * zz[cl_])) +
               (cm1[c] * xz[c] - cm1[cu] * xz[cu]);
        T dw = ((cl[cd] * xx[cd] - cl[c] * xx[c]) + (ca[cd] * zz[cd] - ca[c] * zz[c])) +
               (cm1[cr] * xz[cr] - cm1[c] * xz[c]);
        uu[c] = temp[c] * uu[c] - b[c] * du;
        ww[c] = temp[c] * ww[c] - b1[c] * dw;
      }
    // (2) residual injection at the receivers (:238-242)
    for (int j = 0; j < p.ng; ++j) {
      size_t c = I(p.gz, p.gx + j * p.dg);
      ww[c] = ww[c] + dt * res[(size_t)it + (size_t)j * p.nt];
    }
    // (3) adjoint stress on rows/cols 1..n-2 (:245-248)
    for (int x = 1; x <= NX - 2; ++x)
      for (int z = 1; z <= NZ - 2; ++z) {
        size_t c = I(z, x);
        xx[c] = temp[c] * xx[c] - dtx * (uu[I(z, x + 1)] - uu[c]);
        zz[c] = temp[c] * zz[c] - dtx * (ww[c] - ww[I(z - 1, x)]);
        xz[c] = (temp[c] * xz[c] - dtx * (uu[I(z + 1, x)] - uu[c])) - dtx * (ww[c] - ww[I(z, x - 1)]);
      }
    // (4) free surface (:270)
    for (int x = 0; x < NX; ++x) zz[I(pad_top, x)] = T(0);
    // (5) imaging condition every nt_wf steps (:274-279)
    if (it % p.nt_wf == 0) {
      const size_t off = (size_t)(it / p.nt_wf) * NI;
      for (int x = 0; x < p.nx; ++x)
        for (int z = 0; z < p.nz; ++z) {
          size_t c = I(pad_top + 1 + z, nbc + x);
          size_t o = (size_t)z + (size_t)x * p.nz;
          T fx = wf_fux[off + o], fz = wf_fuz[off + o], bx = wf_bwx[off + o], bz = wf_bwz[off + o];
          T F = fx + bz;
          T tcl = F * (xx[c] + zz[c]);
          T tcm = T(2) * ((xx[c] * fx + zz[c] * bz) + T(0.5) * (xz[c] * (fz + bx)));
          T til = F * F;
          if (accum_fp64) {
            dcl[o] += (double)tcl; dcm[o] += (double)tcm; dil[o] += (double)til;
          } else {
            acl[o] = acl[o] + tcl; acm[o] = acm[o] + tcm; ail[o] = ail[o] + til;
          }
        }
    }
  }
  for (size_t o = 0; o < NI; ++o) {
    cl_img[o] = accum_fp64 ? dcl[o] : (double)acl[o];
    cm_img[o] = accum_fp64 ? dcm[o] : (double)acm[o];
    illum[o] = accum_fp64 ? dil[o] : (double)ail[o];
  }
  return 0;
}

}  // namespace

extern "C" {

// Mirrors eigen_staggerfd_single(iv,temp,ca,cl,cm,cm1,b,b1,s) (core/eigen_staggerfd_single.cpp:68-383).
// wf_* may be NULL (no snapshots kept).
int oracle_staggerfd_f32(const float* iv, int n_iv, const float* temp, const float* ca,
                         const float* cl, const float* cm, const float* cm1, const float* b,
                         const float* b1, const float* s, float* seis_u, float* seis_w,
                         float* fux, float* fuz, float* bwx, float* bwz) {
  return staggerfd<float>(iv, n_iv, temp, ca, cl, cm, cm1, b, b1, s, seis_u, seis_w, fux, fuz, bwx, bwz);
}
int oracle_staggerfd_f64(const double* iv, int n_iv, const double* temp, const double* ca,
                         const double* cl, const double* cm, const double* cm1, const double* b,
                         const double* b1, const double* s, double* seis_u, double* seis_w,
                         double* fux, double* fuz, double* bwx, double* bwz) {
  return staggerfd<double>(iv, n_iv, temp, ca, cl, cm, cm1, b, b1, s, seis_u, seis_w, fux, fuz, bwx, bwz);
}
// Mirrors eigen_e2drtm_single(iv,temp,ca,cl,cm,cm1,b,b1,res,fux,fuz,bwx,bwz) (core/eigen_e2drtm_single.cpp:67-296).
int oracle_e2drtm_f32(const float* iv, int n_iv, const float* temp, const float* ca,
                      const float* cl, const float* cm, const float* cm1, const float* b,
                      const float* b1, const float* res, const float* fux, const float* fuz,
                      const float* bwx, const float* bwz, int accum_fp64, double* cl_img,
                      double* cm_img, double* illum) {
  return e2drtm<float>(iv, n_iv, temp, ca, cl, cm, cm1, b, b1, res, fux, fuz, bwx, bwz, accum_fp64,
                       cl_img, cm_img, illum);
}
int oracle_e2drtm_f64(const double* iv, int n_iv, const double* temp, const double* ca,
                      const double* cl, const double* cm, const double* cm1, const double* b,
                      const double* b1, const double* res, const double* fux, const double* fuz,
                      const double* bwx, const double* bwz, double* cl_img, double* cm_img,
                      double* illum) {
  return e2drtm<double>(iv, n_iv, temp, ca, cl, cm, cm1, b, b1, res, fux, fuz, bwx, bwz, 1, cl_img,
                        cm_img, illum);
}

}  // extern "C"
