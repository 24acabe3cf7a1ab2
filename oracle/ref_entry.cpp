// TEST INFRASTRUCTURE ONLY -- builds ONE unmodified reference MEX source into a shared
// library under oracle/_ref/, with C entry points that call its MexFunction the way
// MATLAB would.  The source is included from where it lies in the reference tree
// (oracle/Makefile passes -I <reference>/core); nothing is copied.
//
//   -DSWDREF_FORWARD  core/eigen_staggerfd_single.cpp  -> swdref_eigen_staggerfd_single
//   -DSWDREF_ADJOINT  core/eigen_e2drtm_single.cpp     -> swdref_eigen_e2drtm_single
//
// Eigen and the MATLAB MEX headers are absent here; oracle/ref_shim/ holds stand-ins
// for the parts of them these sources use.  The two sources each define a global
// class MexFunction, so each one goes into its own library.
//
// Only tests/ and bench.py's reference leg load these libraries; the product never does.
#if defined(SWDREF_FORWARD)
#include "eigen_staggerfd_single.cpp"
#elif defined(SWDREF_ADJOINT)
#include "eigen_e2drtm_single.cpp"
#else
#error "define SWDREF_FORWARD or SWDREF_ADJOINT"
#endif

#include <cstring>
#include <exception>
#include <vector>

namespace {

matlab::data::Array single_array(const float* p, size_t rows, size_t cols) {
  matlab::data::ArrayFactory f;
  return f.createArray<float>({rows, cols}, p, p + rows * cols);
}

void set_err(char* err, int err_len, const char* msg) {
  if (err && err_len > 0) {
    std::strncpy(err, msg, static_cast<size_t>(err_len) - 1);
    err[err_len - 1] = '\0';
  }
}

// copy a single-precision output array into caller memory of n floats
int copy_out(const matlab::data::Array& a, float* dst, size_t n, char* err, int err_len) {
  const auto& p = a.impl();
  if (!p || p->type != matlab::data::ArrayType::SINGLE) {
    set_err(err, err_len, "output is not a single array");
    return 2;
  }
  if (p->f32.size() != n) {
    set_err(err, err_len, "output size differs from the caller's buffer");
    return 2;
  }
  std::memcpy(dst, p->f32.data(), n * sizeof(float));
  return 0;
}

}  // namespace

extern "C" {

#if defined(SWDREF_FORWARD)
// [seismo_u, seismo_w, wavefield_gradient] = eigen_staggerfd_single(iv, temp, ca, cl, cm, cm1, b, b1, s)
// (core/staggerfd_eigen.m:139).  Fields are nzbc x nxbc column-major, s has n_s samples,
// seismograms are nt x ng (n_seis floats each), the four snapshot fields nz x nx x nt/nt_wf
// (n_wf floats each).  Returns 0, 1 (the MEX threw: message in err) or 2 (an output size).
int swdref_eigen_staggerfd_single(const float* iv, int n_iv, int nzbc, int nxbc, const float* temp,
                                  const float* ca, const float* cl, const float* cm, const float* cm1,
                                  const float* b, const float* b1, const float* s, int n_s, float* seismo_u,
                                  float* seismo_w, size_t n_seis, float* fux, float* fuz, float* bwx,
                                  float* bwz, size_t n_wf, char* err, int err_len) {
  try {
    const size_t R = static_cast<size_t>(nzbc), C = static_cast<size_t>(nxbc);
    std::vector<matlab::data::Array> in(9), out(3);
    in[0] = single_array(iv, 1, static_cast<size_t>(n_iv));
    const float* fields[7] = {temp, ca, cl, cm, cm1, b, b1};
    for (int k = 0; k < 7; ++k) in[1 + k] = single_array(fields[k], R, C);
    in[8] = single_array(s, static_cast<size_t>(n_s), 1);
    MexFunction mex;
    mex(matlab::mex::ArgumentList(out.data(), out.size()), matlab::mex::ArgumentList(in.data(), in.size()));
    int rc = copy_out(out[0], seismo_u, n_seis, err, err_len);
    if (!rc) rc = copy_out(out[1], seismo_w, n_seis, err, err_len);
    if (rc) return rc;
    matlab::data::StructArray S(out[2].impl());
    float* wf[4] = {fux, fuz, bwx, bwz};
    const char* names[4] = {"fux", "fuz", "bwx", "bwz"};
    for (int k = 0; k < 4 && !rc; ++k)
      if (wf[k]) rc = copy_out(matlab::data::Array(S[0][names[k]]), wf[k], n_wf, err, err_len);
    return rc;
  } catch (const std::exception& e) {
    set_err(err, err_len, e.what());
    return 1;
  }
}
#endif

#if defined(SWDREF_ADJOINT)
// [cl_img, cm_img, illum_div] = eigen_e2drtm_single(iv, temp, ca, cl, cm, cm1, b, b1, seismo_w,
// fux, fuz, bwx, bwz) (core/e2drtm_eigen.m:122).  seismo_w is nt x ng; the snapshot fields are
// nz x (nx * nrec) as the MEX maps them; the images are nz x nx single (n_img floats each).
int swdref_eigen_e2drtm_single(const float* iv, int n_iv, int nzbc, int nxbc, const float* temp,
                               const float* ca, const float* cl, const float* cm, const float* cm1,
                               const float* b, const float* b1, const float* seismo_w, int nt, int ng,
                               const float* fux, const float* fuz, const float* bwx, const float* bwz, int nz,
                               int nx, int nrec, float* cl_img, float* cm_img, float* illum, size_t n_img,
                               char* err, int err_len) {
  try {
    const size_t R = static_cast<size_t>(nzbc), C = static_cast<size_t>(nxbc);
    std::vector<matlab::data::Array> in(13), out(3);
    in[0] = single_array(iv, 1, static_cast<size_t>(n_iv));
    const float* fields[7] = {temp, ca, cl, cm, cm1, b, b1};
    for (int k = 0; k < 7; ++k) in[1 + k] = single_array(fields[k], R, C);
    in[8] = single_array(seismo_w, static_cast<size_t>(nt), static_cast<size_t>(ng));
    const float* wf[4] = {fux, fuz, bwx, bwz};
    for (int k = 0; k < 4; ++k)
      in[9 + k] = single_array(wf[k], static_cast<size_t>(nz), static_cast<size_t>(nx) * static_cast<size_t>(nrec));
    MexFunction mex;
    mex(matlab::mex::ArgumentList(out.data(), out.size()), matlab::mex::ArgumentList(in.data(), in.size()));
    int rc = copy_out(out[0], cl_img, n_img, err, err_len);
    if (!rc) rc = copy_out(out[1], cm_img, n_img, err, err_len);
    if (!rc) rc = copy_out(out[2], illum, n_img, err, err_len);
    return rc;
  } catch (const std::exception& e) {
    set_err(err, err_len, e.what());
    return 1;
  }
}
#endif

}  // extern "C"
