// TEST INFRASTRUCTURE ONLY -- a compile stand-in for the MATLAB C++ MEX API
// surface (matlab::mex::Function, ArgumentList, MW_NOEXCEPT) used by the reference's
// FD MEX sources, so that they build unmodified into oracle/_ref/.  The C entry points
// that drive a MexFunction live in oracle/ref_entry.cpp.  Written for this repository;
// nothing in the product includes it.
#pragma once

#include <stdexcept>

#include "MatlabDataArray.hpp"

#ifndef MW_NOEXCEPT
#define MW_NOEXCEPT noexcept
#endif

namespace matlab {
namespace mex {

// a view of the caller's argument array (MATLAB passes it by value, as here)
class ArgumentList {
 public:
  ArgumentList(matlab::data::Array* first, size_t n) : a_(first), n_(n) {}
  matlab::data::Array& operator[](size_t i) const {
    if (i >= n_) throw std::runtime_error("MEX argument index out of range");
    return a_[i];
  }
  size_t size() const { return n_; }

 private:
  matlab::data::Array* a_;
  size_t n_;
};

class Function {
 public:
  virtual ~Function() = default;
  virtual void operator()(ArgumentList outputs, ArgumentList inputs) = 0;
};

}  // namespace mex
}  // namespace matlab
