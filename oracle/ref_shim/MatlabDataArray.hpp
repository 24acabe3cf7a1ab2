// TEST INFRASTRUCTURE ONLY -- a compile stand-in for the part of the MATLAB Data
// API (matlab::data) that the reference's FD MEX sources touch
// (core/eigen_staggerfd_single.cpp:46-152,359-383, core/eigen_e2drtm_single.cpp:44-136,
// 284-297), so that they build unmodified into oracle/_ref/.  MATLAB is not
// installed here.  Written for this repository from the API's documented surface;
// nothing in the product includes it.
//
// Kept from the documented behaviour:
//  * Arrays are column-major with a dimension vector; copies share the data.
//  * arr[i] on a numeric array converts element i to the requested arithmetic type
//    (int fields of the MEX input_vector are read by C++ truncation).
//  * TypedArray<T>(Array&&) takes a numeric array of element type T (else throws).
//  * ArrayFactory::createArray<T>(dims, first, last) copies [first, last).
//  * createStructArray(dims, names) gives a struct array whose fields are assigned
//    with S[0]["name"] = array.
#pragma once

#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace matlab {
namespace data {

using ArrayDimensions = std::vector<size_t>;

enum class ArrayType { UNKNOWN, SINGLE, DOUBLE, STRUCT };

namespace detail {
struct Impl {
  ArrayType type = ArrayType::UNKNOWN;
  ArrayDimensions dims;
  std::vector<float> f32;
  std::vector<double> f64;
  std::vector<std::string> names;              // struct arrays (1x1 only)
  std::vector<std::shared_ptr<Impl>> fields;   // one value per name
};

inline size_t count(const ArrayDimensions& d) {
  size_t n = 1;
  for (size_t v : d) n *= v;
  return n;
}
template <class T>
constexpr ArrayType type_of() {
  return std::is_same<T, float>::value ? ArrayType::SINGLE
                                       : (std::is_same<T, double>::value ? ArrayType::DOUBLE : ArrayType::UNKNOWN);
}
template <class T>
std::vector<T>& storage(Impl& a);
template <>
inline std::vector<float>& storage<float>(Impl& a) { return a.f32; }
template <>
inline std::vector<double>& storage<double>(Impl& a) { return a.f64; }
}  // namespace detail

// arr[i] of a numeric array
class ArrayElementRef {
 public:
  ArrayElementRef(const detail::Impl* a, size_t i) : a_(a), i_(i) {}
  template <class T, class = std::enable_if_t<std::is_arithmetic<T>::value>>
  operator T() const {
    if (!a_) throw std::runtime_error("element of an empty array");
    if (a_->type == ArrayType::SINGLE && i_ < a_->f32.size()) return static_cast<T>(a_->f32[i_]);
    if (a_->type == ArrayType::DOUBLE && i_ < a_->f64.size()) return static_cast<T>(a_->f64[i_]);
    throw std::runtime_error("element index outside the array, or not a numeric array");
  }

 private:
  const detail::Impl* a_;
  size_t i_;
};

class Array {
 public:
  Array() = default;
  explicit Array(std::shared_ptr<detail::Impl> p) : p_(std::move(p)) {}
  ArrayElementRef operator[](size_t i) const { return ArrayElementRef(p_.get(), i); }
  ArrayDimensions getDimensions() const { return p_ ? p_->dims : ArrayDimensions{0, 0}; }
  size_t getNumberOfElements() const { return p_ ? detail::count(p_->dims) : 0; }
  ArrayType getType() const { return p_ ? p_->type : ArrayType::UNKNOWN; }
  const std::shared_ptr<detail::Impl>& impl() const { return p_; }

 protected:
  std::shared_ptr<detail::Impl> p_;
};

template <class T>
class TypedIterator {
 public:
  explicit TypedIterator(T* p) : p_(p) {}
  T* operator->() const { return p_; }
  T& operator*() const { return *p_; }

 private:
  T* p_;
};

template <class T>
class TypedArray : public Array {
 public:
  TypedArray(Array&& a) : Array(a.impl()) {
    if (!p_ || p_->type != detail::type_of<T>()) throw std::runtime_error("TypedArray: element type mismatch");
    a = Array();
  }
  TypedIterator<T> begin() { return TypedIterator<T>(detail::storage<T>(*p_).data()); }
  TypedIterator<T> end() { return TypedIterator<T>(detail::storage<T>(*p_).data() + detail::storage<T>(*p_).size()); }
};

class StructArray : public Array {
 public:
  class FieldRef {
   public:
    FieldRef(detail::Impl* s, std::string name) : s_(s), name_(std::move(name)) {}
    FieldRef& operator=(const Array& v) {
      for (size_t k = 0; k < s_->names.size(); ++k)
        if (s_->names[k] == name_) {
          s_->fields[k] = v.impl();
          return *this;
        }
      throw std::runtime_error("no such struct field: " + name_);
    }
    operator Array() const {
      for (size_t k = 0; k < s_->names.size(); ++k)
        if (s_->names[k] == name_) return Array(s_->fields[k]);
      throw std::runtime_error("no such struct field: " + name_);
    }

   private:
    detail::Impl* s_;
    std::string name_;
  };
  class ElementRef {
   public:
    explicit ElementRef(detail::Impl* s) : s_(s) {}
    FieldRef operator[](const std::string& name) const { return FieldRef(s_, name); }

   private:
    detail::Impl* s_;
  };

  explicit StructArray(std::shared_ptr<detail::Impl> p) : Array(std::move(p)) {}
  ElementRef operator[](size_t i) {
    if (i != 0) throw std::runtime_error("only 1x1 struct arrays are supported");
    return ElementRef(p_.get());
  }
};

class ArrayFactory {
 public:
  template <class T, class It>
  TypedArray<T> createArray(ArrayDimensions dims, It first, It last) {
    auto p = std::make_shared<detail::Impl>();
    p->type = detail::type_of<T>();
    p->dims = dims;
    auto& v = detail::storage<T>(*p);
    v.assign(first, last);
    if (v.size() != detail::count(dims)) throw std::runtime_error("createArray: element count does not match dims");
    return TypedArray<T>(Array(p));
  }
  StructArray createStructArray(ArrayDimensions dims, std::vector<std::string> names) {
    if (detail::count(dims) != 1) throw std::runtime_error("only 1x1 struct arrays are supported");
    auto p = std::make_shared<detail::Impl>();
    p->type = ArrayType::STRUCT;
    p->dims = dims;
    p->names = std::move(names);
    p->fields.resize(p->names.size());
    return StructArray(p);
  }
};

}  // namespace data
}  // namespace matlab
