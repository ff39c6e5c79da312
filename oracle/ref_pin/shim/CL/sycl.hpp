// CL/sycl.hpp -- TEST INFRASTRUCTURE: a host-only stand-in for the small part of SYCL 1.2.1 /
// 2020 that the reference's hot-path sources use, so that those sources compile with g++ and
// run their kernel functors serially on the CPU. It is used only by oracle/ref_pin (the
// parity pin of the oracle against the reference's own kernels); nothing in the product
// includes it.
//
// Semantics follow the SYCL 2020 specification:
//   * a buffer owns its storage; one made from a host pointer copies the host data in and
//     writes it back to that pointer when destroyed, unless set_final_data() changed the
//     destination (nullptr: no write-back);
//   * accessors are plain pointers into the buffer's storage; handler::parallel_for runs the
//     kernel for every index in order, so a queue behaves like an in-order queue;
//   * the math built-ins are the SYCL definitions (sign, fmax/fmin as IEEE maxNum/minNum,
//     min/max by comparison, mix, smoothstep, clamp). pow(x, 4/3) -- the only pow of the hot
//     path, whose accuracy SYCL leaves to the implementation -- is, in FP64, the shared
//     division-free sv_math::pow43 that both the oracle and the CUDA path use; FP32 and
//     other exponents go to std::pow, as in the oracle, except an integer exponent of 2,
//     which is the correctly rounded square x * x.
#pragma once

#include <algorithm>
#include <array>
#include <cassert>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <stdexcept>
#include <type_traits>
#include <vector>

#include "../../../../mfcm_b200/csrc/sv_pow43.h"

namespace cl {
namespace sycl {

namespace access {
enum class mode { read, write, read_write, discard_write, discard_read_write, atomic };
enum class target { global_buffer, constant_buffer, local, host_buffer };
enum class placeholder { false_t, true_t };
}  // namespace access

template <int D = 1>
struct range {
  size_t n;
  range(size_t n_ = 0) : n(n_) {}
  size_t size() const { return n; }
  size_t get(int) const { return n; }
  size_t operator[](int) const { return n; }
};

template <int D = 1>
struct id {
  size_t i;
  id(size_t i_ = 0) : i(i_) {}
  size_t operator[](int) const { return i; }
  operator size_t() const { return i; }
};

template <int D = 1, bool WithOffset = false>
struct item {
  size_t i;
  size_t n;
  size_t get_linear_id() const { return i; }
  size_t get_id(int) const { return i; }
  id<D> get_id() const { return id<D>(i); }
  size_t operator[](int) const { return i; }
  range<D> get_range() const { return range<D>(n); }
  operator id<D>() const { return id<D>(i); }
};

class handler;

template <typename T, int D = 1>
class buffer;

template <typename T, int D = 1, access::mode M = access::mode::read_write,
          access::target Tg = access::target::global_buffer, access::placeholder P = access::placeholder::false_t>
class accessor {
 public:
  using value_type = T;
  T* ptr_ = nullptr;
  size_t n_ = 0;
  accessor() = default;
  accessor(buffer<T, D>& b) : ptr_(b.storage()), n_(b.get_count()) {}
  accessor(buffer<T, D>& b, handler&) : ptr_(b.storage()), n_(b.get_count()) {}
  T& operator[](size_t i) const { return ptr_[i]; }
  T& operator[](id<D> i) const { return ptr_[i.i]; }
  size_t size() const { return n_; }
  size_t get_count() const { return n_; }
  size_t get_size() const { return n_ * sizeof(T); }
  T* get_pointer() const { return ptr_; }
};

template <typename T>
class host_accessor {
 public:
  T* ptr_;
  size_t n_;
  T& operator[](size_t i) const { return ptr_[i]; }
  size_t size() const { return n_; }
};

template <typename T, int D>
class buffer {
  std::shared_ptr<std::vector<T>> data_;
  T* final_ = nullptr;

 public:
  using value_type = T;
  explicit buffer(const range<D>& r) : data_(std::make_shared<std::vector<T>>(r.size())) {}
  buffer(T* host, const range<D>& r) : data_(std::make_shared<std::vector<T>>(host, host + r.size())), final_(host) {}
  buffer(const T* host, const range<D>& r) : data_(std::make_shared<std::vector<T>>(host, host + r.size())) {}
  buffer(const buffer&) = delete;
  buffer& operator=(const buffer&) = delete;
  ~buffer() {
    if (final_ && !data_->empty()) std::copy(data_->begin(), data_->end(), final_);
  }
  T* storage() { return data_->data(); }
  size_t get_count() const { return data_->size(); }
  size_t size() const { return data_->size(); }
  range<D> get_range() const { return range<D>(data_->size()); }
  void set_final_data(std::nullptr_t = nullptr) { final_ = nullptr; }
  template <typename It>
  void set_final_data(It it) {
    final_ = &*it;
  }
  template <access::mode M, access::target Tg = access::target::global_buffer>
  accessor<T, D, M, Tg, access::placeholder::false_t> get_access(handler& h) {
    return accessor<T, D, M, Tg, access::placeholder::false_t>(*this, h);
  }
  accessor<T, D, access::mode::read_write, access::target::global_buffer, access::placeholder::false_t> get_access(
      handler& h) {
    return accessor<T, D, access::mode::read_write, access::target::global_buffer, access::placeholder::false_t>(*this,
                                                                                                                  h);
  }
  host_accessor<T> get_host_access() { return host_accessor<T>{data_->data(), data_->size()}; }
};

// sycl::maximum / minimum (SYCL 2020 4.10.2)
template <typename T = void>
struct maximum {
  T operator()(const T& x, const T& y) const { return (x < y) ? y : x; }
};
template <typename T = void>
struct minimum {
  T operator()(const T& x, const T& y) const { return (y < x) ? y : x; }
};
template <typename T = void>
struct plus {
  T operator()(const T& x, const T& y) const { return x + y; }
};

template <typename Acc, typename Op>
struct reduction_t {
  Acc acc;
  Op op;
};
template <typename Acc, typename Op>
reduction_t<Acc, Op> reduction(Acc acc, Op op) {
  return reduction_t<Acc, Op>{acc, op};
}
template <typename T, typename Op>
struct reducer {
  T value;
  Op op;
  void combine(const T& v) { value = op(value, v); }
};

class handler {
 public:
  template <typename K>
  void parallel_for(range<1> r, K k) {
    for (size_t i = 0; i < r.size(); ++i) k(item<1>{i, r.size()});
  }
  // one reduction, combined serially into the buffer's current value
  template <typename Acc, typename Op, typename K>
  void parallel_for(range<1> r, reduction_t<Acc, Op> red, K k) {
    using T = typename Acc::value_type;
    reducer<T, Op> rd{red.acc[0], red.op};
    for (size_t i = 0; i < r.size(); ++i) k(item<1>{i, r.size()}, rd);
    red.acc[0] = rd.value;
  }
  template <typename K>
  void single_task(K k) {
    k();
  }
  template <typename A, typename T>
  void fill(A acc, const T& v) {
    for (size_t i = 0; i < acc.size(); ++i) acc[i] = v;
  }
  template <typename A, typename B>
  void copy(A src, B dst) {
    for (size_t i = 0; i < src.size(); ++i) dst[i] = src[i];
  }
  template <typename A>
  void require(const A&) {}
};

class event {
 public:
  void wait() {}
};

class queue {
 public:
  template <typename F>
  event submit(F f) {
    handler h;
    f(h);
    return event();
  }
  void wait() {}
  void wait_and_throw() {}
  bool operator==(const queue& o) const { return this == &o; }
  bool operator!=(const queue& o) const { return this != &o; }
};

// ---- math built-ins (SYCL 2020 4.17.5-4.17.7) ----------------------------------------------
template <typename T>
T fabs(T x) {
  return std::fabs(x);
}
template <typename T>
T sqrt(T x) {
  return std::sqrt(x);
}
// sign: 1 or -1 for x > 0 or x < 0, the signed zero for a zero, 0 for NaN
template <typename T>
T sign(T x) {
  if (x > T(0)) return T(1);
  if (x < T(0)) return T(-1);
  if (x == x) return x;
  return T(0);
}
// fmax / fmin: IEEE maxNum / minNum (the non-NaN operand)
template <typename T>
T fmax(T x, T y) {
  return std::fmax(x, y);
}
template <typename T>
T fmin(T x, T y) {
  return std::fmin(x, y);
}
// min / max: y if y < x (resp. x < y), else x
template <typename T>
T min(T x, T y) {
  return (y < x) ? y : x;
}
template <typename T>
T max(T x, T y) {
  return (x < y) ? y : x;
}
template <typename T>
T clamp(T x, T lo, T hi) {
  return min(max(x, lo), hi);
}
// mix(x, y, a) = x + (y - x) * a
template <typename T>
T mix(T x, T y, T a) {
  return x + (y - x) * a;
}
// smoothstep(e0, e1, x) = t^2 (3 - 2 t), t = clamp((x - e0) / (e1 - e0), 0, 1)
template <typename T>
T smoothstep(T e0, T e1, T x) {
  T t = clamp((x - e0) / (e1 - e0), T(0), T(1));
  return t * t * (T(3) - T(2) * t);
}
template <typename T>
T pow(T x, T y) {
  if constexpr (std::is_same<T, double>::value)
    if (y == 4.0 / 3.0) return sv_math::pow43(x);
  return std::pow(x, y);
}
// an integer exponent (the Smagorinsky coefficient's pow(..., 2)) converts to the value type;
// the square is the correctly rounded x * x, which is within any accuracy bound SYCL allows
template <typename T, typename I, typename std::enable_if<std::is_integral<I>::value, int>::type = 0>
T pow(T x, I n) {
  if (n == 2) return x * x;
  return pow(x, T(n));
}

}  // namespace sycl
}  // namespace cl
