// Writable host views of solver fields, standing in for the Blitz++ views
// that libmpdata++'s accessors return (concurr_common.hpp:387-433).  A view
// aliases a host mirror owned by the run object; writes through it reach the
// device before the next advance().  Index bases follow the reference:
// advectee views start at 0, advector views at (-1, 0, 0)
// (sharedmem.hpp:431-456, 543-577).
#pragma once

#include <algorithm>
#include <array>
#include <cstddef>
#include <functional>
#include <limits>
#include <stdexcept>
#include <type_traits>

namespace libmpdataxx {

template <class T, int N>
class host_view {
 public:
  host_view() = default;
  host_view(T *data, std::array<int, N> lbound, std::array<int, N> extent) : p_(data), lb_(lbound), ex_(extent) {
    st_[N - 1] = 1;
    for (int d = N - 2; d >= 0; --d) st_[d] = st_[d + 1] * ex_[d + 1];
  }
  int lbound(int d) const { return lb_[d]; }
  int ubound(int d) const { return lb_[d] + ex_[d] - 1; }
  int extent(int d) const { return ex_[d]; }
  std::array<int, N> shape() const { return ex_; }
  size_t size() const {
    size_t n = 1;
    for (int d = 0; d < N; ++d) n *= size_t(ex_[d]);
    return n;
  }
  T *data() const { return p_; }

  template <class... I>
  T &operator()(I... idx) const {
    static_assert(sizeof...(I) == N, "wrong number of indices");
    const int ix[N] = {int(idx)...};
    ptrdiff_t off = 0;
    for (int d = 0; d < N; ++d) off += ptrdiff_t(ix[d] - lb_[d]) * st_[d];
    return p_[off];
  }

  // fill with a value
  host_view &operator=(T v) {
    std::fill(p_, p_ + size(), v);
    return *this;
  }
  // copy another view of the same shape
  host_view &operator=(const host_view &o) {
    if (o.ex_ != ex_) throw std::invalid_argument("host_view: shape mismatch");
    std::copy(o.p_, o.p_ + size(), p_);
    return *this;
  }
  // fill from a function of the indices (the index placeholders of Blitz++
  // expressions become the arguments: run.advectee() = [](int i, int j) {...};)
  template <class F, class = typename std::enable_if<!std::is_arithmetic<F>::value>::type>
  host_view &operator=(F f) {
    assign(f);
    return *this;
  }

 private:
  template <class F>
  void assign(F &f) {
    std::array<int, N> ix;
    for (size_t q = 0, n = size(); q < n; ++q) {
      size_t r = q;
      for (int d = N - 1; d >= 0; --d) {
        ix[d] = lb_[d] + int(r % size_t(ex_[d]));
        r /= size_t(ex_[d]);
      }
      p_[q] = call(f, ix, std::make_integer_sequence<int, N>());
    }
  }
  template <class F, int... D>
  static T call(F &f, const std::array<int, N> &ix, std::integer_sequence<int, D...>) {
    return T(f(ix[D]...));
  }

  T *p_ = nullptr;
  std::array<int, N> lb_{}, ex_{};
  std::array<ptrdiff_t, N> st_{};
};

template <class T, int N> T min(const host_view<T, N> &v) { return *std::min_element(v.data(), v.data() + v.size()); }
template <class T, int N> T max(const host_view<T, N> &v) { return *std::max_element(v.data(), v.data() + v.size()); }
template <class T, int N> double sum(const host_view<T, N> &v) {
  double s = 0;
  for (size_t q = 0; q < v.size(); ++q) s += double(v.data()[q]);
  return s;
}

}  // namespace libmpdataxx
