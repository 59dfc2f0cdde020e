// The part of boost::multi_array that the reference's src/*.cpp files use
// (C-order storage, per-dimension index bases, extents / extent_range,
// chained operator[], shape(), index_bases()), written for this repository so
// that those files compile unmodified without Boost.  TEST INFRASTRUCTURE
// ONLY: compiled into oracle/_ref/libquest_ref.so (the checker).  Like the
// real header it brings in the standard headers the reference's files rely
// on without including them (<cmath> for std::pow in lagrange_set.cpp).
#ifndef QUEST_REF_SHIM_BOOST_MULTI_ARRAY
#define QUEST_REF_SHIM_BOOST_MULTI_ARRAY

#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <functional>
#include <memory>
#include <vector>

namespace boost {

struct extent_range {
  std::ptrdiff_t lo = 0, hi = 0;  // indices lo .. hi-1
  extent_range() = default;
  extent_range(std::ptrdiff_t start, std::ptrdiff_t finish) : lo(start), hi(finish) {}
};

template <std::size_t N>
struct extent_gen {
  std::array<extent_range, N> r{};
  extent_gen<N + 1> operator[](const extent_range &e) const
  {
    extent_gen<N + 1> g;
    for(std::size_t k = 0; k < N; ++k) g.r[k] = r[k];
    g.r[N] = e;
    return g;
  }
  extent_gen<N + 1> operator[](std::ptrdiff_t n) const { return (*this)[extent_range(0, n)]; }
};

namespace {
const extent_gen<0> extents{};
}

namespace shim_detail {
// a view of the last D dimensions starting at p
template <typename T, std::size_t D>
struct sub_ref {
  T *p;
  const std::ptrdiff_t *base;
  const std::ptrdiff_t *stride;
  sub_ref<T, D - 1> operator[](std::ptrdiff_t i) const
  {
    return sub_ref<T, D - 1>{p + (i - base[0]) * stride[0], base + 1, stride + 1};
  }
};
template <typename T>
struct sub_ref<T, 1> {
  T *p;
  const std::ptrdiff_t *base;
  const std::ptrdiff_t *stride;
  T &operator[](std::ptrdiff_t i) const { return p[(i - base[0]) * stride[0]]; }
};
}  // namespace shim_detail

template <typename T, std::size_t N>
class multi_array {
 public:
  typedef T element;
  typedef std::size_t size_type;
  typedef std::ptrdiff_t index;
  typedef boost::extent_range extent_range;

  explicit multi_array(const extent_gen<N> &g)
  {
    std::size_t total = 1;
    for(std::size_t k = 0; k < N; ++k) {
      base_[k] = g.r[k].lo;
      shape_[k] = (size_type)(g.r[k].hi - g.r[k].lo);
      total *= shape_[k];
    }
    std::ptrdiff_t s = 1;
    for(std::size_t k = N; k-- > 0;) {
      stride_[k] = s;
      s *= (std::ptrdiff_t)shape_[k];
    }
    data_.assign(total, T());
  }

  auto operator[](index i) -> decltype(shim_detail::sub_ref<T, N>{nullptr, nullptr, nullptr}[0])
  {
    return shim_detail::sub_ref<T, N>{data_.data(), base_.data(), stride_.data()}[i];
  }
  auto operator[](index i) const -> decltype(shim_detail::sub_ref<const T, N>{nullptr, nullptr, nullptr}[0])
  {
    return shim_detail::sub_ref<const T, N>{data_.data(), base_.data(), stride_.data()}[i];
  }
  const size_type *shape() const { return shape_.data(); }
  const index *index_bases() const { return base_.data(); }
  size_type num_elements() const { return data_.size(); }
  T *data() { return data_.data(); }
  const T *data() const { return data_.data(); }

 private:
  std::vector<T> data_;
  std::array<size_type, N> shape_{};
  std::array<index, N> base_{};
  std::array<index, N> stride_{};
};

}  // namespace boost

#endif
