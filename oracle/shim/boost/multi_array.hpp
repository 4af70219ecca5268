// Minimal stand-in for the part of Boost.MultiArray that the reference's
// iterative core (Core/src of CCPi-Reconstruction) uses, so that the
// reference compiles here without Boost.  Test infrastructure only: it is
// used to build the reference oracle under oracle/_ref, never the product.
//
// Surface covered (grep of Core/src): boost::extents[a][b][c],
// boost::c_storage_order(), multi_array_ref<T,N> (non-owning view over a
// caller buffer), multi_array<T,N,Alloc> (owning, zero-initialised, deep
// copy), chained operator[], data(), shape(), size_type.  Storage is always
// C order (last index fastest), which is the only order the reference asks
// for.
#ifndef ORACLE_SHIM_MULTI_ARRAY_HPP
#define ORACLE_SHIM_MULTI_ARRAY_HPP

#include <cstddef>
#include <cstring>
#include <memory>
#include <type_traits>
// Real Boost pulls these in transitively and the reference relies on it.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

namespace boost {

namespace shim_detail {

template <std::size_t N> struct extent_list {
  std::size_t n[N == 0 ? 1 : N];
  extent_list<N + 1> operator[](std::size_t v) const {
    extent_list<N + 1> r;
    for (std::size_t i = 0; i < N; i++)
      r.n[i] = n[i];
    r.n[N] = v;
    return r;
  }
};

// View of the trailing R dimensions of an array; operator[] peels one.
template <class T, std::size_t R> class sub_view {
public:
  sub_view(T *base, const std::size_t *stride) : base_(base), stride_(stride) {}
  sub_view<T, R - 1> operator[](std::ptrdiff_t i) const {
    return sub_view<T, R - 1>(base_ + i * std::ptrdiff_t(stride_[0]),
                              stride_ + 1);
  }
  T *origin() const { return base_; }

private:
  T *base_;
  const std::size_t *stride_;
};

template <class T> class sub_view<T, 1> {
public:
  sub_view(T *base, const std::size_t *) : base_(base) {}
  T &operator[](std::ptrdiff_t i) const { return base_[i]; }
  T *origin() const { return base_; }

private:
  T *base_;
};

} // namespace shim_detail

static const shim_detail::extent_list<0> extents = shim_detail::extent_list<0>();

struct c_storage_order {};

template <class T, std::size_t N> class multi_array_ref {
public:
  typedef std::size_t size_type;
  typedef T element;

  multi_array_ref(T *data, const shim_detail::extent_list<N> &e,
                  c_storage_order = c_storage_order())
      : data_(data) {
    set_shape(e);
  }

  T *data() { return data_; }
  const T *data() const { return data_; }
  const size_type *shape() const { return shape_; }
  size_type num_elements() const {
    size_type t = 1;
    for (std::size_t i = 0; i < N; i++)
      t *= shape_[i];
    return t;
  }

  // Rank-N indexing peels the first (slowest) dimension.
  typename std::conditional<N == 1, T &, shim_detail::sub_view<T, N - 1> >::type
  operator[](std::ptrdiff_t i) {
    return index<T>(data_, i);
  }
  typename std::conditional<N == 1, const T &,
                            shim_detail::sub_view<const T, N - 1> >::type
  operator[](std::ptrdiff_t i) const {
    return index<const T>(data_, i);
  }

protected:
  multi_array_ref() : data_(0) {
    for (std::size_t i = 0; i < N; i++)
      shape_[i] = stride_[i] = 0;
  }
  void set_shape(const shim_detail::extent_list<N> &e) {
    for (std::size_t i = 0; i < N; i++)
      shape_[i] = e.n[i];
    size_type s = 1;
    for (std::size_t i = N; i-- > 0;) {
      stride_[i] = s;
      s *= shape_[i];
    }
  }

  T *data_;
  size_type shape_[N];
  size_type stride_[N];

private:
  template <class U>
  typename std::conditional<N == 1, U &, shim_detail::sub_view<U, N - 1> >::type
  index(U *base, std::ptrdiff_t i) const {
    return make<U>(base + i * std::ptrdiff_t(stride_[0]),
                   std::integral_constant<bool, N == 1>());
  }
  template <class U> U &make(U *p, std::true_type) const { return *p; }
  template <class U>
  shim_detail::sub_view<U, N - 1> make(U *p, std::false_type) const {
    return shim_detail::sub_view<U, N - 1>(p, stride_ + 1);
  }
};

// Owning array.  Elements are value-initialised (zero for float/double),
// as Boost does, which the reference relies on for its fresh accumulators.
template <class T, std::size_t N, class Alloc = std::allocator<T> >
class multi_array : public multi_array_ref<T, N> {
  typedef multi_array_ref<T, N> base;

public:
  typedef typename base::size_type size_type;

  explicit multi_array(const shim_detail::extent_list<N> &e,
                       c_storage_order = c_storage_order()) {
    this->set_shape(e);
    allocate();
  }
  multi_array(const multi_array &o) : base() {
    for (std::size_t i = 0; i < N; i++) {
      this->shape_[i] = o.shape_[i];
      this->stride_[i] = o.stride_[i];
    }
    allocate();
    if (n_)
      std::memcpy(this->data_, o.data_, n_ * sizeof(T));
  }
  multi_array &operator=(const multi_array &o) {
    if (this != &o) {
      release();
      for (std::size_t i = 0; i < N; i++) {
        this->shape_[i] = o.shape_[i];
        this->stride_[i] = o.stride_[i];
      }
      allocate();
      if (n_)
        std::memcpy(this->data_, o.data_, n_ * sizeof(T));
    }
    return *this;
  }
  ~multi_array() { release(); }

private:
  void allocate() {
    n_ = this->num_elements();
    this->data_ = n_ ? alloc_.allocate(n_) : 0;
    for (size_type i = 0; i < n_; i++)
      this->data_[i] = T();
  }
  void release() {
    if (this->data_)
      alloc_.deallocate(this->data_, n_);
    this->data_ = 0;
    n_ = 0;
  }
  Alloc alloc_;
  size_type n_;
};

} // namespace boost

#endif
