// Minimal stand-in for the part of boost::multi_array the reference uses
// (src/multi_arrays.h: rank-2/3/4 arrays of long double built with
// boost::extents[a][b]..., element access by chained operator[], data(),
// num_elements(), deep-copy value semantics, zero-initialised elements).
// Written for the oracle build of the reference sources only; not part of the
// product.
#ifndef REFSHIM_BOOST_MULTI_ARRAY_HPP
#define REFSHIM_BOOST_MULTI_ARRAY_HPP
#include <cstddef>
#include <vector>

namespace boost {

template <std::size_t K>
struct extent_list {
    std::size_t n[K];
    extent_list<K + 1> operator[](std::size_t e) const {
        extent_list<K + 1> r;
        for (std::size_t i = 0; i < K; i++) r.n[i] = n[i];
        r.n[K] = e;
        return r;
    }
};
template <>
struct extent_list<0> {
    extent_list<1> operator[](std::size_t e) const { extent_list<1> r; r.n[0] = e; return r; }
};
static const extent_list<0> extents = extent_list<0>();

namespace detail {
// view of the trailing K dimensions starting at one element offset
template <class T, std::size_t K>
struct sub_ref {
    T *p; const std::size_t *ext; const std::size_t *stride;
    sub_ref<T, K - 1> operator[](std::size_t i) const { return sub_ref<T, K - 1>{p + i * stride[0], ext + 1, stride + 1}; }
};
template <class T>
struct sub_ref<T, 1> {
    T *p; const std::size_t *ext; const std::size_t *stride;
    T &operator[](std::size_t i) const { return p[i]; }
};
}  // namespace detail

template <class T, std::size_t K>
class multi_array {
public:
    multi_array() { for (std::size_t i = 0; i < K; i++) { ext_[i] = 0; stride_[i] = 0; } }
    multi_array(const extent_list<K> &e) { set(e); }
    multi_array &resize(const extent_list<K> &e) { set(e); return *this; }
    T *data() { return d_.data(); }
    const T *data() const { return d_.data(); }
    std::size_t num_elements() const { return d_.size(); }
    const std::size_t *shape() const { return ext_; }
    detail::sub_ref<T, K - 1> operator[](std::size_t i) {
        return detail::sub_ref<T, K - 1>{d_.data() + i * stride_[0], ext_ + 1, stride_ + 1};
    }
    detail::sub_ref<const T, K - 1> operator[](std::size_t i) const {
        return detail::sub_ref<const T, K - 1>{d_.data() + i * stride_[0], ext_ + 1, stride_ + 1};
    }

private:
    void set(const extent_list<K> &e) {
        std::size_t tot = 1;
        for (std::size_t i = 0; i < K; i++) { ext_[i] = e.n[i]; tot *= e.n[i]; }
        std::size_t s = 1;
        for (std::size_t i = K; i-- > 0;) { stride_[i] = s; s *= ext_[i]; }
        d_.assign(tot, T());
    }
    std::vector<T> d_;
    std::size_t ext_[K];
    std::size_t stride_[K];
};

// rank-1 arrays index straight into the storage
template <class T>
class multi_array<T, 1> {
public:
    multi_array() {}
    multi_array(const extent_list<1> &e) : d_(e.n[0], T()) {}
    T *data() { return d_.data(); }
    const T *data() const { return d_.data(); }
    std::size_t num_elements() const { return d_.size(); }
    T &operator[](std::size_t i) { return d_[i]; }
    const T &operator[](std::size_t i) const { return d_[i]; }

private:
    std::vector<T> d_;
};

}  // namespace boost
#endif
