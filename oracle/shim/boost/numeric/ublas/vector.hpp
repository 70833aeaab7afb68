// Minimal stand-in for the two Boost.uBLAS containers that the CTBB_ICD
// reference uses (Boost itself is not installed in this image).
//
// Test infrastructure only: this header exists so the unmodified reference
// sources can be compiled into the oracle binary under oracle/_ref/.
//
// Semantics that matter for bit-exact parity with the real library:
//  * every vector expression is evaluated element by element, in the order
//    written, with one IEEE operation per operator (uBLAS expression templates
//    evaluate `a*u - b*v - c*w` as ((a*u(i)) - (b*v(i))) - (c*w(i)));
//  * `vector / scalar` divides each element (it does not multiply by a
//    reciprocal);
//  * norm_2 accumulates t += |x_i|*|x_i| from t = 0 in index order and returns
//    sqrt(t) (the unscaled uBLAS norm).
#pragma once

#include <cmath>
#include <cstddef>
#include <vector>

namespace boost {
namespace numeric {
namespace ublas {

template <class T>
class vector {
public:
    typedef std::size_t size_type;
    typedef T value_type;

    vector() {}
    explicit vector(size_type n) : d_(n, T()) {}
    vector(size_type n, const T& init) : d_(n, init) {}

    size_type size() const { return d_.size(); }
    void resize(size_type n, bool preserve = true) {
        if (!preserve) d_.assign(n, T());
        else d_.resize(n, T());
    }
    T& operator()(size_type i) { return d_[i]; }
    const T& operator()(size_type i) const { return d_[i]; }
    T& operator[](size_type i) { return d_[i]; }
    const T& operator[](size_type i) const { return d_[i]; }

private:
    std::vector<T> d_;
};

template <class T>
inline vector<T> operator+(const vector<T>& a, const vector<T>& b) {
    vector<T> r(a.size());
    for (std::size_t i = 0; i < a.size(); ++i) r(i) = a(i) + b(i);
    return r;
}

template <class T>
inline vector<T> operator-(const vector<T>& a, const vector<T>& b) {
    vector<T> r(a.size());
    for (std::size_t i = 0; i < a.size(); ++i) r(i) = a(i) - b(i);
    return r;
}

template <class T>
inline vector<T> operator-(const vector<T>& a) {
    vector<T> r(a.size());
    for (std::size_t i = 0; i < a.size(); ++i) r(i) = -a(i);
    return r;
}

// scalar * vector and vector * scalar: one multiply per element.
template <class T, class S>
inline vector<T> operator*(const S& s, const vector<T>& a) {
    vector<T> r(a.size());
    const T st = static_cast<T>(s);
    for (std::size_t i = 0; i < a.size(); ++i) r(i) = st * a(i);
    return r;
}

template <class T, class S>
inline vector<T> operator*(const vector<T>& a, const S& s) {
    vector<T> r(a.size());
    const T st = static_cast<T>(s);
    for (std::size_t i = 0; i < a.size(); ++i) r(i) = a(i) * st;
    return r;
}

// vector / scalar: element-wise division.
template <class T, class S>
inline vector<T> operator/(const vector<T>& a, const S& s) {
    vector<T> r(a.size());
    const T st = static_cast<T>(s);
    for (std::size_t i = 0; i < a.size(); ++i) r(i) = a(i) / st;
    return r;
}

template <class T>
inline T norm_2(const vector<T>& a) {
    T t = T();
    for (std::size_t i = 0; i < a.size(); ++i) {
        const T u = std::fabs(a(i));
        t += u * u;
    }
    return std::sqrt(t);
}

}  // namespace ublas
}  // namespace numeric
}  // namespace boost
