// Minimal stand-in for boost::numeric::ublas::compressed_vector, covering the
// calls made by the CTBB_ICD reference (generate_system_matrix.cpp:190-193,
// 337-428; icd_iteration.cpp:137).
//
// Test infrastructure only (oracle build). Entries are kept as two parallel
// arrays in push order; push_back insists on strictly increasing indices, the
// same precondition the real container checks, so an out-of-order push in the
// reference aborts loudly instead of silently reordering.
#pragma once

#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "vector.hpp"

namespace boost {
namespace numeric {
namespace ublas {

template <class T>
class compressed_vector {
public:
    typedef std::size_t size_type;

    compressed_vector() : size_(0) {}
    explicit compressed_vector(size_type n) : size_(n) {}
    compressed_vector(size_type n, size_type reserve_nnz) : size_(n) {
        idx_.reserve(reserve_nnz);
        val_.reserve(reserve_nnz);
    }

    size_type size() const { return size_; }
    size_type filled() const { return idx_.size(); }
    size_type nnz() const { return idx_.size(); }

    void resize(size_type n, bool preserve = true) {
        size_ = n;
        if (!preserve) {
            idx_.clear();
            val_.clear();
        }
    }

    void push_back(size_type i, const T& v) {
        if (i >= size_ || (!idx_.empty() && idx_.back() >= i)) {
            std::fprintf(stderr, "compressed_vector::push_back: index %zu out of order\n", i);
            std::abort();
        }
        idx_.push_back(i);
        val_.push_back(v);
    }

    void swap(compressed_vector& o) {
        std::swap(size_, o.size_);
        idx_.swap(o.idx_);
        val_.swap(o.val_);
    }

    class const_iterator {
    public:
        const_iterator(const compressed_vector* v, size_type p) : v_(v), p_(p) {}
        size_type index() const { return v_->idx_[p_]; }
        const T& operator*() const { return v_->val_[p_]; }
        const_iterator& operator++() {
            ++p_;
            return *this;
        }
        bool operator!=(const const_iterator& o) const { return p_ != o.p_; }
        bool operator==(const const_iterator& o) const { return p_ == o.p_; }

    private:
        const compressed_vector* v_;
        size_type p_;
    };
    typedef const_iterator iterator;

    const_iterator begin() const { return const_iterator(this, 0); }
    const_iterator end() const { return const_iterator(this, idx_.size()); }

private:
    size_type size_;
    std::vector<size_type> idx_;
    std::vector<T> val_;
};

}  // namespace ublas
}  // namespace numeric
}  // namespace boost
