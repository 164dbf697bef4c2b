// TEST INFRASTRUCTURE ONLY -- stand-in for the reference's missing counter.h
// (main/optim_par.cpp:1): range<T>(a, b) with counting iterators, used as
// for_each(policy, rng.begin(), rng.end(), functor) at main/optim_par.cpp:633.
#pragma once
#include <cstddef>
#include <iterator>

template <class T>
class range {
 public:
  class iterator {
   public:
    using iterator_category = std::random_access_iterator_tag;
    using value_type = T;
    using difference_type = std::ptrdiff_t;
    using pointer = const T*;
    using reference = const T&;
    explicit iterator(T v = T()) : v_(v) {}
    reference operator*() const { return v_; }
    iterator& operator++() { ++v_; return *this; }
    iterator operator++(int) { iterator t = *this; ++v_; return t; }
    iterator& operator--() { --v_; return *this; }
    iterator& operator+=(difference_type d) { v_ += d; return *this; }
    iterator operator+(difference_type d) const { return iterator(v_ + d); }
    iterator operator-(difference_type d) const { return iterator(v_ - d); }
    difference_type operator-(const iterator& o) const { return difference_type(v_) - difference_type(o.v_); }
    T operator[](difference_type d) const { return v_ + d; }
    bool operator==(const iterator& o) const { return v_ == o.v_; }
    bool operator!=(const iterator& o) const { return v_ != o.v_; }
    bool operator<(const iterator& o) const { return v_ < o.v_; }

   private:
    T v_;
  };
  range(T a, T b) : a_(a), b_(b) {}
  iterator begin() const { return iterator(a_); }
  iterator end() const { return iterator(b_); }

 private:
  T a_, b_;
};
