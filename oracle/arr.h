// Oracle support: Fortran-indexed 3-D and 2-D arrays.
//
// TEST INFRASTRUCTURE ONLY.  This directory is the CPU oracle that the
// parity tests, the smoke check and the CPU-baseline leg of bench.py use as
// the checker.  Nothing in the product library (cress_b200/) links or calls it.
//
// Layout follows the reference's explicit-shape dummies
//   real :: a(0:ni+1, 0:nj+1, 1:nk)       (SrcOrig/hevi.f90:106-160)
// stored column-major with x fastest, so a(i,j,k) sits at
//   i + (ni+2)*(j + (nj+2)*(k-1)).
#pragma once
#include <cstddef>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace oracle {

template <class R>
struct F3 {
  int ni = 0, nj = 0, nk = 0;
  std::vector<R> d;
  F3() = default;
  F3(int ni_, int nj_, int nk_, R v = R(0)) { resize(ni_, nj_, nk_, v); }
  void resize(int ni_, int nj_, int nk_, R v = R(0)) {
    ni = ni_; nj = nj_; nk = nk_;
    d.assign((size_t)(ni + 2) * (nj + 2) * nk, v);
  }
  size_t size() const { return d.size(); }
  inline R& operator()(int i, int j, int k) {
    return d[(size_t)i + (size_t)(ni + 2) * ((size_t)j + (size_t)(nj + 2) * (size_t)(k - 1))];
  }
  inline const R& operator()(int i, int j, int k) const {
    return d[(size_t)i + (size_t)(ni + 2) * ((size_t)j + (size_t)(nj + 2) * (size_t)(k - 1))];
  }
  void fill(R v) { std::fill(d.begin(), d.end(), v); }
  template <class S>
  void load(const S* p) { for (size_t n = 0; n < d.size(); ++n) d[n] = (R)p[n]; }
  template <class S>
  void store(S* p) const { for (size_t n = 0; n < d.size(); ++n) p[n] = (S)d[n]; }
};

// real :: a(0:ni+1, 0:nj+1)
template <class R>
struct F2 {
  int ni = 0, nj = 0;
  std::vector<R> d;
  F2() = default;
  F2(int ni_, int nj_, R v = R(0)) { resize(ni_, nj_, v); }
  void resize(int ni_, int nj_, R v = R(0)) {
    ni = ni_; nj = nj_;
    d.assign((size_t)(ni + 2) * (nj + 2), v);
  }
  inline R& operator()(int i, int j) { return d[(size_t)i + (size_t)(ni + 2) * (size_t)j]; }
  inline const R& operator()(int i, int j) const { return d[(size_t)i + (size_t)(ni + 2) * (size_t)j]; }
  void fill(R v) { std::fill(d.begin(), d.end(), v); }
};

}  // namespace oracle
