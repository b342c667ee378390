// Test infrastructure: the two dense matrix routines of the reference's
// source/matrix_op.cpp (include/matrix_op.h), written here without Eigen
// (absent from this image) so that the reference program builds from its
// own sources for the whole-step pin (oracle/ref_build/build_ref_program.py).
//
//   inverse(mat, N)     mat <- mat^-1, row-major N x N complex (the reference
//                       calls Eigen's inverse(), source/matrix_op.cpp:22-27);
//                       here Gauss-Jordan elimination with partial pivoting
//   m_multi_v(mat, v)   v <- mat v (source/matrix_op.cpp:68-78)
#include <cmath>
#include <complex>
#include <vector>

#include "matrix_op.h"

typedef std::complex<double> zc;

int inverse(cuRPCF::complex* mat, int N) {
  zc* a = reinterpret_cast<zc*>(mat);
  std::vector<zc> inv((size_t)N * N, zc(0.0, 0.0));
  for (int i = 0; i < N; ++i) inv[(size_t)i * N + i] = 1.0;
  for (int k = 0; k < N; ++k) {
    int piv = k;
    double best = std::abs(a[(size_t)k * N + k]);
    for (int i = k + 1; i < N; ++i) {
      const double v = std::abs(a[(size_t)i * N + k]);
      if (v > best) {
        best = v;
        piv = i;
      }
    }
    if (best == 0.0) return 1;
    if (piv != k)
      for (int j = 0; j < N; ++j) {
        std::swap(a[(size_t)k * N + j], a[(size_t)piv * N + j]);
        std::swap(inv[(size_t)k * N + j], inv[(size_t)piv * N + j]);
      }
    const zc d = 1.0 / a[(size_t)k * N + k];
    for (int j = 0; j < N; ++j) {
      a[(size_t)k * N + j] *= d;
      inv[(size_t)k * N + j] *= d;
    }
    for (int i = 0; i < N; ++i) {
      if (i == k) continue;
      const zc f = a[(size_t)i * N + k];
      if (f == zc(0.0, 0.0)) continue;
      for (int j = 0; j < N; ++j) {
        a[(size_t)i * N + j] -= f * a[(size_t)k * N + j];
        inv[(size_t)i * N + j] -= f * inv[(size_t)k * N + j];
      }
    }
  }
  for (size_t i = 0; i < (size_t)N * N; ++i) a[i] = inv[i];
  return 0;
}

int m_multi_v(cuRPCF::complex* mat, cuRPCF::complex* v, const int N) {
  const zc* m = reinterpret_cast<const zc*>(mat);
  zc* x = reinterpret_cast<zc*>(v);
  std::vector<zc> y((size_t)N);
  for (int i = 0; i < N; ++i) {
    zc s(0.0, 0.0);
    for (int j = 0; j < N; ++j) s += m[(size_t)i * N + j] * x[j];
    y[i] = s;
  }
  for (int i = 0; i < N; ++i) x[i] = y[i];
  return 0;
}
