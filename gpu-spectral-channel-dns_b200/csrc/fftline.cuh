// Line-FFT front end used by the pass kernels.
//
// FLine<C, L> with L > 0 uses the compile-time FFT (fft2.cuh: natural-order
// input at padded positions fpos(n)); with L == 0 it falls back to the
// runtime-length FFT (fft.cuh: digit-reversed input, plan in the table).
// with_len() dispatches a runtime length to the compile-time instantiations
// of the grid sizes this library is built for.
#pragma once
#include <type_traits>
#include "fft.cuh"
#include "fft2.cuh"
#include "kernels.cuh"

// lengths instantiated per use: streamwise / spanwise lines, padded and
// unpadded Chebyshev extensions (2 (Py-1) = mz and 2 (Ny-1) = mz/2)
#define FFT_XZ_LENGTHS(X) X(48) X(96) X(144) X(192) X(288) X(384) X(576)
#define FFT_M_LENGTHS(X) X(128) X(192) X(256) X(384) X(512) X(768)
#define FFT_M0_LENGTHS(X) X(64) X(96) X(128) X(192) X(256) X(384)

template <typename C, int L>
struct FLine {
  DNS_HD static int in_pos(const FftTab<C>& t, int n) {
    if (L > 0) return fpos(n);
    return t.drev[n];
  }
  DNS_HD static int out_pos(int k) { return L > 0 ? fpos(k) : k; }
  DNS_HD static int stride(int Lr) { return L > 0 ? fpad_len(L) : Lr; }
#ifdef __CUDACC__
  template <bool INV>
  __device__ __forceinline__ static void fft(C* buf, int nb, int ls, const FftTab<C>& t) {
    if constexpr (L > 0) fft2<C, L, INV>(buf, nb, ls, t.tw);
    else fft_batch<C, INV>(buf, nb, ls, t.plan, t.tw);
  }
#endif
};

#define DNS_LCASE(n) case n: return f(std::integral_constant<int, n>());
template <typename F> cudaError_t with_len_xz(int L, F&& f) {
  switch (L) { FFT_XZ_LENGTHS(DNS_LCASE) default: return f(std::integral_constant<int, 0>()); }
}
template <typename F> cudaError_t with_len_m(int L, F&& f) {
  switch (L) { FFT_M_LENGTHS(DNS_LCASE) default: return f(std::integral_constant<int, 0>()); }
}
template <typename F> cudaError_t with_len_m0(int L, F&& f) {
  switch (L) { FFT_M0_LENGTHS(DNS_LCASE) default: return f(std::integral_constant<int, 0>()); }
}
