// Launchers of the spanwise / streamwise pass kernels (zxpass.cu).
#pragma once
#include "kernels.cuh"

template <typename C>
cudaError_t launch_zb(PencilArr in, RowArr out, int nf, DnsGeom g, FftTab<C> tab, cudaStream_t st,
                      int* status = nullptr, int variant = VAR_AUTO, bool probe = false);
template <typename C>
cudaError_t launch_zf(RowArr in, PencilArr out, int nf, DnsGeom g, FftTab<C> tab, cudaStream_t st,
                      int* status = nullptr, int variant = VAR_AUTO, bool probe = false);
template <typename C>
cudaError_t launch_x_fused(RowArr in, RowArr out, DnsGeom g, FftTab<C> tab, const double* Uy,
                           double Ro, int* status, cudaStream_t st, int variant = VAR_AUTO,
                           bool probe = false, const double* runs = nullptr);
template <typename C>
cudaError_t launch_x_c2r(RowArr in, T_of<C>* outr, long long rps, long long nrows, DnsGeom g,
                         FftTab<C> tab, cudaStream_t st);
template <typename C>
cudaError_t launch_x_r2c(const T_of<C>* inr, long long rps, RowArr out, long long nrows,
                         DnsGeom g, FftTab<C> tab, double scale, cudaStream_t st);
cudaError_t launch_lamb_rows(const double* const in6[6], double* const out3[3], long long rps,
                             long long nrows, DnsGeom g, const double* Uy, double Ro,
                             cudaStream_t st);
