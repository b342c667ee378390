// Launchers of the wall-normal pass kernels (ypass.cu).
#pragma once
#include "kernels.cuh"

template <typename C>
cudaError_t launch_cheby_inplace(PencilArr arr, long long npencils, int mode, int Ny,
                                 FftTab<C> tab, cudaStream_t st);
cudaError_t launch_get_uvw(double2* const f[6], long long ps, DnsGeom g, PhysParams ph,
                           cudaStream_t st);
cudaError_t launch_rhs_nonlinear(double2* lx, double2* ly, const double2* lz, long long ps,
                                 DnsGeom g, PhysParams ph, cudaStream_t st);
cudaError_t launch_solve_eq(const double2* inv, double2* rhs, long long ps, int N,
                            long long npencils, cudaStream_t st);
template <typename C>
cudaError_t launch_y3(const double2* V, const double2* O, PencilArr out, DnsGeom g,
                      PhysParams ph, FftTab<C> tab, int* status, cudaStream_t st, int variant = VAR_AUTO,
                      bool probe = false);
// rows of the integrated right-hand sides written by y1 for the wall solve
struct RhsDims {
  int nv, no;       // rows per pencil (v / omega systems)
  long long gp;     // pencil pitch (complex)
};
// device tables for the integrated right-hand sides (y1)
struct RhsTabs {
  const double* bkcv;  // 4 x nv: rows 4.. of B^4 C_m, m = 0, 1, N-1, N (C_m cardinal polynomial of y_m)
  const double* bkco;  // 2 x no: rows 2.. of B^2 C_m, m = 0, N
  const double* cosk;  // cos(k pi / N), k = 0..N
  const double* b4;    // 5 x nv: [d][r], row r of B^4 restricted to rows 4..: weight of f_{r+4+2d-4}
  const double* b2;    // 3 x nv: [d][r], row r of B^2 restricted to rows 2..: weight of f_{r+2+2d-2}
};
template <typename C>
cudaError_t launch_y1(PencilArr lam, const double2* V, const double2* O, double2* Nvp,
                      double2* Nop, double2* gv, double2* go, RhsDims rd, RhsTabs tb, DnsGeom g,
                      PhysParams ph, FftTab<C> tabP, int boot, int* status, cudaStream_t st,
                      int variant = VAR_AUTO, bool probe = false);
// tensor-core form of y3 (y3tc.cu): Ny = 129, FP32 output; cudaErrorNotSupported
// for other sizes
cudaError_t launch_y3tc(const double2* V, const double2* O, PencilArr out, DnsGeom g, PhysParams ph,
                        const uint32_t* atab, int* status, cudaStream_t st);
// its Chebyshev table (TF32 hi/lo words, y3tc_table_words() of them)
size_t y3tc_table_words();
void y3tc_table(uint32_t* w);
