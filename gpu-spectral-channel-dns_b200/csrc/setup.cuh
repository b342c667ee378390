// Operator setup and reference-layout transpose (setup.cu).
#pragma once
#include "kernels.cuh"

void host_T_matrix(int N, double* T0, double* T2, double* T4);
void host_base_flow(int n, double U0, double U1, double U2, double* U, double* dU, double* ddU);
int gj_cluster_size(int N);
cudaError_t launch_gj_invert(int mode, long long unit0, long long nunits, DnsGeom g, PhysParams ph,
                             const double* T0, const double* T2, const double* T4,
                             const double* U, const double* ddU, double2* outAT,
                             double2* outV, double2* outO, int* status, cudaStream_t st);
cudaError_t launch_transpose_ref(int dir, double2* xyz, long long ps, double2* zxy, long long tps,
                                 DnsGeom g, cudaStream_t st);
cudaError_t launch_operator_matrices(long long p0, long long np, DnsGeom g, PhysParams ph,
                                     const double* T0, const double* T2, const double* T4,
                                     const double* U, const double* ddU, double2* outV,
                                     double2* outO, cudaStream_t st);
cudaError_t launch_solve_residual(const double2* bv, const double2* bo, const double2* xv, const double2* xo,
                                  long long ps, DnsGeom g, PhysParams ph, const double* T0,
                                  const double* T2, const double* T4, const double* U, const double* ddU,
                                  double* per, cudaStream_t st);
