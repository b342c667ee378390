// C entry points over the reference's own CPU operator / right-hand-side
// functions (source/coefficient.cu, source/linear.cpp), compiled from the
// reference's sources by oracle/ref_build/Makefile into oracle/_ref.
// TEST INFRASTRUCTURE ONLY: used by tests/test_oracle_vs_reference.py to
// check the NumPy oracle against the reference's code, value for value.
#include "data.h"
#include "coefficient.cuh"
#include "linear.h"

extern "C" {
int ref_get_T_matrix(int N, double* T0, double* T2, double* T4) { return get_T_matrix(N, T0, T2, T4); }
int ref_get_U(int N, double* U, double* dU, double* ddU) { return get_U(N, U, dU, ddU); }
int ref_coef_v(void* m, int N, double* U, double* ddU, double* T0, double* T2, double* T4,
               double Re, double dt, double kmn, double alpha) {
  return _get_coefficient_v((cuRPCF::complex*)m, N, U, ddU, T0, T2, T4, Re, dt, kmn, alpha);
}
int ref_coef_omega(void* m, int N, double* U, double* T0, double* T2, double* T4, double Re,
                   double dt, double kmn, double alpha) {
  return _get_coefficient_omega((cuRPCF::complex*)m, N, U, T0, T2, T4, Re, dt, kmn, alpha);
}
int ref_coef_u0(void* m, int N, double* T0, double* T2, double Re, double dt) {
  return _get_coef_u0((cuRPCF::complex*)m, N, T0, T2, Re, dt);
}
int ref_linear_v(void* rhs_v, void* nl, void* nl_p, void* rhs_v_p, int N, double* U, double* ddU,
                 double* T0, double* T2, double* T4, double Re, double dt, double kmn, double alpha) {
  return _get_linear_v((cuRPCF::complex*)rhs_v, (cuRPCF::complex*)nl, (cuRPCF::complex*)nl_p,
                       (cuRPCF::complex*)rhs_v_p, N, U, ddU, T0, T2, T4, Re, dt, kmn, alpha);
}
int ref_linear_omega_y(void* rhs_o, void* nl, void* nl_p, void* rhs_v, void* rhs_v_p, int N,
                       double* U, double* dU, double* T0, double* T2, double Re, double dt,
                       double kmn, double alpha, double beta) {
  return _get_linear_omega_y((cuRPCF::complex*)rhs_o, (cuRPCF::complex*)nl, (cuRPCF::complex*)nl_p,
                             (cuRPCF::complex*)rhs_v, (cuRPCF::complex*)rhs_v_p, N, U, dU, T0, T2,
                             Re, dt, kmn, alpha, beta);
}
int ref_linear_u0(void* rhs_u0, void* l0, void* l0_p, int N, double* T0, double* T2, double Re, double dt) {
  return _get_linear_u0((cuRPCF::complex*)rhs_u0, (cuRPCF::complex*)l0, (cuRPCF::complex*)l0_p, N,
                        T0, T2, Re, dt);
}
}
