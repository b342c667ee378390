// Banded form of the wall-normal Crank-Nicolson systems of the v-omega_y step.
//
// The reference solves, per Fourier mode, the dense Chebyshev collocation
// systems built by _get_coefficient_v / _get_coefficient_omega /
// _get_coef_u0 (source/coefficient.cu:7-86) through explicit inverses
// (source/solver.cpp:107-123, matrix_op.cpp:22-78).  The same solutions are
// obtained here from an equivalent sparse formulation:
//
//   * unknowns: coefficients b_j of a basis that satisfies the wall
//     conditions exactly (v: phi_j = T_j - 2(j+2)/(j+3) T_{j+2}
//     + (j+1)/(j+3) T_{j+4}, clamped; omega_y and the mean modes:
//     phi_j = T_{j+2} - T_j, Dirichlet), plus the few coefficients of the
//     residual that the collocation leaves free (h_l multiplying
//     T_N'(y) T_l(y), l = 0..deg(U)+1, and for v the two cardinal-like
//     polynomials T_N'(y)/(y - y_m), m = 1, N-1, at the two interior
//     Gauss-Lobatto points v does not collocate);
//   * equations: the K-fold Chebyshev integral (K = 4 for v, 2 otherwise)
//     of  L u - R = residual,  R the interpolant of the collocation
//     right-hand side, rows K .. K+n-1.
//
// Integration turns D^K into the identity and y, y^2 (the base flow) and
// the lower derivatives into a few diagonals, so each system is banded
// (v: kl = deg U + 4, ku = 2 deg U + 8, two dense trailing columns; omega:
// kl = deg U + 2, ku = 2 deg U + 4) and is factorised without pivoting.
// Host code only: construction, factorisation, packing.  The per-step
// solve runs on the device (wallsolve.cu).
#pragma once
#include <string>
#include <vector>

namespace wall {

struct cx {
  double re, im;
};

enum { EQ_V = 0, EQ_OMEGA = 1, EQ_MEAN = 2 };

// One equation family: system matrix = sum_t sigma_t G_t + F, with G_t
// pencil-independent real matrices acting on the basis unknowns and F the
// fixed residual columns.
struct Family {
  int eq = 0, N = 0, K = 0, delta = 0;
  int n = 0;    // unknowns = equations
  int nb = 0;   // basis unknowns (the rest are residual coefficients)
  int nd = 0;   // dense trailing columns (2 for v)
  int nterms = 0;
  std::vector<int> term;  // index of each term in the family's full term list
  std::vector<double> G;  // nterms x n x n, row-major
  std::vector<double> F;  // n x n
};

// Storage shape of one packed system: n rows, lower band kl, upper band ku
// over the first n - nd columns, nd dense trailing columns.
struct Shape {
  int n, kl, ku, nd;
};

// degree of the base-flow polynomial U0 + U1 y + U2 y^2
int base_degree(double U1, double U2);

void build_family(int eq, int N, int delta, Family& f);

// band actually occupied by the family (over columns < n - nd)
void family_band(const Family& f, int nd, int* kl, int* ku);

// pencil weights sigma_t for wavenumber^2 kmn and streamwise wavenumber al
void sigma(const Family& f, double Re, double dt, double kmn, double al, double U0, double U1,
           double U2, cx* s);

// The family's matrices in band storage for one packed shape: the family
// sits in the top-left corner of an sh.n x sh.n system (identity on the rest
// of the diagonal).  prepare() fails if an entry falls outside the shape.
struct Prepared {
  Shape sh;
  int nf = 0, nterms = 0;
  std::vector<double> band;   // (nterms + 1) x n x (kl + ku + 1); term nterms is F
  std::vector<double> dense;  // (nterms + 1) x n x nd
};
bool prepare(const Family& f, const Shape& sh, Prepared& p);

// Assemble sum_t sig_t G_t + F and factor it without pivoting.
// L: n x kl (row i, entry e <-> column i - kl + e),
// U: n x (1 + ku + nd) (1/diagonal, upper band, dense columns).
// Returns false on a zero pivot.
bool factor(const Prepared& p, const cx* sig, cx* L, cx* U);

// Reference solve with factors from factor(): g (n) -> x (n)
void solve(const Shape& sh, const cx* L, const cx* U, const cx* g, cx* x);

// rows K .. K+n-1 of B^K rho, rho of length N+1 (B: Chebyshev integration)
void integrate_rows(int K, int N, const cx* rho, int n, cx* g);

// rows K .. K+n-1 of B^K C_m, C_m the coefficients of the cardinal
// polynomial of the Gauss-Lobatto point y_m (1 at y_m, 0 at the others)
void cardinal_rows(int N, int m, int K, int n, double* out);

// Rows 4..4+n-1 of B^4 and 2..2+n-1 of B^2 as stencils on an (N+1)-coefficient
// vector f: (B^4 f)_{r+4} = sum_d b4[5r + d/2 + 2] f_{r+4+d}, d = -4,-2,0,2,4;
// (B^2 f)_{r+2} = sum_d b2[3r + d/2 + 1] f_{r+2+d}, d = -2,0,2.
void integration_stencils(int N, int n, double* b4, double* b2);

// Chebyshev coefficients (N+1) from basis unknowns: v or Dirichlet recombination
void recombine(int eq, int N, const cx* x, cx* a);

// Tilting operator of the omega_y equation in integrated form:
// T_r = sum_j Q[7 r + j] w_{r-1+j}, r = 0..n-1, is row r+2 of B^2 applied to
// the Gauss-Lobatto interpolant of U'(y) w(y) (w given by its N+1
// coefficients).  Returns false if an entry falls outside the 7 diagonals.
bool tilting_table(int N, int n, double U1, double U2, double* Q);

// Number of streamed records (rows x entries) per slot for the packed
// v and omega shapes, and the packing of one group of 16 slots.
struct Packing {
  Shape v, o;
  int e0, e1, e2, e3;  // entries per row: v forward, v backward, omega forward, omega backward
  long long group_complex;  // complex values per group of 16 slots
};
Packing make_packing(const Shape& v, const Shape& o);
// write slot q (0..15) of a group: v factors (Lv, Uv) and omega factors (Lo, Uo)
void pack_slot(const Packing& pk, int q, const cx* Lv, const cx* Uv, const cx* Lo, const cx* Uo,
               cx* group);

// Operator slots of a grid: (kx, kz'), kx in [0, Kx), kz' in [0, Kh), slot
// kz' * Kx + kx; the pencils kz' and Nz - kz' share a slot (the operators
// depend on the spanwise wavenumber only through its square).
struct Grid {
  int N, Kx, Nz, Kh;
  double aphi, beta, Re, dt, U0, U1, U2;
  int kz0 = 0, nkz = -1;  // the slots kz' in [kz0, kz0 + nkz) only (nkz < 0: all Kh)
};
// Factor every slot for the packed shapes v and o and write the groups of 16
// slots (slot 0, the mean modes, holds the mean-mode system in both shapes;
// padding slots of the last group hold identity factors).  Returns "" or an
// error message.
std::string pack_grid(const Grid& gr, const Shape& v, const Shape& o, std::vector<cx>& out,
                      int threads);

}  // namespace wall
