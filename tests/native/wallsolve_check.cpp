// CPU test wrapper around the host half of the banded wall-normal solve
// (gpu-spectral-channel-dns_b200/csrc/wallsolve_host.cpp).  Built by
// tests/test_wallsolve_host.py with g++ into a temporary shared library and
// compared there with the oracle's dense collocation systems.
#include <cmath>
#include <vector>

#include "../../gpu-spectral-channel-dns_b200/csrc/wallsolve.h"

using wall::cx;

namespace {
// Gauss-Lobatto values -> Chebyshev coefficients (the reference's no-pad
// p2s, source/transform.cu:680-748), evaluated directly in long double
void p2s(int N, const cx* v, cx* c) {
  const long double PI = 3.141592653589793238462643383279502884L;
  for (int k = 0; k <= N; ++k) {
    long double sr = 0, si = 0;
    for (int j = 0; j <= N; ++j) {
      const long double w = (j == 0 || j == N) ? 0.5L : 1.0L;
      const long double cs = cosl(PI * (long double)(((long long)j * k) % (2LL * N)) / N);
      sr += w * v[j].re * cs;
      si += w * v[j].im * cs;
    }
    long double s = 2.0L / N;
    if (k == 0 || k == N) s *= 0.5L;
    c[k] = cx{(double)(sr * s), (double)(si * s)};
  }
}
}  // namespace

extern "C" {

// band of a family: out = {n, nb, nd, kl, ku}
int ws_band(int eq, int N, int delta, int* out) {
  wall::Family f;
  wall::build_family(eq, N, delta, f);
  int kl, ku;
  wall::family_band(f, f.nd, &kl, &ku);
  out[0] = f.n; out[1] = f.nb; out[2] = f.nd; out[3] = kl; out[4] = ku;
  return 0;
}

// Solve the collocation system of equation family `eq` for the right-hand
// side rows r (N+1 complex, the reference's row layout: rows below the
// first equation row are boundary rows and ignored).  The system is stored
// in the shape of family `shape_eq` (a different family embeds the mean
// modes the way the device packing does).  a: N+1 Chebyshev coefficients.
int ws_solve(int eq, int shape_eq, int N, int delta, double Re, double dt, double kmn, double al,
             double U0, double U1, double U2, const double* r, double* a) {
  wall::Family f, fs;
  wall::build_family(eq, N, delta, f);
  wall::build_family(shape_eq, N, delta, fs);
  int kl, ku, kl2, ku2;
  wall::family_band(fs, fs.nd, &kl, &ku);
  wall::family_band(f, fs.nd, &kl2, &ku2);
  wall::Shape sh{fs.n, kl > kl2 ? kl : kl2, ku > ku2 ? ku : ku2, fs.nd};
  wall::Prepared p;
  if (!wall::prepare(f, sh, p)) return 1;
  std::vector<cx> sig(f.nterms), L((size_t)sh.n * sh.kl), U((size_t)sh.n * (1 + sh.ku + sh.nd));
  wall::sigma(f, Re, dt, kmn, al, U0, U1, U2, sig.data());
  if (!wall::factor(p, sig.data(), L.data(), U.data())) return 2;
  // rows -> values at the collocated Gauss-Lobatto points, zero elsewhere
  const int off = (eq == wall::EQ_V) ? 2 : 1;
  const int m0 = off, m1 = N - off;
  std::vector<cx> vals(N + 1, cx{0, 0}), rho(N + 1), g(sh.n, cx{0, 0}), x(sh.n), c(N + 1);
  for (int m = m0; m <= m1; ++m) vals[m] = cx{r[2 * (m + off)], r[2 * (m + off) + 1]};
  p2s(N, vals.data(), rho.data());
  wall::integrate_rows(f.K, N, rho.data(), f.n, g.data());
  wall::solve(sh, L.data(), U.data(), g.data(), x.data());
  wall::recombine(eq, N, x.data(), c.data());
  for (int k = 0; k <= N; ++k) { a[2 * k] = c[k].re; a[2 * k + 1] = c[k].im; }
  return 0;
}

// Q w for the tilting table (n rows), w: N+1 complex coefficients
int ws_tilt(int N, int n, double U1, double U2, const double* w, double* out) {
  std::vector<double> Q((size_t)7 * n);
  if (!wall::tilting_table(N, n, U1, U2, Q.data())) return 1;
  for (int r = 0; r < n; ++r) {
    double sr = 0, si = 0;
    for (int j = 0; j < 7; ++j) {
      const int k = r - 1 + j;
      if (k < 0 || k > N) continue;
      sr += Q[(size_t)7 * r + j] * w[2 * k];
      si += Q[(size_t)7 * r + j] * w[2 * k + 1];
    }
    out[2 * r] = sr;
    out[2 * r + 1] = si;
  }
  return 0;
}

// rows K .. K+n-1 of B^K applied to the interpolant of Gauss-Lobatto values
int ws_integrate_values(int K, int N, int n, const double* vals, double* g) {
  std::vector<cx> v(N + 1), rho(N + 1), gg(n);
  for (int k = 0; k <= N; ++k) v[k] = cx{vals[2 * k], vals[2 * k + 1]};
  p2s(N, v.data(), rho.data());
  wall::integrate_rows(K, N, rho.data(), n, gg.data());
  for (int r = 0; r < n; ++r) { g[2 * r] = gg[r].re; g[2 * r + 1] = gg[r].im; }
  return 0;
}

// max |stencil - integrate_rows| over random vectors, K = 4 and 2
double ws_stencil_err(int N, int n) {
  std::vector<double> b4((size_t)5 * n), b2((size_t)3 * n);
  wall::integration_stencils(N, n, b4.data(), b2.data());
  std::vector<cx> f(N + 1), g4(n), g2(n);
  unsigned s = 12345;
  for (auto& x : f) {
    s = s * 1103515245u + 12345u;
    x.re = (double)(s >> 8) / (1 << 24) - 0.5;
    s = s * 1103515245u + 12345u;
    x.im = (double)(s >> 8) / (1 << 24) - 0.5;
  }
  wall::integrate_rows(4, N, f.data(), n, g4.data());
  wall::integrate_rows(2, N, f.data(), n, g2.data());
  auto fg = [&](int k) { return (k >= 0 && k <= N) ? f[k] : cx{0, 0}; };
  double err = 0, mx = 0;
  for (int r = 0; r < n; ++r) {
    cx a{0, 0}, b{0, 0};
    for (int d = 0; d < 5; ++d) {
      const cx v = fg(r + 4 + 2 * d - 4);
      a.re += v.re * b4[5 * r + d];
      a.im += v.im * b4[5 * r + d];
    }
    for (int d = 0; d < 3; ++d) {
      const cx v = fg(r + 2 + 2 * d - 2);
      b.re += v.re * b2[3 * r + d];
      b.im += v.im * b2[3 * r + d];
    }
    err = std::fmax(err, std::fmax(std::hypot(a.re - g4[r].re, a.im - g4[r].im),
                                   std::hypot(b.re - g2[r].re, b.im - g2[r].im)));
    mx = std::fmax(mx, std::fmax(std::hypot(g4[r].re, g4[r].im), std::hypot(g2[r].re, g2[r].im)));
  }
  return err / mx;
}

}  // extern "C"
