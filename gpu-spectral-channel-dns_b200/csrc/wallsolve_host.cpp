// Host side of the banded wall-normal solve: family construction,
// factorisation without pivoting, tilting table and packing for the device.
// The systems restated here are those of source/coefficient.cu:7-86 (v,
// omega_y, mean modes) with the right-hand sides of source/linear.cpp:86-205;
// see wallsolve.h for the formulation.
#include "wallsolve.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>

namespace wall {
namespace {

inline cx cadd(cx a, cx b) { return cx{a.re + b.re, a.im + b.im}; }
inline cx csub(cx a, cx b) { return cx{a.re - b.re, a.im - b.im}; }
inline cx cmul(cx a, cx b) { return cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cx cscale(cx a, double s) { return cx{a.re * s, a.im * s}; }
inline cx cinv(cx a) {
  const double d = a.re * a.re + a.im * a.im;
  return cx{a.re / d, -a.im / d};
}
inline bool cnz(cx a) { return a.re != 0.0 || a.im != 0.0; }

typedef std::vector<double> Vec;

// Chebyshev integration: (B x)_k = (c_{k-1} x_{k-1} - x_{k+1}) / (2k), k >= 1,
// c_0 = 2, (B x)_0 = 0 (the integration constant is not represented).
Vec int_B(const Vec& x) {
  const size_t m = x.size();
  Vec y(m, 0.0);
  for (size_t k = 1; k < m; ++k) {
    const double ck1 = (k == 1) ? 2.0 : 1.0;
    const double xp = (k + 1 < m) ? x[k + 1] : 0.0;
    y[k] = (ck1 * x[k - 1] - xp) / (2.0 * (double)k);
  }
  return y;
}

// multiplication by y: y T_0 = T_1, y T_j = (T_{j+1} + T_{j-1}) / 2
Vec mul_y(const Vec& x) {
  const size_t m = x.size();
  Vec y(m, 0.0);
  for (size_t j = 0; j < m; ++j) {
    if (x[j] == 0.0) continue;
    if (j == 0) {
      if (m > 1) y[1] += x[0];
    } else {
      if (j + 1 < m) y[j + 1] += 0.5 * x[j];
      y[j - 1] += 0.5 * x[j];
    }
  }
  return y;
}

Vec int_B_pow(Vec x, int p) {
  for (int i = 0; i < p; ++i) x = int_B(x);
  return x;
}

// T_N T_l = (T_{N+l} + T_{|N-l|}) / 2
void add_TN_times(int N, int l, double s, Vec& out) {
  out[N + l] += 0.5 * s;
  out[std::abs(N - l)] += 0.5 * s;
}

// basis column j: coefficients of phi_j
Vec basis(int eq, int j, size_t m) {
  Vec v(m, 0.0);
  if (eq == EQ_V) {
    v[j] = 1.0;
    v[j + 2] = -2.0 * (j + 2) / (double)(j + 3);
    v[j + 4] = (double)(j + 1) / (double)(j + 3);
  } else {
    v[j] = -1.0;
    v[j + 2] = 1.0;
  }
  return v;
}

// Chebyshev coefficients of l_m(y) = T_N'(y) / (y - y_m) from its values at
// the Gauss-Lobatto points: N^2/(1-y_m) at y=1, (-1)^(N+1) N^2/(-1-y_m) at
// y=-1, T_N''(y_m) = -(-1)^m N^2 / sin^2(m pi/N) at y_m, zero elsewhere.
Vec cardinal_coeffs(int N, int m) {
  const long double PI = 3.141592653589793238462643383279502884L;
  const long double NN = (long double)N * N;
  const long double th = PI * m / N;
  const long double s_half = sinl(th / 2), c_half = cosl(th / 2);
  const long double v0 = NN / (2 * s_half * s_half);               // N^2 / (1 - y_m)
  const long double vN = ((N + 1) % 2 ? -1.0L : 1.0L) * NN / (-2 * c_half * c_half);
  const long double sm = sinl(th);
  const long double vm = -((m % 2) ? -1.0L : 1.0L) * NN / (sm * sm);
  Vec c(N + 1);
  for (int k = 0; k <= N; ++k) {
    const long long r = ((long long)m * k) % (2LL * N);
    const long double ck = (v0 + ((k % 2) ? -vN : vN)) / N + 2.0L / N * vm * cosl(PI * r / N);
    c[k] = (double)((k == 0 || k == N) ? ck / 2 : ck);
  }
  return c;
}

}  // namespace

int base_degree(double U1, double U2) { return U2 != 0.0 ? 2 : (U1 != 0.0 ? 1 : 0); }

void build_family(int eq, int N, int delta, Family& f) {
  if (eq == EQ_MEAN) delta = 0;
  f.eq = eq;
  f.N = N;
  f.delta = delta;
  f.K = (eq == EQ_V) ? 4 : 2;
  f.n = N + delta + 1;
  f.nb = (eq == EQ_V) ? N - 3 : N - 1;
  f.nd = (eq == EQ_V) ? 2 : 0;
  // full term lists: (power of B, power of y, base-flow degree the weight
  // needs); term 0 is the identity (the integrated highest derivative).
  // Terms whose weight vanishes for this base flow are left out.
  static const int tv[9][3] = {{0, 0, 0}, {2, 0, 0}, {2, 1, 1}, {2, 2, 2}, {3, 0, 1},
                               {3, 1, 2}, {4, 0, 0}, {4, 1, 1}, {4, 2, 2}};
  static const int to[4][3] = {{0, 0, 0}, {2, 0, 0}, {2, 1, 1}, {2, 2, 2}};
  static const int tm[2][3] = {{0, 0, 0}, {2, 0, 0}};
  const int(*all)[3] = (eq == EQ_V) ? tv : (eq == EQ_OMEGA ? to : tm);
  const int nall = (eq == EQ_V) ? 9 : (eq == EQ_OMEGA ? 4 : 2);
  f.term.clear();
  for (int t = 0; t < nall; ++t)
    if (all[t][2] <= delta) f.term.push_back(t);
  f.nterms = (int)f.term.size();
  const int n = f.n, K = f.K;
  const size_t m = (size_t)N + delta + K + 12;
  f.G.assign((size_t)f.nterms * n * n, 0.0);
  f.F.assign((size_t)n * n, 0.0);
  for (int j = 0; j < f.nb; ++j) {
    const Vec phi = basis(eq, j, m);
    for (int t = 0; t < f.nterms; ++t) {
      Vec v = phi;
      for (int q = 0; q < all[f.term[t]][1]; ++q) v = mul_y(v);
      v = int_B_pow(v, all[f.term[t]][0]);
      for (int r = 0; r < n; ++r) f.G[((size_t)t * n + r) * n + j] = v[K + r];
    }
  }
  // residual columns h_l: -B^K (T_N' T_l) = -(B^{K-1}(T_N T_l) - B^K(T_N T_l')) on rows >= K
  for (int l = 0; l < delta + 2; ++l) {
    Vec p(m, 0.0), q(m, 0.0);
    add_TN_times(N, l, 1.0, p);
    for (int i = l - 1; i >= 0; i -= 2) add_TN_times(N, i, (i == 0 ? 0.5 : 1.0) * 2.0 * l, q);
    const Vec a = int_B_pow(p, K - 1), b = int_B_pow(q, K);
    for (int r = 0; r < n; ++r) f.F[(size_t)r * n + f.nb + l] = -(a[K + r] - b[K + r]);
  }
  if (eq == EQ_V) {
    const int ms[2] = {1, N - 1};
    for (int d = 0; d < 2; ++d) {
      Vec c = cardinal_coeffs(N, ms[d]);
      c.resize(m, 0.0);
      const Vec b = int_B_pow(c, K);
      for (int r = 0; r < n; ++r) f.F[(size_t)r * n + n - 2 + d] = -b[K + r];
    }
  }
}

void family_band(const Family& f, int nd, int* kl, int* ku) {
  int lo = 0, up = 0;
  const int n = f.n;
  for (int t = 0; t <= f.nterms; ++t) {
    const double* M = (t < f.nterms) ? &f.G[(size_t)t * n * n] : f.F.data();
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n - nd; ++j)
        if (M[(size_t)i * n + j] != 0.0) {
          lo = std::max(lo, i - j);
          up = std::max(up, j - i);
        }
  }
  *kl = lo;
  *ku = up;
}

void sigma(const Family& f, double Re, double dt, double kmn, double al, double U0, double U1,
           double U2, cx* s) {
  const double c = dt * 0.5 / Re;
  const double g = al * dt * 0.5;
  cx w[9];
  if (f.eq == EQ_MEAN) {
    w[0] = cx{-c, 0.0};
    w[1] = cx{1.0, 0.0};
  } else if (f.eq == EQ_OMEGA) {
    const double sd = 1.0 + kmn * dt * 0.5 / Re;
    w[0] = cx{-c, 0.0};
    w[1] = cx{sd, g * U0};
    w[2] = cx{0.0, g * U1};
    w[3] = cx{0.0, g * U2};
  } else {
    const double s2 = 1.0 + kmn * dt / Re;
    const double s0 = kmn * (1.0 + kmn * dt * 0.5 / Re);
    w[0] = cx{-c, 0.0};
    w[1] = cx{s2, g * U0};
    w[2] = cx{0.0, g * U1};
    w[3] = cx{0.0, g * U2};
    w[4] = cx{0.0, -2.0 * g * U1};
    w[5] = cx{0.0, -4.0 * g * U2};
    w[6] = cx{-s0, -g * kmn * U0};
    w[7] = cx{0.0, -g * kmn * U1};
    w[8] = cx{0.0, -g * kmn * U2};
  }
  for (int t = 0; t < f.nterms; ++t) s[t] = w[f.term[t]];
}

bool prepare(const Family& f, const Shape& sh, Prepared& p) {
  const int n = sh.n, kl = sh.kl, ku = sh.ku, nd = sh.nd, nf = f.n;
  if (nf > n) return false;
  const int bw = kl + ku + 1;
  p.sh = sh;
  p.nf = nf;
  p.nterms = f.nterms;
  p.band.assign((size_t)(f.nterms + 1) * n * bw, 0.0);
  p.dense.assign((size_t)(f.nterms + 1) * n * std::max(nd, 1), 0.0);
  for (int t = 0; t <= f.nterms; ++t) {
    const double* M = (t < f.nterms) ? &f.G[(size_t)t * nf * nf] : f.F.data();
    for (int i = 0; i < nf; ++i)
      for (int j = 0; j < nf; ++j) {
        const double v = M[(size_t)i * nf + j];
        if (v == 0.0) continue;
        if (j >= n - nd) {
          p.dense[((size_t)t * n + i) * nd + (j - (n - nd))] = v;
        } else {
          const int d = j - i;
          if (d < -kl || d > ku) return false;
          p.band[((size_t)t * n + i) * bw + d + kl] = v;
        }
      }
  }
  return true;
}

bool factor(const Prepared& p, const cx* sig, cx* L, cx* U) {
  const int n = p.sh.n, kl = p.sh.kl, ku = p.sh.ku, nd = p.sh.nd;
  const int bw = kl + ku + 1, nc = n - nd, ue = 1 + ku + nd;
  std::vector<cx> W((size_t)n * bw, cx{0, 0}), D((size_t)n * std::max(nd, 1), cx{0, 0});
  for (int t = 0; t <= p.nterms; ++t) {
    const cx s = (t < p.nterms) ? sig[t] : cx{1.0, 0.0};
    const double* B = &p.band[(size_t)t * n * bw];
    for (size_t k = 0; k < (size_t)n * bw; ++k)
      if (B[k] != 0.0) W[k] = cadd(W[k], cscale(s, B[k]));
    if (nd) {
      const double* Dd = &p.dense[(size_t)t * n * nd];
      for (size_t k = 0; k < (size_t)n * nd; ++k)
        if (Dd[k] != 0.0) D[k] = cadd(D[k], cscale(s, Dd[k]));
    }
  }
  for (int i = p.nf; i < n; ++i) {  // identity on the padding
    if (i < nc) W[(size_t)i * bw + kl] = cx{1.0, 0.0};
    else D[(size_t)i * nd + (i - nc)] = cx{1.0, 0.0};
  }
  std::fill(L, L + (size_t)n * kl, cx{0, 0});
  std::fill(U, U + (size_t)n * ue, cx{0, 0});
  for (int j = 0; j < n; ++j) {
    const cx piv = (j < nc) ? W[(size_t)j * bw + kl] : D[(size_t)j * nd + (j - nc)];
    if (!cnz(piv)) return false;
    const cx ip = cinv(piv);
    const int iend = std::min(n - 1, j + kl);
    for (int i = j + 1; i <= iend; ++i) {
      const cx a = (j < nc) ? W[(size_t)i * bw + (j - i + kl)] : D[(size_t)i * nd + (j - nc)];
      const cx l = cmul(a, ip);
      L[(size_t)i * kl + (j - i + kl)] = l;
      if (!cnz(l)) continue;
      const int cend = std::min(j + ku, nc - 1);
      for (int c = j + 1; c <= cend; ++c)
        W[(size_t)i * bw + (c - i + kl)] =
            csub(W[(size_t)i * bw + (c - i + kl)], cmul(l, W[(size_t)j * bw + (c - j + kl)]));
      for (int d = 0; d < nd; ++d)
        if (nc + d > j) D[(size_t)i * nd + d] = csub(D[(size_t)i * nd + d], cmul(l, D[(size_t)j * nd + d]));
    }
    cx* u = U + (size_t)j * ue;
    u[0] = ip;
    for (int e = 1; e <= ku; ++e)
      if (j + e < nc) u[e] = W[(size_t)j * bw + kl + e];
    for (int d = 0; d < nd; ++d)
      if (nc + d > j) u[1 + ku + d] = D[(size_t)j * nd + d];
  }
  return true;
}

void solve(const Shape& sh, const cx* L, const cx* U, const cx* g, cx* x) {
  const int n = sh.n, kl = sh.kl, ku = sh.ku, nd = sh.nd, ue = 1 + ku + nd;
  std::vector<cx> y(n);
  for (int i = 0; i < n; ++i) {
    cx s = g[i];
    for (int e = 0; e < kl; ++e) {
      const int j = i - kl + e;
      if (j >= 0) s = csub(s, cmul(L[(size_t)i * kl + e], y[j]));
    }
    y[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {
    const cx* u = U + (size_t)i * ue;
    cx s = y[i];
    for (int e = 1; e <= ku; ++e)
      if (i + e < n) s = csub(s, cmul(u[e], x[i + e]));
    for (int d = 0; d < nd; ++d) s = csub(s, cmul(u[1 + ku + d], x[n - nd + d]));
    x[i] = cmul(u[0], s);
  }
}

void integrate_rows(int K, int N, const cx* rho, int n, cx* g) {
  const size_t m = (size_t)N + K + n + 4;
  Vec re(m, 0.0), im(m, 0.0);
  for (int k = 0; k <= N; ++k) {
    re[k] = rho[k].re;
    im[k] = rho[k].im;
  }
  re = int_B_pow(re, K);
  im = int_B_pow(im, K);
  for (int r = 0; r < n; ++r) g[r] = cx{re[K + r], im[K + r]};
}

void cardinal_rows(int N, int m, int K, int n, double* out) {
  const long double PI = 3.141592653589793238462643383279502884L;
  std::vector<cx> rho(N + 1), g(n);
  const long double wm = (m == 0 || m == N) ? 0.5L : 1.0L;
  for (int k = 0; k <= N; ++k) {
    const long long r = ((long long)m * k) % (2LL * N);
    long double c = 2.0L / N * wm * cosl(PI * r / N);
    if (k == 0 || k == N) c *= 0.5L;
    rho[k] = cx{(double)c, 0.0};
  }
  integrate_rows(K, N, rho.data(), n, g.data());
  for (int r = 0; r < n; ++r) out[r] = g[r].re;
}

void integration_stencils(int N, int n, double* b4, double* b2) {
  std::fill(b4, b4 + (size_t)5 * n, 0.0);
  std::fill(b2, b2 + (size_t)3 * n, 0.0);
  const size_t m = (size_t)N + n + 12;
  for (int k = 0; k <= N; ++k) {
    Vec e(m, 0.0);
    e[k] = 1.0;
    const Vec e2 = int_B_pow(e, 2), e4 = int_B_pow(e2, 2);
    for (int r = 0; r < n; ++r) {
      const int d4 = k - (r + 4), d2 = k - (r + 2);
      if (e4[r + 4] != 0.0 && d4 >= -4 && d4 <= 4 && (d4 & 1) == 0) b4[(size_t)5 * r + d4 / 2 + 2] = e4[r + 4];
      if (e2[r + 2] != 0.0 && d2 >= -2 && d2 <= 2 && (d2 & 1) == 0) b2[(size_t)3 * r + d2 / 2 + 1] = e2[r + 2];
    }
  }
}

void recombine(int eq, int N, const cx* x, cx* a) {
  const int nb = (eq == EQ_V) ? N - 3 : N - 1;
  auto b = [&](int j) { return (j >= 0 && j < nb) ? x[j] : cx{0, 0}; };
  for (int k = 0; k <= N; ++k) {
    if (eq == EQ_V) {
      cx s = b(k);
      if (k >= 2) s = csub(s, cscale(b(k - 2), 2.0 * k / (double)(k + 1)));
      if (k >= 4) s = cadd(s, cscale(b(k - 4), (double)(k - 3) / (double)(k - 1)));
      a[k] = s;
    } else {
      cx s = cscale(b(k), -1.0);
      if (k >= 2) s = cadd(s, b(k - 2));
      a[k] = s;
    }
  }
}

bool tilting_table(int N, int n, double U1, double U2, double* Q) {
  std::fill(Q, Q + (size_t)7 * n, 0.0);
  const size_t m = (size_t)N + n + 12;
  for (int k = 0; k <= N; ++k) {
    Vec w(m, 0.0);
    w[k] = 1.0;
    const Vec yw = mul_y(w);
    Vec f(m, 0.0);
    for (size_t i = 0; i < m; ++i) f[i] = U1 * w[i] + 2.0 * U2 * yw[i];
    // Gauss-Lobatto interpolation folds T_{N+1} onto T_{N-1}
    f[N - 1] += f[N + 1];
    f[N + 1] = 0.0;
    const Vec h = int_B_pow(f, 2);
    for (int r = 0; r < n; ++r) {
      const double v = h[r + 2];
      if (v == 0.0) continue;
      const int j = k - r + 1;
      if (j < 0 || j > 6) return false;
      Q[(size_t)7 * r + j] = v;
    }
  }
  return true;
}

Packing make_packing(const Shape& v, const Shape& o) {
  Packing p;
  p.v = v;
  p.o = o;
  p.e0 = v.kl;
  p.e1 = 1 + v.ku + v.nd;
  p.e2 = o.kl;
  p.e3 = 1 + o.ku + o.nd;
  p.group_complex = 16LL * ((long long)v.n * (p.e0 + p.e1) + (long long)o.n * (p.e2 + p.e3));
  return p;
}

void pack_slot(const Packing& pk, int q, const cx* Lv, const cx* Uv, const cx* Lo, const cx* Uo,
               cx* group) {
  const int nv = pk.v.n, no = pk.o.n;
  size_t off = 0;
  for (int i = 0; i < nv; ++i)
    for (int e = 0; e < pk.e0; ++e) group[off + ((size_t)i * pk.e0 + e) * 16 + q] = Lv[(size_t)i * pk.e0 + e];
  off += (size_t)16 * nv * pk.e0;
  for (int r = 0; r < nv; ++r) {
    const int i = nv - 1 - r;
    for (int e = 0; e < pk.e1; ++e) group[off + ((size_t)r * pk.e1 + e) * 16 + q] = Uv[(size_t)i * pk.e1 + e];
  }
  off += (size_t)16 * nv * pk.e1;
  for (int i = 0; i < no; ++i)
    for (int e = 0; e < pk.e2; ++e) group[off + ((size_t)i * pk.e2 + e) * 16 + q] = Lo[(size_t)i * pk.e2 + e];
  off += (size_t)16 * no * pk.e2;
  for (int r = 0; r < no; ++r) {
    const int i = no - 1 - r;
    for (int e = 0; e < pk.e3; ++e) group[off + ((size_t)r * pk.e3 + e) * 16 + q] = Uo[(size_t)i * pk.e3 + e];
  }
}

std::string pack_grid(const Grid& gr, const Shape& v, const Shape& o, std::vector<cx>& out,
                      int threads) {
  const int N = gr.N;
  const int delta = base_degree(gr.U1, gr.U2);
  Family fv, fo, fm;
  build_family(EQ_V, N, delta, fv);
  build_family(EQ_OMEGA, N, delta, fo);
  build_family(EQ_MEAN, N, 0, fm);
  Prepared pv, po, pmv, pmo;
  if (!prepare(fv, v, pv) || !prepare(fo, o, po) || !prepare(fm, v, pmv) || !prepare(fm, o, pmo))
    return "wall-normal operator outside its packed band";
  const Packing pk = make_packing(v, o);
  const long long nslots = (long long)gr.Kx * (gr.nkz < 0 ? gr.Kh : gr.nkz);
  const long long s0 = (long long)gr.Kx * gr.kz0;  // global slot of local slot 0
  const long long ngroups = (nslots + 15) / 16;
  out.assign((size_t)(ngroups * pk.group_complex), cx{0, 0});
  if (threads < 1) threads = 1;
  std::vector<std::string> errs(threads);
  auto work = [&](int t) {
    std::vector<cx> Lv((size_t)v.n * v.kl), Uv((size_t)v.n * pk.e1), Lo((size_t)o.n * o.kl),
        Uo((size_t)o.n * pk.e3), sig(16);
    for (long long grp = t; grp < ngroups; grp += threads) {
      cx* group = out.data() + grp * pk.group_complex;
      for (int q = 0; q < 16; ++q) {
        const long long sl = grp * 16 + q, s = s0 + sl;
        if (sl >= nslots) {  // identity factors
          std::fill(Lv.begin(), Lv.end(), cx{0, 0});
          std::fill(Uv.begin(), Uv.end(), cx{0, 0});
          std::fill(Lo.begin(), Lo.end(), cx{0, 0});
          std::fill(Uo.begin(), Uo.end(), cx{0, 0});
          for (int i = 0; i < v.n; ++i) Uv[(size_t)i * pk.e1] = cx{1, 0};
          for (int i = 0; i < o.n; ++i) Uo[(size_t)i * pk.e3] = cx{1, 0};
        } else if (s == 0) {
          sigma(fm, gr.Re, gr.dt, 0.0, 0.0, gr.U0, gr.U1, gr.U2, sig.data());
          if (!factor(pmv, sig.data(), Lv.data(), Uv.data()) ||
              !factor(pmo, sig.data(), Lo.data(), Uo.data())) {
            errs[t] = "zero pivot in the mean-mode operator";
            return;
          }
        } else {
          const int kx = (int)(s % gr.Kx), kz = (int)(s / gr.Kx);
          const double ia = (double)kx / gr.aphi, ib = (double)kz / gr.beta;
          const double kmn = ia * ia + ib * ib;
          sigma(fv, gr.Re, gr.dt, kmn, ia, gr.U0, gr.U1, gr.U2, sig.data());
          if (!factor(pv, sig.data(), Lv.data(), Uv.data())) {
            errs[t] = "zero pivot in a v operator";
            return;
          }
          sigma(fo, gr.Re, gr.dt, kmn, ia, gr.U0, gr.U1, gr.U2, sig.data());
          if (!factor(po, sig.data(), Lo.data(), Uo.data())) {
            errs[t] = "zero pivot in an omega_y operator";
            return;
          }
        }
        pack_slot(pk, q, Lv.data(), Uv.data(), Lo.data(), Uo.data(), group);
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
  for (auto& e : errs)
    if (!e.empty()) return e;
  return "";
}

}  // namespace wall
