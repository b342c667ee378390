// Host run of the warp FFT (csrc/wfft.cuh): every pass executed lane by lane
// with the same load/store index arithmetic as the device, compared with a
// long-double DFT.  Built and run by tests/test_fft_host.py.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "../../gpu-spectral-channel-dns_b200/csrc/wfft.cuh"

template <typename C, int L, int NL, bool INV, int Ns, int R, int... Rest>
struct HRun {
  static void go(C* buf, const C* tw) {
    typedef WPass<C, L, NL, INV, R, Ns> P;
    std::vector<C> v(32 * P::B * R);
    for (int lane = 0; lane < 32; ++lane)
      for (int q = 0; q < P::B; ++q)
        if (P::on(lane, q)) P::load(buf, wlen<C>(L), tw, lane, q, &v[(lane * P::B + q) * R]);
    for (int lane = 0; lane < 32; ++lane)
      for (int q = 0; q < P::B; ++q)
        if (P::on(lane, q)) P::store(buf, wlen<C>(L), lane, q, &v[(lane * P::B + q) * R]);
    if constexpr (sizeof...(Rest) > 0) HRun<C, L, NL, INV, Ns * R, Rest...>::go(buf, tw);
  }
};
template <typename C, int L, int NL, bool INV, typename RS> struct HDo;
template <typename C, int L, int NL, bool INV, int... Rs>
struct HDo<C, L, NL, INV, Radices<Rs...>> {
  static void go(C* buf, const C* tw) { HRun<C, L, NL, INV, 1, Rs...>::go(buf, tw); }
};

// fused-IO form: first pass reads a separate input, last pass writes a separate output
template <typename C, int L, int NL, bool INV, int Ns, bool FIRST, int R, int... Rest>
struct HRunIO {
  template <class LD, class ST>
  static void go(C* buf, const C* tw, LD& ld, ST& st) {
    typedef WPass<C, L, NL, INV, R, Ns> P;
    constexpr bool LAST = sizeof...(Rest) == 0;
    std::vector<C> v(32 * P::B * R);
    for (int lane = 0; lane < 32; ++lane)
      for (int q = 0; q < P::B; ++q) {
        if (!P::on(lane, q)) continue;
        if constexpr (FIRST) P::load_fn(ld, lane, q, &v[(lane * P::B + q) * R]);
        else P::load(buf, wlen<C>(L), tw, lane, q, &v[(lane * P::B + q) * R]);
      }
    for (int lane = 0; lane < 32; ++lane)
      for (int q = 0; q < P::B; ++q) {
        if (!P::on(lane, q)) continue;
        if constexpr (LAST) P::store_fn(st, lane, q, &v[(lane * P::B + q) * R]);
        else P::store(buf, wlen<C>(L), lane, q, &v[(lane * P::B + q) * R]);
      }
    if constexpr (!LAST) HRunIO<C, L, NL, INV, Ns * R, false, Rest...>::go(buf, tw, ld, st);
  }
};
template <typename C, int L, int NL, bool INV, typename RS> struct HDoIO;
template <typename C, int L, int NL, bool INV, int... Rs>
struct HDoIO<C, L, NL, INV, Radices<Rs...>> {
  template <class LD, class ST>
  static void go(C* buf, const C* tw, LD& ld, ST& st) { HRunIO<C, L, NL, INV, 1, true, Rs...>::go(buf, tw, ld, st); }
};

template <typename C, int L, int NL, bool INV, bool IO = false>
double check() {
  const long double PI = 3.141592653589793238462643383279502884L;
  constexpr int LW = wlen<C>(L);
  std::vector<C> tw(L), buf(NL * LW, cmk<C>(1e30, 1e30));
  for (int j = 0; j < L; ++j) tw[j] = cmk<C>((double)cosl(-2 * PI * j / L), (double)sinl(-2 * PI * j / L));
  std::mt19937 rng(L * 7 + NL);
  std::normal_distribution<double> nd;
  std::vector<long double> xr(NL * L), xi(NL * L);
  for (int i = 0; i < NL * L; ++i) {
    xr[i] = (T_of<C>)nd(rng);
    xi[i] = (T_of<C>)nd(rng);
  }
  std::vector<C> in(NL * L), outv(NL * L);
  for (int l = 0; l < NL; ++l)
    for (int n = 0; n < L; ++n) {
      in[l * L + n] = cmk<C>((double)xr[l * L + n], (double)xi[l * L + n]);
      buf[l * LW + wsw<C>(n)] = in[l * L + n];
    }
  typedef typename WPlan<L, NL, FftMaxRadix<C>::v>::R RS;
  // FP32 passes read the plan's pass-by-pass table, FP64 passes W_L^j
  if (FftMaxRadix<C>::v != 8) {
    std::vector<C> wt;
    wtw_table<C, L, NL>(wt);
    wt.push_back(cmk<C>(0.0, 0.0));  // never empty
    tw = wt;
  }
  if (IO) {
    auto ld = [&](int l, int n) { return in[l * L + n]; };
    auto st = [&](int l, int k, C v) { outv[l * L + k] = v; };
    HDoIO<C, L, NL, INV, RS>::go(buf.data(), tw.data(), ld, st);
    for (int l = 0; l < NL; ++l)
      for (int k = 0; k < L; ++k) buf[l * LW + wsw<C>(k)] = outv[l * L + k];
  } else {
    HDo<C, L, NL, INV, RS>::go(buf.data(), tw.data());
  }
  double err = 0, nrm = 0;
  for (int l = 0; l < NL; ++l)
    for (int k = 0; k < L; ++k) {
      long double sr = 0, si = 0;
      for (int n = 0; n < L; ++n) {
        const long double a = (INV ? 2 : -2) * PI * (long double)((long long)n * k % L) / L;
        const long double c = cosl(a), s = sinl(a);
        sr += xr[l * L + n] * c - xi[l * L + n] * s;
        si += xr[l * L + n] * s + xi[l * L + n] * c;
      }
      const C got = buf[l * LW + wsw<C>(k)];
      err = fmax(err, (double)hypotl(got.x - sr, got.y - si));
      nrm = fmax(nrm, (double)hypotl(sr, si));
    }
  return err / nrm;
}

#define CASE(C, L, NL)                                                                    \
  {                                                                                       \
    const double ef = check<C, L, NL, false>(), eb = check<C, L, NL, true>();             \
    const double ei = check<C, L, NL, false, true>(), ej = check<C, L, NL, true, true>(); \
    printf("%s %d %d %.3e %.3e\n", #C, L, NL, ef > ei ? ef : ei, eb > ej ? eb : ej);     \
  }

// every plan of wfft.cuh, both precisions (ragged rounds at 48, 96, 144 and 192 x 1)
#define ALL_PLANS(C)                                                                              \
  CASE(C, 128, 1) CASE(C, 256, 1) CASE(C, 384, 1) CASE(C, 512, 1) CASE(C, 768, 1) CASE(C, 192, 1) \
  CASE(C, 128, 2) CASE(C, 192, 2) CASE(C, 256, 2) CASE(C, 384, 2) CASE(C, 512, 2)                 \
  CASE(C, 768, 2) CASE(C, 384, 3) CASE(C, 384, 4) CASE(C, 192, 4)                                 \
  CASE(C, 48, 1) CASE(C, 48, 2) CASE(C, 48, 4) CASE(C, 96, 1) CASE(C, 96, 2) CASE(C, 96, 4)       \
  CASE(C, 144, 1) CASE(C, 144, 2) CASE(C, 144, 4)

int main() {
  ALL_PLANS(float2)
  ALL_PLANS(double2)
  return 0;
}
