// CPU check of fft2.cuh (compile-time-length FFT): runs each pass's
// butterflies sequentially (all loads, then all stores, as the block does)
// and prints the transform of a test vector.  Usage: fft2_check L inv prec
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "../../gpu-spectral-channel-dns_b200/csrc/fft2.cuh"

template <typename C, int L, bool INV, int Ns, int R>
void host_pass(std::vector<C>& line, const std::vector<C>& tw) {
  typedef FftPass<L, R, Ns, INV, C> P;
  std::vector<C> regs((size_t)P::NB * R);
  for (int j = 0; j < P::NB; ++j) P::load(line.data(), j, &regs[(size_t)j * R], tw.data());
  for (int j = 0; j < P::NB; ++j) P::store(line.data(), j, &regs[(size_t)j * R]);
}
template <typename C, int L, bool INV, int Ns, int R, int... Rest>
struct HostRun {
  static void go(std::vector<C>& line, const std::vector<C>& tw) {
    host_pass<C, L, INV, Ns, R>(line, tw);
    HostRun<C, L, INV, Ns * R, Rest...>::go(line, tw);
  }
};
template <typename C, int L, bool INV, int Ns, int R>
struct HostRun<C, L, INV, Ns, R> {
  static void go(std::vector<C>& line, const std::vector<C>& tw) { host_pass<C, L, INV, Ns, R>(line, tw); }
};
template <typename C, int L, bool INV, typename RS> struct HostDo;
template <typename C, int L, bool INV, int... Rs>
struct HostDo<C, L, INV, Radices<Rs...>> {
  static void go(std::vector<C>& line, const std::vector<C>& tw) { HostRun<C, L, INV, 1, Rs...>::go(line, tw); }
};

template <typename C, int L>
void run(bool inv) {
  std::vector<C> tw(L), line(fpad_len(L));
  for (int j = 0; j < L; ++j) {
    long double a = -2.0L * 3.14159265358979323846264338327950288L * j / L;
    tw[j] = cmk<C>((double)cosl(a), (double)sinl(a));
    line[fpos(j)] = cmk<C>(std::sin(0.37 * j * j + 1.0), std::cos(1.3 * j) - 0.25);
  }
  typedef typename FftPlanL<L, FftMaxRadix<C>::v>::R RS;
  if (inv) HostDo<C, L, true, RS>::go(line, tw);
  else HostDo<C, L, false, RS>::go(line, tw);
  for (int k = 0; k < L; ++k) printf("%.17g %.17g\n", (double)line[fpos(k)].x, (double)line[fpos(k)].y);
}

int main(int argc, char** argv) {
  int L = atoi(argv[1]);
  bool inv = atoi(argv[2]) != 0;
  bool f = argv[3][0] == 'f';
#define CASE(n) case n: if (f) run<float2, n>(inv); else run<double2, n>(inv); break;
  switch (L) { FFT2_LENGTHS(CASE) default: printf("bad\n"); }
  return 0;
}
