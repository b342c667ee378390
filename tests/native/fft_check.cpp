// CPU check of the shared-memory FFT plan and butterflies (fft.cuh): runs
// every stage's butterflies sequentially (they are independent within a
// stage) and prints the transform of a test vector for comparison with
// numpy.fft.  Usage: fft_check L inverse(0|1) prec(d|f)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "../../gpu-spectral-channel-dns_b200/csrc/fft.cuh"

template <typename C>
static void run(int L, bool inv) {
  FftPlan P;
  if (!fft_make_plan(L, &P)) { printf("noplan\n"); return; }
  std::vector<C> tw(L), x(L), buf(L);
  for (int j = 0; j < L; ++j) {
    long double a = -2.0L * 3.14159265358979323846264338327950288L * j / L;
    tw[j] = cmk<C>((double)cosl(a), (double)sinl(a));
    x[j] = cmk<C>(std::sin(0.37 * j * j + 1.0), std::cos(1.3 * j) - 0.25);
  }
  for (int n = 0; n < L; ++n) buf[fft_digitrev(P, n)] = x[n];
  for (int s = 0; s < P.S; ++s) {
    int nbf = L / P.R[s];
    for (int t = 0; t < nbf; ++t) {
      if (inv) fft_butterfly<C, true>(buf.data(), P, s, t, tw.data());
      else fft_butterfly<C, false>(buf.data(), P, s, t, tw.data());
    }
  }
  for (int k = 0; k < L; ++k) printf("%.17g %.17g\n", (double)buf[k].x, (double)buf[k].y);
}

int main(int argc, char** argv) {
  int L = atoi(argv[1]);
  bool inv = atoi(argv[2]) != 0;
  if (argv[3][0] == 'f') run<float2>(L, inv); else run<double2>(L, inv);
  return 0;
}
