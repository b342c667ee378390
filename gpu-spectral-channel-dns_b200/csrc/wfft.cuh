// Warp-synchronous line FFT: one warp transforms NL lines of length L held
// in shared memory, with no block-wide barrier.
//
// Each pass is a Stockham autosort step (as in fft2.cuh): with Ns = product
// of the previous radices, butterfly j in [0, L/R) reads x[j + r L/R],
// applies W_{Ns R}^{r (j mod Ns)}, takes the R-point DFT in registers and
// writes y[(j/Ns) Ns R + (j mod Ns) + r Ns].  The NL L / R butterflies of a
// pass are dealt to the 32 lanes in rounds of 32 (where NL L / R is not a
// multiple of 32 the last round leaves lanes idle); a lane loads all its
// inputs before the warp synchronises and writes, so the transform runs in
// place.
//
// Layout: element i of a line sits at wsw(i) = i + i / 2^S, one padding
// slot after every 2^S elements (2^S x the element size = 128 bytes), which
// spreads the strided accesses of the early passes over the banks.  The map
// is linear within runs that do not cross a 2^S boundary, so where a pass's
// R accesses of a butterfly are i = b + c_r with compile-time c_r and no
// carry from the low S bits of b into c_r (checked at compile time for all
// butterflies of the pass), wsw(b + c_r) = wsw(b) + wsw(c_r): one address
// per butterfly and immediate offsets.  Lines are wlen(L) elements apart
// unless the caller passes another stride.
#pragma once
#include <cmath>
#include <vector>

#include "fft2.cuh"

// butterfly index range hint for the device compiler (lets it resolve, per
// compile-time r, which branch of a first-pass load function applies)
#ifdef __CUDA_ARCH__
#define WFFT_ASSUME(c) __builtin_assume(c)
#else
#define WFFT_ASSUME(c) ((void)0)
#endif

template <typename C> struct WSwz { enum { S = 4 }; };
template <> struct WSwz<double2> { enum { S = 3 }; };
template <typename C> DNS_HD constexpr int wsw(int i) { return i + (i >> WSwz<C>::S); }
// line length covering positions wsw(0..L-1)
template <typename C> DNS_HD constexpr int wlen(int L) { return L + (L >> WSwz<C>::S); }

// plans: radices (up to 48 FP32, 8 FP64 for register pressure); a radix
// that divides NL L / 32 keeps every lane busy in every round
template <int L, int NL, int MAXR> struct WPlan { enum { ok = 0 }; };
#define WPLAN(L, NL, MAXR, ...) \
  template <> struct WPlan<L, NL, MAXR> { enum { ok = 1 }; typedef Radices<__VA_ARGS__> R; };
// FP32
WPLAN(128, 1, 16, 4, 4, 4, 2)
WPLAN(256, 1, 16, 8, 8, 4)
WPLAN(384, 1, 16, 8, 8, 6)
WPLAN(512, 1, 16, 8, 8, 8)
WPLAN(768, 1, 16, 8, 8, 12)
WPLAN(128, 2, 16, 8, 4, 4)
WPLAN(192, 2, 16, 16, 12)
WPLAN(256, 2, 16, 16, 16)
WPLAN(384, 2, 16, 16, 24)
WPLAN(512, 2, 16, 32, 16)
WPLAN(768, 2, 16, 16, 48)
WPLAN(384, 3, 16, 12, 4, 4, 2)
WPLAN(384, 4, 16, 16, 24)
WPLAN(192, 4, 16, 8, 24)
WPLAN(192, 1, 16, 8, 8, 3)
// the ensemble grids' streamwise and spanwise lengths (ragged rounds)
WPLAN(48, 1, 16, 6, 8)
WPLAN(48, 2, 16, 6, 8)
WPLAN(48, 4, 16, 6, 8)
WPLAN(96, 1, 16, 12, 8)
WPLAN(96, 2, 16, 12, 8)
WPLAN(96, 4, 16, 12, 8)
WPLAN(144, 1, 16, 12, 12)
WPLAN(144, 2, 16, 12, 12)
WPLAN(144, 4, 16, 12, 12)
// FP64
WPLAN(128, 1, 8, 4, 4, 4, 2)
WPLAN(256, 1, 8, 8, 8, 4)
WPLAN(384, 1, 8, 6, 4, 4, 4)
WPLAN(512, 1, 8, 8, 8, 8)
WPLAN(768, 1, 8, 8, 8, 4, 3)
WPLAN(128, 2, 8, 8, 4, 4)
WPLAN(192, 2, 8, 4, 4, 4, 3)
WPLAN(256, 2, 8, 8, 8, 4)
WPLAN(384, 2, 8, 8, 8, 6)
WPLAN(512, 2, 8, 8, 8, 8)
WPLAN(768, 2, 8, 8, 8, 4, 3)
WPLAN(384, 3, 8, 6, 4, 4, 4)
WPLAN(384, 4, 8, 8, 8, 6)
WPLAN(192, 4, 8, 8, 4, 6)
WPLAN(192, 1, 8, 8, 8, 3)
WPLAN(48, 1, 8, 6, 8)
WPLAN(48, 2, 8, 6, 8)
WPLAN(48, 4, 8, 6, 8)
WPLAN(96, 1, 8, 4, 4, 6)
WPLAN(96, 2, 8, 4, 4, 6)
WPLAN(96, 4, 8, 4, 4, 6)
WPLAN(144, 1, 8, 4, 6, 6)
WPLAN(144, 2, 8, 4, 6, 6)
WPLAN(144, 4, 8, 4, 6, 6)
#undef WPLAN

// One pass, split into the load (inputs of the lane's butterfly q, twiddled,
// transformed) and the store of its outputs, so that host code can run the
// same index arithmetic lane by lane.
// true when no butterfly j < NB of a pass stores across a 2^S boundary
// from its first output: (base(j) mod 2^S) + (r Ns mod 2^S) < 2^S for all r
constexpr bool wlin_store(int M, int NB, int Ns, int R) {
  for (int j = 0; j < NB; ++j) {
    const int b = ((j / Ns) * Ns * R + j % Ns) & M;
    for (int r = 0; r < R; ++r)
      if (b + ((r * Ns) & M) > M) return false;
  }
  return true;
}

// FP32 twiddles: one table per plan, pass by pass (passes with Ns > 1), the
// (R - 1) Ns values W_L^{r k L/(Ns R)}, r = 1..R-1, k < Ns, stored [r][k]:
// the lanes of a pass (consecutive k) read consecutive entries.  FP64 passes
// use W_L^j, j < L, and a product recurrence instead.
template <int... Rs> constexpr int wtw_offset(Radices<Rs...>, int Ns) {
  const int rs[] = {Rs...};
  int off = 0, ns = 1;
  for (int i = 0; i < (int)sizeof...(Rs) && ns != Ns; ++i) {
    if (ns > 1) off += (rs[i] - 1) * ns;
    ns *= rs[i];
  }
  return off;
}
template <int... Rs> constexpr int wtw_size(Radices<Rs...>) {
  const int rs[] = {Rs...};
  int off = 0, ns = 1;
  for (int i = 0; i < (int)sizeof...(Rs); ++i) {
    if (ns > 1) off += (rs[i] - 1) * ns;
    ns *= rs[i];
  }
  return off;
}

template <typename C, int L, int NL, bool INV, int R, int Ns>
struct WPass {
  static constexpr int NB = L / R;           // butterflies per line
  static constexpr int NT = NL * NB;         // butterflies of the pass
  static constexpr int B = (NT + 31) / 32;   // rounds: butterfly lane + 32 q in round q
  static_assert(L % R == 0, "radix does not divide the length");
  // lanes past the last butterfly idle in the last round
  DNS_HD static bool on(int lane, int q) { return NT % 32 == 0 || lane + 32 * q < NT; }
  static constexpr int S = WSwz<C>::S, M = (1 << S) - 1;
  // loads i = j + r NB: no carry for any j when NB is a multiple of 2^S
  static constexpr bool LIN_LD = (NB & M) == 0;
  // stores i = base(j) + r Ns, base(j) = (j / Ns) Ns R + j mod Ns
  static constexpr bool LIN_ST = wlin_store(M, NB, Ns, R);
  static constexpr int TWO = wtw_offset(typename WPlan<L, NL, FftMaxRadix<C>::v>::R(), Ns);
  DNS_HD static void load(const C* buf, int ls, const C* tw, int lane, int q, C* v) {
    const int w = lane + 32 * q;
    const int line = w / NB;
    const int j = w - line * NB;
    WFFT_ASSUME(j >= 0 && j < NB);
    const C* x = buf + line * ls;
    if constexpr (LIN_LD) {
      const C* xb = x + wsw<C>(j);
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = xb[wsw<C>(r * NB)];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = x[wsw<C>(j + r * NB)];
    }
    if (Ns > 1) {
      const int k = j % Ns;
      if (k > 0) {
        constexpr int step = L / (Ns * R);
        if constexpr (FftMaxRadix<C>::v == 8) {
          const C w1 = tw[k * step];
          C wr = w1;
#pragma unroll
          for (int r = 1; r < R; ++r) {
            if (r > 1) wr = cmul(wr, w1);
            v[r] = INV ? cmulc(v[r], wr) : cmul(v[r], wr);
          }
        } else {
          const C* tk = tw + TWO + k;  // entry (r, k) at tk[(r - 1) Ns]
#pragma unroll
          for (int r = 1; r < R; ++r) {
            const C wr = tk[(r - 1) * Ns];
            v[r] = INV ? cmulc(v[r], wr) : cmul(v[r], wr);
          }
        }
      }
    }
    Codelet<R, INV, C>::run(v);
  }
  // first pass (Ns = 1, no twiddles) reading element n of line l from ld(l, n)
  template <class LD> DNS_HD static void load_fn(LD& ld, int lane, int q, C* v) {
    const int w = lane + 32 * q;
    const int line = w / NB;
    const int j = w - line * NB;
    WFFT_ASSUME(j >= 0 && j < NB);
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = ld(line, j + r * NB);
    Codelet<R, INV, C>::run(v);
  }
  // last pass handing output k of line l to st(l, k, value)
  template <class ST> DNS_HD static void store_fn(ST& st, int lane, int q, const C* v) {
    const int w = lane + 32 * q;
    const int line = w / NB;
    const int j = w - line * NB;
    WFFT_ASSUME(j >= 0 && j < NB);
    const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
    for (int r = 0; r < R; ++r) st(line, base + r * Ns, v[r]);
  }
  DNS_HD static void store(C* buf, int ls, int lane, int q, const C* v) {
    const int w = lane + 32 * q;
    const int line = w / NB;
    const int j = w - line * NB;
    WFFT_ASSUME(j >= 0 && j < NB);
    C* y = buf + line * ls;
    const int base = (j / Ns) * Ns * R + (j % Ns);
    if constexpr (LIN_ST) {
      C* yb = y + wsw<C>(base);
#pragma unroll
      for (int r = 0; r < R; ++r) yb[wsw<C>(r * Ns)] = v[r];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) y[wsw<C>(base + r * Ns)] = v[r];
    }
  }
};

// host: the FP32 twiddle table of plan (L, NL) (wtw_size entries), values
// rounded from long double like the W_L^j table; -1 if there is no plan
template <typename C, int L, int NL, int... Rs>
void wtw_fill_radices(Radices<Rs...>, C* out) {
  const long double PI = 3.141592653589793238462643383279502884L;
  const int rs[] = {Rs...};
  int off = 0, ns = 1;
  for (int i = 0; i < (int)sizeof...(Rs); ++i) {
    const int R = rs[i];
    if (ns > 1) {
      const int step = L / (ns * R);
      for (int r = 1; r < R; ++r)
        for (int k = 0; k < ns; ++k) {
          const long double a = -2.0L * PI * (long double)(r * k * step) / (long double)L;
          out[off + (r - 1) * ns + k] = cmk<C>((double)cosl(a), (double)sinl(a));
        }
      off += (R - 1) * ns;
    }
    ns *= R;
  }
}
template <typename C, int L, int NL> int wtw_table(std::vector<C>& out) {
  if constexpr (WPlan<L, NL, FftMaxRadix<C>::v>::ok) {
    typedef typename WPlan<L, NL, FftMaxRadix<C>::v>::R RS;
    out.assign(wtw_size(RS()), cmk<C>(0.0, 0.0));
    wtw_fill_radices<C, L, NL>(RS(), out.data());
    return (int)out.size();
  } else {
    return -1;
  }
}
// runtime length: the lengths that have warp plans
template <typename C, int NL> int wtw_table_any(int L, std::vector<C>& out) {
  switch (L) {
    case 48: return wtw_table<C, 48, NL>(out);
    case 96: return wtw_table<C, 96, NL>(out);
    case 144: return wtw_table<C, 144, NL>(out);
    case 128: return wtw_table<C, 128, NL>(out);
    case 192: return wtw_table<C, 192, NL>(out);
    case 256: return wtw_table<C, 256, NL>(out);
    case 384: return wtw_table<C, 384, NL>(out);
    case 512: return wtw_table<C, 512, NL>(out);
    case 768: return wtw_table<C, 768, NL>(out);
  }
  return -1;
}

#ifdef __CUDACC__
template <typename C, int L, int NL, bool INV, int R, int Ns>
__device__ __forceinline__ void wfft_pass(C* buf, int ls, const C* __restrict__ tw, int lane) {
  typedef WPass<C, L, NL, INV, R, Ns> P;
  C v[P::B][R];
#pragma unroll
  for (int q = 0; q < P::B; ++q)
    if (P::on(lane, q)) P::load(buf, ls, tw, lane, q, v[q]);
  __syncwarp();
#pragma unroll
  for (int q = 0; q < P::B; ++q)
    if (P::on(lane, q)) P::store(buf, ls, lane, q, v[q]);
  __syncwarp();
}

template <typename C, int L, int NL, bool INV, int Ns, int R, int... Rest>
struct WRun {
  __device__ __forceinline__ static void go(C* buf, int ls, const C* tw, int lane) {
    wfft_pass<C, L, NL, INV, R, Ns>(buf, ls, tw, lane);
    WRun<C, L, NL, INV, Ns * R, Rest...>::go(buf, ls, tw, lane);
  }
};
template <typename C, int L, int NL, bool INV, int Ns, int R>
struct WRun<C, L, NL, INV, Ns, R> {
  __device__ __forceinline__ static void go(C* buf, int ls, const C* tw, int lane) {
    wfft_pass<C, L, NL, INV, R, Ns>(buf, ls, tw, lane);
  }
};
template <typename C, int L, int NL, bool INV, typename RS> struct WDo;
template <typename C, int L, int NL, bool INV, int... Rs>
struct WDo<C, L, NL, INV, Radices<Rs...>> {
  __device__ __forceinline__ static void go(C* buf, int ls, const C* tw, int lane) {
    WRun<C, L, NL, INV, 1, Rs...>::go(buf, ls, tw, lane);
  }
};

// Variant with the input and output fused into the first and last passes:
// the first pass reads ld(line, n), the last hands st(line, k, value) every
// output; buf (NL lines, ls >= wlen(L) apart) holds the intermediate passes only.
template <typename C, int L, int NL, bool INV, int Ns, bool FIRST, int R, int... Rest>
struct WRunIO {
  template <class LD, class ST>
  __device__ __forceinline__ static void go(C* buf, int ls, const C* tw, int lane, LD& ld, ST& st) {
    typedef WPass<C, L, NL, INV, R, Ns> P;
    constexpr bool LAST = sizeof...(Rest) == 0;
    C v[P::B][R];
#pragma unroll
    for (int q = 0; q < P::B; ++q) {
      if (!P::on(lane, q)) continue;
      if constexpr (FIRST) P::template load_fn<LD>(ld, lane, q, v[q]);
      else P::load(buf, ls, tw, lane, q, v[q]);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < P::B; ++q) {
      if (!P::on(lane, q)) continue;
      if constexpr (LAST) P::template store_fn<ST>(st, lane, q, v[q]);
      else P::store(buf, ls, lane, q, v[q]);
    }
    __syncwarp();
    if constexpr (!LAST) WRunIO<C, L, NL, INV, Ns * R, false, Rest...>::go(buf, ls, tw, lane, ld, st);
  }
};
template <typename C, int L, int NL, bool INV, typename RS> struct WDoIO;
template <typename C, int L, int NL, bool INV, int... Rs>
struct WDoIO<C, L, NL, INV, Radices<Rs...>> {
  template <class LD, class ST>
  __device__ __forceinline__ static void go(C* buf, int ls, const C* tw, int lane, LD& ld, ST& st) {
    WRunIO<C, L, NL, INV, 1, true, Rs...>::go(buf, ls, tw, lane, ld, st);
  }
};
template <typename C, int L, int NL, bool INV, class LD, class ST>
__device__ __forceinline__ void wfft_io(C* buf, const C* __restrict__ tw, LD ld, ST st, int ls = wlen<C>(L)) {
  WDoIO<C, L, NL, INV, typename WPlan<L, NL, FftMaxRadix<C>::v>::R>::go(buf, ls, tw, threadIdx.x & 31, ld, st);
}

// Transform the NL lines at buf (line stride ls >= wlen(L), positions wsw(i)) by
// the calling warp.  The lines must have been written by this warp (or be
// visible to it after a barrier); a __syncwarp is taken first.
// tw: the plan's twiddle table (FP32, wtw_table) or W_L^j, j < L (FP64).
template <typename C, int L, int NL, bool INV>
__device__ __forceinline__ void wfft(C* buf, const C* __restrict__ tw, int ls = wlen<C>(L)) {
  __syncwarp();
  WDo<C, L, NL, INV, typename WPlan<L, NL, FftMaxRadix<C>::v>::R>::go(buf, ls, tw, threadIdx.x & 31);
}
#endif
