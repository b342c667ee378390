// Compile-time-length shared-memory FFT built from register codelets.
//
// L = R_1 * R_2 * ... * R_P with every radix R_p <= 16 (codelets 2, 3, 4, 6,
// 8, 12, 16).  Pass p is a Stockham autosort step: with Ns = R_1 ... R_{p-1},
// butterfly j in [0, L/R) reads x[j + r L/R] (r < R), multiplies by
// W_{Ns R}^{r (j mod Ns)}, takes the R-point DFT in registers and writes
// y[(j/Ns) Ns R + (j mod Ns) + r Ns].  Every thread reads all its butterfly
// inputs, the block synchronises, then every thread writes, so one buffer
// suffices.  Input and output are in natural order.
//
// Shared-memory positions go through fpos(i) = i + i/16 (one pad element
// every 16) so the strided accesses of the early passes spread over banks.
// Pass twiddles come from the table W_L^j (host long double); codelet
// constants are the exact values cos, sin (2 pi m / R) for R <= 16.
#pragma once
#include <type_traits>
#include "dns_common.cuh"

DNS_HD int fpos(int i) { return i + (i >> 4); }
DNS_HD int fpad_len(int L) { return L + (L >> 4) + 1; }

template <int... Rs> struct Radices {};

// Radix plans: MAXR 16 (fewer passes, FP32 data) or 8 (fewer registers per
// butterfly, FP64 data).
template <int L, int MAXR> struct FftPlanL;
template <> struct FftPlanL<48, 16> { typedef Radices<16, 3> R; };
template <> struct FftPlanL<64, 16> { typedef Radices<8, 8> R; };
template <> struct FftPlanL<96, 16> { typedef Radices<16, 6> R; };
template <> struct FftPlanL<128, 16> { typedef Radices<16, 8> R; };
template <> struct FftPlanL<144, 16> { typedef Radices<12, 12> R; };
template <> struct FftPlanL<192, 16> { typedef Radices<16, 12> R; };
template <> struct FftPlanL<256, 16> { typedef Radices<16, 16> R; };
template <> struct FftPlanL<288, 16> { typedef Radices<16, 6, 3> R; };
template <> struct FftPlanL<384, 16> { typedef Radices<16, 8, 3> R; };
template <> struct FftPlanL<512, 16> { typedef Radices<8, 8, 8> R; };
template <> struct FftPlanL<576, 16> { typedef Radices<16, 12, 3> R; };
template <> struct FftPlanL<768, 16> { typedef Radices<16, 16, 3> R; };
template <> struct FftPlanL<48, 8> { typedef Radices<8, 6> R; };
template <> struct FftPlanL<64, 8> { typedef Radices<8, 8> R; };
template <> struct FftPlanL<96, 8> { typedef Radices<8, 4, 3> R; };
template <> struct FftPlanL<128, 8> { typedef Radices<8, 4, 4> R; };
template <> struct FftPlanL<144, 8> { typedef Radices<8, 6, 3> R; };
template <> struct FftPlanL<192, 8> { typedef Radices<8, 8, 3> R; };
template <> struct FftPlanL<256, 8> { typedef Radices<8, 8, 4> R; };
template <> struct FftPlanL<288, 8> { typedef Radices<8, 6, 6> R; };
template <> struct FftPlanL<384, 8> { typedef Radices<8, 8, 6> R; };
template <> struct FftPlanL<512, 8> { typedef Radices<8, 8, 8> R; };
template <> struct FftPlanL<576, 8> { typedef Radices<8, 6, 4, 3> R; };
template <> struct FftPlanL<768, 8> { typedef Radices<8, 8, 4, 3> R; };
template <typename C> struct FftMaxRadix { enum { v = 16 }; };
template <> struct FftMaxRadix<double2> { enum { v = 8 }; };

#define FFT2_LENGTHS(X) X(48) X(64) X(96) X(128) X(144) X(192) X(256) X(288) X(384) X(512) X(576) X(768)

// ---------------------------------------------------------------------------
// register codelets: out-of-place R-point DFT, v[] -> v[] (forward sign -)
// ---------------------------------------------------------------------------
template <int R> struct CodeletConst;
// cos / sin of 2 pi m / R
template <> struct CodeletConst<8> {
  DNS_HD static double c(int m) {
    const double t[8] = {1.0, 0.70710678118654752440084436210485, 0.0, -0.70710678118654752440084436210485,
                         -1.0, -0.70710678118654752440084436210485, 0.0, 0.70710678118654752440084436210485};
    return t[m & 7];
  }
  DNS_HD static double s(int m) { return c((m + 6) & 7); }
};
template <> struct CodeletConst<16> {
  DNS_HD static double c(int m) {
    const double a = 0.92387953251128675612818318939679, b = 0.38268343236508977172845998403040,
                 h = 0.70710678118654752440084436210485;
    const double t[16] = {1.0, a, h, b, 0.0, -b, -h, -a, -1.0, -a, -h, -b, 0.0, b, h, a};
    return t[m & 15];
  }
  DNS_HD static double s(int m) { return c((m + 12) & 15); }
};
template <> struct CodeletConst<12> {
  DNS_HD static double c(int m) {
    const double r = 0.86602540378443864676372317075294;
    const double t[12] = {1.0, r, 0.5, 0.0, -0.5, -r, -1.0, -r, -0.5, 0.0, 0.5, r};
    return t[m % 12];
  }
  DNS_HD static double s(int m) { return c((m + 9) % 12); }
};
template <> struct CodeletConst<6> {
  DNS_HD static double c(int m) {
    const double t[6] = {1.0, 0.5, -0.5, -1.0, -0.5, 0.5};
    return t[m % 6];
  }
  DNS_HD static double s(int m) {
    const double r = 0.86602540378443864676372317075294;
    const double t[6] = {0.0, r, r, 0.0, -r, -r};
    return t[m % 6];
  }
};

// radices 24, 32, 48: quarter-wave tables (correctly rounded) and symmetry
template <int R> struct CodeletQuarter;
template <> struct CodeletQuarter<24> {
  DNS_HD static double q(int m) {
    const double t[7] = {1.0, 0.9659258262890683, 0.8660254037844386, 0.7071067811865476, 0.5,
                         0.25881904510252074, 0.0};
    return t[m];
  }
};
template <> struct CodeletQuarter<32> {
  DNS_HD static double q(int m) {
    const double t[9] = {1.0, 0.9807852804032304, 0.9238795325112867, 0.8314696123025452,
                         0.7071067811865476, 0.5555702330196022, 0.3826834323650898,
                         0.19509032201612828, 0.0};
    return t[m];
  }
};
template <> struct CodeletQuarter<48> {
  DNS_HD static double q(int m) {
    const double t[13] = {1.0, 0.9914448613738104, 0.9659258262890683, 0.9238795325112867,
                          0.8660254037844386, 0.7933533402912352, 0.7071067811865476,
                          0.6087614290087207, 0.5, 0.3826834323650898, 0.25881904510252074,
                          0.1305261922200516, 0.0};
    return t[m];
  }
};
template <int R> struct CodeletConstQ {
  DNS_HD static double c(int m) {
    m %= R;
    if (m <= R / 4) return CodeletQuarter<R>::q(m);
    if (m <= R / 2) return -CodeletQuarter<R>::q(R / 2 - m);
    if (m <= 3 * R / 4) return -CodeletQuarter<R>::q(m - R / 2);
    return CodeletQuarter<R>::q(R - m);
  }
  DNS_HD static double s(int m) { return c(m + 3 * R / 4); }
};
template <> struct CodeletConst<24> : CodeletConstQ<24> {};
template <> struct CodeletConst<32> : CodeletConstQ<32> {};
template <> struct CodeletConst<48> : CodeletConstQ<48> {};

// W_R^m (forward: exp(-2 pi i m / R)); INV conjugates
template <int R, bool INV, typename C>
DNS_HD C wconst(int m) {
  typedef T_of<C> T;
  const double cc = CodeletConst<R>::c(m);
  const double ss = CodeletConst<R>::s(m);
  C w;
  w.x = (T)cc;
  w.y = (T)(INV ? ss : -ss);
  return w;
}

template <bool INV, typename C>
DNS_HD void dft2(C& a, C& b) {
  C t = a - b;
  a = a + b;
  b = t;
}

template <bool INV, typename C>
DNS_HD void dft3(C& y0, C& y1, C& y2) {
  typedef T_of<C> T;
  const T c3 = (T)(-0.5);
  const T s3 = (T)0.86602540378443864676372317075294;
  C t1 = y1 + y2;
  C t2 = y1 - y2;
  C base = y0 + t1 * c3;
  C its = muli(t2) * s3;
  y0 = y0 + t1;
  if (INV) { y1 = base + its; y2 = base - its; }
  else { y1 = base - its; y2 = base + its; }
}

template <bool INV, typename C>
DNS_HD void dft4(C& y0, C& y1, C& y2, C& y3) {
  C a = y0 + y2, b = y0 - y2, c = y1 + y3, d = y1 - y3;
  C id = muli(d);
  y0 = a + c;
  y2 = a - c;
  if (INV) { y1 = b + id; y3 = b - id; }
  else { y1 = b - id; y3 = b + id; }
}

// FP32 radix-2, -3 and -4 butterflies on packed pairs: a complex value's
// (re, im) is one 64-bit register pair, so a complex add or subtract is one
// add/sub.rn.f32x2 (sm_100) instead of two scalar instructions, b -+ i d is
// one fma.rn.f32x2 of the swapped d with (+-1, -+1), and radix 3's products
// with constants are one mul/fma.rn.f32x2 (the same roundings as the scalar
// form: the results equal it bit for bit).  Host code takes the scalar form.
#if defined(__CUDA_ARCH__)
__device__ __forceinline__ unsigned long long f2u(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 u2f(unsigned long long u) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(u));
  return r;
}
__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
// (y.im, y.re)
__device__ __forceinline__ unsigned long long swap2(unsigned long long a) {
  unsigned long long r;
  asm("{\n\t.reg .b32 lo, hi;\n\tmov.b64 {lo, hi}, %1;\n\tmov.b64 %0, {hi, lo};\n\t}" : "=l"(r) : "l"(a));
  return r;
}
template <bool INV>
__device__ __forceinline__ void dft2_f32x2(float2& a, float2& b) {
  const unsigned long long ua = f2u(a), ub = f2u(b);
  a = u2f(add2(ua, ub));
  b = u2f(sub2(ua, ub));
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long pair2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
template <bool INV>
__device__ __forceinline__ void dft3_f32x2(float2& y0, float2& y1, float2& y2) {
  const float c3 = -0.5f, s3 = 0.86602540378443864676372317075294f;
  const unsigned long long u0 = f2u(y0), u1 = f2u(y1), u2 = f2u(y2);
  const unsigned long long t1 = add2(u1, u2), t2 = sub2(u1, u2);
  const unsigned long long base = fma2(t1, pair2(c3, c3), u0);
  const unsigned long long its = mul2(swap2(t2), pair2(-s3, s3));  // i t2 s3
  y0 = u2f(add2(u0, t1));
  if (INV) { y1 = u2f(add2(base, its)); y2 = u2f(sub2(base, its)); }
  else { y1 = u2f(sub2(base, its)); y2 = u2f(add2(base, its)); }
}
template <bool INV>
__device__ __forceinline__ void dft4_f32x2(float2& y0, float2& y1, float2& y2, float2& y3) {
  const unsigned long long u0 = f2u(y0), u1 = f2u(y1), u2 = f2u(y2), u3 = f2u(y3);
  const unsigned long long a = add2(u0, u2), b = sub2(u0, u2), c = add2(u1, u3), d = sub2(u1, u3);
  const unsigned long long ds = swap2(d);
  // (1, -1) and (-1, 1) as f32x2 bit patterns (low word = re)
  const unsigned long long pm = 0xBF8000003F800000ull, mp = 0x3F800000BF800000ull;
  y0 = u2f(add2(a, c));
  y2 = u2f(sub2(a, c));
  // forward: y1 = b - i d = (b.re + d.im, b.im - d.re), y3 = b + i d
  y1 = u2f(fma2(ds, INV ? mp : pm, b));
  y3 = u2f(fma2(ds, INV ? pm : mp, b));
}
#endif

// Generic R = R1 * R2 codelet: x[r2 + R2 r1] -> X[k1 + R1 k2]
template <int R, bool INV, typename C> struct Codelet;

template <bool INV, typename C> struct Codelet<2, INV, C> {
  DNS_HD static void run(C* v) {
#if defined(__CUDA_ARCH__)
    if constexpr (std::is_same<C, float2>::value) {
      dft2_f32x2<INV>(v[0], v[1]);
      return;
    }
#endif
    dft2<INV>(v[0], v[1]);
  }
};
template <bool INV, typename C> struct Codelet<3, INV, C> {
  DNS_HD static void run(C* v) {
#if defined(__CUDA_ARCH__)
    if constexpr (std::is_same<C, float2>::value) {
      dft3_f32x2<INV>(v[0], v[1], v[2]);
      return;
    }
#endif
    dft3<INV>(v[0], v[1], v[2]);
  }
};
template <bool INV, typename C> struct Codelet<4, INV, C> {
  DNS_HD static void run(C* v) {
#if defined(__CUDA_ARCH__)
    if constexpr (std::is_same<C, float2>::value) {
      dft4_f32x2<INV>(v[0], v[1], v[2], v[3]);
      return;
    }
#endif
    dft4<INV>(v[0], v[1], v[2], v[3]);
  }
};

template <int R1, int R2, int R, bool INV, typename C>
DNS_HD void codelet_split(C* v) {
  // step 1: R2 DFTs of size R1 over r1 (stride R2), twiddle W_R^{r2 k1}
  C t[R];
#pragma unroll
  for (int r2 = 0; r2 < R2; ++r2) {
    C a[R1];
#pragma unroll
    for (int r1 = 0; r1 < R1; ++r1) a[r1] = v[r2 + R2 * r1];
    Codelet<R1, INV, C>::run(a);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      C x = a[k1];
      if (r2 * k1) x = cmul(x, wconst<R, INV, C>(r2 * k1));
      t[k1 * R2 + r2] = x;
    }
  }
  // step 2: R1 DFTs of size R2 over r2, output X[k1 + R1 k2]
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    C b[R2];
#pragma unroll
    for (int r2 = 0; r2 < R2; ++r2) b[r2] = t[k1 * R2 + r2];
    Codelet<R2, INV, C>::run(b);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = b[k2];
  }
}

template <bool INV, typename C> struct Codelet<6, INV, C> {
  DNS_HD static void run(C* v) { codelet_split<2, 3, 6, INV, C>(v); }
};
template <bool INV, typename C> struct Codelet<8, INV, C> {
  DNS_HD static void run(C* v) { codelet_split<2, 4, 8, INV, C>(v); }
};
template <bool INV, typename C> struct Codelet<12, INV, C> {
  DNS_HD static void run(C* v) { codelet_split<4, 3, 12, INV, C>(v); }
};
template <bool INV, typename C> struct Codelet<16, INV, C> {
  DNS_HD static void run(C* v) { codelet_split<4, 4, 16, INV, C>(v); }
};
template <bool INV, typename C> struct Codelet<24, INV, C> {
  DNS_HD static void run(C* v) { codelet_split<8, 3, 24, INV, C>(v); }
};
template <bool INV, typename C> struct Codelet<32, INV, C> {
  DNS_HD static void run(C* v) { codelet_split<4, 8, 32, INV, C>(v); }
};
template <bool INV, typename C> struct Codelet<48, INV, C> {
  DNS_HD static void run(C* v) { codelet_split<16, 3, 48, INV, C>(v); }
};

// ---------------------------------------------------------------------------
// one Stockham pass; Ns = product of the previous radices
// ---------------------------------------------------------------------------
template <int L, int R, int Ns, bool INV, typename C>
struct FftPass {
  static constexpr int NB = L / R;  // butterflies per line
  // read inputs of butterfly j of one line into v, twiddled
  DNS_HD static void load(const C* line, int j, C* v, const C* tw) {
    const int k = j % Ns;
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = line[fpos(j + r * NB)];
    if (Ns > 1 && k > 0) {
      // FP64: W^r from one table load by products (error ~ r eps, far below
      // the FP64 budget, and cheaper than R-1 loads through L1); FP32: exact
      // table values for every r.
      const C w1 = tw[k * (L / (Ns * R))];
      C wr = w1;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        if (FftMaxRadix<C>::v == 8) {
          if (r > 1) wr = cmul(wr, w1);
        } else {
          wr = tw[(r * k) * (L / (Ns * R))];
        }
        v[r] = INV ? cmulc(v[r], wr) : cmul(v[r], wr);
      }
    }
    Codelet<R, INV, C>::run(v);
  }
  DNS_HD static void store(C* line, int j, const C* v) {
    const int k = j % Ns;
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) line[fpos(base + r * Ns)] = v[r];
  }
};

#ifdef __CUDACC__
// One pass over nb lines (line stride ls >= fpad_len(L)) by the whole block.
// A thread keeps KMAX butterflies in registers; a round covers whole lines,
// so all reads of a line precede all writes to it.
template <typename C, int L, bool INV, int R, int Ns>
__device__ __forceinline__ void fft2_pass(C* buf, int nb, int ls, const C* __restrict__ tw) {
  typedef FftPass<L, R, Ns, INV, C> P;
  // complex values a thread keeps in registers per round: the max radix
  constexpr int KMAX = (FftMaxRadix<C>::v / R) > 0 ? FftMaxRadix<C>::v / R : 1;
  const int per_round = (KMAX * (int)blockDim.x) / P::NB;
  for (int l0 = 0; l0 < nb; l0 += per_round) {
    const int total = min(per_round, nb - l0) * P::NB;
    C v[KMAX][R];
#pragma unroll
    for (int q = 0; q < KMAX; ++q) {
      const int w = q * blockDim.x + threadIdx.x;
      if (w < total) {
        const int line = w / P::NB;
        const int j = w - line * P::NB;
        P::load(buf + (size_t)(l0 + line) * ls, j, v[q], tw);
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < KMAX; ++q) {
      const int w = q * blockDim.x + threadIdx.x;
      if (w < total) {
        const int line = w / P::NB;
        const int j = w - line * P::NB;
        P::store(buf + (size_t)(l0 + line) * ls, j, v[q]);
      }
    }
    __syncthreads();
  }
}

template <typename C, int L, bool INV, int Ns, int R, int... Rest>
struct FftRun {
  __device__ __forceinline__ static void go(C* buf, int nb, int ls, const C* tw) {
    fft2_pass<C, L, INV, R, Ns>(buf, nb, ls, tw);
    FftRun<C, L, INV, Ns * R, Rest...>::go(buf, nb, ls, tw);
  }
};
template <typename C, int L, bool INV, int Ns, int R>
struct FftRun<C, L, INV, Ns, R> {
  __device__ __forceinline__ static void go(C* buf, int nb, int ls, const C* tw) {
    fft2_pass<C, L, INV, R, Ns>(buf, nb, ls, tw);
  }
};

template <typename C, int L, bool INV, typename RS> struct FftDo;
template <typename C, int L, bool INV, int... Rs>
struct FftDo<C, L, INV, Radices<Rs...>> {
  __device__ __forceinline__ static void go(C* buf, int nb, int ls, const C* tw) {
    FftRun<C, L, INV, 1, Rs...>::go(buf, nb, ls, tw);
  }
};

// Entry: the lines must be written (at fpos positions) before the call;
// a barrier is taken first, and the result is complete on return.
template <typename C, int L, bool INV>
__device__ __forceinline__ void fft2(C* buf, int nb, int ls, const C* __restrict__ tw) {
  __syncthreads();
  FftDo<C, L, INV, typename FftPlanL<L, FftMaxRadix<C>::v>::R>::go(buf, nb, ls, tw);
}
#endif
