// Shared-memory mixed-radix FFT (radix 4, 2, 3), in place, decimation in
// time with the input loaded in digit-reversed order.
//
// A plan factors L = R_1 * ... * R_S (radices 4, 2, 3).  With
// m_0 = 1 and m_s = R_1 ... R_s, stage s combines R_s sub-transforms of size
// m_{s-1} into one of size m_s: for block b and k < m_{s-1} the elements at
// b*m_s + k + r*m_{s-1} (r < R_s) are multiplied by W_{m_s}^{r k} and
// replaced by their R_s-point DFT.  The natural index n goes to position
// digitrev(n) (mixed-radix digits of n, least significant first in R_S,
// ..., R_1, become the most significant first).  Twiddles come from a table
// W_L^j = exp(-2 pi i j / L), j < L, computed on the host in long double.
//
// All threads of the block cooperate on a batch of lines; every stage ends
// with a block barrier.  The per-butterfly body is __host__ __device__ so
// the plan and the index arithmetic are tested on the CPU.
#pragma once
#include "dns_common.cuh"

#define FFT_MAX_STAGES 12

struct FftPlan {
  int L;
  int S;
  int R[FFT_MAX_STAGES];
  int m[FFT_MAX_STAGES + 1];
};

static inline bool fft_make_plan(int L, FftPlan* p) {
  p->L = L;
  p->S = 0;
  p->m[0] = 1;
  int rem = L;
  int radix_seq[FFT_MAX_STAGES];
  int ns = 0;
  while (rem % 4 == 0) { radix_seq[ns++] = 4; rem /= 4; if (ns >= FFT_MAX_STAGES) return false; }
  while (rem % 2 == 0) { radix_seq[ns++] = 2; rem /= 2; if (ns >= FFT_MAX_STAGES) return false; }
  while (rem % 3 == 0) { radix_seq[ns++] = 3; rem /= 3; if (ns >= FFT_MAX_STAGES) return false; }
  if (rem != 1 || L < 2) return false;
  p->S = ns;
  for (int s = 0; s < ns; ++s) {
    p->R[s] = radix_seq[s];
    p->m[s + 1] = p->m[s] * radix_seq[s];
  }
  return true;
}

DNS_HD int fft_digitrev(const FftPlan& P, int n) {
  int pos = 0;
  int rem = n;
  for (int s = P.S - 1; s >= 0; --s) {
    int r = rem % P.R[s];
    rem /= P.R[s];
    pos += r * P.m[s];
  }
  return pos;
}

// One butterfly: stage s, butterfly t in [0, L/R_s), on one line.
template <typename C, bool INV>
DNS_HD void fft_butterfly(C* line, const FftPlan& P, int s, int t, const C* tw) {
  const int R = P.R[s];
  const int mp = P.m[s];
  const int mc = mp * R;
  const int b = t / mp;
  const int k = t - b * mp;
  const int tstride = P.L / mc;
  C* x = line + b * mc + k;
  typedef decltype(x->x) T;
  if (R == 4) {
    C y0 = x[0];
    C y1 = x[mp];
    C y2 = x[2 * mp];
    C y3 = x[3 * mp];
    if (k) {
      C w1 = tw[k * tstride], w2 = tw[2 * k * tstride], w3 = tw[3 * k * tstride];
      if (INV) { y1 = cmulc(y1, w1); y2 = cmulc(y2, w2); y3 = cmulc(y3, w3); }
      else { y1 = cmul(y1, w1); y2 = cmul(y2, w2); y3 = cmul(y3, w3); }
    }
    C a = y0 + y2, bb = y0 - y2, c = y1 + y3, d = y1 - y3;
    C id = muli(d);
    x[0] = a + c;
    x[2 * mp] = a - c;
    if (INV) { x[mp] = bb + id; x[3 * mp] = bb - id; }
    else { x[mp] = bb - id; x[3 * mp] = bb + id; }
  } else if (R == 2) {
    C y0 = x[0];
    C y1 = x[mp];
    if (k) {
      C w1 = tw[k * tstride];
      y1 = INV ? cmulc(y1, w1) : cmul(y1, w1);
    }
    x[0] = y0 + y1;
    x[mp] = y0 - y1;
  } else {  // R == 3
    C y0 = x[0];
    C y1 = x[mp];
    C y2 = x[2 * mp];
    if (k) {
      C w1 = tw[k * tstride], w2 = tw[2 * k * tstride];
      if (INV) { y1 = cmulc(y1, w1); y2 = cmulc(y2, w2); }
      else { y1 = cmul(y1, w1); y2 = cmul(y2, w2); }
    }
    const T c3 = (T)(-0.5);
    const T s3 = (T)0.86602540378443864676372317075294;
    C t1 = y1 + y2;
    C t2 = y1 - y2;
    C base = y0 + t1 * c3;
    C its = muli(t2) * s3;  // i * s * (y1 - y2)
    x[0] = y0 + t1;
    if (INV) { x[mp] = base + its; x[2 * mp] = base - its; }
    else { x[mp] = base - its; x[2 * mp] = base + its; }
  }
}

#ifdef __CUDACC__
// Batched in-place FFT over nb lines of stride ls (elements) in shared
// memory.  Lines must already hold their input in digit-reversed order.
// Starts and ends with a block barrier.
template <typename C, bool INV>
__device__ void fft_batch(C* buf, int nb, int ls, const FftPlan& P, const C* __restrict__ tw) {
  for (int s = 0; s < P.S; ++s) {
    __syncthreads();
    const int nbf = P.L / P.R[s];
    const int total = nb * nbf;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
      const int line = w / nbf;
      const int t = w - line * nbf;
      fft_butterfly<C, INV>(buf + (size_t)line * ls, P, s, t, tw);
    }
  }
  __syncthreads();
}
#endif
