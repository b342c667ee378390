// Wall-normal (Chebyshev) pass kernels: one pencil (kx, kz) per CTA.
//
// Reference counterparts:
//   cheby_s2p / cheby_p2s ........ source/transform.cu:416-748
//   getUVW ....................... source/velocity.cu:22-170
//   ddz_sm ....................... source/RPCFKernels.cu:476-520
//   rhsNonlinear ................. source/nonlinear.cu:130-242
//   worker s2p(No_Padding) ....... source/rhs.cpp:95-97
//   _get_linear_v / _omega_y / u0  source/linear.cpp:86-205
//   AB2 add ...................... source/rhs.cpp:205-215
//   solveEq / m_multi_v .......... source/solver.cpp:107-123, matrix_op.cpp:68-78
//
// The Chebyshev transforms are DCT-I evaluated as complex FFTs of the even
// extension, as the reference does with cuFFT, but in shared memory with the
// project's own FFT (fft.cuh).  Collocation-point values of v, v'', v'''',
// omega, omega'' (the reference's T0/T2/T4 matrix products) are obtained the
// same way: coefficient-space derivatives, then the no-pad DCT.
#include "fftline.cuh"
#include "kernels.cuh"
#include "ypass.cuh"

namespace {

struct Carve {
  char* p;
  __device__ explicit Carve(void* b) : p((char*)b) {}
  template <class T> __device__ T* take(size_t n) {
    T* r = (T*)p;
    p += (n * sizeof(T) + 15) & ~(size_t)15;
    return r;
  }
};

// Chebyshev coefficient derivative executed by one full warp:
// b_i = sum_{j>i, j-i odd} 2 j a_j, b_0 halved (source/RPCFKernels.cu:476-520),
// evaluated as parity-split suffix sums.  a, b in shared memory, no alias.
__device__ void ddz_warp(const double2* a, double2* b, int N) {
  const int lane = threadIdx.x & 31;
  const int c = (N + 31) / 32;
  const int j0 = lane * c;
  const int j1 = min(j0 + c, N);
  double er = 0, ei = 0, orr = 0, oi = 0;
  for (int j = j0; j < j1; ++j) {
    double2 v = a[j];
    double f = 2.0 * j;
    if (j & 1) { orr += f * v.x; oi += f * v.y; }
    else { er += f * v.x; ei += f * v.y; }
  }
  double s0 = er, s1 = ei, s2 = orr, s3 = oi;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    double t0 = __shfl_down_sync(0xffffffffu, s0, d);
    double t1 = __shfl_down_sync(0xffffffffu, s1, d);
    double t2 = __shfl_down_sync(0xffffffffu, s2, d);
    double t3 = __shfl_down_sync(0xffffffffu, s3, d);
    if (lane + d < 32) { s0 += t0; s1 += t1; s2 += t2; s3 += t3; }
  }
  double re_e = s0 - er, im_e = s1 - ei, re_o = s2 - orr, im_o = s3 - oi;
  for (int j = j1 - 1; j >= j0; --j) {
    double2 v = a[j];
    double f = 2.0 * j;
    double2 out = (j & 1) ? make_double2(re_e, im_e) : make_double2(re_o, im_o);
    if (j == 0) out = out * 0.5;
    b[j] = out;
    if (j & 1) { re_o += f * v.x; im_o += f * v.y; }
    else { re_e += f * v.x; im_e += f * v.y; }
  }
}

// even extension for the padded s2p (cheby_pre_s2p_pad): e[0] = c0,
// e[k] = e[M-k] = c_k/2 for 1 <= k <= Ny-1, zero otherwise; M = 4(Ny-1).
template <typename C>
__device__ __forceinline__ double2 ext_s2p_pad(const double2* c, int n, int M, int Ny) {
  if (n == 0) return c[0];
  if (n <= Ny - 1) return c[n] * 0.5;
  if (n >= M - (Ny - 1)) return c[M - n] * 0.5;
  return make_double2(0.0, 0.0);
}

// even extension for the no-pad s2p (cheby_pre_s2p_noPad): M0 = 2(Ny-1);
// e[0] = c0, e[Ny-1] = c_{Ny-1}, e[k] = e[M0-k] = c_k/2 otherwise.
__device__ __forceinline__ double2 ext_s2p_nopad(const double2* c, int n, int M0, int Ny) {
  if (n == 0) return c[0];
  if (n < Ny - 1) return c[n] * 0.5;
  if (n == Ny - 1) return c[n];
  return c[M0 - n] * 0.5;
}

template <typename C>
__device__ __forceinline__ C* pencil_ptr(const PencilArr& a, int f, long long p) {
  return (C*)a.base + (long long)f * a.fs + p * a.ps;
}

}  // namespace

// ---------------------------------------------------------------------------
// Reference-layout in-place Chebyshev transforms (drop-in cheby_s2p/p2s)
// mode 0: s2p pad (FFT length mz), 1: s2p no-pad (mz/2),
// mode 2: p2s pad (mz), 3: p2s no-pad (mz/2).
// ---------------------------------------------------------------------------
template <typename C>
__global__ void k_cheby_inplace(PencilArr arr, long long npencils, int mode, int Ny,
                                FftTab<C> tab, int PB) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* lines = (C*)smem_raw;
  const int L = tab.plan.L;
  const long long p0 = (long long)blockIdx.x * PB;
  const int P = (mode == 2) ? L / 2 + 1 : Ny;  // p2s input points
  for (int w = threadIdx.x; w < PB * L; w += blockDim.x) {
    const int b = w / L;
    const int n = w - b * L;
    const long long p = p0 + b;
    C val = cmk<C>(0.0, 0.0);
    if (p < npencils) {
      const C* src = pencil_ptr<C>(arr, 0, p);
      if (mode == 0) {
        const int nzl = Ny - 1;
        if (n == 0) val = src[0];
        else if (n <= nzl) val = src[n] * (decltype(val.x))0.5;
        else if (n >= L - nzl) val = src[L - n] * (decltype(val.x))0.5;
      } else if (mode == 1) {
        const int nzl = Ny - 1;
        if (n == 0) val = src[0];
        else if (n < nzl) val = src[n] * (decltype(val.x))0.5;
        else if (n == nzl) val = src[n];
        else val = src[L - n] * (decltype(val.x))0.5;
      } else {
        const int Pm = (mode == 2) ? P : Ny;
        val = (n < Pm) ? src[n] : src[L - n];
      }
    }
    lines[(size_t)b * L + tab.drev[n]] = val;
  }
  fft_batch<C, false>(lines, PB, L, tab.plan, tab.tw);
  for (int w = threadIdx.x; w < PB * L; w += blockDim.x) {
    const int b = w / L;
    const int k = w - b * L;
    const long long p = p0 + b;
    if (p >= npencils) continue;
    C v = lines[(size_t)b * L + k];
    if (mode >= 2) {
      const int Pm = L / 2 + 1;
      if (k < Pm) {
        v = v * (decltype(v.x))(1.0 / (Pm - 1));
        if (k == 0 || k == Pm - 1) v = v * (decltype(v.x))0.5;
      }
    }
    pencil_ptr<C>(arr, 0, p)[k] = v;
  }
}

// ---------------------------------------------------------------------------
// getUVW on reference-layout pencils (six fields, FP64)
// ---------------------------------------------------------------------------
struct SixPtr {
  double2* f[6];  // u, v(span), w(wall), omega_x, omega_y, omega_z(wall)
  long long ps;
};

__global__ void k_get_uvw(SixPtr a, DnsGeom g, PhysParams ph) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Ny = g.Ny;
  Carve cv(smem_raw);
  double2* w = cv.take<double2>(Ny);
  double2* oz = cv.take<double2>(Ny);
  double2* Dw = cv.take<double2>(Ny);
  double2* u = cv.take<double2>(Ny);
  double2* v = cv.take<double2>(Ny);
  double2* Du = cv.take<double2>(Ny);
  double2* Dv = cv.take<double2>(Ny);
  const long long p = blockIdx.x;
  const int kx = (int)(p % g.Kx);
  const int kz = (int)(p / g.Kx);
  const bool zero = (kx == 0 && kz == 0);
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = kmn_of(ia, ib);
  const double kmn1 = zero ? 0.0 : 1.0 / kmn;
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    w[n] = a.f[2][p * a.ps + n];
    oz[n] = a.f[5][p * a.ps + n];
  }
  __syncthreads();
  if (!zero && threadIdx.x < 32) ddz_warp(w, Dw, Ny);
  __syncthreads();
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    if (zero) {
      u[n] = w[n];
      v[n] = oz[n];
    } else {
      const double2 d = Dw[n], o = oz[n];
      // u = i(ia/k^2) Dw - i(ib/k^2) oz ; v = i(ib/k^2) Dw + i(ia/k^2) oz
      u[n] = muli(d * (ia * kmn1)) - muli(o * (ib * kmn1));
      v[n] = muli(d * (ib * kmn1)) + muli(o * (ia * kmn1));
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  if (warp == 0) ddz_warp(v, Dv, Ny);
  if (warp == 1) ddz_warp(u, Du, Ny);
  __syncthreads();
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    const double2 wn = w[n];
    a.f[0][p * a.ps + n] = u[n];
    a.f[1][p * a.ps + n] = v[n];
    const double2 ox = Dv[n] - muli(wn * ib);
    const double2 oy = muli(wn * ia) - Du[n];
    a.f[3][p * a.ps + n] = ox;
    a.f[4][p * a.ps + n] = oy;
    if (zero) {
      a.f[2][p * a.ps + n] = make_double2(0.0, 0.0);
      a.f[5][p * a.ps + n] = make_double2(0.0, 0.0);
    }
  }
}

// ---------------------------------------------------------------------------
// rhsNonlinear on reference-layout pencils (FP64)
// ---------------------------------------------------------------------------
__global__ void k_rhs_nonlinear(double2* lx, double2* ly, const double2* lz, long long ps,
                                DnsGeom g, PhysParams ph) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Ny = g.Ny;
  Carve cv(smem_raw);
  double2* ax = cv.take<double2>(Ny);
  double2* ay = cv.take<double2>(Ny);
  double2* Dx = cv.take<double2>(Ny);
  double2* Dy = cv.take<double2>(Ny);
  const long long p = blockIdx.x;
  const int kx = (int)(p % g.Kx);
  const int kz = (int)(p / g.Kx);
  if (kx == 0 && kz == 0) return;  // source/nonlinear.cu:157
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = kmn_of(ia, ib);
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    ax[n] = lx[p * ps + n];
    ay[n] = ly[p * ps + n];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  if (warp == 0) ddz_warp(ax, Dx, Ny);
  if (warp == 1) ddz_warp(ay, Dy, Ny);
  __syncthreads();
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    const double2 hv = lz[p * ps + n] * kmn + muli(Dx[n] * ia) + muli(Dy[n] * ib);
    const double2 ho = muli(ay[n] * ia) - muli(ax[n] * ib);
    lx[p * ps + n] = hv;
    ly[p * ps + n] = ho;
  }
}

// ---------------------------------------------------------------------------
// solveEq: rhs <- inv * rhs per pencil, inverses row-major [pencil][N][N]
// (source/solver.cpp:107-123).  One warp per row, lanes over columns.
// ---------------------------------------------------------------------------
__global__ void k_solve_eq(const double2* __restrict__ inv, double2* rhs, long long ps,
                           int N, long long npencils) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* r = (double2*)smem_raw;
  double2* x = r + N;
  const long long p = blockIdx.x;
  if (p >= npencils) return;
  for (int n = threadIdx.x; n < N; n += blockDim.x) r[n] = rhs[p * ps + n];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  const double2* A = inv + p * (long long)N * N;
  for (int i = threadIdx.x >> 5; i < N; i += nw) {
    double sr = 0, si = 0;
    for (int j = lane; j < N; j += 32) {
      const double2 a = __ldg(A + (long long)i * N + j);
      const double2 b = r[j];
      sr += a.x * b.x - a.y * b.y;
      si += a.x * b.y + a.y * b.x;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      sr += __shfl_down_sync(0xffffffffu, sr, d);
      si += __shfl_down_sync(0xffffffffu, si, d);
    }
    if (lane == 0) x[i] = make_double2(sr, si);
  }
  __syncthreads();
  for (int n = threadIdx.x; n < N; n += blockDim.x) rhs[p * ps + n] = x[n];
}

// ---------------------------------------------------------------------------
// Fused backward wall-normal pass (step start): getUVW from the FP64 state
// then the padded s2p of all six fields, written pencil-major for the
// spanwise pass.  Fields: u, v(span), w(wall), omega_x, omega_y, omega_z.
// ---------------------------------------------------------------------------
template <typename C, int LM>
__global__ void __launch_bounds__(256, 3) k_y3(const double2* __restrict__ V, const double2* __restrict__ O,
                     PencilArr out, DnsGeom g, PhysParams ph, FftTab<C> tab) {
  typedef FLine<C, LM> FL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Ny = g.Ny;
  const int M = tab.plan.L;  // 4 (Ny - 1)
  const int ls = FL::stride(M);
  Carve cv(smem_raw);
  double2* w = cv.take<double2>(Ny);
  double2* oz = cv.take<double2>(Ny);
  double2* Dw = cv.take<double2>(Ny);
  double2* u = cv.take<double2>(Ny);
  double2* v = cv.take<double2>(Ny);
  double2* Du = cv.take<double2>(Ny);
  double2* Dv = cv.take<double2>(Ny);
  double2* ox = cv.take<double2>(Ny);
  double2* oy = cv.take<double2>(Ny);
  C* lines = cv.take<C>((size_t)6 * ls);
  const long long p = blockIdx.x;
  const int kx = (int)(p % g.Kx);
  const int kz = (int)(p / g.Kx);
  const bool zero = (kx == 0 && kz == 0);
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = kmn_of(ia, ib);
  const double kmn1 = zero ? 0.0 : 1.0 / kmn;
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    w[n] = V[p * Ny + n];
    oz[n] = O[p * Ny + n];
  }
  __syncthreads();
  if (!zero && threadIdx.x < 32) ddz_warp(w, Dw, Ny);
  __syncthreads();
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    if (zero) {
      u[n] = w[n];
      v[n] = oz[n];
    } else {
      const double2 d = Dw[n], o = oz[n];
      u[n] = muli(d * (ia * kmn1)) - muli(o * (ib * kmn1));
      v[n] = muli(d * (ib * kmn1)) + muli(o * (ia * kmn1));
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  if (warp == 0) ddz_warp(v, Dv, Ny);
  if (warp == 1) ddz_warp(u, Du, Ny);
  __syncthreads();
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    const double2 wn = w[n];
    ox[n] = Dv[n] - muli(wn * ib);
    oy[n] = muli(wn * ia) - Du[n];
    if (zero) { w[n] = make_double2(0.0, 0.0); oz[n] = make_double2(0.0, 0.0); }
  }
  __syncthreads();
  const double2* src[6] = {u, v, w, ox, oy, oz};
  for (int t = threadIdx.x; t < 6 * M; t += blockDim.x) {
    const int f = t / M;
    const int n = t - f * M;
    lines[(size_t)f * ls + FL::in_pos(tab, n)] = from_d2<C>(ext_s2p_pad<C>(src[f], n, M, Ny));
  }
  FL::template fft<false>(lines, 6, ls, tab);
  const int Py = g.Py;
  for (int t = threadIdx.x; t < 6 * Py; t += blockDim.x) {
    const int f = t / Py;
    const int j = t - f * Py;
    pencil_ptr<C>(out, f, p)[j] = lines[(size_t)f * ls + FL::out_pos(j)];
  }
}

// ---------------------------------------------------------------------------
// Fused forward wall-normal pass: padded p2s of the three Lamb components,
// rhsNonlinear, no-pad s2p to collocation values, then (unless boot) the
// CN explicit operators and AB2 for v, omega_y and the mean modes.
//   boot: only store the nonlinear terms as the AB2 history (the effect of
//         the reference's "extra previous step", source/main_loop.cpp:39-52).
// ---------------------------------------------------------------------------
template <typename C, int LM, int LM0>
__global__ void __launch_bounds__(256, 3) k_y1(PencilArr lam, const double2* __restrict__ V, const double2* __restrict__ O,
                     double2* Nvp, double2* Nop, double2* rv, double2* ro,
                     const double* __restrict__ Ut, const double* __restrict__ ddUt,
                     DnsGeom g, PhysParams ph, FftTab<C> tabP, FftTab<double2> tab0,
                     int boot) {
  typedef FLine<C, LM> FP;
  typedef FLine<double2, LM0> F0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Ny = g.Ny;
  const int Py = g.Py;
  const int M = tabP.plan.L;   // 2 (Py - 1)
  const int M0 = tab0.plan.L;  // 2 (Ny - 1)
  const int lsP = FP::stride(M);
  const int ls0 = F0::stride(M0);
  Carve cv(smem_raw);
  double2* lc = cv.take<double2>((size_t)3 * Ny);  // lambda coefficients
  double2* D1 = cv.take<double2>((size_t)2 * Ny);  // D lambda_x, D lambda_y
  double2* Hv = cv.take<double2>(Ny);
  double2* Ho = cv.take<double2>(Ny);
  double2* Vc = cv.take<double2>(Ny);
  double2* Oc = cv.take<double2>(Ny);
  double2* t1 = cv.take<double2>(Ny);
  double2* t3 = cv.take<double2>(Ny);
  double2* D2V = cv.take<double2>(Ny);
  double2* D2O = cv.take<double2>(Ny);
  double2* t2 = cv.take<double2>(Ny);
  double2* D4V = cv.take<double2>(Ny);
  double2* nvp = cv.take<double2>(Ny);
  double2* nop = cv.take<double2>(Ny);
  const size_t bytesP = (size_t)3 * lsP * sizeof(C);
  const size_t bytes0 = (size_t)7 * ls0 * sizeof(double2);
  unsigned char* region = (unsigned char*)cv.take<unsigned char>(bytesP > bytes0 ? bytesP : bytes0);
  C* linesP = (C*)region;
  double2* lines0 = (double2*)region;

  const long long p = blockIdx.x;
  const int kx = (int)(p % g.Kx);
  const int kz = (int)(p / g.Kx);
  const bool zero = (kx == 0 && kz == 0);
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = kmn_of(ia, ib);

  // 1. load Lamb pencils as even extensions (DCT-I of Py points); state
  for (int t = threadIdx.x; t < 3 * M; t += blockDim.x) {
    const int f = t / M;
    const int n = t - f * M;
    const C* src = pencil_ptr<C>(lam, f, p);
    linesP[(size_t)f * lsP + FP::in_pos(tabP, n)] = (n < Py) ? src[n] : src[M - n];
  }
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    Vc[n] = V[p * Ny + n];
    Oc[n] = O[p * Ny + n];
    nvp[n] = Nvp[p * Ny + n];
    nop[n] = Nop[p * Ny + n];
  }
  FP::template fft<false>(linesP, 3, lsP, tabP);
  const double sc = 1.0 / (Py - 1);
  for (int t = threadIdx.x; t < 3 * Ny; t += blockDim.x) {
    const int f = t / Ny;
    const int k = t - f * Ny;
    double2 c = to_d2(linesP[(size_t)f * lsP + FP::out_pos(k)]) * sc;
    if (k == 0) c = c * 0.5;
    lc[t] = c;
  }
  __syncthreads();
  // 2. derivatives (independent chains on separate warps)
  const int warp = threadIdx.x >> 5;
  if (warp == 0) ddz_warp(lc, D1, Ny);
  if (warp == 1) ddz_warp(lc + Ny, D1 + Ny, Ny);
  if (!boot) {
    if (warp == 2) ddz_warp(Vc, t1, Ny);
    if (warp == 3) ddz_warp(Oc, t3, Ny);
  }
  __syncthreads();
  if (!boot) {
    if (warp == 0) ddz_warp(t1, D2V, Ny);
    if (warp == 1) ddz_warp(t3, D2O, Ny);
    __syncthreads();
    if (warp == 0) ddz_warp(D2V, t2, Ny);
    __syncthreads();
    if (warp == 0) ddz_warp(t2, D4V, Ny);
  }
  // 3. nonlinear terms in coefficient space
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    if (zero) {
      Hv[n] = lc[n];
      Ho[n] = lc[Ny + n];
    } else {
      Hv[n] = lc[2 * Ny + n] * kmn + muli(D1[n] * ia) + muli(D1[Ny + n] * ib);
      Ho[n] = muli(lc[Ny + n] * ia) - muli(lc[n] * ib);
    }
  }
  __syncthreads();
  // 4. no-pad s2p: collocation values of Hv, Ho, V, V'', V'''', O, O''
  const int nl = boot ? 2 : 7;
  const double2* srcs[7] = {Hv, Ho, Vc, D2V, D4V, Oc, D2O};
  for (int t = threadIdx.x; t < nl * M0; t += blockDim.x) {
    const int f = t / M0;
    const int n = t - f * M0;
    lines0[(size_t)f * ls0 + F0::in_pos(tab0, n)] = ext_s2p_nopad(srcs[f], n, M0, Ny);
  }
  F0::template fft<false>(lines0, nl, ls0, tab0);
  // collocation value at point m of line f (natural order)
  auto col = [&](int f, int m) { return lines0[(size_t)f * ls0 + F0::out_pos(m)]; };
  if (boot) {
    for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
      Nvp[p * Ny + n] = col(0, n);
      Nop[p * Ny + n] = col(1, n);
    }
    return;
  }
  const double dt = ph.dt, Re = ph.Re, al = ia;
  const int N = Ny - 1;
  // lines: 0 Nv, 1 No, 2 v, 3 v'', 4 v(4), 5 omega, 6 omega''
  for (int i = threadIdx.x; i < Ny; i += blockDim.x) {
    double2 rvi = make_double2(0.0, 0.0), roi = make_double2(0.0, 0.0);
    if (zero) {
      // _get_linear_u0 / _w0: rows 2..N at point i-1
      if (i >= 2) {
        const int m = i - 1;
        rvi = col(2, m) + col(3, m) * (dt * 0.5 / Re) - (col(0, m) * 1.5 - nvp[m] * 0.5) * dt;
        roi = col(5, m) + col(6, m) * (dt * 0.5 / Re) - (col(1, m) * 1.5 - nop[m] * 0.5) * dt;
      }
    } else {
      if (i >= 4 && i <= N) {
        const int m = i - 2;
        const double Um = Ut[m];
        const double2 P0 = col(2, m), P2 = col(3, m), P4 = col(4, m);
        const double2 re = P4 * (dt * 0.5 / Re) + P2 * (1 - kmn * dt / Re)
                           - P0 * (kmn * (1 - kmn * dt * 0.5 / Re));
        const double2 im = P2 * (-al * dt * 0.5 * Um)
                           + P0 * (kmn * al * dt * 0.5 * Um + al * dt * 0.5 * ddUt[m]);
        rvi = re + muli(im) + (col(0, m) * 1.5 - nvp[m] * 0.5) * dt;
      }
      if (i >= 2) {
        const int m = i - 1;
        const double2 Q0 = col(5, m), Q2 = col(6, m);
        const double2 re = Q2 * (0.5 / Re * dt) + Q0 * (1 - kmn * dt * 0.5 / Re);
        const double2 im = Q0 * (-al * dt * 0.5 * Ut[m]);
        roi = re + muli(im) + (col(1, m) * 1.5 - nop[m] * 0.5) * dt;
      }
    }
    rv[p * Ny + i] = rvi;
    ro[p * Ny + i] = roi;
    Nvp[p * Ny + i] = col(0, i);
    Nop[p * Ny + i] = col(1, i);
  }
}

// ---------------------------------------------------------------------------
// Per-mode solves.  One CTA per operator slot (kx, kz'), kz' in [0, Nz/2];
// the operator depends on kz only through beta^2, so pencils kz' and Nz-kz'
// share it.  Explicit inverses are stored transposed, AT[slot][eq][j][i],
// and streamed through a shared-memory ring with cp.async.bulk + mbarrier.
// Between the v and omega solves the tilting term -i beta U' dt/2 (v^{n+1}
// + v^n) of source/linear.cpp:147-151 is added at the collocation points.
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// Bounded wait: gives up after `limit` SM clock cycles (about a second), or
// at once when another CTA has already reported a timeout in *status
// (status == nullptr: no early exit, used to drain copies in flight).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit,
                                                  const int* status) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
    if (status && (*(volatile const int*)status & 1)) return false;
  }
  return true;
}
}  // namespace

#define Y2_WAIT_LIMIT (1LL << 31)

template <int LM0>
__global__ void k_y2(const double2* __restrict__ AT, double2* V, double2* O,
                     const double2* __restrict__ rv, const double2* __restrict__ ro,
                     const double* __restrict__ dUt, DnsGeom g, PhysParams ph,
                     FftTab<double2> tab0, int CH, int NST, int* status) {
  typedef FLine<double2, LM0> F0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Ny = g.Ny;
  const int M0 = tab0.plan.L;
  const int ls0 = F0::stride(M0);
  Carve cv(smem_raw);
  uint64_t* full = cv.take<uint64_t>(NST);
  double2* ring = cv.take<double2>((size_t)NST * CH * Ny);
  double2* r = cv.take<double2>((size_t)2 * Ny);    // current right-hand sides
  double2* ro_s = cv.take<double2>((size_t)2 * Ny); // omega right-hand sides
  double2* vold = cv.take<double2>((size_t)2 * Ny);
  double2* xv = cv.take<double2>((size_t)2 * Ny);
  double2* lines = cv.take<double2>((size_t)2 * ls0);

  const int kx = blockIdx.x % g.Kx;
  const int kzs = blockIdx.x / g.Kx;  // slot kz' in [0, Nz/2]
  const long long slot = blockIdx.x;
  const int npen = (kzs == 0 || kzs == g.Nz / 2) ? 1 : 2;
  long long pen[2];
  pen[0] = (long long)kzs * g.Kx + kx;
  pen[1] = (long long)(g.Nz - kzs) * g.Kx + kx;
  const bool zero = (kx == 0 && kzs == 0);
  const long long NN = (long long)Ny * Ny;
  const double2* Av = AT + slot * 2 * NN;
  const double2* Ao = Av + NN;
  const int nch = (Ny + CH - 1) / CH;
  const int nchunks = 2 * nch;
  const int tid = threadIdx.x;

  if (tid == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  for (int t = tid; t < npen * Ny; t += blockDim.x) {
    const int b = t / Ny;
    const int n = t - b * Ny;
    r[t] = rv[pen[b] * Ny + n];
    ro_s[t] = ro[pen[b] * Ny + n];
    vold[t] = V[pen[b] * Ny + n];
  }
  __syncthreads();
  auto issue = [&](int c) {
    const int s = c % NST;
    const int e = c / nch;
    const int j0 = (c - e * nch) * CH;
    const int ncol = min(CH, Ny - j0);
    const uint32_t bytes = (uint32_t)(ncol * Ny * sizeof(double2));
    const double2* src = (e == 0 ? Av : Ao) + (long long)j0 * Ny;
    mbar_expect_tx(&full[s], bytes);
    bulk_g2s(ring + (size_t)s * CH * Ny, src, bytes, &full[s]);
  };
  if (tid == 0)
    for (int c = 0; c < min(NST, nchunks); ++c) issue(c);

  const int b = tid / Ny;        // right-hand side handled by this thread
  const int i = tid - b * Ny;    // output row
  const bool active = (b < npen);
  double2 acc = make_double2(0.0, 0.0);
  for (int c = 0; c < nchunks; ++c) {
    if (c == nch) {
      // v solved: keep it, then add the tilting term to the omega rhs
      if (active) xv[b * Ny + i] = acc;
      acc = make_double2(0.0, 0.0);
      __syncthreads();
      if (!zero) {
        for (int t = tid; t < npen * M0; t += blockDim.x) {
          const int bb = t / M0;
          const int n = t - bb * M0;
          // S = v^{n+1} + v^n, even extension for the no-pad s2p
          int src;
          double sc;
          if (n == 0) { src = 0; sc = 1.0; }
          else if (n < Ny - 1) { src = n; sc = 0.5; }
          else if (n == Ny - 1) { src = n; sc = 1.0; }
          else { src = M0 - n; sc = 0.5; }
          const double2 sv = (xv[bb * Ny + src] + vold[bb * Ny + src]) * sc;
          lines[(size_t)bb * ls0 + F0::in_pos(tab0, n)] = sv;
        }
        F0::template fft<false>(lines, npen, ls0, tab0);
        if (active && i >= 2) {
          const int m = i - 1;
          const int kzp = (b == 0) ? kzs : g.Nz - kzs;
          double iab, ibb;
          wavenumbers(kx, kzp, g.Nz, ph.aphi, ph.beta, iab, ibb);
          const double coef = -0.5 * ibb * dUt[m] * ph.dt;
          ro_s[b * Ny + i] = ro_s[b * Ny + i] + muli(lines[(size_t)b * ls0 + F0::out_pos(m)] * coef);
        }
      }
      __syncthreads();
    }
    const int s = c % NST;
    const uint32_t par = (uint32_t)((c / NST) & 1);
    const bool ok = mbar_wait_bounded(&full[s], par, Y2_WAIT_LIMIT, status);
    const int e = c / nch;
    const int j0 = (c - e * nch) * CH;
    const int ncol = min(CH, Ny - j0);
    if (ok && active) {
      const double2* rr = (e == 0 ? r : ro_s) + b * Ny + j0;
      const double2* A = ring + (size_t)s * CH * Ny;
      double ar = acc.x, ai = acc.y;
      for (int jj = 0; jj < ncol; ++jj) {
        const double2 a = A[jj * Ny + i];
        const double2 x = rr[jj];
        ar += a.x * x.x - a.y * x.y;
        ai += a.x * x.y + a.y * x.x;
      }
      acc = make_double2(ar, ai);
    }
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicOr(status, 1);
        // let the copies already in flight land before the CTA exits
        for (int cc = c; cc < min(c + NST, nchunks); ++cc)
          mbar_wait_bounded(&full[cc % NST], (uint32_t)((cc / NST) & 1), Y2_WAIT_LIMIT, nullptr);
      }
      return;
    }
    if (tid == 0 && c + NST < nchunks) issue(c + NST);
  }
  if (active) {
    V[pen[b] * Ny + i] = xv[b * Ny + i];
    O[pen[b] * Ny + i] = acc;
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
size_t y3_smem(int Ny, int ls, size_t csz) {
  auto a = [](size_t b) { return (b + 15) & ~(size_t)15; };
  return 9 * a((size_t)Ny * 16) + a((size_t)6 * ls * csz);
}
size_t y1_smem(int Ny, int lsP, int ls0, size_t csz) {
  auto a = [](size_t b) { return (b + 15) & ~(size_t)15; };
  size_t s = a((size_t)3 * Ny * 16) + a((size_t)2 * Ny * 16) + 12 * a((size_t)Ny * 16);
  size_t bp = (size_t)3 * lsP * csz, b0 = (size_t)7 * ls0 * 16;
  return s + a(bp > b0 ? bp : b0);
}
size_t y2_smem(int Ny, int ls0, int CH, int NST) {
  auto a = [](size_t b) { return (b + 15) & ~(size_t)15; };
  return a((size_t)NST * 8) + a((size_t)NST * CH * Ny * 16) + 4 * a((size_t)2 * Ny * 16) +
         a((size_t)2 * ls0 * 16);
}

template <typename C>
cudaError_t launch_cheby_inplace(PencilArr arr, long long npencils, int mode, int Ny,
                                 FftTab<C> tab, cudaStream_t st) {
  const int L = tab.plan.L;
  int PB = (int)(32768 / ((size_t)L * sizeof(C)));
  if (PB < 1) PB = 1;
  if (PB > 8) PB = 8;
  const size_t sm = (size_t)PB * L * sizeof(C);
  cudaFuncSetAttribute(k_cheby_inplace<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const long long nb = (npencils + PB - 1) / PB;
  k_cheby_inplace<C><<<(unsigned)nb, 256, sm, st>>>(arr, npencils, mode, Ny, tab, PB);
  return cudaGetLastError();
}
template cudaError_t launch_cheby_inplace<double2>(PencilArr, long long, int, int, FftTab<double2>, cudaStream_t);

cudaError_t launch_get_uvw(double2* const f[6], long long ps, DnsGeom g, PhysParams ph,
                           cudaStream_t st) {
  SixPtr a;
  for (int i = 0; i < 6; ++i) a.f[i] = f[i];
  a.ps = ps;
  const size_t sm = 7 * (((size_t)g.Ny * 16 + 15) & ~(size_t)15);
  cudaFuncSetAttribute(k_get_uvw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_get_uvw<<<(unsigned)g.H, 128, sm, st>>>(a, g, ph);
  return cudaGetLastError();
}

cudaError_t launch_rhs_nonlinear(double2* lx, double2* ly, const double2* lz, long long ps,
                                 DnsGeom g, PhysParams ph, cudaStream_t st) {
  const size_t sm = 4 * (((size_t)g.Ny * 16 + 15) & ~(size_t)15);
  cudaFuncSetAttribute(k_rhs_nonlinear, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_rhs_nonlinear<<<(unsigned)g.H, 128, sm, st>>>(lx, ly, lz, ps, g, ph);
  return cudaGetLastError();
}

cudaError_t launch_solve_eq(const double2* inv, double2* rhs, long long ps, int N,
                            long long npencils, cudaStream_t st) {
  const size_t sm = (size_t)2 * N * 16;
  cudaFuncSetAttribute(k_solve_eq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_solve_eq<<<(unsigned)npencils, 256, sm, st>>>(inv, rhs, ps, N, npencils);
  return cudaGetLastError();
}

template <typename C>
cudaError_t launch_y3(const double2* V, const double2* O, PencilArr out, DnsGeom g,
                      PhysParams ph, FftTab<C> tab, cudaStream_t st) {
  return with_len_m(tab.plan.L, [&](auto LL) {
    constexpr int L = decltype(LL)::value;
    const size_t sm = y3_smem(g.Ny, FLine<C, L>::stride(tab.plan.L), sizeof(C));
    cudaFuncSetAttribute(k_y3<C, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_y3<C, L><<<(unsigned)g.H, 256, sm, st>>>(V, O, out, g, ph, tab);
    return cudaGetLastError();
  });
}
template cudaError_t launch_y3<double2>(const double2*, const double2*, PencilArr, DnsGeom, PhysParams, FftTab<double2>, cudaStream_t);
template cudaError_t launch_y3<float2>(const double2*, const double2*, PencilArr, DnsGeom, PhysParams, FftTab<float2>, cudaStream_t);

template <typename C>
cudaError_t launch_y1(PencilArr lam, const double2* V, const double2* O, double2* Nvp,
                      double2* Nop, double2* rv, double2* ro, const double* Ut,
                      const double* ddUt, DnsGeom g, PhysParams ph, FftTab<C> tabP,
                      FftTab<double2> tab0, int boot, cudaStream_t st) {
  return with_len_m(tabP.plan.L, [&](auto LL) {
    constexpr int L = decltype(LL)::value;
    constexpr int L0 = L / 2;  // the no-pad extension is half the padded one
    const size_t sm = y1_smem(g.Ny, FLine<C, L>::stride(tabP.plan.L),
                              FLine<double2, L0>::stride(tab0.plan.L), sizeof(C));
    cudaFuncSetAttribute(k_y1<C, L, L0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_y1<C, L, L0><<<(unsigned)g.H, 256, sm, st>>>(lam, V, O, Nvp, Nop, rv, ro, Ut, ddUt, g, ph,
                                                   tabP, tab0, boot);
    return cudaGetLastError();
  });
}
template cudaError_t launch_y1<double2>(PencilArr, const double2*, const double2*, double2*, double2*, double2*, double2*, const double*, const double*, DnsGeom, PhysParams, FftTab<double2>, FftTab<double2>, int, cudaStream_t);
template cudaError_t launch_y1<float2>(PencilArr, const double2*, const double2*, double2*, double2*, double2*, double2*, const double*, const double*, DnsGeom, PhysParams, FftTab<float2>, FftTab<double2>, int, cudaStream_t);

cudaError_t launch_y2(const double2* AT, double2* V, double2* O, const double2* rv,
                      const double2* ro, const double* dUt, DnsGeom g, PhysParams ph,
                      FftTab<double2> tab0, int* status, cudaStream_t st) {
  const int CH = 8;
  const int NST = 4;
  // the tilting transform is a small part of this kernel: the runtime-length
  // FFT keeps its register footprint (and so the occupancy) low
  return with_len_m0(0, [&](auto LL) {
    constexpr int L = decltype(LL)::value;
    const size_t sm = y2_smem(g.Ny, FLine<double2, L>::stride(tab0.plan.L), CH, NST);
    cudaFuncSetAttribute(k_y2<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int threads = ((2 * g.Ny + 31) / 32) * 32;
    if (threads < 64) threads = 64;
    const unsigned nslots = (unsigned)(g.Kx * g.Kh);
    k_y2<L><<<nslots, threads, sm, st>>>(AT, V, O, rv, ro, dUt, g, ph, tab0, CH, NST, status);
    return cudaGetLastError();
  });
}
