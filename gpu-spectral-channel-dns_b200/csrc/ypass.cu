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
//                                  (reference-layout op; the time step solves
//                                  the banded systems of wallsolve.cu)
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
// CN explicit operators, AB2 and the v^n half of the tilting term for v,
// omega_y and the mean modes at the collocation points; finally the values
// (zero at the points an equation does not use) go back to coefficients
// (no-pad p2s) and are integrated K times (K = 4 for v, 2 for omega_y and
// the mean modes): the right-hand sides of the banded systems of
// wallsolve.h, rows K .. K+n-1.
//   boot: only store the nonlinear terms as the AB2 history (the effect of
//         the reference's "extra previous step", source/main_loop.cpp:39-52).
// ---------------------------------------------------------------------------
template <typename C, int LM, int LM0>
__global__ void __launch_bounds__(256, 3) k_y1(PencilArr lam, const double2* __restrict__ V, const double2* __restrict__ O,
                     double2* Nvp, double2* Nop, double2* gv, double2* go, RhsDims rd,
                     const double* __restrict__ Ut, const double* __restrict__ dUt,
                     const double* __restrict__ ddUt,
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
  // work region of 15 Ny: coefficient-space arrays, reused at the end for the
  // right-hand-side values and their integration
  double2* wk = cv.take<double2>((size_t)15 * Ny);
  double2* lc = wk;              // lambda coefficients (3 Ny)
  double2* D1 = wk + 3 * Ny;     // D lambda_x, D lambda_y (2 Ny)
  double2* Hv = wk + 5 * Ny;
  double2* Ho = wk + 6 * Ny;
  double2* Vc = wk + 7 * Ny;
  double2* Oc = wk + 8 * Ny;
  double2* t1 = wk + 9 * Ny;
  double2* t3 = wk + 10 * Ny;
  double2* D2V = wk + 11 * Ny;
  double2* D2O = wk + 12 * Ny;
  double2* t2 = wk + 13 * Ny;
  double2* D4V = wk + 14 * Ny;
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
  const double kap = -0.5 * ib * dt;  // tilting weight (source/linear.cpp:147-151)
  double2* vv = wk;        // collocation values of the v (mean: u0) right-hand side
  double2* vo = wk + Ny;   // ... of the omega_y (mean: w0) right-hand side
  // lines: 0 Nv, 1 No, 2 v, 3 v'', 4 v(4), 5 omega, 6 omega''
  for (int i = threadIdx.x; i < Ny; i += blockDim.x) {
    double2 rvi = make_double2(0.0, 0.0), roi = make_double2(0.0, 0.0);
    if (zero) {
      // _get_linear_u0 / _w0: rows 2..N at point i-1
      if (i >= 2) {
        const int m = i - 1;
        rvi = col(2, m) + col(3, m) * (dt * 0.5 / Re) - (col(0, m) * 1.5 - nvp[m] * 0.5) * dt;
        roi = col(5, m) + col(6, m) * (dt * 0.5 / Re) - (col(1, m) * 1.5 - nop[m] * 0.5) * dt;
        vv[m] = rvi;
        vo[m] = roi;
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
        vv[m] = rvi;
      }
      if (i >= 2) {
        const int m = i - 1;
        const double2 Q0 = col(5, m), Q2 = col(6, m);
        const double2 re = Q2 * (0.5 / Re * dt) + Q0 * (1 - kmn * dt * 0.5 / Re);
        const double2 im = Q0 * (-al * dt * 0.5 * Ut[m]);
        roi = re + muli(im) + (col(1, m) * 1.5 - nop[m] * 0.5) * dt + muli(col(2, m) * (kap * dUt[m]));
        vo[m] = roi;
      }
    }
    Nvp[p * Ny + i] = col(0, i);
    Nop[p * Ny + i] = col(1, i);
  }
  if (threadIdx.x == 0) {
    const double2 z = make_double2(0.0, 0.0);
    vv[0] = z; vv[N] = z; vo[0] = z; vo[N] = z;
    if (!zero) { vv[1] = z; vv[N - 1] = z; }
  }
  __syncthreads();
  // no-pad p2s of the two value vectors (even extension, FFT, 1/N, ends halved)
  for (int t = threadIdx.x; t < 2 * M0; t += blockDim.x) {
    const int f = t / M0;
    const int n = t - f * M0;
    const double2* src = f ? vo : vv;
    lines0[(size_t)f * ls0 + F0::in_pos(tab0, n)] = (n <= N) ? src[n] : src[M0 - n];
  }
  F0::template fft<false>(lines0, 2, ls0, tab0);
  const int LB = Ny + 8;
  double2* av = wk + 2 * Ny;
  double2* bv = av + LB;
  double2* ao = bv + LB;
  double2* bo = ao + LB;
  for (int t = threadIdx.x; t < 2 * LB; t += blockDim.x) {
    const int f = t / LB;
    const int k = t - f * LB;
    double2 cval = make_double2(0.0, 0.0);
    if (k <= N) {
      cval = lines0[(size_t)f * ls0 + F0::out_pos(k)] * (1.0 / N);
      if (k == 0 || k == N) cval = cval * 0.5;
    }
    (f ? ao : av)[k] = cval;
  }
  __syncthreads();
  // Chebyshev integration (B x)_k = (c_{k-1} x_{k-1} - x_{k+1}) / (2k), (B x)_0 = 0
  const int Kv = zero ? 2 : 4;
  for (int it = 0; it < Kv; ++it) {
    const int nf = (it < 2) ? 2 : 1;
    for (int t = threadIdx.x; t < nf * LB; t += blockDim.x) {
      const int f = t / LB;
      const int k = t - f * LB;
      const double2* x = f ? ao : av;
      double2* y = f ? bo : bv;
      double2 r = make_double2(0.0, 0.0);
      if (k >= 1) {
        const double2 xm = x[k - 1] * (k == 1 ? 2.0 : 1.0);
        const double2 xp = (k + 1 < LB) ? x[k + 1] : make_double2(0.0, 0.0);
        r = (xm - xp) * (1.0 / (2.0 * k));
      }
      y[k] = r;
    }
    __syncthreads();
    double2* tmp = av; av = bv; bv = tmp;
    if (it < 2) { tmp = ao; ao = bo; bo = tmp; }
  }
  for (int r = threadIdx.x; r < rd.nv; r += blockDim.x)
    gv[p * rd.gp + r] = (Kv + r < LB) ? av[Kv + r] : make_double2(0.0, 0.0);
  for (int r = threadIdx.x; r < rd.no; r += blockDim.x)
    go[p * rd.gp + r] = (2 + r < LB) ? ao[2 + r] : make_double2(0.0, 0.0);
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
                      double2* Nop, double2* gv, double2* go, RhsDims rd, const double* Ut,
                      const double* dUt, const double* ddUt, DnsGeom g, PhysParams ph,
                      FftTab<C> tabP, FftTab<double2> tab0, int boot, cudaStream_t st) {
  return with_len_m(tabP.plan.L, [&](auto LL) {
    constexpr int L = decltype(LL)::value;
    constexpr int L0 = L / 2;  // the no-pad extension is half the padded one
    const size_t sm = y1_smem(g.Ny, FLine<C, L>::stride(tabP.plan.L),
                              FLine<double2, L0>::stride(tab0.plan.L), sizeof(C));
    cudaFuncSetAttribute(k_y1<C, L, L0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_y1<C, L, L0><<<(unsigned)g.H, 256, sm, st>>>(lam, V, O, Nvp, Nop, gv, go, rd, Ut, dUt, ddUt,
                                                   g, ph, tabP, tab0, boot);
    return cudaGetLastError();
  });
}
template cudaError_t launch_y1<double2>(PencilArr, const double2*, const double2*, double2*, double2*, double2*, double2*, RhsDims, const double*, const double*, const double*, DnsGeom, PhysParams, FftTab<double2>, FftTab<double2>, int, cudaStream_t);
template cudaError_t launch_y1<float2>(PencilArr, const double2*, const double2*, double2*, double2*, double2*, double2*, RhsDims, const double*, const double*, const double*, DnsGeom, PhysParams, FftTab<float2>, FftTab<double2>, int, cudaStream_t);
