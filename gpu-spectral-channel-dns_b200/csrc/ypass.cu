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
#include "mbar.cuh"
#include "wfft.cuh"
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
__device__ __noinline__ void ddz_warp(const double2* a, double2* b, int N) {
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

// The same derivative with CH (even) coefficients per lane: every lane's
// run starts at an even index, so the parity of each of its elements is
// known at compile time (the sums split by parity without divergent
// branches), and the run stays in registers between the two sweeps.  E is
// the element type: double2, or float2 where the result feeds FP32
// transforms only.
template <int CH, typename E = double2>
__device__ __noinline__ void ddz_fast(const E* __restrict__ a, E* __restrict__ b, int N) {
  static_assert(CH % 2 == 0, "runs of even length");
  typedef T_of<E> S;
  const int lane = threadIdx.x & 31;
  const int j0 = lane * CH;
  E v[CH];
#pragma unroll
  for (int i = 0; i < CH; ++i) v[i] = (j0 + i < N) ? a[j0 + i] : cmk<E>(0.0, 0.0);
  E te = cmk<E>(0.0, 0.0), to = te;  // this run's sums of 2 j a_j, even / odd j
#pragma unroll
  for (int i = 0; i < CH; ++i) {
    const S f = (S)(2 * (j0 + i));
    if (i & 1) to = to + v[i] * f;
    else te = te + v[i] * f;
  }
  S s0 = te.x, s1 = te.y, s2 = to.x, s3 = to.y;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const S t0 = __shfl_down_sync(0xffffffffu, s0, d);
    const S t1 = __shfl_down_sync(0xffffffffu, s1, d);
    const S t2 = __shfl_down_sync(0xffffffffu, s2, d);
    const S t3 = __shfl_down_sync(0xffffffffu, s3, d);
    if (lane + d < 32) { s0 += t0; s1 += t1; s2 += t2; s3 += t3; }
  }
  // sums over the runs of the lanes above, then down this run
  E re = cmk<E>(s0 - te.x, s1 - te.y), ro = cmk<E>(s2 - to.x, s3 - to.y);
#pragma unroll
  for (int i = CH - 1; i >= 0; --i) {
    const int j = j0 + i;
    E out = (i & 1) ? re : ro;  // j' > j of the other parity
    if (j == 0) out = out * (S)0.5;
    if (j < N) b[j] = out;
    const S f = (S)(2 * j);
    if (i & 1) ro = ro + v[i] * f;
    else re = re + v[i] * f;
  }
}

// Second derivative of a Chebyshev series by one warp in one sweep, CH
// (even) coefficients per lane: b_i = (1 / c_i) sum_{j >= i+2, j - i even}
// j (j^2 - i^2) a_j (c_0 = 2, else 1), the composition of two ddz_warp
// steps, as parity-split suffix sums of j a_j and j^3 a_j.  The lane's run
// is read twice from shared memory rather than held in registers.
template <int CH>
__device__ __noinline__ void d2z_fast(const double2* __restrict__ a, double2* __restrict__ b, int N) {
  static_assert(CH % 2 == 0, "runs of even length");
  const int lane = threadIdx.x & 31;
  const int j0 = lane * CH;
  double t[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // (j a_j, j^3 a_j) x (even, odd j), re / im
#pragma unroll
  for (int i = 0; i < CH; ++i) {
    if (j0 + i < N) {
      const double2 v = a[j0 + i];
      const double j = (double)(j0 + i), j3 = j * j * j;
      const int o = (i & 1) * 4;
      t[o + 0] += j * v.x;
      t[o + 1] += j * v.y;
      t[o + 2] += j3 * v.x;
      t[o + 3] += j3 * v.y;
    }
  }
  // inclusive suffix sums over the lanes, then those of the lanes above
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const double x = __shfl_down_sync(0xffffffffu, t[k], d);
      if (lane + d < 32) t[k] += x;
    }
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const double x = __shfl_down_sync(0xffffffffu, t[k], 1);
    t[k] = lane < 31 ? x : 0.0;
  }
#pragma unroll
  for (int i = CH - 1; i >= 0; --i) {
    const int jj = j0 + i;
    if (jj < N) {
      const double j = (double)jj, j2 = j * j;
      const int o = (i & 1) * 4;  // j' >= j + 2 of the same parity
      double2 out = make_double2(t[o + 2] - j2 * t[o + 0], t[o + 3] - j2 * t[o + 1]);
      if (jj == 0) out = out * 0.5;
      const double2 v = a[jj];
      b[jj] = out;
      t[o + 0] += j * v.x;
      t[o + 1] += j * v.y;
      t[o + 2] += j * j2 * v.x;
      t[o + 3] += j * j2 * v.y;
    }
  }
}
// lanes' run length for Ny coefficients
__host__ __device__ constexpr int ddz_run(int Ny) { return 2 * ((Ny + 63) / 64); }

// even extension for the padded s2p (cheby_pre_s2p_pad): e[0] = c0,
// e[k] = e[M-k] = c_k/2 for 1 <= k <= Ny-1, zero otherwise; M = 4(Ny-1).
template <typename C>
__device__ __forceinline__ double2 ext_s2p_pad(const double2* c, int n, int M, int Ny) {
  if (n == 0) return c[0];
  if (n <= Ny - 1) return c[n] * 0.5;
  if (n >= M - (Ny - 1)) return c[M - n] * 0.5;
  return make_double2(0.0, 0.0);
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
  int run, kx, kz;
  pencil_modes(g, p, run, kx, kz);
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
  int run, kx, kz;
  pencil_modes(g, p, run, kx, kz);
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
  int run, kx, kz;
  pencil_modes(g, p, run, kx, kz);
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

// Same pass with the warp FFT: three warps per pencil, two of the six lines
// per warp, no block barrier inside the transforms; twiddles from the
// plan's table through L1.
template <typename C, int M>
__global__ void __launch_bounds__(96) k_y3w(const double2* __restrict__ V, const double2* __restrict__ O,
                                           PencilArr out, DnsGeom g, PhysParams ph, FftTab<C> tab,
                                           int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int Ny = M / 4 + 1;  // the launcher checks g.Ny, g.Py against M
  // everything lives in the six line buffers (two per warp): the FP64 state
  // and derivatives (w, omega_z; D w, D^2 w, D omega_z), then the six
  // fields in the transform's precision, ready for the even extension
  // (c_0, c_n / 2), two in the lines of the warp that transforms them
  // (u, v | w, omega_x | omega_y, omega_z), which its first FFT pass reads
  // before it writes the lines
  constexpr int MW = wlen<C>(M);
  C* lines = (C*)smem_raw;
  constexpr size_t VS = (Ny * 16 + 15) / 16;             // FP64 vector slot (double2)
  constexpr size_t FS = (Ny * sizeof(C) + 15) / 16 * 16;  // field slot (bytes)
  static_assert(2 * VS * 16 + 2 * FS <= (size_t)2 * MW * sizeof(C), "vectors do not fit the lines");
  unsigned char* rb0 = (unsigned char*)lines;
  unsigned char* rb1 = (unsigned char*)(lines + (size_t)2 * MW);
  unsigned char* rb2 = (unsigned char*)(lines + (size_t)4 * MW);
  double2 *Dw = (double2*)rb0, *D2w = Dw + VS, *w = (double2*)rb1, *Doz = w + VS, *oz = (double2*)rb2;
  C* fu = (C*)(rb0 + 2 * VS * 16);
  C* fv = (C*)(rb0 + 2 * VS * 16 + FS);
  C* fw = (C*)(rb1 + 2 * VS * 16);
  C* fox = (C*)(rb1 + 2 * VS * 16 + FS);
  C* foy = (C*)(rb2 + 2 * VS * 16);
  C* foz = (C*)(rb2 + 2 * VS * 16 + FS);
  const long long p = blockIdx.x;
  int run, kx, kz;
  pencil_modes(g, p, run, kx, kz);
  const bool zero = (kx == 0 && kz == 0);
  // the pencil's wavenumbers and 1 / k^2: the FP64 divisions once per CTA
  // (thread 0, under the copies), shared through shared memory
  __shared__ double pen[3];
  // twiddles and the pencil's state by bulk copies on one barrier
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
    mbar_expect_tx(&bar, (uint32_t)(2 * Ny * 16));
    bulk_g2s(w, V + p * Ny, (uint32_t)(Ny * 16), &bar);
    bulk_g2s(oz, O + p * Ny, (uint32_t)(Ny * 16), &bar);
    double a, b;
    wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, a, b);
    pen[0] = a;
    pen[1] = b;
    pen[2] = zero ? 0.0 : 1.0 / kmn_of(a, b);
  }
  __syncthreads();
  const double ia = pen[0], ib = pen[1], kmn1 = pen[2];
  if (!__syncthreads_and(mbar_wait_bounded(&bar, 0, ph.wait_limit, status))) {
    if (threadIdx.x == 0) {
      atomicOr(status, 1);
      mbar_wait_bounded(&bar, 0, DNS_WAIT_LIMIT, nullptr);  // let the copies land before leaving
    }
    return;
  }
  // derivatives: D w, D^2 w (warp 0) and D omega_z (warp 1); then, by
  // linearity, u = i(ia Dw - ib oz)/k^2, v = i(ib Dw + ia oz)/k^2 and their
  // derivatives from D^2 w, D oz (source/velocity.cu:90-170).  The mean
  // mode holds u0, w0 in (w, oz): u = w, v = oz, omega_x = D oz, omega_y = -D w.
  // The FP32 form takes the state to FP32 first and forms the velocities
  // and vorticities in FP32: they feed FP32 transforms only.
  typedef typename std::conditional<sizeof(C) == 8, float2, double2>::type E;
  typedef T_of<E> S;
  E *ew = (E*)w, *eDw = (E*)Dw, *eD2w = (E*)D2w, *eoz = (E*)oz, *eDoz = (E*)Doz;
  if constexpr (sizeof(C) == 8) {
    // in place: element n of the FP32 copy lies below element n of the
    // FP64 vector, so the conversion runs in one pass per warp
    const int warp0 = threadIdx.x >> 5, lane0 = threadIdx.x & 31;
    if (warp0 < 2) {
      const double2* src = warp0 ? oz : w;
      E* dst = warp0 ? eoz : ew;
      for (int n0 = 0; n0 < Ny; n0 += 32) {
        const int n = n0 + lane0;
        const double2 x = n < Ny ? src[n] : make_double2(0.0, 0.0);
        __syncwarp();
        if (n < Ny) dst[n] = make_float2((float)x.x, (float)x.y);
      }
    }
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5;
  constexpr int CH = ddz_run(Ny);
  if (warp == 0) {
    ddz_fast<CH, E>(ew, eDw, Ny);
    __syncwarp();
    if (!zero) ddz_fast<CH, E>(eDw, eD2w, Ny);
  } else if (warp == 1) {
    ddz_fast<CH, E>(eoz, eDoz, Ny);
  }
  __syncthreads();
  const S sia = (S)(ia * kmn1), sib = (S)(ib * kmn1), fia = (S)ia, fib = (S)ib;
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    const E wn = ew[n], on = eoz[n], d1 = eDw[n], dz = eDoz[n];
    E u, v, ox, oy;
    if (zero) {
      u = wn;
      v = on;
      ox = dz;
      oy = cmk<E>(-d1.x, -d1.y);
    } else {
      const E d2 = eD2w[n];
      u = muli(d1 * sia) - muli(on * sib);
      v = muli(d1 * sib) + muli(on * sia);
      const E du = muli(d2 * sia) - muli(dz * sib);
      const E dv = muli(d2 * sib) + muli(dz * sia);
      ox = dv - muli(wn * fib);
      oy = muli(wn * fia) - du;
    }
    const S h = n ? (S)0.5 : (S)1.0;  // even extension: c_0, then c_n / 2
    fu[n] = from_e<C>(u * h);
    fv[n] = from_e<C>(v * h);
    fw[n] = from_e<C>(wn * h);
    fox[n] = from_e<C>(ox * h);
    foy[n] = from_e<C>(oy * h);
    foz[n] = from_e<C>(on * h);
  }
  __syncthreads();
  // this warp's two lines: fields 2 warp, 2 warp + 1; the first FFT pass
  // reads the even extensions e[0] = c_0, e[n] = e[M-n] = c_n / 2 (n < Ny),
  // zero elsewhere, the last one writes the Py values
  C* wl = lines + (size_t)2 * warp * MW;
  const C* s0 = (warp == 0) ? fu : (warp == 1 ? fw : foy);
  const C* s1 = (warp == 0) ? fv : (warp == 1 ? fox : foz);
  // w (line 2) and omega_z (line 5) vanish for the mean mode
  const bool z0 = zero && warp == 1, z1 = zero && warp == 2;
  auto ld = [&](int l, int n) -> C {
    const C* src = l ? s1 : s0;
    C e = cmk<C>(0.0, 0.0);
    if (!(l ? z1 : z0)) {
      if (n < Ny) e = src[n];
      else if (n > M - Ny) e = src[M - n];
    }
    return e;
  };
  constexpr int Py = M / 2 + 1;
  C* d0 = pencil_ptr<C>(out, 2 * warp, p);
  C* d1 = pencil_ptr<C>(out, 2 * warp + 1, p);
  auto st = [&](int l, int k, C val) {
    if (k < Py) (l ? d1 : d0)[k] = val;
  };
  wfft_io<C, M, 2, false>(wl, wtw_of(tab, 1), ld, st);
}

// ---------------------------------------------------------------------------
// Fused forward wall-normal pass: padded p2s of the three Lamb components,
// rhsNonlinear, then (unless boot) the right-hand sides of the banded
// wall-normal systems (wallsolve.h), all in Chebyshev coefficient space:
//
//   f = interpolant, at the Gauss-Lobatto points, of the reference's
//       collocation right-hand side (CN explicit operators, AB2 of the
//       nonlinear terms, v^n half of the tilting term; source/linear.cpp:
//       86-205, rhs.cpp:205-215).  Every term is a polynomial: derivatives
//       come from the coefficient recurrence, products with U(y), U'(y)
//       from multiplication by y, and the degrees above N fold back
//       (T_{N+j} = T_{N-j} at the Gauss-Lobatto points);
//   the equations do not use the walls (and, for v, the points next to
//       them): the interpolant with those values set to zero is f minus
//       f(y_m) times the cardinal polynomial of each such point y_m;
//   g = rows K .. K+n-1 of the K-fold Chebyshev integral (K = 4 for v, 2
//       for omega_y and the mean modes), the cardinal corrections taken from
//       precomputed integrated tables.
//
// The AB2 history is kept as Chebyshev coefficients of the nonlinear terms.
//   boot: only store the nonlinear terms as the AB2 history (the effect of
//         the reference's "extra previous step", source/main_loop.cpp:39-52).
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ double2 cget(const double2* X, int j, int N) {
  return (j >= 0 && j <= N) ? X[j] : make_double2(0.0, 0.0);
}
// coefficient j of y X (y T_0 = T_1, y T_i = (T_{i+1} + T_{i-1}) / 2)
__device__ __forceinline__ double2 ymul(const double2* X, int j, int N) {
  if (j < 0) return make_double2(0.0, 0.0);
  if (j == 0) return cget(X, 1, N) * 0.5;
  return (cget(X, j - 1, N) * (j == 1 ? 2.0 : 1.0) + cget(X, j + 1, N)) * 0.5;
}
__device__ __forceinline__ double2 y2mul(const double2* X, int j, int N) {
  if (j < 0) return make_double2(0.0, 0.0);
  if (j == 0) return ymul(X, 1, N) * 0.5;
  return (ymul(X, j - 1, N) * (j == 1 ? 2.0 : 1.0) + ymul(X, j + 1, N)) * 0.5;
}
// coefficient k of the Gauss-Lobatto interpolant of U(y) X(y)
__device__ __forceinline__ double2 umul_gl(const double2* X, int k, int N, const PhysParams& ph) {
  const bool quad = ph.U2 != 0.0;
  auto u = [&](int j) {
    double2 r = cget(X, j, N) * ph.U0 + ymul(X, j, N) * ph.U1;
    if (quad) r = r + y2mul(X, j, N) * ph.U2;
    return r;
  };
  double2 r = u(k);
  if (k == N - 1 || k == N - 2) r = r + u(2 * N - k);
  return r;
}
// the same for X given element-wise by a functor (X(j) for 0 <= j <= N):
// one interpolant of a combination in place of a combination of interpolants
template <class F>
__device__ __forceinline__ double2 umul_fn(F X, int k, int N, const PhysParams& ph) {
  const double2 z = make_double2(0.0, 0.0);
  auto xm = [&](int j) { return (j >= 0 && j <= N) ? X(j) : z; };
  auto ym = [&](int j) {
    if (j < 0) return z;
    if (j == 0) return xm(1) * 0.5;
    return (xm(j - 1) * (j == 1 ? 2.0 : 1.0) + xm(j + 1)) * 0.5;
  };
  auto u = [&](int j) {
    double2 r = xm(j) * ph.U0 + ym(j) * ph.U1;
    if (ph.U2 != 0.0) {
      const double2 y2 = (j < 0) ? z
                         : (j == 0) ? ym(1) * 0.5
                                    : (ym(j - 1) * (j == 1 ? 2.0 : 1.0) + ym(j + 1)) * 0.5;
      r = r + y2 * ph.U2;
    }
    return r;
  };
  double2 r = u(k);
  if (k == N - 1 || k == N - 2) r = r + u(2 * N - k);
  return r;
}
// ... of U'(y) X(y)
__device__ __forceinline__ double2 upmul_gl(const double2* X, int k, int N, const PhysParams& ph) {
  auto u = [&](int j) { return cget(X, j, N) * ph.U1 + ymul(X, j, N) * (2.0 * ph.U2); };
  double2 r = u(k);
  if (k == N - 1) r = r + u(N + 1);
  return r;
}
__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, d);
    v.y += __shfl_down_sync(0xffffffffu, v.y, d);
  }
  return v;
}
}  // namespace

template <typename C, int LM>
__global__ void __launch_bounds__(256, 3) k_y1(PencilArr lam, const double2* __restrict__ V,
                                                const double2* __restrict__ O, double2* Nvp,
                                                double2* Nop, double2* gv, double2* go, RhsDims rd,
                                                RhsTabs tb, DnsGeom g, PhysParams ph,
                                                FftTab<C> tabP, int boot) {
  typedef FLine<C, LM> FP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Ny = g.Ny;
  const int Py = g.Py;
  const int N = Ny - 1;
  const int M = tabP.plan.L;  // 2 (Py - 1)
  const int lsP = FP::stride(M);
  const int LB = Ny + 8;
  Carve cv(smem_raw);
  double2* lc = cv.take<double2>((size_t)3 * Ny);  // lambda coefficients, then fv, fo
  double2* D1 = cv.take<double2>((size_t)2 * Ny);  // D lambda_x, D lambda_y
  double2* Vc = cv.take<double2>(Ny);
  double2* Oc = cv.take<double2>(Ny);
  double2* nvc = cv.take<double2>(Ny);
  double2* noc = cv.take<double2>(Ny);
  double2* DV = cv.take<double2>(Ny);
  double2* D2V = cv.take<double2>(Ny);
  double2* D3V = cv.take<double2>(Ny);
  double2* D4V = cv.take<double2>(Ny);
  double2* DO = cv.take<double2>(Ny);
  double2* D2O = cv.take<double2>(Ny);
  double2* red = cv.take<double2>(8);  // values of fv, fo at the unused points
  const size_t bytesP = (size_t)3 * lsP * sizeof(C), bytesI = (size_t)4 * LB * 16;
  unsigned char* region = cv.take<unsigned char>(bytesP > bytesI ? bytesP : bytesI);
  C* linesP = (C*)region;

  const long long p = blockIdx.x;
  int run, kx, kz;
  pencil_modes(g, p, run, kx, kz);
  const bool zero = (kx == 0 && kz == 0);
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = kmn_of(ia, ib);

  // 1. Lamb pencils as even extensions (DCT-I of Py points); state, history
  for (int t = threadIdx.x; t < 3 * M; t += blockDim.x) {
    const int f = t / M;
    const int n = t - f * M;
    const C* src = pencil_ptr<C>(lam, f, p);
    linesP[(size_t)f * lsP + FP::in_pos(tabP, n)] = (n < Py) ? src[n] : src[M - n];
  }
  if (!boot)
    for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
      Vc[n] = V[p * Ny + n];
      Oc[n] = O[p * Ny + n];
      nvc[n] = Nvp[p * Ny + n];
      noc[n] = Nop[p * Ny + n];
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
    if (warp == 2) {
      ddz_warp(Vc, DV, Ny);
      __syncwarp();
      ddz_warp(DV, D2V, Ny);
      __syncwarp();
      ddz_warp(D2V, D3V, Ny);
      __syncwarp();
      ddz_warp(D3V, D4V, Ny);
    }
    if (warp == 3) {
      ddz_warp(Oc, DO, Ny);
      __syncwarp();
      ddz_warp(DO, D2O, Ny);
    }
  }
  __syncthreads();
  // 3. nonlinear terms (coefficients) -> history; interpolated right-hand sides
  const double dt = run_dt(ph, run), Re = run_Re(ph, run), gam = ia * dt * 0.5;
  const double kap = -0.5 * ib * dt;  // tilting weight (source/linear.cpp:147-151)
  double2* fv = lc;
  double2* fo = lc + Ny;
  for (int k = threadIdx.x; k < Ny; k += blockDim.x) {
    double2 hv, ho;
    if (zero) {
      hv = lc[k];
      ho = lc[Ny + k];
    } else {
      hv = lc[2 * Ny + k] * kmn + muli(D1[k] * ia) + muli(D1[Ny + k] * ib);
      ho = muli(lc[Ny + k] * ia) - muli(lc[k] * ib);
    }
    Nvp[p * Ny + k] = hv;
    Nop[p * Ny + k] = ho;
    if (boot) continue;
    double2 a, b;
    if (zero) {
      // _get_linear_u0 / _w0
      a = Vc[k] + D2V[k] * (dt * 0.5 / Re) - (hv * 1.5 - nvc[k] * 0.5) * dt;
      b = Oc[k] + D2O[k] * (dt * 0.5 / Re) - (ho * 1.5 - noc[k] * 0.5) * dt;
    } else {
      const double2 re = D4V[k] * (dt * 0.5 / Re) + D2V[k] * (1 - kmn * dt / Re)
                         - Vc[k] * (kmn * (1 - kmn * dt * 0.5 / Re));
      const double2 im = umul_gl(D2V, k, N, ph) * (-gam) + umul_gl(Vc, k, N, ph) * (kmn * gam)
                         + Vc[k] * (gam * 2.0 * ph.U2);
      a = re + muli(im) + (hv * 1.5 - nvc[k] * 0.5) * dt;
      const double2 ro = D2O[k] * (0.5 / Re * dt) + Oc[k] * (1 - kmn * dt * 0.5 / Re);
      b = ro + muli(umul_gl(Oc, k, N, ph) * (-gam)) + (ho * 1.5 - noc[k] * 0.5) * dt
          + muli(upmul_gl(Vc, k, N, ph) * kap);
    }
    fv[k] = a;
    fo[k] = b;
  }
  if (boot) return;
  __syncthreads();
  // 4. values at the points the equations leave out; integration buffers
  double2* av = (double2*)region;
  double2* bv = av + LB;
  double2* ao = bv + LB;
  double2* bo = ao + LB;
  const int lane = threadIdx.x & 31;
  if (warp < 2) {
    const double2* f = warp ? fo : fv;
    double2 s0 = make_double2(0.0, 0.0), sN = s0, s1 = s0, sN1 = s0;
    for (int k = lane; k < Ny; k += 32) {
      const double2 v = f[k];
      const double cs = __ldg(tb.cosk + k);
      const double sg = (k & 1) ? -1.0 : 1.0;
      s0 = s0 + v;
      sN = sN + v * sg;
      s1 = s1 + v * cs;
      sN1 = sN1 + v * (sg * cs);
    }
    s0 = warp_sum(s0);
    sN = warp_sum(sN);
    s1 = warp_sum(s1);
    sN1 = warp_sum(sN1);
    if (lane == 0) {
      red[4 * warp + 0] = s0;   // y = 1
      red[4 * warp + 1] = s1;   // y_1
      red[4 * warp + 2] = sN1;  // y_{N-1}
      red[4 * warp + 3] = sN;   // y = -1
    }
  } else {
    for (int t = threadIdx.x - 64; t < 2 * LB; t += blockDim.x - 64) {
      const int f = t / LB;
      const int k = t - f * LB;
      (f ? ao : av)[k] = (k <= N) ? (f ? fo : fv)[k] : make_double2(0.0, 0.0);
    }
  }
  __syncthreads();
  // 5. Chebyshev integration (B x)_k = (c_{k-1} x_{k-1} - x_{k+1}) / (2k), (B x)_0 = 0
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
  // 6. rows K .. K+n-1 minus the integrated cardinal corrections
  for (int r = threadIdx.x; r < rd.nv; r += blockDim.x) {
    double2 v = (Kv + r < LB) ? av[Kv + r] : make_double2(0.0, 0.0);
    if (zero) {
      v = v - red[0] * __ldg(tb.bkco + r) - red[3] * __ldg(tb.bkco + rd.no + r);
    } else {
#pragma unroll
      for (int m = 0; m < 4; ++m) v = v - red[m] * __ldg(tb.bkcv + (size_t)m * rd.nv + r);
    }
    gv[p * rd.gp + r] = v;
  }
  for (int r = threadIdx.x; r < rd.no; r += blockDim.x) {
    double2 v = (2 + r < LB) ? ao[2 + r] : make_double2(0.0, 0.0);
    v = v - red[4] * __ldg(tb.bkco + r) - red[7] * __ldg(tb.bkco + rd.no + r);
    go[p * rd.gp + r] = v;
  }
}

// Same pass with warp FFTs: warps 0-2 transform one Lamb line each (0 and 1
// also differentiate theirs), while warp 3 forms D^2 v and D^4 v (two
// second-derivative sweeps) and warp 4 D^2 omega_y; no block barrier inside
// the transforms.
template <typename C, int M>
__global__ void __launch_bounds__(160, sizeof(C) == 8 ? 6 : 4) k_y1w(PencilArr lam, const double2* __restrict__ V,
                                            const double2* __restrict__ O, double2* Nvp,
                                            double2* Nop, double2* gv, double2* go, RhsDims rd,
                                            RhsTabs tb, DnsGeom g, PhysParams ph,
                                            FftTab<C> tabP, int boot, int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int Ny = M / 4 + 1;  // the launcher checks g.Ny, g.Py against M
  constexpr int Py = M / 2 + 1;
  constexpr int N = Ny - 1;
  const int LB = Ny + 8;
  Carve cv(smem_raw);
  double2* Vc = cv.take<double2>(Ny);
  double2* Oc = cv.take<double2>(Ny);
  double2* nvc = cv.take<double2>(Ny);
  double2* noc = cv.take<double2>(Ny);
  double2* D2V = cv.take<double2>(Ny);
  double2* D4V = cv.take<double2>(Ny);
  double2* D2O = cv.take<double2>(Ny);
  double2* red = cv.take<double2>(8);
  const size_t bytesL = (size_t)3 * wlen<C>(M) * sizeof(C), bytesI = (size_t)4 * LB * 16;
  unsigned char* region = cv.take<unsigned char>(bytesL > bytesI ? bytesL : bytesI);
  C* lines = (C*)region;
  // in the line buffer of warp w < 3, after its transform: the coefficients
  // of lambda_w, then (w < 2) their derivative; fv and fo later take the
  // slots of lambda_x, lambda_y element by element
  constexpr size_t VS = (Ny * 16 + 15) / 16;  // vector slot (double2)
  static_assert((size_t)2 * VS * 16 <= (size_t)wlen<C>(M) * sizeof(C), "vectors do not fit a line");
  double2* lx = (double2*)lines;
  double2* ly = (double2*)(lines + (size_t)wlen<C>(M));
  double2* lz = (double2*)(lines + (size_t)2 * wlen<C>(M));
  double2* D1x = lx + VS;
  double2* D1y = ly + VS;

  const long long p = blockIdx.x;
  int run, kx, kz;
  pencil_modes(g, p, run, kx, kz);
  const bool zero = (kx == 0 && kz == 0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // the pencil's wavenumbers, k^2, dt and dt / (2 Re): the FP64 divisions
  // once per CTA (thread 0, under the copies), shared through shared memory
  __shared__ double pen[5];

  // 1. bulk copies on one barrier: the three Lamb pencils (Py
  //    values, natural order, at the start of each warp's line: the first
  //    FFT pass reads them all before it writes the line), state, history
  const uint32_t lamb = (uint32_t)(((Py + 1) & ~1) * sizeof(C));
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
    mbar_expect_tx(&bar, 3 * lamb + (boot ? 0u : (uint32_t)(4 * Ny * 16)));
    for (int f = 0; f < 3; ++f) bulk_g2s(lines + (size_t)f * wlen<C>(M), pencil_ptr<C>(lam, f, p), lamb, &bar);
    if (!boot) {
      bulk_g2s(Vc, V + p * Ny, (uint32_t)(Ny * 16), &bar);
      bulk_g2s(Oc, O + p * Ny, (uint32_t)(Ny * 16), &bar);
      bulk_g2s(nvc, Nvp + p * Ny, (uint32_t)(Ny * 16), &bar);
      bulk_g2s(noc, Nop + p * Ny, (uint32_t)(Ny * 16), &bar);
    }
    double a, b;
    wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, a, b);
    const double dt = run_dt(ph, run), Re = run_Re(ph, run);
    pen[0] = a;
    pen[1] = b;
    pen[2] = kmn_of(a, b);
    pen[3] = dt;
    pen[4] = dt * 0.5 / Re;
  }
  __syncthreads();
  const double ia = pen[0], ib = pen[1], kmn = pen[2];
  if (!__syncthreads_and(mbar_wait_bounded(&bar, 0, ph.wait_limit, status))) {
    if (threadIdx.x == 0) {
      atomicOr(status, 1);
      mbar_wait_bounded(&bar, 0, DNS_WAIT_LIMIT, nullptr);  // let the copies land before leaving
    }
    return;
  }
  // 2. transforms, one Lamb line per warp (0: lambda_x, 1: lambda_y,
  //    2: lambda_z), read from the pencils as even extensions, coefficients
  //    written to lc, and the warp's own derivative (D lambda_x, D lambda_y);
  //    warps 3 and 4 build the derivative chains of v and omega_y meanwhile
  const double sc = 1.0 / (Py - 1);
  if (warp < 3) {
    C* wline = lines + (size_t)warp * wlen<C>(M);
    const C* src = wline;  // staged pencil
    double2* lf = (double2*)wline;  // coefficients over the consumed lines
    auto ld = [&](int, int n) -> C { return (n < Py) ? src[n] : src[M - n]; };
    auto st = [&](int, int k, C val) {
      if (k < Ny) {
        double2 c = to_d2(val) * sc;
        if (k == 0) c = c * 0.5;
        lf[k] = c;
      }
    };
    wfft_io<C, M, 1, false>(wline, wtw_of(tabP, 0), ld, st);
    if (warp < 2) ddz_fast<ddz_run(Ny)>(lf, lf + VS, Ny);
  } else if (!boot && warp == 3) {
    // D^2 v in one sweep, D^4 v = D^2 (D^2 v)
    d2z_fast<ddz_run(Ny)>(Vc, D2V, Ny);
    __syncwarp();
    d2z_fast<ddz_run(Ny)>(D2V, D4V, Ny);
  } else if (!boot && warp == 4) {
    d2z_fast<ddz_run(Ny)>(Oc, D2O, Ny);
  }
  __syncthreads();
  // 3. nonlinear terms (coefficients) -> history; interpolated right-hand sides
  const double dt = pen[3], gam = ia * dt * 0.5;
  const double kap = -0.5 * ib * dt;  // tilting weight (source/linear.cpp:147-151)
  // the CN operators' coefficients
  const double h = pen[4], c2v = 1 - 2.0 * kmn * h, c0v = kmn * (1 - kmn * h), c0o = 1 - kmn * h;
  double2* fv = lx;
  double2* fo = ly;
  for (int k = threadIdx.x; k < Ny; k += blockDim.x) {
    double2 hv, ho;
    if (zero) {
      hv = lx[k];
      ho = ly[k];
    } else {
      hv = lz[k] * kmn + muli(D1x[k] * ia) + muli(D1y[k] * ib);
      ho = muli(ly[k] * ia) - muli(lx[k] * ib);
    }
    Nvp[p * Ny + k] = hv;
    Nop[p * Ny + k] = ho;
    if (boot) continue;
    double2 a, b;
    if (zero) {
      a = Vc[k] + D2V[k] * h - (hv * 1.5 - nvc[k] * 0.5) * dt;
      b = Oc[k] + D2O[k] * h - (ho * 1.5 - noc[k] * 0.5) * dt;
    } else {
      const double2 re = D4V[k] * h + D2V[k] * c2v - Vc[k] * c0v;
      // U (-gam D^2 v + k^2 gam v) as one interpolant
      const double2 im = umul_fn([&](int j) { return D2V[j] * (-gam) + Vc[j] * (kmn * gam); }, k, N, ph)
                         + Vc[k] * (gam * 2.0 * ph.U2);
      a = re + muli(im) + (hv * 1.5 - nvc[k] * 0.5) * dt;
      const double2 ro = D2O[k] * h + Oc[k] * c0o;
      b = ro + muli(umul_gl(Oc, k, N, ph) * (-gam)) + (ho * 1.5 - noc[k] * 0.5) * dt
          + muli(upmul_gl(Vc, k, N, ph) * kap);
    }
    fv[k] = a;
    fo[k] = b;
  }
  if (boot) return;
  __syncthreads();
  // 4. values at the points the equations leave out and the K-fold
  //    integrals of fv, fo by their banded stencils (all threads); the
  //    values by three warps, two sums each: warp 0 fv at y = +-1, warp 2
  //    fv at y_1, y_{N-1}, warp 1 fo at y = +-1 (omega does not use y_1,
  //    y_{N-1})
  if (warp < 3) {
    const double2* f = (warp == 1) ? fo : fv;
    const bool inner = warp == 2;
    double2 sa = make_double2(0.0, 0.0), sb = sa;
    for (int k = lane; k < Ny; k += 32) {
      const double2 v = f[k];
      const double sg = (k & 1) ? -1.0 : 1.0;
      const double cs = inner ? __ldg(tb.cosk + k) : 1.0;
      sa = sa + v * cs;
      sb = sb + v * (sg * cs);
    }
    sa = warp_sum(sa);
    sb = warp_sum(sb);
    if (lane == 0) {
      const int ia0 = inner ? 1 : 4 * warp;      // y = 1 or y_1
      const int ib0 = inner ? 2 : 4 * warp + 3;  // y = -1 or y_{N-1}
      red[ia0] = sa;
      red[ib0] = sb;
    }
  }
  auto fget = [&](const double2* f, int k) { return (k >= 0 && k <= N) ? f[k] : make_double2(0.0, 0.0); };
  constexpr int RPT = (Ny + 2 + 159) / 160;  // rows per thread (n <= Ny + 2, 160 threads)
  double2 iv[RPT], io[RPT];
#pragma unroll
  for (int t = 0; t < RPT; ++t) {
    const int r = threadIdx.x + t * blockDim.x;
    iv[t] = make_double2(0.0, 0.0);
    io[t] = make_double2(0.0, 0.0);
    if (r < rd.nv) {
      if (zero) {
#pragma unroll
        for (int d = 0; d < 3; ++d) iv[t] = iv[t] + fget(fv, r + 2 + 2 * d - 2) * __ldg(tb.b2 + (size_t)d * rd.nv + r);
      } else {
#pragma unroll
        for (int d = 0; d < 5; ++d) iv[t] = iv[t] + fget(fv, r + 4 + 2 * d - 4) * __ldg(tb.b4 + (size_t)d * rd.nv + r);
      }
    }
    if (r < rd.no) {
#pragma unroll
      for (int d = 0; d < 3; ++d) io[t] = io[t] + fget(fo, r + 2 + 2 * d - 2) * __ldg(tb.b2 + (size_t)d * rd.nv + r);
    }
  }
  __syncthreads();
  // 5. minus the integrated cardinal corrections, out
#pragma unroll
  for (int t = 0; t < RPT; ++t) {
    const int r = threadIdx.x + t * blockDim.x;
    if (r < rd.nv) {
      double2 v = iv[t];
      if (zero) {
        v = v - red[0] * __ldg(tb.bkco + r) - red[3] * __ldg(tb.bkco + rd.no + r);
      } else {
#pragma unroll
        for (int m = 0; m < 4; ++m) v = v - red[m] * __ldg(tb.bkcv + (size_t)m * rd.nv + r);
      }
      gv[p * rd.gp + r] = v;
    }
    if (r < rd.no) go[p * rd.gp + r] = io[t] - red[4] * __ldg(tb.bkco + r) - red[7] * __ldg(tb.bkco + rd.no + r);
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
size_t y3_smem(int Ny, int ls, size_t csz) {
  auto a = [](size_t b) { return (b + 15) & ~(size_t)15; };
  return 9 * a((size_t)Ny * 16) + a((size_t)6 * ls * csz);
}
size_t y1_smem(int Ny, int lsP, size_t csz) {
  auto a = [](size_t b) { return (b + 15) & ~(size_t)15; };
  size_t s = a((size_t)3 * Ny * 16) + a((size_t)2 * Ny * 16) + 10 * a((size_t)Ny * 16) + a(8 * 16);
  size_t bp = (size_t)3 * lsP * csz, bi = (size_t)4 * (Ny + 8) * 16;
  return s + a(bp > bi ? bp : bi);
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
                      PhysParams ph, FftTab<C> tab, int* status, cudaStream_t st, int variant, bool probe) {
  const bool any = variant == VAR_AUTO;
  // the warp form stages its inputs by bulk copies (16-byte aligned
  // sources) and takes Ny = M/4 + 1, Py = M/2 + 1 as compile-time constants
  const bool bulk_ok = aligned16(V) && aligned16(O) && wtw_of(tab, 1) &&
                       g.Ny == tab.plan.L / 4 + 1 && g.Py == tab.plan.L / 2 + 1;
  return with_len_m(tab.plan.L, [&](auto LL) -> cudaError_t {
    constexpr int L = decltype(LL)::value;
    if constexpr (L > 0 && WPlan<L, 2, FftMaxRadix<C>::v>::ok) {
     if ((any || variant == DNS_Y3_FFT) && bulk_ok) {
      if (probe) return cudaSuccess;
      const size_t sm = (size_t)6 * wlen<C>(L) * sizeof(C);
      cudaFuncSetAttribute(k_y3w<C, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k_y3w<C, L><<<(unsigned)g.H, 96, sm, st>>>(V, O, out, g, ph, tab, status);
      return cudaGetLastError();
     }
    }
    if (!any && variant != DNS_Y3_BLOCK) return cudaErrorNotSupported;
    if (probe) return cudaSuccess;
    const size_t sm = y3_smem(g.Ny, FLine<C, L>::stride(tab.plan.L), sizeof(C));
    cudaFuncSetAttribute(k_y3<C, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_y3<C, L><<<(unsigned)g.H, 256, sm, st>>>(V, O, out, g, ph, tab);
    return cudaGetLastError();
  });
}
template cudaError_t launch_y3<double2>(const double2*, const double2*, PencilArr, DnsGeom, PhysParams, FftTab<double2>, int*, cudaStream_t, int, bool);
template cudaError_t launch_y3<float2>(const double2*, const double2*, PencilArr, DnsGeom, PhysParams, FftTab<float2>, int*, cudaStream_t, int, bool);

template <typename C>
cudaError_t launch_y1(PencilArr lam, const double2* V, const double2* O, double2* Nvp,
                      double2* Nop, double2* gv, double2* go, RhsDims rd, RhsTabs tb, DnsGeom g,
                      PhysParams ph, FftTab<C> tabP, int boot, int* status, cudaStream_t st, int variant,
                      bool probe) {
  const bool any = variant == VAR_AUTO;
  // the warp form stages its inputs by bulk copies (16-byte aligned pencils
  // with room for Py rounded up to even) and takes Ny = M/4 + 1,
  // Py = M/2 + 1 as compile-time constants
  const bool bulk_ok = aligned16(lam.base) && (lam.ps * sizeof(C)) % 16 == 0 &&
                       (lam.fs * sizeof(C)) % 16 == 0 && lam.ps >= ((g.Py + 1) & ~1) && aligned16(V) &&
                       aligned16(O) && aligned16(Nvp) && aligned16(Nop) && wtw_of(tabP, 0) &&
                       g.Ny == tabP.plan.L / 4 + 1 && g.Py == tabP.plan.L / 2 + 1;
  return with_len_m(tabP.plan.L, [&](auto LL) -> cudaError_t {
    constexpr int L = decltype(LL)::value;
    if constexpr (L > 0 && WPlan<L, 1, FftMaxRadix<C>::v>::ok) {
     if ((any || variant == DNS_Y1_WARP) && bulk_ok) {
      if (probe) return cudaSuccess;
      auto a = [](size_t b) { return (b + 15) & ~(size_t)15; };
      const size_t bl = (size_t)3 * wlen<C>(L) * sizeof(C), bi = (size_t)4 * (g.Ny + 8) * 16;
      const size_t sm = 7 * a((size_t)g.Ny * 16) + a(8 * 16) + a(bl > bi ? bl : bi);
      cudaFuncSetAttribute(k_y1w<C, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k_y1w<C, L><<<(unsigned)g.H, 160, sm, st>>>(lam, V, O, Nvp, Nop, gv, go, rd, tb, g, ph, tabP, boot,
                                                    status);
      return cudaGetLastError();
     }
    }
    if (!any && variant != DNS_Y1_BLOCK) return cudaErrorNotSupported;
    if (probe) return cudaSuccess;
    const size_t sm = y1_smem(g.Ny, FLine<C, L>::stride(tabP.plan.L), sizeof(C));
    cudaFuncSetAttribute(k_y1<C, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_y1<C, L><<<(unsigned)g.H, 256, sm, st>>>(lam, V, O, Nvp, Nop, gv, go, rd, tb, g, ph, tabP, boot);
    return cudaGetLastError();
  });
}
template cudaError_t launch_y1<double2>(PencilArr, const double2*, const double2*, double2*, double2*, double2*, double2*, RhsDims, RhsTabs, DnsGeom, PhysParams, FftTab<double2>, int, int*, cudaStream_t, int, bool);
template cudaError_t launch_y1<float2>(PencilArr, const double2*, const double2*, double2*, double2*, double2*, double2*, RhsDims, RhsTabs, DnsGeom, PhysParams, FftTab<float2>, int, int*, cudaStream_t, int, bool);
