// Solve-only entry of the wall-normal systems: the reference's solveEq
// (source/solver.cpp:107-123) for the v and the omega_y system of every
// Fourier mode, with the banded factors of wallsolve.h in place of the
// explicit inverses (source/matrix_op.cpp:68-78).
//
// The right-hand sides arrive in the reference's collocation form
// (source/coefficient.cu:7-86): for v, rows 0..3 are the wall values v(1),
// v(-1), v'(1), v'(-1) and rows 4..N the values at the Gauss-Lobatto points
// y_2..y_{N-2}; for omega_y and for the mean modes (pencil (0,0) of both
// arrays) rows 0..1 are the wall values and rows 2..N the values at
// y_1..y_{N-1}.  Per pencil:
//   1. p = the Chebyshev polynomial of lowest degree that meets the wall rows
//      (cubic for v, linear otherwise);
//   2. f = the interior rows minus (A p) at their points, zero at the points
//      the equation leaves out, and the coefficients of its interpolant
//      (DCT-I over the Gauss-Lobatto points: the FFT of the even extension,
//      the library's no-padding p2s);
//   3. rows K .. K+n-1 of the K-fold Chebyshev integral (K = 4 for v, 2
//      otherwise), the input of the banded solve, which then runs without
//      the tilting term;
//   4. x = the banded solution + p, written over the right-hand side.
// A p is evaluated from the operator rows of the reference's matrices:
//   v:     Re part  (1 + k^2 dt/Re) p'' - k^2 (1 + k^2 dt/(2Re)) p   (p'''' = 0)
//          Im part  a dt/2 U p'' - (k^2 a dt/2 U + a dt/2 U'') p
//   omega: (1 + k^2 dt/(2Re)) p + i a dt/2 U p                       (p'' = 0)
//   mean:  p                                                          (p'' = 0)
// with a = kx/aphi the streamwise wavenumber and k^2 = a^2 + b^2.
#include <algorithm>
#include <type_traits>

#include "kernels.cuh"
#include "mbar.cuh"
#include "wallsolve_dev.cuh"
#include "wfft.cuh"

namespace {

__device__ __forceinline__ double2 cx(double a, double b) { return make_double2(a, b); }

// 1-2. wall polynomial and the point values of the interior right-hand side
// minus A p, zero where the equation has no row; written as Gauss-Lobatto
// values (m = 0..N, pitch sp) for the DCT-I that follows
__global__ void __launch_bounds__(128) k_colloc_prep(const double2* __restrict__ bv,
                                                     const double2* __restrict__ bo, long long bp,
                                                     double2* sv, double2* so, long long sp,
                                                     double2* pbc, const double* __restrict__ cosk,
                                                     const double* __restrict__ Ut,
                                                     const double* __restrict__ ddUt, DnsGeom g,
                                                     PhysParams ph) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Ny = g.Ny, N = Ny - 1;
  const long long p = blockIdx.x;
  const int kx = (int)(p % g.Kx), kz = (int)(p / g.Kx);
  const bool zero = p == 0;
  double2* rv = (double2*)smem_raw;
  double2* ro = rv + Ny;
  __shared__ double2 pc[6];
  for (int k = threadIdx.x; k < Ny; k += blockDim.x) {
    rv[k] = bv[p * bp + k];
    ro[k] = bo[p * bp + k];
  }
  __syncthreads();
  // wall polynomial: T_j(+-1) = (+-1)^j, T_j'(1) = j^2, T_j'(-1) = (-1)^(j+1) j^2
  if (threadIdx.x == 0) {
    const double2 e = (rv[0] + rv[1]) * 0.5, o = (rv[0] - rv[1]) * 0.5;
    if (zero) {
      pc[0] = e; pc[1] = o; pc[2] = cx(0, 0); pc[3] = cx(0, 0);
    } else {
      const double2 c2 = (rv[2] - rv[3]) * 0.125;
      const double2 c3 = ((rv[2] + rv[3]) * 0.5 - o) * 0.125;
      pc[0] = e - c2; pc[1] = o - c3; pc[2] = c2; pc[3] = c3;
    }
    pc[4] = (ro[0] + ro[1]) * 0.5;
    pc[5] = (ro[0] - ro[1]) * 0.5;
    for (int j = 0; j < 6; ++j) pbc[p * 6 + j] = pc[j];
  }
  __syncthreads();
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = ia * ia + ib * ib, dt = ph.dt, Re = ph.Re;
  for (int m = threadIdx.x; m <= N; m += blockDim.x) {
    double2 fv = cx(0, 0), fo = cx(0, 0);
    const double y = __ldg(cosk + m);
    if (zero) {
      if (m >= 1 && m <= N - 1) {
        fv = rv[m + 1] - (pc[0] + pc[1] * y);
        fo = ro[m + 1] - (pc[4] + pc[5] * y);
      }
    } else {
      if (m >= 2 && m <= N - 2) {
        const double2 P0 = pc[0] + pc[1] * y + pc[2] * (2 * y * y - 1) + pc[3] * (y * (4 * y * y - 3));
        const double2 P2 = pc[2] * 4.0 + pc[3] * (24.0 * y);
        const double U = Ut[m], ddU = ddUt[m];
        const double2 re = P2 * (1 + kmn * dt / Re) - P0 * (kmn * (1 + kmn * dt * 0.5 / Re));
        const double2 im = P2 * (ia * dt * 0.5 * U) - P0 * (kmn * ia * dt * 0.5 * U + ia * dt * 0.5 * ddU);
        fv = rv[m + 2] - (re + muli(im));
      }
      if (m >= 1 && m <= N - 1) {
        const double2 P0 = pc[4] + pc[5] * y;
        fo = ro[m + 1] - (P0 * (1 + kmn * dt * 0.5 / Re) + muli(P0 * (ia * dt * 0.5 * Ut[m])));
      }
    }
    sv[p * sp + m] = fv;
    so[p * sp + m] = fo;
  }
}

// 3. rows K .. K+n-1 of the K-fold Chebyshev integral of the interpolant
// coefficients a_0..a_N (K = 4 for v, 2 for omega_y and the mean modes):
// (B x)_k = (c_{k-1} x_{k-1} - x_{k+1}) / (2k), (B x)_0 = 0
__global__ void __launch_bounds__(128) k_colloc_integrate(const double2* __restrict__ cv,
                                                          const double2* __restrict__ co, long long cp,
                                                          double2* gv, double2* go, int nv, int no,
                                                          long long gp, DnsGeom g) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Ny = g.Ny, N = Ny - 1, LB = Ny + 8;
  const long long p = blockIdx.x;
  const bool zero = p == 0;
  double2* av = (double2*)smem_raw;
  double2* sv = av + LB;
  double2* ao = sv + LB;
  double2* so = ao + LB;
  for (int k = threadIdx.x; k < LB; k += blockDim.x) {
    av[k] = k <= N ? cv[p * cp + k] : cx(0, 0);
    ao[k] = k <= N ? co[p * cp + k] : cx(0, 0);
  }
  __syncthreads();
  const int Kv = zero ? 2 : 4;
  for (int it = 0; it < Kv; ++it) {
    const int nf = (it < 2) ? 2 : 1;
    for (int t = threadIdx.x; t < nf * LB; t += blockDim.x) {
      const int f = t / LB;
      const int k = t - f * LB;
      const double2* x = f ? ao : av;
      double2* y = f ? so : sv;
      double2 r = cx(0, 0);
      if (k >= 1) {
        const double2 xm = x[k - 1] * (k == 1 ? 2.0 : 1.0);
        const double2 xp = (k + 1 < LB) ? x[k + 1] : cx(0, 0);
        r = (xm - xp) * (1.0 / (2.0 * k));
      }
      y[k] = r;
    }
    __syncthreads();
    double2* tmp = av; av = sv; sv = tmp;
    if (it < 2) { tmp = ao; ao = so; so = tmp; }
  }
  for (int r = threadIdx.x; r < nv; r += blockDim.x) gv[p * gp + r] = (Kv + r < LB) ? av[Kv + r] : cx(0, 0);
  for (int r = threadIdx.x; r < no; r += blockDim.x) go[p * gp + r] = (2 + r < LB) ? ao[2 + r] : cx(0, 0);
}

// 4. x = banded solution + wall polynomial, into the caller's pencils
__global__ void __launch_bounds__(256) k_colloc_finish(const double2* __restrict__ Xv,
                                                       const double2* __restrict__ Xo,
                                                       const double2* __restrict__ pbc, double2* ov,
                                                       double2* oo, long long op, int Ny, long long H) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= H * Ny) return;
  const long long p = i / Ny;
  const int k = (int)(i - p * Ny);
  double2 a = Xv[i], b = Xo[i];
  if (k < 4) a = a + pbc[p * 6 + k];
  if (k < 2) b = b + pbc[p * 6 + 4 + k];
  if (ov) ov[p * op + k] = a;
  if (oo) oo[p * op + k] = b;
}

// any non-finite real or imaginary part in a or b sets *flag
__global__ void __launch_bounds__(256) k_nonfinite(const double2* __restrict__ a,
                                                   const double2* __restrict__ b, long long n,
                                                   int* flag) {
  bool bad = false;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 x = a[i], y = b[i];
    bad |= !(isfinite(x.x) && isfinite(x.y) && isfinite(y.x) && isfinite(y.y));
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

// 1-3 fused, one CTA per pencil, one warp per system (0: v, 1: omega_y):
// the point values of step 2 are formed in the first pass of a warp FFT of
// the even extension (the DCT-I over the Gauss-Lobatto points, length
// L = 2N), its coefficients written over the consumed line, and the K-fold
// integration runs in place of the line (two halves as ping-pong buffers).
// Compile-time L = 2 (Ny - 1); the launcher falls back to the three kernels
// above for lengths without a warp plan.
template <int L>
__global__ void __launch_bounds__(64, 16) k_colloc_fused(const double2* __restrict__ bv, const double2* __restrict__ bo,
                                                     long long bp, double2* pbc, const double* __restrict__ cosk,
                                                     const double* __restrict__ Ut, const double* __restrict__ ddUt,
                                                     double2* gv, double2* go, int nv, int no, long long gp,
                                                     DnsGeom g, PhysParams ph, FftTab<double2> tab, int* status) {
  constexpr int N = L / 2, Ny = N + 1, LB = Ny + 8;
  constexpr int LS = (wlen<double2>(L) > 2 * LB) ? wlen<double2>(L) : 2 * LB;  // line stride
  static_assert(LS - Ny >= Ny, "the staged right-hand side lies above the point values");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint64_t bars[2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2* line = (double2*)smem_raw + (size_t)warp * LS;
  const long long p = blockIdx.x;
  const int kx = (int)(p % g.Kx), kz = (int)(p / g.Kx);
  const bool zero = p == 0;
  // this warp's right-hand side (Ny point values) by one bulk copy into the
  // top of its line, above the point values the next loop writes (the
  // launcher checks the 16-byte alignment)
  const double2* b = line + (LS - Ny);
  {
    uint64_t* bar = &bars[warp];
    if (lane == 0) {
      mbar_init(bar, 1);
      fence_mbar_init();
      mbar_expect_tx(bar, (uint32_t)(Ny * 16));
      bulk_g2s(line + (LS - Ny), (warp ? bo : bv) + p * bp, (uint32_t)(Ny * 16), bar);
    }
    __syncwarp();
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(bar, 0, ph.wait_limit, status))) {
      if (lane == 0) {
        atomicOr(status, 1);
        mbar_wait_bounded(bar, 0, DNS_WAIT_LIMIT, nullptr);  // let the copy land before leaving
      }
      return;
    }
  }
  // wall polynomial (every lane; rows 0..3 of the right-hand side)
  double2 pc0, pc1, pc2 = cx(0, 0), pc3 = cx(0, 0);
  {
    const double2 r0 = b[0], r1 = b[1];
    const double2 e = (r0 + r1) * 0.5, o = (r0 - r1) * 0.5;
    pc0 = e;
    pc1 = o;
    if (warp == 0 && !zero) {
      const double2 r2 = b[2], r3 = b[3];
      pc2 = (r2 - r3) * 0.125;
      pc3 = ((r2 + r3) * 0.5 - o) * 0.125;
      pc0 = e - pc2;
      pc1 = o - pc3;
    }
    if (lane == 0) {
      if (warp == 0) {
        pbc[p * 6 + 0] = pc0; pbc[p * 6 + 1] = pc1; pbc[p * 6 + 2] = pc2; pbc[p * 6 + 3] = pc3;
      } else {
        pbc[p * 6 + 4] = pc0; pbc[p * 6 + 5] = pc1;
      }
    }
  }
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = ia * ia + ib * ib, dt = ph.dt, Re = ph.Re;
  // the operator's constants (the same expressions as the three-kernel path)
  const double cv2 = 1 + kmn * dt / Re, cv0 = kmn * (1 + kmn * dt * 0.5 / Re), co0 = 1 + kmn * dt * 0.5 / Re;
  const double ah = ia * dt * 0.5;
  // point value m of the interior right-hand side minus A p (zero where the
  // equation has no row), staged at line[m] in natural order: the FFT's
  // first pass reads them all before it writes the line
  for (int m = lane; m <= N; m += 32) {
    const double y = __ldg(cosk + m);
    double2 f = cx(0, 0);
    if (zero || warp == 1) {
      if (m >= 1 && m <= N - 1) {
        const double2 P0 = pc0 + pc1 * y;
        f = zero ? b[m + 1] - P0 : b[m + 1] - (P0 * co0 + muli(P0 * (ah * __ldg(Ut + m))));
      }
    } else if (m >= 2 && m <= N - 2) {
      const double2 P0 = pc0 + pc1 * y + pc2 * (2 * y * y - 1) + pc3 * (y * (4 * y * y - 3));
      const double2 P2 = pc2 * 4.0 + pc3 * (24.0 * y);
      const double U = __ldg(Ut + m), ddU = __ldg(ddUt + m);
      const double2 re = P2 * cv2 - P0 * cv0;
      const double2 im = P2 * (ah * U) - P0 * (kmn * ah * U + ah * ddU);
      f = b[m + 2] - (re + muli(im));
    }
    line[m] = f;
  }
  __syncwarp();
  // DCT-I: FFT of the even extension; coefficient k = value / N, halved at
  // k = 0 and k = N, written over the line (its last pass read it all)
  auto ld = [&](int, int n) -> double2 { return line[n <= N ? n : L - n]; };
  auto st = [&](int, int k, double2 v) {
    if (k <= N) line[k] = v * ((k == 0 || k == N) ? 0.5 / N : 1.0 / N);
  };
  wfft_io<double2, L, 1, false>(line, wtw_of(tab, 0), ld, st, LS);
  __syncwarp();
  for (int k = Ny + lane; k < LB; k += 32) line[k] = cx(0, 0);
  // K-fold integration: (B x)_k = (c_{k-1} x_{k-1} - x_{k+1}) / (2k), (B x)_0 = 0;
  // each lane keeps the weights 1 / (2k) of its elements k = lane + 32 i
  // (the divisions once, not once per sweep)
  const int K = (warp == 0 && !zero) ? 4 : 2;
  constexpr int KPL = (LB + 31) / 32;
  double w2k[KPL];
#pragma unroll
  for (int i = 0; i < KPL; ++i) {
    const int k = lane + 32 * i;
    w2k[i] = k >= 1 ? 1.0 / (2.0 * k) : 0.0;
  }
  double2* x = line;
  double2* yb = line + LB;
  for (int it = 0; it < K; ++it) {
    __syncwarp();
#pragma unroll
    for (int i = 0; i < KPL; ++i) {
      const int k = lane + 32 * i;
      if (k >= LB) break;
      double2 r = cx(0, 0);
      if (k >= 1) {
        const double2 xm = x[k - 1] * (k == 1 ? 2.0 : 1.0);
        const double2 xp = (k + 1 < LB) ? x[k + 1] : cx(0, 0);
        r = (xm - xp) * w2k[i];
      }
      yb[k] = r;
    }
    double2* t = x;
    x = yb;
    yb = t;
  }
  __syncwarp();
  double2* out = (warp ? go : gv) + p * gp;
  const int n = warp ? no : nv;
  for (int r = lane; r < n; r += 32) out[r] = (K + r < LB) ? x[K + r] : cx(0, 0);
}

}  // namespace

cudaError_t launch_nonfinite(const double2* a, const double2* b, long long n, int* flag,
                             cudaStream_t st) {
  const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 8);
  k_nonfinite<<<(unsigned)std::max<long long>(blocks, 1), 256, 0, st>>>(a, b, n, flag);
  return cudaGetLastError();
}

cudaError_t launch_colloc_prep(const double2* bv, const double2* bo, long long bp, double2* sv,
                               double2* so, long long sp, double2* pbc, const double* cosk,
                               const double* Ut, const double* ddUt, const DnsGeom& g,
                               const PhysParams& ph, cudaStream_t st) {
  const size_t sm = (size_t)32 * g.Ny;
  if (sm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_colloc_prep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e) return e;
  }
  k_colloc_prep<<<(unsigned)g.H, 128, sm, st>>>(bv, bo, bp, sv, so, sp, pbc, cosk, Ut, ddUt, g, ph);
  return cudaGetLastError();
}

cudaError_t launch_colloc_integrate(const double2* cv, const double2* co, long long cp, double2* gv,
                                    double2* go, const WallDims& wd, const DnsGeom& g, cudaStream_t st) {
  const size_t sm = (size_t)64 * (g.Ny + 8);
  if (sm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_colloc_integrate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e) return e;
  }
  k_colloc_integrate<<<(unsigned)g.H, 128, sm, st>>>(cv, co, cp, gv, go, wd.nv, wd.no, wd.gp, g);
  return cudaGetLastError();
}

cudaError_t launch_colloc_finish(const double2* Xv, const double2* Xo, const double2* pbc,
                                 double2* ov, double2* oo, long long op, const DnsGeom& g,
                                 cudaStream_t st) {
  const long long n = g.H * g.Ny;
  k_colloc_finish<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(Xv, Xo, pbc, ov, oo, op, g.Ny, g.H);
  return cudaGetLastError();
}

cudaError_t launch_colloc_fused(const double2* bv, const double2* bo, long long bp, double2* pbc,
                                const double* cosk, const double* Ut, const double* ddUt, double2* gv,
                                double2* go, const WallDims& wd, const DnsGeom& g, const PhysParams& ph,
                                FftTab<double2> tab, int* status, cudaStream_t st) {
  auto go1 = [&](auto LL) -> cudaError_t {
    constexpr int L = decltype(LL)::value;
    if constexpr (WPlan<L, 1, FftMaxRadix<double2>::v>::ok) {
      if (tab.plan.L != L || g.Ny != L / 2 + 1 || !tab.tw || !status || !aligned16(bv) || !aligned16(bo))
        return cudaErrorNotSupported;
      constexpr int LB = L / 2 + 9;
      constexpr int LS = (wlen<double2>(L) > 2 * LB) ? wlen<double2>(L) : 2 * LB;
      const size_t sm = (size_t)2 * LS * 16;
      cudaFuncSetAttribute(k_colloc_fused<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k_colloc_fused<L><<<(unsigned)g.H, 64, sm, st>>>(bv, bo, bp, pbc, cosk, Ut, ddUt, gv, go, wd.nv, wd.no,
                                                       wd.gp, g, ph, tab, status);
      return cudaGetLastError();
    }
    return cudaErrorNotSupported;
  };
  switch (tab.plan.L) {
    case 128: return go1(std::integral_constant<int, 128>());
    case 256: return go1(std::integral_constant<int, 256>());
    case 384: return go1(std::integral_constant<int, 384>());
    case 512: return go1(std::integral_constant<int, 512>());
    case 768: return go1(std::integral_constant<int, 768>());
  }
  return cudaErrorNotSupported;
}
