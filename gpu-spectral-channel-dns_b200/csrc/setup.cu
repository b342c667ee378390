// Operator setup: Chebyshev tables, base flow, collocation operators and
// their explicit inverses; also the plain reference-layout transpose.
//
// Reference counterparts:
//   get_T_matrix / get_U ...................... source/coefficient.cu:88-159
//   _get_coefficient_v / _omega / _coef_u0 .... source/coefficient.cu:7-86
//   initAuxMatrix (operators + inverse()) ..... source/solver.cpp:260-320,
//                                               source/matrix_op.cpp:22-27
//   cuda_transpose ............................ source/transpose.cu:115-166
//
// The operators are assembled on the device with explicitly rounded
// arithmetic (__dmul_rn/__dadd_rn/__ddiv_rn) in the reference's evaluation
// order, from tables computed on the host exactly as the reference does, so
// each matrix entry equals the reference's.  Each matrix is inverted in place
// by Gauss-Jordan elimination with partial (row) pivoting on a thread-block
// cluster: its rows are spread over the cluster's CTAs and the pivot search,
// row swaps and pivot-row broadcast go through distributed shared memory.
#include <cooperative_groups.h>
#include <cmath>
#include <vector>
#include "kernels.cuh"
#include "setup.cuh"

namespace cg = cooperative_groups;

void host_T_matrix(int N, double* T0, double* T2, double* T4) {
  const double PI = 4.0 * atan(1.0);
  const int n1 = N + 1;
  std::vector<double> T1((size_t)n1 * n1), T3((size_t)n1 * n1);
  for (int i = 0; i <= N; i++)
    for (int j = 0; j <= N; j++) T0[(size_t)n1 * i + j] = cos(j * PI * i / N);
  for (int j = 0; j <= 3; j++)
    for (int i = 0; i <= N; i++) {
      size_t inc = (size_t)n1 * i + j;
      T1[inc] = 0.0; T2[inc] = 0.0; T3[inc] = 0.0; T4[inc] = 0.0;
    }
  for (int i = 0; i <= N; i++) T1[(size_t)n1 * i + 1] = T0[(size_t)n1 * i + 0];
  for (int i = 0; i <= N; i++) {
    T2[(size_t)n1 * i + 2] = 4 * T0[(size_t)n1 * i + 0];
    T1[(size_t)n1 * i + 2] = 4 * T0[(size_t)n1 * i + 1];
  }
  for (int j = 3; j <= N; j++)
    for (int i = 0; i <= N; i++) {
      size_t J = (size_t)n1 * i + j, J1 = J - 1, J2 = J - 2;
      T1[J] = 2 * j * T0[J1] + j * T1[J2] / (j - 2);
      T2[J] = 2 * j * T1[J1] + j * T2[J2] / (j - 2);
      T3[J] = 2 * j * T2[J1] + j * T3[J2] / (j - 2);
      T4[J] = 2 * j * T3[J1] + j * T4[J2] / (j - 2);
    }
}

// U, U', U'' of U(y) = U0 + U1 y + U2 y^2 at n Gauss-Lobatto points
// y_i = cos(pi i/(n-1)); the Couette default (0.5, 0.5, 0) is evaluated as
// the reference does, 0.5*(1+z) (source/coefficient.cu:149-159).
void host_base_flow(int n, double U0, double U1, double U2, double* U, double* dU, double* ddU) {
  const double PI = 4.0 * atan(1.0);
  const bool ref = (U0 == 0.5 && U1 == 0.5 && U2 == 0.0);
  for (int i = 0; i < n; i++) {
    double z = cos((double)i / (n - 1) * PI);
    U[i] = ref ? 0.5 * (1 + z) : U0 + U1 * z + U2 * z * z;
    if (dU) dU[i] = U1 + 2 * U2 * z;
    if (ddU) ddU[i] = 2 * U2;
  }
}

namespace {
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dv(double a, double b) { return __ddiv_rn(a, b); }

// operator entry (row i, column j); eq 0 = v, 1 = omega; zero = (0,0) mode
__device__ double2 op_entry(int eq, bool zero, int i, int j, int N1, const double* T0,
                            const double* T2, const double* T4, const double* U,
                            const double* ddU, double Re, double dt, double kmn, double al) {
  const double jj = (double)j;
  if (zero || eq == 1) {
    if (i == 0) return make_double2(1.0, 0.0);
    if (i == 1) return make_double2((j % 2 == 0) ? 1.0 : -1.0, 0.0);
    const size_t c = (size_t)N1 * (i - 1) + j;
    if (zero)  // -T2*dt*0.5/Re + T0
      return make_double2(add(dv(mul(mul(-T2[c], dt), 0.5), Re), T0[c]), 0.0);
    // -T2*dt*0.5/Re + (1 + kmn*dt*0.5/Re)*T0 ; alpha*dt*0.5*U*T0
    const double re = add(dv(mul(mul(-T2[c], dt), 0.5), Re),
                          mul(add(1.0, dv(mul(mul(kmn, dt), 0.5), Re)), T0[c]));
    const double im = mul(mul(mul(mul(al, dt), 0.5), U[i - 1]), T0[c]);
    return make_double2(re, im);
  }
  if (i == 0) return make_double2(1.0, 0.0);
  if (i == 1) return make_double2((j % 2 == 0) ? 1.0 : -1.0, 0.0);
  if (i == 2) return make_double2(jj * jj, 0.0);
  if (i == 3) return make_double2(((j % 2 == 0) ? -1.0 : 1.0) * jj * jj, 0.0);
  const size_t c = (size_t)N1 * (i - 2) + j;
  // -T4*dt*0.5/Re + (1 + kmn*dt/Re)*T2 - kmn*(1 + kmn*dt*0.5/Re)*T0
  const double a1 = dv(mul(mul(-T4[c], dt), 0.5), Re);
  const double a2 = mul(add(1.0, dv(mul(kmn, dt), Re)), T2[c]);
  const double a3 = mul(mul(kmn, add(1.0, dv(mul(mul(kmn, dt), 0.5), Re))), T0[c]);
  const double re = sub(add(a1, a2), a3);
  // alpha*dt*U*0.5*T2 - (kmn*alpha*dt*0.5*U + alpha*dt*0.5*ddU)*T0
  const double Ui = U[i - 2], ddUi = ddU[i - 2];
  const double b1 = mul(mul(mul(mul(al, dt), Ui), 0.5), T2[c]);
  const double b2 = add(mul(mul(mul(mul(kmn, al), dt), 0.5), Ui), mul(mul(mul(al, dt), 0.5), ddUi));
  const double im = sub(b1, mul(b2, T0[c]));
  return make_double2(re, im);
}

__device__ __forceinline__ double2 cdiv1(double2 a) {  // 1/a
  const double d = a.x * a.x + a.y * a.y;
  return make_double2(a.x / d, -a.y / d);
}
}  // namespace

// mode 0: operator slots (kx, kz'), kz' <= Nz/2, output transposed AT[u][eq][j][i]
// mode 1: every pencil p = kz*Kx + kx, output row-major out{v,o}[p][i][j]
__global__ void __launch_bounds__(256) k_gj_invert(int mode, long long unit0, DnsGeom g, PhysParams ph,
                                                    const double* T0, const double* T2,
                                                    const double* T4, const double* U,
                                                    const double* ddU, double2* outAT,
                                                    double2* outV, double2* outO, int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int N = g.Ny;
  const int RB = (N + C - 1) / C;
  const int lo = rank * RB;
  const int nown = max(0, min(N - lo, RB));
  double2* A = (double2*)smem_raw;               // RB x N
  double2* piv = A + (size_t)RB * N;             // N
  double2* tmp = piv + N;                        // N
  double2* fcol = tmp + N;                       // RB
  int* perm = (int*)(fcol + RB);                 // N
  double* cval = (double*)(perm + ((N + 3) & ~3));  // 1 (+pad)
  int* cidx = (int*)(cval + 2);
  __shared__ double wv[32];
  __shared__ int wi[32];
  __shared__ double2 s_pinv;

  const long long mid = blockIdx.x / C;
  const int eq = (int)(mid & 1);
  const long long lunit = mid >> 1;  // index within this launch (output)
  const long long unit = unit0 + lunit;
  const int kx = (int)(unit % g.Kx);
  const int kz = (int)(unit / g.Kx);
  const bool zero = (kx == 0 && kz == 0);
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = kmn_of(ia, ib);
  const int tid = threadIdx.x, nt = blockDim.x;

  for (int t = tid; t < nown * N; t += nt) {
    const int il = t / N, j = t - il * N;
    A[t] = op_entry(eq, zero, lo + il, j, N, T0, T2, T4, U, ddU, ph.Re, ph.dt, kmn, ia);
  }
  __syncthreads();

  for (int k = 0; k < N; ++k) {
    // 1. local pivot candidate among rows >= k
    double best = -1.0;
    int bi = N;
    for (int il = tid; il < nown; il += nt) {
      const int i = lo + il;
      if (i < k) continue;
      const double2 a = A[(size_t)il * N + k];
      const double m = a.x * a.x + a.y * a.y;
      if (m > best || (m == best && i < bi)) { best = m; bi = i; }
    }
    for (int d = 16; d > 0; d >>= 1) {
      const double ob = __shfl_down_sync(0xffffffffu, best, d);
      const int oi = __shfl_down_sync(0xffffffffu, bi, d);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if ((tid & 31) == 0) { wv[tid >> 5] = best; wi[tid >> 5] = bi; }
    __syncthreads();
    if (tid == 0) {
      for (int w = 1; w < nt / 32; ++w)
        if (wv[w] > best || (wv[w] == best && wi[w] < bi)) { best = wv[w]; bi = wi[w]; }
      *cval = best;
      *cidx = bi;
    }
    cl.sync();
    // 2. global pivot (same result in every CTA)
    double gb = -1.0;
    int p = N;
    for (int r = 0; r < C; ++r) {
      const double v = *cl.map_shared_rank(cval, r);
      const int ix = *cl.map_shared_rank(cidx, r);
      if (v > gb || (v == gb && ix < p)) { gb = v; p = ix; }
    }
    if (p >= N || !(gb > 0.0)) {  // singular: flag and leave the matrix as is
      if (tid == 0 && rank == 0) atomicOr(status, 2);
      p = k;
    }
    if (tid == 0) perm[k] = p;
    // 3. swap rows k and p
    const int ok = k / RB, op = p / RB;
    if (p != k) {
      if (ok == op) {
        if (rank == ok) {
          for (int j = tid; j < N; j += nt) {
            double2 a = A[(size_t)(k - lo) * N + j];
            A[(size_t)(k - lo) * N + j] = A[(size_t)(p - lo) * N + j];
            A[(size_t)(p - lo) * N + j] = a;
          }
        }
      } else {
        if (rank == ok) {
          const double2* rem = cl.map_shared_rank(A, op) + (size_t)(p - op * RB) * N;
          for (int j = tid; j < N; j += nt) tmp[j] = rem[j];
        }
        if (rank == op) {
          const double2* rem = cl.map_shared_rank(A, ok) + (size_t)(k - ok * RB) * N;
          for (int j = tid; j < N; j += nt) tmp[j] = rem[j];
        }
        cl.sync();
        if (rank == ok)
          for (int j = tid; j < N; j += nt) A[(size_t)(k - lo) * N + j] = tmp[j];
        if (rank == op)
          for (int j = tid; j < N; j += nt) A[(size_t)(p - lo) * N + j] = tmp[j];
      }
    }
    __syncthreads();
    // 4. normalise the pivot row
    if (rank == ok) {
      double2* rk = A + (size_t)(k - lo) * N;
      if (tid == 0) s_pinv = cdiv1(rk[k]);
      __syncthreads();
      const double2 pinv = s_pinv;
      for (int j = tid; j < N; j += nt) rk[j] = (j == k) ? pinv : cmul(rk[j], pinv);
    }
    cl.sync();
    // 5. broadcast the pivot row and eliminate the own rows
    {
      const double2* src = cl.map_shared_rank(A, ok) + (size_t)(k - ok * RB) * N;
      for (int j = tid; j < N; j += nt) piv[j] = src[j];
      for (int il = tid; il < nown; il += nt) fcol[il] = A[(size_t)il * N + k];
    }
    __syncthreads();
    for (int t = tid; t < nown * N; t += nt) {
      const int il = t / N, j = t - il * N;
      if (lo + il == k) continue;
      const double2 f = fcol[il];
      if (j == k) A[t] = make_double2(0.0, 0.0) - cmul(f, piv[j]);
      else A[t] = A[t] - cmul(f, piv[j]);
    }
    __syncthreads();
  }
  // 6. undo the column permutation
  for (int il = tid; il < nown; il += nt) {
    double2* row = A + (size_t)il * N;
    for (int k = N - 1; k >= 0; --k) {
      const int p = perm[k];
      if (p != k) { double2 a = row[k]; row[k] = row[p]; row[p] = a; }
    }
  }
  __syncthreads();
  // 7. store
  const long long NN = (long long)N * N;
  if (mode == 0) {
    double2* dst = outAT + (lunit * 2 + eq) * NN;
    for (int t = tid; t < nown * N; t += nt) {
      const int j = t / nown, il = t - j * nown;
      dst[(long long)j * N + lo + il] = A[(size_t)il * N + j];
    }
  } else {
    double2* dst = (eq == 0 ? outV : outO) + lunit * NN;
    for (int t = tid; t < nown * N; t += nt) dst[(long long)lo * N + t] = A[t];
  }
  cl.sync();  // keep the shared memory alive until every remote reader is done
}

int gj_cluster_size(int N) {
  for (int C = 1; C <= 8; C *= 2) {
    const int RB = (N + C - 1) / C;
    if ((size_t)RB * N * 16 <= 160 * 1024) return C;
  }
  return -1;
}

size_t gj_smem(int N, int C) {
  const int RB = (N + C - 1) / C;
  return (size_t)RB * N * 16 + 2 * (size_t)N * 16 + (size_t)RB * 16 + (size_t)((N + 3) & ~3) * 4 + 32;
}

cudaError_t launch_gj_invert(int mode, long long unit0, long long nunits, DnsGeom g, PhysParams ph,
                             const double* T0, const double* T2, const double* T4,
                             const double* U, const double* ddU, double2* outAT,
                             double2* outV, double2* outO, int* status, cudaStream_t st) {
  const int C = gj_cluster_size(g.Ny);
  if (C < 0) return cudaErrorInvalidValue;
  const size_t sm = gj_smem(g.Ny, C);
  cudaError_t e = cudaFuncSetAttribute(k_gj_invert, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nunits * 2 * C), 1, 1);
  cfg.blockDim = dim3(256, 1, 1);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_gj_invert, mode, unit0, g, ph, T0, T2, T4, U, ddU, outAT, outV,
                            outO, status);
}

// ---------------------------------------------------------------------------
// cuda_transpose (source/transpose.cu:223-257, 358-382): XYZ complex
// [z][ky'][kx] (pitch bytes) <-> ZXY [ky][kx][z] (tpitch bytes) for kx < Kx,
// ky < Nz, z < Py; ky' = ky for ky <= Nz/2 else ky + Pz - Nz.  BACKWARD
// leaves the unmapped XYZ entries untouched, as the reference does.
// ---------------------------------------------------------------------------
__global__ void k_transpose_ref(int dir, double2* xyz, long long ps, double2* zxy, long long tps,
                                DnsGeom g) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)g.H * g.Py;
  if (idx >= total) return;
  const int z = (int)(idx % g.Py);
  const long long p = idx / g.Py;
  const int kx = (int)(p % g.Kx);
  const int ky = (int)(p / g.Kx);
  const int kyp = (ky > g.Nz / 2) ? ky + (g.Pz - g.Nz) : ky;
  double2* a = xyz + ((long long)z * g.Pz + kyp) * ps + kx;
  double2* b = zxy + p * tps + z;
  if (dir == 0) *b = *a;
  else *a = *b;
}

cudaError_t launch_transpose_ref(int dir, double2* xyz, long long ps, double2* zxy, long long tps,
                                 DnsGeom g, cudaStream_t st) {
  const long long total = (long long)g.H * g.Py;
  k_transpose_ref<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(dir, xyz, ps, zxy, tps, g);
  return cudaGetLastError();
}

// The collocation operators themselves, row-major out{v,o}[p][i][j] for the
// pencils p0 .. p0 + gridDim.x - 1 (initAuxMatrix with inversed = false,
// source/solver.cpp:275-313): the same entries k_gj_invert inverts.
__global__ void k_operator_matrices(long long p0, DnsGeom g, PhysParams ph, const double* T0,
                                    const double* T2, const double* T4, const double* U,
                                    const double* ddU, double2* outV, double2* outO) {
  const long long lp = blockIdx.x;
  const long long p = p0 + lp;
  const int kx = (int)(p % g.Kx), kz = (int)(p / g.Kx);
  const bool zero = (kx == 0 && kz == 0);
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = kmn_of(ia, ib);
  const int N = g.Ny;
  const size_t NN = (size_t)N * N;
  for (int t = threadIdx.x; t < N * N; t += blockDim.x) {
    const int i = t / N, j = t - i * N;
    outV[lp * NN + t] = op_entry(0, zero, i, j, N, T0, T2, T4, U, ddU, ph.Re, ph.dt, kmn, ia);
    outO[lp * NN + t] = op_entry(1, zero, i, j, N, T0, T2, T4, U, ddU, ph.Re, ph.dt, kmn, ia);
  }
}

cudaError_t launch_operator_matrices(long long p0, long long np, DnsGeom g, PhysParams ph,
                                     const double* T0, const double* T2, const double* T4,
                                     const double* U, const double* ddU, double2* outV,
                                     double2* outO, cudaStream_t st) {
  if (np <= 0) return cudaSuccess;
  k_operator_matrices<<<(unsigned)np, 256, 0, st>>>(p0, g, ph, T0, T2, T4, U, ddU, outV, outO);
  return cudaGetLastError();
}

// Residual of solved collocation systems, one CTA per pencil: r = A x - b
// with A the reference's operator (the same entries as k_gj_invert's) for
// the v (eq 0) and omega (eq 1) systems.  per[p] = {|r_v|^2, |b_v|^2,
// |r_o|^2, |b_o|^2, normwise backward error of v and of omega:
// max|r| / (max_i sum_j |A_ij| max|x| + max|b|)}.
__global__ void __launch_bounds__(128) k_solve_residual(const double2* __restrict__ bv,
                                                        const double2* __restrict__ bo,
                                                        const double2* __restrict__ xv,
                                                        const double2* __restrict__ xo, long long ps,
                                                        DnsGeom g, PhysParams ph, const double* T0,
                                                        const double* T2, const double* T4,
                                                        const double* U, const double* ddU, double* per) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = g.Ny;
  double2* x = (double2*)smem_raw;  // [eq][N]
  __shared__ double red[4][6];      // per warp: |r|^2, |b|^2, max|r|, max rowsum, max|x|, max|b|
  const long long p = blockIdx.x;
  const int kx = (int)(p % g.Kx), kz = (int)(p / g.Kx);
  const bool zero = kx == 0 && kz == 0;
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = kmn_of(ia, ib);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int eq = 0; eq < 2; ++eq) {
    const double2* xs = eq ? xo : xv;
    const double2* bs = eq ? bo : bv;
    for (int j = threadIdx.x; j < N; j += blockDim.x) x[j] = xs[p * ps + j];
    __syncthreads();
    double r2 = 0, b2 = 0, rmax = 0, amax = 0, xmax = 0, bmax = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      double2 s = make_double2(0.0, 0.0);
      double rs = 0;
      for (int j = 0; j < N; ++j) {
        const double2 a = op_entry(eq, zero, i, j, N, T0, T2, T4, U, ddU, ph.Re, ph.dt, kmn, ia);
        s = s + cmul(a, x[j]);
        rs += hypot(a.x, a.y);
      }
      const double2 b = bs[p * ps + i];
      const double2 r = s - b;
      r2 += r.x * r.x + r.y * r.y;
      b2 += b.x * b.x + b.y * b.y;
      rmax = fmax(rmax, hypot(r.x, r.y));
      amax = fmax(amax, rs);
      bmax = fmax(bmax, hypot(b.x, b.y));
      xmax = fmax(xmax, hypot(x[i].x, x[i].y));
    }
    for (int o = 16; o; o >>= 1) {
      r2 += __shfl_xor_sync(0xffffffffu, r2, o);
      b2 += __shfl_xor_sync(0xffffffffu, b2, o);
      rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
      amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
      xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
      bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
    }
    if (lane == 0) {
      red[warp][0] = r2; red[warp][1] = b2; red[warp][2] = rmax;
      red[warp][3] = amax; red[warp][4] = xmax; red[warp][5] = bmax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t[6] = {0, 0, 0, 0, 0, 0};
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        t[0] += red[w][0]; t[1] += red[w][1];
        for (int k = 2; k < 6; ++k) t[k] = fmax(t[k], red[w][k]);
      }
      const double den = t[3] * t[4] + t[5];
      per[p * 6 + 2 * eq] = t[0];
      per[p * 6 + 2 * eq + 1] = t[1];
      per[p * 6 + 4 + eq] = den > 0 ? t[2] / den : 0.0;
    }
    __syncthreads();
  }
}

cudaError_t launch_solve_residual(const double2* bv, const double2* bo, const double2* xv, const double2* xo,
                                  long long ps, DnsGeom g, PhysParams ph, const double* T0,
                                  const double* T2, const double* T4, const double* U, const double* ddU,
                                  double* per, cudaStream_t st) {
  k_solve_residual<<<(unsigned)g.H, 128, (size_t)g.Ny * 16, st>>>(bv, bo, xv, xo, ps, g, ph, T0, T2, T4, U, ddU,
                                                                  per);
  return cudaGetLastError();
}
