// Reference-layout right-hand sides of the Crank-Nicolson / AB2 step, for
// callers that run the reference's step sequence function by function
// (get_rhs_v -> solveEq -> get_rhs_omega -> solveEq):
//
//   dns_rhs_v ......... get_linear_v + the AB2 loop of get_rhs_v
//                       (source/linear.cpp:7-41,86-125, source/rhs.cpp:185-219)
//   dns_rhs_omega ..... get_linear_omega_y (source/linear.cpp:52-84,127-171)
//   dns_rhs_mean ...... get_linear_zero_wave_u_w (source/linear.cpp:43-50,173-205)
//   dns_operator_tables / dns_operator_matrices ... the T matrices, U profile
//                       and collocation operators initAuxMatrix stores
//                       (source/solver.cpp:260-320, source/coefficient.cu)
//
// The fused time step does not use these kernels: it forms the same right-
// hand sides in Chebyshev coefficient space inside its y1 pass.  Here each
// pencil's right-hand side is the reference's collocation form, evaluated on
// the GPU: one CTA per pencil, one warp per collocation row, lanes over the
// Chebyshev index (coalesced rows of the T tables), FP64 throughout.
#include <algorithm>
#include <string>

#include "../../include/dns_b200.h"
#include "context_impl.cuh"

namespace {

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double2 warp_sum(double2 v) {
  return make_double2(warp_sum(v.x), warp_sum(v.y));
}

// rows 4..N: the explicit half of the CN v operator applied to v^n at the
// collocation point r = i - 2, plus AB2; rows 0..3 (wall rows) zero; v^n is
// saved to rvp (the reference's rhs_v_p).  Pencil (0,0) is left alone.
__global__ void k_rhs_v(double2* rv, double2* rvp, const double2* nv, const double2* nvp,
                        long long ps, const double* T0, const double* T2, const double* T4,
                        const double* U, const double* ddU, DnsGeom g, PhysParams ph) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* v = (double2*)smem_raw;
  const int Ny = g.Ny;
  const long long p = blockIdx.x;
  const int kx = (int)(p % g.Kx), kz = (int)(p / g.Kx);
  if (kx == 0 && kz == 0) return;
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = kmn_of(ia, ib);
  const double dt = ph.dt, Re = ph.Re;
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    v[n] = rv[p * ps + n];
    rvp[p * ps + n] = v[n];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double a4 = dt * 0.5 / Re, a2 = 1 - kmn * dt / Re, a0 = -kmn * (1 - kmn * dt * 0.5 / Re);
  for (int i = warp; i < Ny; i += nw) {
    double2 out = make_double2(0.0, 0.0);
    if (i >= 4) {
      const int r = i - 2;
      double2 P0 = make_double2(0, 0), P2 = P0, P4 = P0;
      for (int j = lane; j < Ny; j += 32) {
        const size_t c = (size_t)r * Ny + j;
        P0 = P0 + v[j] * T0[c];
        P2 = P2 + v[j] * T2[c];
        P4 = P4 + v[j] * T4[c];
      }
      P0 = warp_sum(P0);
      P2 = warp_sum(P2);
      P4 = warp_sum(P4);
      const double b2 = -ia * dt * 0.5 * U[r];
      const double b0 = kmn * ia * dt * 0.5 * U[r] + ia * dt * 0.5 * ddU[r];
      out = P4 * a4 + P2 * a2 + P0 * a0 + muli(P2 * b2 + P0 * b0);
      out = out + (nv[p * ps + r] * 1.5 - nvp[p * ps + r] * 0.5) * dt;
    }
    if (lane == 0) rv[p * ps + i] = out;
  }
}

// rows 2..N: the explicit half of the CN omega operator at r = i - 1, the
// tilting term -i beta U' dt/2 (v^{n+1} + v^n) and AB2; rows 0, 1 zero.
__global__ void k_rhs_omega(double2* ro, const double2* no, const double2* nop, const double2* vn1,
                            const double2* vn, long long ps, const double* T0, const double* T2,
                            const double* U, const double* dU, DnsGeom g, PhysParams ph) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* o = (double2*)smem_raw;
  double2* s = o + g.Ny;
  const int Ny = g.Ny;
  const long long p = blockIdx.x;
  const int kx = (int)(p % g.Kx), kz = (int)(p / g.Kx);
  if (kx == 0 && kz == 0) return;
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kmn = kmn_of(ia, ib);
  const double dt = ph.dt, Re = ph.Re;
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) {
    o[n] = ro[p * ps + n];
    s[n] = vn[p * ps + n] + vn1[p * ps + n];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double a2 = 0.5 / Re * dt, a0 = 1 - kmn * dt * 0.5 / Re;
  for (int i = warp; i < Ny; i += nw) {
    double2 out = make_double2(0.0, 0.0);
    if (i >= 2) {
      const int r = i - 1;
      double2 Q0 = make_double2(0, 0), Q2 = Q0, S0 = Q0;
      for (int j = lane; j < Ny; j += 32) {
        const size_t c = (size_t)r * Ny + j;
        Q0 = Q0 + o[j] * T0[c];
        Q2 = Q2 + o[j] * T2[c];
        S0 = S0 + s[j] * T0[c];
      }
      Q0 = warp_sum(Q0);
      Q2 = warp_sum(Q2);
      S0 = warp_sum(S0);
      out = Q2 * a2 + Q0 * a0 + muli(Q0 * (-ia * dt * 0.5 * U[r]) + S0 * (-0.5 * ib * dU[r] * dt));
      out = out + (no[p * ps + r] * 1.5 - nop[p * ps + r] * 0.5) * dt;
    }
    if (lane == 0) ro[p * ps + i] = out;
  }
}

// the mean modes u0 (block 0) and w0 (block 1): rows 2..N of
// (T0 + dt/(2 Re) T2) x - dt (1.5 lambda - 0.5 lambda_p) at r = i - 1;
// rows 0, 1 (Dirichlet) zero
__global__ void k_rhs_mean(double2* u0, const double2* lx, const double2* lxp, double2* w0,
                           const double2* lz, const double2* lzp, int Ny, const double* T0,
                           const double* T2, double Re, double dt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* x = (double2*)smem_raw;
  double2* vec = blockIdx.x == 0 ? u0 : w0;
  const double2* l = blockIdx.x == 0 ? lx : lz;
  const double2* lp = blockIdx.x == 0 ? lxp : lzp;
  for (int n = threadIdx.x; n < Ny; n += blockDim.x) x[n] = vec[n];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int i = warp; i < Ny; i += nw) {
    double2 out = make_double2(0.0, 0.0);
    if (i >= 2) {
      const int r = i - 1;
      double2 a = make_double2(0, 0);
      for (int j = lane; j < Ny; j += 32) {
        const size_t c = (size_t)r * Ny + j;
        a = a + x[j] * (T0[c] + dt * 0.5 / Re * T2[c]);
      }
      a = warp_sum(a);
      out = a - (l[r] * 1.5 - lp[r] * 0.5) * dt;
    }
    if (lane == 0) vec[i] = out;
  }
}

struct Stage {
  // a pencil field of the caller: pointer, read by the kernel, written by it
  const void* src;
  bool in, out;
};

// Run `launch(ptrs, ps)` on the caller's pencils: in place for device
// buffers, through the context's staging vectors (pitch Ny) for host ones.
template <typename F>
dns_status staged(dns_ctx* c, Stage* f, int n, size_t tpitch, int where, F launch) {
  const DnsGeom& g = c->g;
  const size_t row = (size_t)g.Ny * 16;
  if (where != DNS_HOST && where != DNS_DEVICE)
    return dns_internal_fail(DNS_ERR_ARG, "where must be DNS_HOST or DNS_DEVICE");
  if (tpitch % 16 || tpitch < row)
    return dns_internal_fail(DNS_ERR_ARG, "tpitch must be a multiple of 16 and hold Ny complex values");
  if (cudaSetDevice(c->P.device)) return dns_internal_fail(DNS_ERR_CUDA, "cudaSetDevice");
  double2* ptr[6];
  if (where == DNS_DEVICE) {
    for (int i = 0; i < n; ++i) ptr[i] = (double2*)f[i].src;
    cudaError_t e = launch(ptr, (long long)(tpitch / 16));
    if (e) return dns_internal_fail(DNS_ERR_CUDA, cudaGetErrorString(e));
    return DNS_OK;
  }
  const size_t hn = (size_t)g.H * g.Ny;
  if (!c->rhs_io && c->alloc(&c->rhs_io, 6 * hn))
    return dns_internal_fail(DNS_ERR_CUDA, "staging allocation");
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < n && !e; ++i) {
    ptr[i] = c->rhs_io + i * hn;
    if (f[i].in)
      e = cudaMemcpy2DAsync(ptr[i], row, f[i].src, tpitch, row, g.H, cudaMemcpyHostToDevice, c->st);
  }
  if (!e) e = launch(ptr, (long long)g.Ny);
  for (int i = 0; i < n && !e; ++i)
    if (f[i].out)
      e = cudaMemcpy2DAsync((void*)f[i].src, tpitch, ptr[i], row, row, g.H, cudaMemcpyDeviceToHost, c->st);
  if (!e) e = cudaStreamSynchronize(c->st);
  if (e) return dns_internal_fail(DNS_ERR_CUDA, cudaGetErrorString(e));
  return DNS_OK;
}

unsigned threads_for(int Ny) { return (unsigned)std::min(256, std::max(64, (Ny + 31) / 32 * 32)); }

}  // namespace

extern "C" {

dns_status dns_rhs_v(dns_ctx* c, void* rhs_v, void* rhs_v_p, const void* nv, const void* nv_p,
                     size_t tpitch, int where) {
  if (!c || !rhs_v || !rhs_v_p || !nv || !nv_p) return dns_internal_fail(DNS_ERR_ARG, "null argument");
  // rhs_v_p is copied in too: pencil (0,0) keeps its value
  Stage f[4] = {{rhs_v, true, true}, {rhs_v_p, true, true}, {nv, true, false}, {nv_p, true, false}};
  const DnsGeom g = c->g;
  const PhysParams ph = c->ph;
  const size_t sm = (size_t)g.Ny * 16;
  return staged(c, f, 4, tpitch, where, [&](double2** q, long long ps) {
    k_rhs_v<<<(unsigned)g.H, threads_for(g.Ny), sm, c->st>>>(q[0], q[1], q[2], q[3], ps, c->T0, c->T2,
                                                            c->T4, c->Ut, c->ddUt, g, ph);
    return cudaGetLastError();
  });
}

dns_status dns_rhs_omega(dns_ctx* c, void* rhs_omega, const void* nomega, const void* nomega_p,
                         const void* rhs_v, const void* rhs_v_p, size_t tpitch, int where) {
  if (!c || !rhs_omega || !nomega || !nomega_p || !rhs_v || !rhs_v_p)
    return dns_internal_fail(DNS_ERR_ARG, "null argument");
  Stage f[5] = {{rhs_omega, true, true}, {nomega, true, false}, {nomega_p, true, false},
                {rhs_v, true, false}, {rhs_v_p, true, false}};
  const DnsGeom g = c->g;
  const PhysParams ph = c->ph;
  const size_t sm = (size_t)2 * g.Ny * 16;
  return staged(c, f, 5, tpitch, where, [&](double2** q, long long ps) {
    k_rhs_omega<<<(unsigned)g.H, threads_for(g.Ny), sm, c->st>>>(q[0], q[1], q[2], q[3], q[4], ps,
                                                                c->T0, c->T2, c->Ut, c->dUt, g, ph);
    return cudaGetLastError();
  });
}

dns_status dns_rhs_mean(dns_ctx* c, void* u0, const void* lambx0, const void* lambx0_p, void* w0,
                        const void* lambz0, const void* lambz0_p, int where) {
  if (!c || !u0 || !lambx0 || !lambx0_p || !w0 || !lambz0 || !lambz0_p)
    return dns_internal_fail(DNS_ERR_ARG, "null argument");
  if (where != DNS_HOST && where != DNS_DEVICE)
    return dns_internal_fail(DNS_ERR_ARG, "where must be DNS_HOST or DNS_DEVICE");
  if (cudaSetDevice(c->P.device)) return dns_internal_fail(DNS_ERR_CUDA, "cudaSetDevice");
  const int Ny = c->g.Ny;
  const size_t vb = (size_t)Ny * 16;
  const void* src[6] = {u0, lambx0, lambx0_p, w0, lambz0, lambz0_p};
  double2* q[6];
  cudaError_t e = cudaSuccess;
  if (where == DNS_HOST) {
    const size_t hn = (size_t)c->g.H * Ny;
    if (!c->rhs_io && c->alloc(&c->rhs_io, 6 * hn))
      return dns_internal_fail(DNS_ERR_CUDA, "staging allocation");
    for (int i = 0; i < 6 && !e; ++i) {
      q[i] = c->rhs_io + (size_t)i * Ny;
      e = cudaMemcpyAsync(q[i], src[i], vb, cudaMemcpyHostToDevice, c->st);
    }
  } else {
    for (int i = 0; i < 6; ++i) q[i] = (double2*)src[i];
  }
  if (!e) {
    k_rhs_mean<<<2, threads_for(Ny), vb, c->st>>>(q[0], q[1], q[2], q[3], q[4], q[5], Ny, c->T0, c->T2,
                                                c->ph.Re, c->ph.dt);
    e = cudaGetLastError();
  }
  if (!e && where == DNS_HOST) {
    e = cudaMemcpyAsync(u0, q[0], vb, cudaMemcpyDeviceToHost, c->st);
    if (!e) e = cudaMemcpyAsync(w0, q[3], vb, cudaMemcpyDeviceToHost, c->st);
    if (!e) e = cudaStreamSynchronize(c->st);
  }
  if (e) return dns_internal_fail(DNS_ERR_CUDA, cudaGetErrorString(e));
  return DNS_OK;
}

dns_status dns_operator_tables(dns_ctx* c, double* T0, double* T2, double* T4, double* U, double* dU,
                               double* ddU) {
  if (!c) return dns_internal_fail(DNS_ERR_ARG, "null context");
  if (cudaSetDevice(c->P.device)) return dns_internal_fail(DNS_ERR_CUDA, "cudaSetDevice");
  const size_t Ny = (size_t)c->g.Ny;
  struct { void* dst; const double* src; size_t n; } cp[6] = {
      {T0, c->T0, Ny * Ny}, {T2, c->T2, Ny * Ny}, {T4, c->T4, Ny * Ny},
      {U, c->Ut, Ny}, {dU, c->dUt, Ny}, {ddU, c->ddUt, Ny}};
  for (auto& x : cp)
    if (x.dst && cudaMemcpy(x.dst, x.src, x.n * 8, cudaMemcpyDeviceToHost))
      return dns_internal_fail(DNS_ERR_CUDA, "table copy");
  return DNS_OK;
}

}  // extern "C"
