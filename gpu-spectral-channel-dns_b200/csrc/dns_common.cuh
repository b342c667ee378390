// Common types and helpers for the B200 DNS kernels.
//
// Complex numbers are CUDA vector types (double2 / float2), 16 / 8 bytes,
// layout-compatible with the reference's cuRPCF::complex (include/data.h:37-79)
// so buffers in the reference's pitched layouts can be read directly.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DNS_HD __host__ __device__ __forceinline__

template <typename T> struct cplx;
template <> struct cplx<double> { typedef double2 t; };
template <> struct cplx<float> { typedef float2 t; };

template <typename C> struct scalar_of;
template <> struct scalar_of<double2> { typedef double t; };
template <> struct scalar_of<float2> { typedef float t; };
template <typename C> using T_of = typename scalar_of<C>::t;

template <typename C> DNS_HD C cmk(double re, double im) {
  C r; r.x = (decltype(r.x))re; r.y = (decltype(r.y))im; return r;
}
DNS_HD double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
DNS_HD double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
DNS_HD double2 operator*(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
DNS_HD double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
DNS_HD double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
DNS_HD double2 conj(double2 a) { return make_double2(a.x, -a.y); }
DNS_HD double2 muli(double2 a) { return make_double2(-a.y, a.x); }  // i*a

DNS_HD float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
DNS_HD float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
DNS_HD float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
DNS_HD float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
DNS_HD float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
DNS_HD float2 conj(float2 a) { return make_float2(a.x, -a.y); }
DNS_HD float2 muli(float2 a) { return make_float2(-a.y, a.x); }

DNS_HD double2 to_d2(double2 a) { return a; }
DNS_HD double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
template <typename C> DNS_HD C from_d2(double2 a);
template <> DNS_HD double2 from_d2<double2>(double2 a) { return a; }
template <> DNS_HD float2 from_d2<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }

// Problem geometry derived from the reference's parameter triple
// (mx, my, mz) (source/data.cpp:3-13, include/data.h:312-328).
struct DnsGeom {
  int mx, my, mz;   // reference parameters: padded x, padded span, 4*(Ny-1)
  int Nx, Nz, Ny;   // Fourier modes (x, span) and Chebyshev modes
  int Kx;           // streamwise modes kept: Nx/2 + 1 (reference hnx)
  int Px, Pz, Py;   // physical points: mx, my, 2*Ny - 1 (reference pz)
  long long H;      // number of pencils Kx * Nz (of a launch: the pencils it covers)
  int Kh;           // spanwise pencils that own an operator: Nz/2 + 1
  int kz0;          // spanwise index of a launch's first pencil (wall-normal passes
                    // on a run of pencils kz0 .. kz0 + H/Kx - 1; 0 for the whole grid)
  long long Hrun;   // pencils per member of a batch of runs (= H for one run): pencil
                    // p of a launch is pencil p mod Hrun of member p / Hrun
  int nrun;         // members of a batch (1 for one run)
};

static inline DnsGeom dns_make_geom(int mx, int my, int mz) {
  DnsGeom g;
  g.mx = mx; g.my = my; g.mz = mz;
  g.Nx = mx / 3 * 2; g.Nz = my / 3 * 2; g.Ny = mz / 4 + 1;
  g.Kx = g.Nx / 2 + 1;
  g.Px = mx; g.Pz = my; g.Py = mz / 2 + 1;
  g.H = (long long)g.Kx * g.Nz;
  g.Kh = g.Nz / 2 + 1;
  g.kz0 = 0;
  g.Hrun = g.H;
  g.nrun = 1;
  return g;
}

// member, streamwise and spanwise index of pencil p of a wall-normal launch
// (32-bit arithmetic: a launch covers fewer than 2^31 pencils, checked when
// the context is created)
DNS_HD void pencil_modes(const DnsGeom& g, long long p, int& run, int& kx, int& kz) {
  const unsigned pu = (unsigned)p, hr = (unsigned)g.Hrun, K = (unsigned)g.Kx;
  const unsigned r = g.nrun > 1 ? pu / hr : 0u;
  const unsigned q = pu - r * hr;
  run = (int)r;
  kx = (int)(q % K);
  kz = g.kz0 + (int)(q / K);
}

// ia^2 + ib^2 rounded like the reference's host code (no FMA contraction)
DNS_HD double kmn_of(double ia, double ib) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(__dmul_rn(ia, ia), __dmul_rn(ib, ib));
#else
  return ia * ia + ib * ib;
#endif
}

// streamwise / spanwise wavenumbers of a pencil (source/RPCFKernels.cu:522-532)
DNS_HD void wavenumbers(int kx, int kz, int Nz, double aphi, double beta,
                        double& ia, double& ib) {
  ia = (double)kx / aphi;
  ib = (kz >= Nz / 2 + 1) ? (double)(kz - Nz) / beta : (double)kz / beta;
}

// a complex value of element type E (float2 / double2) as C
template <typename C, typename E> DNS_HD C from_e(E a) { return cmk<C>(a.x, a.y); }
