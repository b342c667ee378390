// The reference's analytic initial condition (initFlow,
// source/RPCFKernels.cu:358-431; fields :142-309, grid :311-356).
//
// Only the wall-normal velocity w and the wall-normal vorticity omega_z enter
// the state (the reference copies their transforms into rhs_v / rhs_omega_y
// and recomputes the other four components with getUVW), so the kernel
// evaluates those two on the no-padding grid: mx x my points, nz Gauss-Lobatto
// planes z_k = cos(pi k / (nz - 1)), zero on the two wall planes.  They are
// then taken to spectral space by the forward transform without padding.
#include <cmath>

#include "../../include/dns_b200.h"
#include "context_impl.cuh"

namespace {

constexpr double kEpsInit = 0.005;  // EPSILON_INIT, source/RPCFKernels.cu:132

// w(x, y, z) and omega_z(x, y, z), the three-mode perturbation written out
__device__ void init_w_oz(double xx, double yy, double zz, double lx, double ly, double* w,
                          double* oz) {
  const double pi = 3.141592653589793;
  const double a1 = 2.0 * pi * xx / lx, a2 = 4.0 * pi * xx / lx;
  const double b1 = 2.0 * pi * yy / ly, b2 = 4.0 * pi * yy / ly;
  const double sa1 = sin(a1), sa2 = sin(a2), ca1 = cos(a1), ca2 = cos(a2);
  const double sb1 = sin(b1), sb2 = sin(b2), cb1 = cos(b1), cb2 = cos(b2);
  const double s15 = sin(1.5 * pi * zz), c15 = cos(1.5 * pi * zz);
  *w = kEpsInit * (-2.0 / 3.0) * (1.0 + c15) * (sa1 * sb1 + sa2 * sb1 + sa1 * sb2);
  *oz = kEpsInit * 2.0 * pi * s15 *
        (lx / ly * (ca1 * cb1 + 0.5 * ca2 * cb1 + 2.0 * ca1 * cb2) +
         ly / lx * (0.5 * ca1 * cb1 + ca2 * cb1 + 0.25 * ca1 * cb2));
}

// one thread per point of an x row; rows [z][y] of pitch rp doubles
__global__ void k_init_flow(double* __restrict__ w, double* __restrict__ oz, long long rp, int px,
                            int py, int nz, double lx, double ly) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  if (x >= px) return;
  const long long at = rp * ((long long)py * z + y) + x;
  if (z == 0 || z == nz - 1) {
    w[at] = 0.0;
    oz[at] = 0.0;
    return;
  }
  const double pi = 3.141592653589793;
  const double xx = (x * 1.0) / px * lx, yy = (y * 1.0) / py * ly, zz = cos(pi * z / (nz - 1));
  init_w_oz(xx, yy, zz, lx, ly, &w[at], &oz[at]);
}

}  // namespace

extern "C" dns_status dns_init_flow(dns_ctx* c) {
  if (c && (c->g.nrun > 1 || c->slab))
    return dns_internal_fail(DNS_ERR_STATE, "a batch or slab context: this entry point takes one whole run");
  if (!c) return dns_internal_fail(DNS_ERR_ARG, "null context");
  if (cudaSetDevice(c->P.device)) return dns_internal_fail(DNS_ERR_CUDA, "cudaSetDevice");
  const DnsGeom& g = c->g;
  // two physical fields (all Py planes, the unused ones zero) and two
  // spectral fields of pitch mz complex
  const size_t pitch = (size_t)(g.Px / 2 + 1) * 16, tpitch = (size_t)g.mz * 16;
  const size_t psz = pitch * (size_t)g.Pz * g.Py, tsz = tpitch * (size_t)g.H;
  unsigned char* buf = nullptr;
  if (cudaMalloc(&buf, 2 * psz + 2 * tsz)) return dns_internal_fail(DNS_ERR_CUDA, "init flow: device memory");
  struct Guard {
    void* p;
    ~Guard() { cudaFree(p); }
  } guard{buf};
  double* w = (double*)buf;
  double* oz = (double*)(buf + psz);
  unsigned char* tw = buf + 2 * psz;
  unsigned char* toz = tw + tsz;
  if (cudaMemsetAsync(buf, 0, 2 * psz, c->st)) return dns_internal_fail(DNS_ERR_CUDA, "init flow: memset");
  const double lx = 2.0 * 3.141592653589793 * c->ph.aphi, ly = 2.0 * 3.141592653589793 * c->ph.beta;
  dim3 grid((g.Px + 127) / 128, g.Pz, g.Ny);
  k_init_flow<<<grid, 128, 0, c->st>>>(w, oz, (long long)(pitch / 8), g.Px, g.Pz, g.Ny, lx, ly);
  if (cudaGetLastError()) return dns_internal_fail(DNS_ERR_CUDA, "init flow: launch");
  dns_status s = dns_transform_3d_one(c, DNS_FORWARD, w, pitch, tw, tpitch, DNS_NO_PADDING);
  if (s == DNS_OK) s = dns_transform_3d_one(c, DNS_FORWARD, oz, pitch, toz, tpitch, DNS_NO_PADDING);
  if (s == DNS_OK) s = dns_synchronize(c);
  if (s == DNS_OK) s = dns_set_state(c, tw, toz, tpitch, DNS_DEVICE);
  return s;
}
