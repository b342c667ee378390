// dns_transform_3d_one_noalloc: the reference-layout 3D transform without
// any device allocation at call time.
//
// Why: dns_transform_3d_one needs a work buffer of one complex row per
// (wall-normal point, spanwise point) and allocates it with cudaMalloc on its
// first call.  Some callers cannot allow that: an application that has
// already carved almost all device memory into its own arena (a late
// cudaMalloc would fail or fragment it), or a time-critical loop where the
// implicit device synchronisation of cudaMalloc is not acceptable.  This
// variant keeps its work buffer in a file-scope device array, reserved once
// when the library's device code is loaded, and runs the same kernels as
// dns_transform_3d_one over slabs of wall-normal planes that fit in it, so
// its results are identical.
//
// The device array is DNS_NOALLOC_SCRATCH_BYTES (16 MiB) per GPU that loads
// the library, held until the process exits.  Limit: one wall-normal plane of
// streamwise rows, my x roundup(mx/2+1, 8) complex doubles, must fit in it;
// larger grids are rejected with DNS_ERR_ARG.  The buffer is shared by every
// call on a device and keeps the previous call's contents; each slab writes
// every entry it later reads, so nothing needs clearing, but calls that
// overlap on the GPU (different streams, contexts or threads) race on it.
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current, and again after the
// device's context has been reset and created anew; make that first call
// before any stream capture.
#include <mutex>
#include <string>

#include "context_impl.cuh"
#include "kernels.cuh"
#include "ypass.cuh"
#include "zxpass.cuh"

#define DNS_NOALLOC_SCRATCH_BYTES (16u << 20)
#define DNS_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[DNS_NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_addr[DNS_NOALLOC_MAX_DEVICES];
void* g_noalloc_ctx[DNS_NOALLOC_MAX_DEVICES];  // the context the address belongs to

// the driver's cuCtxGetCurrent, through the runtime (no link against libcuda)
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = []() -> CtxGetCurrentFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return (CtxGetCurrentFn)p;
  }();
  return fn;
}

// device address of g_noalloc_scratch on the current device, looked up once
// per device and context: a context that was reset (cudaDeviceReset) and
// created again loads the module again, at a possibly different address
cudaError_t noalloc_scratch(int dev, void** out) {
  if (dev < 0 || dev >= DNS_NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  void* ctx = nullptr;
  if (CtxGetCurrentFn f = ctx_get_current()) f(&ctx);
  if (!g_noalloc_addr[dev] || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[dev] = p;
    g_noalloc_ctx[dev] = ctx;
  }
  *out = g_noalloc_addr[dev];
  return cudaSuccess;
}
}  // namespace

extern "C" dns_status dns_transform_3d_one_noalloc(dns_ctx* c, int dir, void* phys, size_t pitch,
                                                   void* spec, size_t tpitch, int pad) {
  auto fail = [](dns_status s, const std::string& m) { return dns_internal_fail(s, m.c_str()); };
  if (!c || !phys || !spec) return fail(DNS_ERR_ARG, "null argument");
  if ((dir != DNS_FORWARD && dir != DNS_BACKWARD) || (pad != DNS_PADDING && pad != DNS_NO_PADDING))
    return fail(DNS_ERR_ARG, "bad direction or padding mode");
  const DnsGeom& g = c->g;
  if (tpitch % 16 || tpitch < (size_t)c->P.mz * 16)
    return fail(DNS_ERR_ARG, "tpitch must be a multiple of 16 and hold mz complex values");
  if (pitch % 16 || pitch < (size_t)(g.Px / 2 + 1) * 16)
    return fail(DNS_ERR_ARG, "pitch must be a multiple of 16 and hold mx/2+1 complex values");
  const size_t plane_bytes = (size_t)g.Pz * (size_t)c->RS * 16;
  if (plane_bytes > DNS_NOALLOC_SCRATCH_BYTES)
    return fail(DNS_ERR_ARG, "grid too large for the 16 MiB static work buffer: one wall-normal "
                             "plane (my x roundup(mx/2+1,8) complex doubles) must fit");
  cudaError_t e = cudaSetDevice(c->P.device);
  if (e != cudaSuccess) return fail(DNS_ERR_CUDA, cudaGetErrorString(e));
  void* scr = nullptr;
  e = noalloc_scratch(c->P.device, &scr);
  if (e != cudaSuccess) return fail(DNS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));

  // wall-normal planes per slab; row pairs of the streamwise transform never
  // straddle a slab because Pz is even
  const int S = (int)(DNS_NOALLOC_SCRATCH_BYTES / plane_bytes);
  const long long ps = (long long)(tpitch / 16);
  const long long rps = (long long)(pitch / 8);
  PencilArr sp{spec, ps, 0};
  RowArr sr{scr, c->RS, 0};
  auto ck = [&](cudaError_t err) { return err == cudaSuccess ? DNS_OK : fail(DNS_ERR_CUDA, cudaGetErrorString(err)); };
  dns_status st = DNS_OK;
  if (dir == DNS_BACKWARD) {
    if (pad == DNS_PADDING) st = ck(launch_cheby_inplace<double2>(sp, g.H, 0, g.Ny, c->fyP_d.tab(), c->st));
    else st = ck(launch_cheby_inplace<double2>(sp, g.H, 1, g.Ny, c->fy0_d.tab(), c->st));
    for (int y0 = 0; y0 < g.Py && st == DNS_OK; y0 += S) {
      DnsGeom gs = g;
      gs.Py = (g.Py - y0 < S) ? g.Py - y0 : S;
      PencilArr slab_in{(double2*)spec + y0, ps, 0};
      double* out = (double*)phys + (long long)y0 * g.Pz * rps;
      st = ck(launch_zb<double2>(slab_in, sr, 1, gs, c->fz_d.tab(), c->st, nullptr, DNS_Z_BLOCK));
      if (st == DNS_OK)
        st = ck(launch_x_c2r<double2>(sr, out, rps, (long long)gs.Py * g.Pz, gs, c->fx_d.tab(), c->st));
    }
  } else {
    for (int y0 = 0; y0 < g.Py && st == DNS_OK; y0 += S) {
      DnsGeom gs = g;
      gs.Py = (g.Py - y0 < S) ? g.Py - y0 : S;
      const double* in = (const double*)phys + (long long)y0 * g.Pz * rps;
      PencilArr slab_out{(double2*)spec + y0, ps, 0};
      st = ck(launch_x_r2c<double2>(in, rps, sr, (long long)gs.Py * g.Pz, gs, c->fx_d.tab(),
                                     1.0 / g.Px / g.Pz, c->st));
      if (st == DNS_OK) st = ck(launch_zf<double2>(sr, slab_out, 1, gs, c->fz_d.tab(), c->st, nullptr, DNS_Z_BLOCK));
    }
    if (st == DNS_OK) {
      if (pad == DNS_PADDING) st = ck(launch_cheby_inplace<double2>(sp, g.H, 2, g.Ny, c->fyP_d.tab(), c->st));
      else st = ck(launch_cheby_inplace<double2>(sp, g.H, 3, g.Ny, c->fy0_d.tab(), c->st));
    }
  }
  return st;
}
