// Recovery files and physical field output in the reference's formats.
//
//   write_recover_data / read_recover_data ... source/output.cpp:105-178
//   output_velocity / write_velocity ......... source/output.cpp:19-103
//
// Sizes follow the reference's allocator (source/operation.cpp:152-180):
// the pitches come from cudaMalloc3D with the same extents it uses, so the
// byte counts equal the reference's on the same device.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dns_b200.h"
#include "context_impl.cuh"

namespace {

struct RefPitches {
  size_t pitch, tpitch, psize, tsize;
};

cudaError_t ref_pitches(const DnsGeom& g, RefPitches& r) {
  cudaPitchedPtr t;
  cudaError_t e = cudaMalloc3D(&t, make_cudaExtent(16 * (size_t)(g.mx / 2 + 1), g.my, g.Py));
  if (e) return e;
  r.pitch = t.pitch;
  cudaFree(t.ptr);
  e = cudaMalloc3D(&t, make_cudaExtent(16 * (size_t)g.mz, g.Kx, g.Nz));
  if (e) return e;
  r.tpitch = t.pitch;
  cudaFree(t.ptr);
  r.psize = r.pitch * (size_t)g.my * g.Py;
  r.tsize = r.tpitch * (size_t)g.Kx * g.Nz;
  return cudaSuccess;
}

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

}  // namespace

extern "C" {

dns_status dns_write_recovery(dns_ctx* c, const char* path) {
  if (c && (c->g.nrun > 1 || c->slab))
    return dns_internal_fail(DNS_ERR_STATE, "a batch or slab context: this entry point takes one whole run");
  if (!c || !path) return dns_internal_fail(DNS_ERR_ARG, "null argument");
  if (cudaSetDevice(c->P.device)) return dns_internal_fail(DNS_ERR_CUDA, "cudaSetDevice");
  const DnsGeom& g = c->g;
  RefPitches rp;
  if (ref_pitches(g, rp)) return dns_internal_fail(DNS_ERR_CUDA, "pitch query");
  const size_t ny16 = (size_t)g.Ny * 16;
  std::vector<unsigned char> v(rp.tsize, 0), o(rp.tsize, 0), nv(rp.tsize, 0), no(rp.tsize, 0);
  dns_status s = dns_get_state(c, v.data(), o.data(), rp.tpitch, DNS_HOST);
  if (s == DNS_OK) s = dns_get_history(c, nv.data(), no.data(), rp.tpitch, DNS_HOST);
  if (s != DNS_OK) return s;
  File f;
  f.f = fopen(path, "wb");
  if (!f.f) return dns_internal_fail(DNS_ERR_IO, (std::string("cannot open ") + path).c_str());
  const int dims[3] = {g.mx, g.my, g.mz};
  bool ok = fwrite(dims, sizeof(int), 3, f.f) == 3;
  ok = ok && fwrite(&rp.psize, sizeof(size_t), 1, f.f) == 1;
  ok = ok && fwrite(&rp.tsize, sizeof(size_t), 1, f.f) == 1;
  // mean-mode history lambx0, lambz0 (the (0,0) pencil of the nonlinear
  // terms), their previous values (not used on restart: the next step swaps
  // them out; the current ones are written), mean modes tv0, tomega_y_0
  const unsigned char* mean[6] = {nv.data(), no.data(), nv.data(), no.data(), v.data(), o.data()};
  for (int i = 0; i < 6 && ok; ++i) ok = fwrite(mean[i], 1, ny16, f.f) == ny16;
  // rhs_v, rhs_v_p (previous state: not used on restart, the next step
  // overwrites it; the current state is written), rhs_omega_y, nonlinear_v,
  // nonlinear_omega_y
  const unsigned char* bufs[5] = {v.data(), v.data(), o.data(), nv.data(), no.data()};
  for (int i = 0; i < 5 && ok; ++i) ok = fwrite(bufs[i], 1, rp.tsize, f.f) == rp.tsize;
  if (!ok) return dns_internal_fail(DNS_ERR_IO, "recovery file: write failed");
  return DNS_OK;
}

dns_status dns_read_recovery(dns_ctx* c, const char* path) {
  if (c && (c->g.nrun > 1 || c->slab))
    return dns_internal_fail(DNS_ERR_STATE, "a batch or slab context: this entry point takes one whole run");
  if (!c || !path) return dns_internal_fail(DNS_ERR_ARG, "null argument");
  if (cudaSetDevice(c->P.device)) return dns_internal_fail(DNS_ERR_CUDA, "cudaSetDevice");
  const DnsGeom& g = c->g;
  File f;
  f.f = fopen(path, "rb");
  if (!f.f) return dns_internal_fail(DNS_ERR_IO, (std::string("cannot open ") + path).c_str());
  int dims[3];
  size_t psize, tsize;
  if (fread(dims, sizeof(int), 3, f.f) != 3 || fread(&psize, sizeof(size_t), 1, f.f) != 1 ||
      fread(&tsize, sizeof(size_t), 1, f.f) != 1)
    return dns_internal_fail(DNS_ERR_IO, "recovery file: short header");
  if (dims[0] != g.mx || dims[1] != g.my || dims[2] != g.mz)
    return dns_internal_fail(DNS_ERR_ARG, "recovery file: mx, my, mz differ from the context");
  // the pencil pitch of the writer (its device's cudaMalloc3D alignment)
  const size_t npen = (size_t)g.Kx * g.Nz;
  if (tsize % npen || tsize / npen < (size_t)g.mz * 16 || (tsize / npen) % 16)
    return dns_internal_fail(DNS_ERR_IO, "recovery file: inconsistent tSize");
  const size_t tpitch = tsize / npen, ny16 = (size_t)g.Ny * 16;
  std::vector<unsigned char> skip(6 * ny16), v(tsize), vp(tsize), o(tsize), nv(tsize), no(tsize);
  unsigned char* bufs[6] = {skip.data(), v.data(), vp.data(), o.data(), nv.data(), no.data()};
  const size_t sizes[6] = {6 * ny16, tsize, tsize, tsize, tsize, tsize};
  for (int i = 0; i < 6; ++i)
    if (fread(bufs[i], 1, sizes[i], f.f) != sizes[i])
      return dns_internal_fail(DNS_ERR_IO, "recovery file: truncated");
  dns_status s = dns_set_state(c, v.data(), o.data(), tpitch, DNS_HOST);
  if (s == DNS_OK) s = dns_set_history(c, nv.data(), no.data(), tpitch, DNS_HOST);
  return s;
}

dns_status dns_write_fields(dns_ctx* c, const char* velocity_path, const char* vorticity_path) {
  if (c && (c->g.nrun > 1 || c->slab))
    return dns_internal_fail(DNS_ERR_STATE, "a batch or slab context: this entry point takes one whole run");
  if (!c || (!velocity_path && !vorticity_path)) return dns_internal_fail(DNS_ERR_ARG, "null argument");
  if (cudaSetDevice(c->P.device)) return dns_internal_fail(DNS_ERR_CUDA, "cudaSetDevice");
  const DnsGeom& g = c->g;
  // six spectral fields (getUVW of the state) in ZXY pencils of mz complex,
  // one physical field at a time in XYZ rows of mx/2+1 complex
  const size_t tpitch = (size_t)g.mz * 16, pitch = ((size_t)(g.mx / 2 + 1) * 16 + 15) & ~(size_t)15;
  const size_t tsz = tpitch * (size_t)g.H, psz = pitch * (size_t)g.Pz * g.Py;
  unsigned char* spec = nullptr;
  unsigned char* phys = nullptr;
  if (cudaMalloc(&spec, 6 * tsz)) return dns_internal_fail(DNS_ERR_CUDA, "field output: device memory");
  if (cudaMalloc(&phys, psz)) {
    cudaFree(spec);
    return dns_internal_fail(DNS_ERR_CUDA, "field output: device memory");
  }
  struct Guard {
    unsigned char *a, *b;
    ~Guard() { cudaFree(a); cudaFree(b); }
  } guard{spec, phys};
  void* f6[6];
  for (int i = 0; i < 6; ++i) f6[i] = spec + i * tsz;
  // getUVW reads w (f[2]) = v-hat and omega_z (f[5]) = omega_y-hat
  dns_status s = dns_get_state(c, f6[2], f6[5], tpitch, DNS_DEVICE);
  if (s == DNS_OK) s = dns_get_uvw(c, f6, tpitch);
  if (s != DNS_OK) return s;
  std::vector<unsigned char> host(psz);
  const char* paths[2] = {velocity_path, vorticity_path};
  for (int file = 0; file < 2; ++file) {
    if (!paths[file]) continue;
    File f;
    f.f = fopen(paths[file], "wb");
    if (!f.f) return dns_internal_fail(DNS_ERR_IO, (std::string("cannot open ") + paths[file]).c_str());
    for (int comp = 0; comp < 3; ++comp) {
      // the backward transform works on its spectral input in place; each
      // field is transformed once
      unsigned char* tmp = spec + (size_t)(3 * file + comp) * tsz;
      s = dns_transform_3d_one(c, DNS_BACKWARD, phys, pitch, tmp, tpitch, DNS_PADDING);
      if (s == DNS_OK) s = dns_synchronize(c);
      if (s != DNS_OK) return s;
      if (cudaMemcpy(host.data(), phys, psz, cudaMemcpyDeviceToHost))
        return dns_internal_fail(DNS_ERR_CUDA, "field output: copy");
      // pz planes x my rows x mx doubles, unpitched (source/output.cpp:67-103)
      for (int k = 0; k < g.Py; ++k)
        for (int j = 0; j < g.Pz; ++j) {
          const unsigned char* r = host.data() + pitch * ((size_t)g.Pz * k + j);
          if (fwrite(r, sizeof(double), (size_t)g.Px, f.f) != (size_t)g.Px)
            return dns_internal_fail(DNS_ERR_IO, "field output: write failed");
        }
    }
  }
  return DNS_OK;
}

}  // extern "C"
