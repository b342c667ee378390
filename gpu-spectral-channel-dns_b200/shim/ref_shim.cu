// The reference's hot-path entry points, and the set-up calls of its driver,
// defined over libdnsb200's C ABI.
//
// Compiled against the reference's own include/ directory, so each definition
// matches the reference's declaration exactly.  Linked with the reference's
// unchanged source/main_loop.cpp (run_simulation), operation.cpp (parameter
// reader, cuCheck, device arena), data.cpp and transform_multi_gpu.cpp, and
// with -ldnsb200, in place of transform.cu, transpose.cu, velocity.cu,
// nonlinear.cu, rhs.cpp, linear.cpp, solver.cpp, matrix_op.cpp,
// coefficient.cu, RPCFKernels.cu and output.cpp.  Not part of libdnsb200 (it
// needs the reference's headers); shim/build_ref_main.py builds the two
// executables below from it.
//
// nextStep comes in two forms:
//   default: the fused step (dns_step, one CUDA graph; the state and AB2
//     history stay on the device).  After each step the host state
//     (rhs_v, rhs_omega_y, tv0, tomega_y_0) and the device spectral fields
//     (dptr_tu .. dptr_tomega_z, getUVW of the state) are mirrored, as the
//     reference leaves them.  The first nextStep of a fresh run stands for
//     the reference's "extra previous step" (source/main_loop.cpp:39-52): it
//     stores the nonlinear term of the initial state as the AB2 history
//     (dns_bootstrap) before stepping, so the reference's unchanged sequence
//     initFlow, nextStep, initFlow, nextStep... runs as it does there.
//   -DDNS_SHIM_FUNCTION_BY_FUNCTION: the reference's own sequence
//     (source/solver.cpp:35-101): get_rhs_v (the worker's getNonlinear and
//     no-pad s2p, the history swaps, the linear v right-hand side and AB2),
//     solveEq with the explicit inverses on the host buffers, get_rhs_omega,
//     solveEq, save_0_v_omega_y, getUVW -- each piece on the GPU through the
//     per-function drop-ins, every buffer where the reference keeps it.
//
// The device arena of the reference (operation.cpp) still owns the problem's
// spectral and physical fields; these definitions keep its last-in, first-
// out discipline.  Errors exit the process, as cuCheck does.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "cuRPCF.h"
#include "data.h"
#include "nonlinear.cuh"
#include "operation.h"
#include "output.h"
#include "RPCFKernels.cuh"
#include "rhs.cuh"
#include "solver.h"
#include "transform.cuh"
#include "transpose.cuh"
#include "velocity.h"

#include "dns_b200.h"

#ifdef DNS_SHIM_FUNCTION_BY_FUNCTION
static const bool kFunctionByFunction = true;
#else
static const bool kFunctionByFunction = false;
#endif

static dns_ctx* g_ctx = nullptr;
static bool g_booted = false;        // the fused step has its AB2 history
static void* g_phys = nullptr;       // getNonlinear's six physical work fields

static void check(dns_status s, const char* what) {
  if (s != DNS_OK) {
    std::fprintf(stderr, "dns_b200: %s: %s\n", what, dns_last_error());
    std::exit((int)s);
  }
}

static int dir_of(DIRECTION d) { return d == FORWARD ? DNS_FORWARD : DNS_BACKWARD; }
static int pad_of(Padding_mode p) { return p == Padding ? DNS_PADDING : DNS_NO_PADDING; }

static cudaPitchedPtr* spectral_fields(problem& pb, int i) {
  cudaPitchedPtr* f[6] = {&pb.dptr_tu, &pb.dptr_tv, &pb.dptr_tw,
                          &pb.dptr_tomega_x, &pb.dptr_tomega_y, &pb.dptr_tomega_z};
  return f[i];
}
static cudaPitchedPtr* physical_fields(problem& pb, int i) {
  cudaPitchedPtr* f[6] = {&pb.dptr_u, &pb.dptr_v, &pb.dptr_w,
                          &pb.dptr_omega_x, &pb.dptr_omega_y, &pb.dptr_omega_z};
  return f[i];
}

// Release arena fields in the order the arena requires (the last one handed
// out first): ZXY fields grow down from the top of the arena, XYZ fields up
// from the bottom.
static void arena_free(std::vector<cudaPitchedPtr*> f, myCudaMemType type) {
  f.erase(std::remove_if(f.begin(), f.end(), [](cudaPitchedPtr* p) { return p->ptr == nullptr; }),
          f.end());
  std::sort(f.begin(), f.end(), [&](cudaPitchedPtr* a, cudaPitchedPtr* b) {
    return type == ZXY_3D ? a->ptr < b->ptr : a->ptr > b->ptr;
  });
  for (cudaPitchedPtr* p : f) cuCheck(myCudaFree(*p, type), "arena free");
}

// the six spectral fields allocated (and the physical ones released), the
// arena state the reference is in after initFlow, getUVW and nextStep
static void ensure_spectral_fields(problem& pb) {
  std::vector<cudaPitchedPtr*> phys;
  for (int i = 0; i < 6; ++i) phys.push_back(physical_fields(pb, i));
  arena_free(phys, XYZ_3D);
  for (int i = 5; i >= 0; --i)
    if (spectral_fields(pb, i)->ptr == nullptr)
      cuCheck(myCudaMalloc(*spectral_fields(pb, i), ZXY_3D), "arena allocation");
}

// device spectral fields from the context's state: w, omega_z <- (v, omega_y),
// then getUVW for the other four
static void mirror_device_fields(problem& pb) {
  cuCheck(cudaMemset(pb.dptr_tw.ptr, 0, pb.tSize), "memset");
  cuCheck(cudaMemset(pb.dptr_tomega_z.ptr, 0, pb.tSize), "memset");
  check(dns_get_state(g_ctx, pb.dptr_tw.ptr, pb.dptr_tomega_z.ptr, pb.tPitch, DNS_DEVICE), "state");
  getUVW(pb);
}

// host state rhs_v / rhs_omega_y from the context, with tv0 / tomega_y_0
static void mirror_host_state(problem& pb) {
  check(dns_get_state(g_ctx, pb.rhs_v, pb.rhs_omega_y, pb.tPitch, DNS_HOST), "state");
  save_0_v_omega_y(pb);
}

// ---- set-up (source/RPCFKernels.cu:17-128, source/transform.cu:18-93,
// ---- source/solver.cpp:216-320) -------------------------------------------

// source/RPCFKernels.cu:17: device report; no worker thread is started
__host__ void getDeviceInfo(problem& pb) {
  int dev = 0, n = 0;
  cudaDeviceProp prop;
  size_t free_b = 0, total_b = 0;
  cuCheck(cudaGetDevice(&dev), "device");
  cuCheck(cudaGetDeviceProperties(&prop, dev), "device properties");
  cuCheck(cudaMemGetInfo(&free_b, &total_b), "memory info");
  cuCheck(cudaGetDeviceCount(&n), "device count");
  std::printf("Using CUDA device %d: %s (PCI bus %d), %.0f MB of %.0f MB free, %d device(s)\n", dev,
              prop.name, prop.pciBusID, free_b / 1.024e6, total_b / 1.024e6, n);
  launch_subthread(pb);
}

// source/RPCFKernels.cu:47: the reference's extents, pitches, sizes and
// arena, with the six physical fields taken from it and every spectral
// field unset -- the problem layout the reference's callers rely on
__host__ int allocDeviceMem(problem& pb) {
  pb.extent = make_cudaExtent(2 * (pb.mx / 2 + 1) * sizeof(REAL), pb.my, pb.mz);
  pb.tExtent = make_cudaExtent(pb.mz * sizeof(cuRPCF::complex), pb.nx / 2 + 1, pb.ny);
  pb.pExtent = make_cudaExtent(2 * (pb.mx / 2 + 1) * sizeof(REAL), pb.my, pb.pz);
  cudaPitchedPtr probe;
  cuCheck(cudaMalloc3D(&probe, pb.tExtent), "pitch query");
  pb.tPitch = probe.pitch;
  cuCheck(cudaFree(probe.ptr), "pitch query");
  initMyCudaMalloc(dim3(pb.mx, pb.my, pb.mz));
  for (int i = 0; i < 6; ++i) cuCheck(myCudaMalloc(*physical_fields(pb, i), XYZ_3D), "allocate");
  for (int i = 0; i < 6; ++i) spectral_fields(pb, i)->ptr = nullptr;
  cudaPitchedPtr* rest[6] = {&pb.dptr_lamb_x, &pb.dptr_lamb_y, &pb.dptr_lamb_z,
                             &pb.dptr_tLamb_x, &pb.dptr_tLamb_y, &pb.dptr_tLamb_z};
  for (cudaPitchedPtr* p : rest) p->ptr = nullptr;
  pb.pitch = pb.dptr_u.pitch;
  pb.size = pb.pitch * pb.my * pb.mz;
  pb.pSize = pb.pitch * pb.my * pb.pz;
  pb.tSize = pb.tPitch * (pb.nx / 2 + 1) * pb.ny;
  return 0;
}

// source/transform.cu:18: one library context holds the tables and state
__host__ int initFFT(problem& pb) {
  dns_params p;
  check(dns_params_default(&p), "parameters");
  p.mx = pb.mx;
  p.my = pb.my;
  p.mz = pb.mz;
  p.n_pi_x = pb.para.numPara.n_pi_x;
  p.n_pi_y = pb.para.numPara.n_pi_y;
  p.Re = pb.Re;
  p.Ro = pb.Ro;
  p.dt = pb.dt;
  cuCheck(cudaGetDevice(&p.device), "device");
  if (g_ctx) check(dns_destroy(g_ctx), "destroy");
  check(dns_create(&p, &g_ctx), "create");
  g_booted = false;
  return 0;
}

// source/solver.cpp:216: the reference's host buffers (pinned where it pins
// them), zero-filled
int allocHostMemory(problem& pb) {
  const size_t tSize = pb.tSize, nz = (size_t)pb.nz;
  const size_t mSize = nz * nz * (pb.nx / 2 + 1) * pb.ny * sizeof(cuRPCF::complex);
  auto host = [](size_t n) {
    void* p = std::calloc(1, n);
    if (!p) { std::fprintf(stderr, "dns_b200: host allocation of %zu bytes failed\n", n); std::exit(2); }
    return p;
  };
  auto pinned = [](size_t n) {
    void* p = nullptr;
    cuCheck(cudaMallocHost(&p, n), "pinned allocation");
    std::memset(p, 0, n);
    return p;
  };
  pb.matrix_coeff_v = (cuRPCF::complex*)host(mSize);
  pb.matrix_coeff_omega = (cuRPCF::complex*)host(mSize);
  cuRPCF::complex** pin_t[7] = {&pb.nonlinear_v, &pb.nonlinear_v_p, &pb.nonlinear_omega_y,
                                &pb.nonlinear_omega_y_p, &pb.rhs_v, &pb.rhs_v_p, &pb.rhs_omega_y};
  for (auto q : pin_t) *q = (cuRPCF::complex*)pinned(tSize);
  cuRPCF::complex** pin_z[4] = {&pb.lambx0, &pb.lambx0_p, &pb.lambz0, &pb.lambz0_p};
  for (auto q : pin_z) *q = (cuRPCF::complex*)pinned(nz * sizeof(cuRPCF::complex));
  pb.tv0 = (cuRPCF::complex*)host(nz * sizeof(cuRPCF::complex));
  pb.tomega_y_0 = (cuRPCF::complex*)host(nz * sizeof(cuRPCF::complex));
  pb._U0 = (REAL*)host(nz * sizeof(REAL));
  pb._dU0 = (REAL*)host(nz * sizeof(REAL));
  pb._ddU0 = (REAL*)host(nz * sizeof(REAL));
  pb.T0 = (REAL*)host(nz * nz * sizeof(REAL));
  pb.T2 = (REAL*)host(nz * nz * sizeof(REAL));
  pb.T4 = (REAL*)host(nz * nz * sizeof(REAL));
  return 0;
}

// source/solver.cpp:260: the T tables, U profile and the operators (their
// explicit inverses by default) in the reference's host buffers
int initAuxMatrix(problem& pb, bool inversed) {
  check(dns_operator_tables(g_ctx, pb.T0, pb.T2, pb.T4, pb._U0, pb._dU0, pb._ddU0), "tables");
  if (inversed)
    check(dns_init_aux_matrix(g_ctx, pb.matrix_coeff_v, pb.matrix_coeff_omega, DNS_HOST), "inverses");
  else
    check(dns_operator_matrices(g_ctx, pb.matrix_coeff_v, pb.matrix_coeff_omega, DNS_HOST), "operators");
  pb.currenStep = pb.para.stepPara.start_step;
  return 0;
}

// ---- transforms (source/transform.cu, source/transpose.cu) ----------------

// source/transform.cu:95
__host__ int transform_3d_one(DIRECTION dir, cudaPitchedPtr& Ptr, cudaPitchedPtr& tPtr, int* dim,
                              int* tDim, Padding_mode pd, bool isOutput) {
  check(dns_transform_3d_one(g_ctx, dir_of(dir), Ptr.ptr, Ptr.pitch, tPtr.ptr, tPtr.pitch, pad_of(pd)),
        "transform_3d_one");
  check(dns_synchronize(g_ctx), "transform_3d_one");
  return 0;
}

// source/transform.cu:321: six fields backward, three forward
__host__ int transform(DIRECTION dir, problem& pb) {
  if (dir == BACKWARD) {
    void* phys[6];
    void* spec[6];
    for (int i = 0; i < 6; ++i) {
      phys[i] = physical_fields(pb, i)->ptr;
      spec[i] = spectral_fields(pb, i)->ptr;
    }
    check(dns_transform(g_ctx, DNS_BACKWARD, 6, phys, pb.pitch, spec, pb.tPitch), "transform");
  } else {
    void* phys[3] = {pb.dptr_lamb_x.ptr, pb.dptr_lamb_y.ptr, pb.dptr_lamb_z.ptr};
    void* spec[3] = {pb.dptr_tLamb_x.ptr, pb.dptr_tLamb_y.ptr, pb.dptr_tLamb_z.ptr};
    check(dns_transform(g_ctx, DNS_FORWARD, 3, phys, pb.pitch, spec, pb.tPitch), "transform");
  }
  check(dns_synchronize(g_ctx), "transform");
  return 0;
}

// source/transpose.cu:115
__host__ int cuda_transpose(DIRECTION dir, cudaPitchedPtr& input, cudaPitchedPtr& tPtr, int* dim,
                            int* tDim) {
  check(dns_cuda_transpose(g_ctx, dir_of(dir), input.ptr, input.pitch, tPtr.ptr, tPtr.pitch),
        "cuda_transpose");
  check(dns_synchronize(g_ctx), "cuda_transpose");
  return 0;
}

// source/transform.cu:538-748
__host__ void cheby_s2p(cudaPitchedPtr tPtr, int mx, int my, int mz, Padding_mode padding) {
  check(dns_cheby_s2p(g_ctx, tPtr.ptr, tPtr.pitch, pad_of(padding)), "cheby_s2p");
  check(dns_synchronize(g_ctx), "cheby_s2p");
}
__host__ void cheby_p2s(cudaPitchedPtr tPtr, int mx, int my, int mz, Padding_mode padding) {
  check(dns_cheby_p2s(g_ctx, tPtr.ptr, tPtr.pitch, pad_of(padding)), "cheby_p2s");
  check(dns_synchronize(g_ctx), "cheby_p2s");
}

// ---- velocity and nonlinear terms (source/velocity.cu, nonlinear.cu) -------

// source/velocity.cu:22
int getUVW(problem& pb) {
  void* f[6];
  for (int i = 0; i < 6; ++i) f[i] = spectral_fields(pb, i)->ptr;
  check(dns_get_uvw(g_ctx, f, pb.tPitch), "getUVW");
  check(dns_synchronize(g_ctx), "getUVW");
  return 0;
}

// source/nonlinear.cu:307: lambda over the u, v, w storage, as the reference
// aliases it
__host__ int computeLambVector(problem& pb) {
  void* in[6];
  for (int i = 0; i < 6; ++i) in[i] = physical_fields(pb, i)->ptr;
  pb.dptr_lamb_x = pb.dptr_u;
  pb.dptr_lamb_y = pb.dptr_v;
  pb.dptr_lamb_z = pb.dptr_w;
  void* out[3] = {pb.dptr_lamb_x.ptr, pb.dptr_lamb_y.ptr, pb.dptr_lamb_z.ptr};
  check(dns_compute_lamb(g_ctx, in, out, pb.pitch), "computeLambVector");
  check(dns_synchronize(g_ctx), "computeLambVector");
  return 0;
}

// source/nonlinear.cu:130
__host__ int rhsNonlinear(problem& pb) {
  check(dns_rhs_nonlinear(g_ctx, pb.dptr_tLamb_x.ptr, pb.dptr_tLamb_y.ptr, pb.dptr_tLamb_z.ptr,
                          pb.tPitch),
        "rhsNonlinear");
  check(dns_synchronize(g_ctx), "rhsNonlinear");
  return 0;
}

// source/nonlinear.cu:25: from the six spectral fields (getUVW of the state)
// to the nonlinear terms H_v, H_omega (coefficients) in dptr_tLamb_x /
// dptr_tLamb_y, lambda_z in dptr_tLamb_z.  As in the reference the spectral
// fields are consumed and released and the three lambda fields taken from
// the arena; the physical fields are the shim's own work buffers.
__host__ int getNonlinear(problem& pb) {
  if (!g_phys) cuCheck(cudaMalloc(&g_phys, 6 * pb.pSize), "nonlinear work fields");
  void* phys[6];
  void* spec[6];
  for (int i = 0; i < 6; ++i) {
    phys[i] = (char*)g_phys + i * pb.pSize;
    spec[i] = spectral_fields(pb, i)->ptr;
  }
  check(dns_transform(g_ctx, DNS_BACKWARD, 6, phys, pb.pitch, spec, pb.tPitch), "transform");
  check(dns_compute_lamb(g_ctx, phys, phys, pb.pitch), "computeLambVector");
  std::vector<cudaPitchedPtr*> spectral;
  for (int i = 0; i < 6; ++i) spectral.push_back(spectral_fields(pb, i));
  check(dns_synchronize(g_ctx), "getNonlinear");
  arena_free(spectral, ZXY_3D);
  cuCheck(myCudaMalloc(pb.dptr_tLamb_z, ZXY_3D), "allocate");
  cuCheck(myCudaMalloc(pb.dptr_tLamb_y, ZXY_3D), "allocate");
  cuCheck(myCudaMalloc(pb.dptr_tLamb_x, ZXY_3D), "allocate");
  void* lam[3] = {pb.dptr_tLamb_x.ptr, pb.dptr_tLamb_y.ptr, pb.dptr_tLamb_z.ptr};
  check(dns_transform(g_ctx, DNS_FORWARD, 3, phys, pb.pitch, lam, pb.tPitch), "transform");
  return rhsNonlinear(pb);
}

// ---- right-hand sides and solves (source/rhs.cpp, linear.cpp, solver.cpp) --

// source/rhs.cpp:15-54: one stream, no worker thread
void launch_subthread(problem& pb) {}
void synchronizeGPUsolver() { check(dns_synchronize(g_ctx), "synchronize"); }

// source/rhs.cpp:185: the worker's half first (source/rhs.cpp:60-183:
// getNonlinear, no-pad s2p of H_v and H_omega, history swap, copy to the
// host, mean-mode lambda), then get_linear_v with AB2 and the mean modes
__host__ int get_rhs_v(problem& pb) {
  getNonlinear(pb);
  cheby_s2p(pb.dptr_tLamb_x, pb.mx / 2 + 1, pb.my, pb.mz, No_Padding);
  cheby_s2p(pb.dptr_tLamb_y, pb.mx / 2 + 1, pb.my, pb.mz, No_Padding);
  std::swap(pb.nonlinear_omega_y, pb.nonlinear_omega_y_p);
  std::swap(pb.nonlinear_v, pb.nonlinear_v_p);
  cuCheck(cudaMemcpy(pb.nonlinear_v, pb.dptr_tLamb_x.ptr, pb.tSize, cudaMemcpyDeviceToHost), "memcpy");
  cuCheck(cudaMemcpy(pb.nonlinear_omega_y, pb.dptr_tLamb_y.ptr, pb.tSize, cudaMemcpyDeviceToHost),
          "memcpy");
  std::swap(pb.lambx0, pb.lambx0_p);
  std::swap(pb.lambz0, pb.lambz0_p);
  std::memcpy(pb.lambx0, pb.nonlinear_v, pb.nz * sizeof(cuRPCF::complex));
  std::memcpy(pb.lambz0, pb.nonlinear_omega_y, pb.nz * sizeof(cuRPCF::complex));
  arena_free({&pb.dptr_tLamb_x, &pb.dptr_tLamb_y, &pb.dptr_tLamb_z}, ZXY_3D);
  ensure_spectral_fields(pb);
  check(dns_rhs_v(g_ctx, pb.rhs_v, pb.rhs_v_p, pb.nonlinear_v, pb.nonlinear_v_p, pb.tPitch, DNS_HOST),
        "get_rhs_v");
  check(dns_rhs_mean(g_ctx, pb.tv0, pb.lambx0, pb.lambx0_p, pb.tomega_y_0, pb.lambz0, pb.lambz0_p,
                     DNS_HOST),
        "mean modes");
  std::memcpy(pb.rhs_v, pb.tv0, pb.nz * sizeof(cuRPCF::complex));
  std::memcpy(pb.rhs_omega_y, pb.tomega_y_0, pb.nz * sizeof(cuRPCF::complex));
  return 0;
}

// source/rhs.cpp:221: rhs_v holds v^{n+1} (solved), rhs_v_p v^n
__host__ int get_rhs_omega(problem& pb) {
  check(dns_rhs_omega(g_ctx, pb.rhs_omega_y, pb.nonlinear_omega_y, pb.nonlinear_omega_y_p, pb.rhs_v,
                      pb.rhs_v_p, pb.tPitch, DNS_HOST),
        "get_rhs_omega");
  return 0;
}

// source/solver.cpp:107: the inverses and right-hand sides where the caller
// keeps them (the reference: host memory)
int solveEq(cuRPCF::complex* inv_coef, cuRPCF::complex* rhs, int N, size_t pitch, int nx, int ny) {
  cudaPointerAttributes a{}, b{};
  const bool dev = cudaPointerGetAttributes(&a, inv_coef) == cudaSuccess &&
                   cudaPointerGetAttributes(&b, rhs) == cudaSuccess &&
                   a.type == cudaMemoryTypeDevice && b.type == cudaMemoryTypeDevice;
  cudaGetLastError();
  check(dns_solve_eq(g_ctx, inv_coef, rhs, N, pitch, dev ? DNS_DEVICE : DNS_HOST), "solveEq");
  if (dev) check(dns_synchronize(g_ctx), "solveEq");
  return 0;
}

// source/solver.cpp:332: u0 / w0 of the solved state
void save_0_v_omega_y(problem& pb) {
  std::memcpy(pb.tv0, pb.rhs_v, pb.nz * sizeof(cuRPCF::complex));
  std::memcpy(pb.tomega_y_0, pb.rhs_omega_y, pb.nz * sizeof(cuRPCF::complex));
}

// source/solver.cpp:35
int nextStep(problem& pb) {
  if (kFunctionByFunction) {
    get_rhs_v(pb);
    solveEq(pb.matrix_coeff_v, pb.rhs_v, pb.nz, pb.tPitch, pb.mx, pb.my);
    get_rhs_omega(pb);
    solveEq(pb.matrix_coeff_omega, pb.rhs_omega_y, pb.nz, pb.tPitch, pb.mx, pb.my);
    save_0_v_omega_y(pb);
    synchronizeGPUsolver();
    cuCheck(cudaMemcpy(pb.dptr_tw.ptr, pb.rhs_v, pb.tSize, cudaMemcpyHostToDevice), "memcpy");
    cuCheck(cudaMemcpy(pb.dptr_tomega_z.ptr, pb.rhs_omega_y, pb.tSize, cudaMemcpyHostToDevice), "memcpy");
    getUVW(pb);
    // the context follows the run, for the field and recovery output
    check(dns_set_state(g_ctx, pb.rhs_v, pb.rhs_omega_y, pb.tPitch, DNS_HOST), "state");
    check(dns_set_history(g_ctx, pb.nonlinear_v, pb.nonlinear_omega_y, pb.tPitch, DNS_HOST), "history");
    return 0;
  }
  if (!g_booted) {
    check(dns_bootstrap(g_ctx), "extra previous step");
    g_booted = true;
  }
  check(dns_step(g_ctx, 1), "nextStep");
  mirror_host_state(pb);
  ensure_spectral_fields(pb);
  mirror_device_fields(pb);
  return 0;  // the caller's loop advances pb.currenStep, as in the reference
}

// source/RPCFKernels.cu:358: the analytic start, then the reference's
// bookkeeping (tv0, tomega_y_0, rhs_v_p) and getUVW on the device fields.
// The AB2 history is kept, so the reference's second initFlow after the
// extra previous step leaves the bootstrap in place.
__host__ int initFlow(problem& pb) {
  check(dns_init_flow(g_ctx), "initFlow");
  mirror_host_state(pb);
  std::memcpy(pb.rhs_v_p, pb.rhs_v, pb.tSize);
  ensure_spectral_fields(pb);
  mirror_device_fields(pb);
  return 0;
}

// ---- output (source/output.cpp) --------------------------------------------

// source/output.cpp:19
void output_velocity(problem& pb) {
  const std::string s = std::to_string(pb.currenStep);
  const std::string pre = pb.para.ioPara.output_file_prefix;
  check(dns_write_fields(g_ctx, (pre + "_velocity." + s + ".dat").c_str(),
                         (pre + "_vortricity." + s + ".dat").c_str()),
        "output_velocity");
}

// source/output.cpp:105-178: state and the full AB2 history
void write_recover_data(problem& pb, char* filename) {
  check(dns_write_recovery(g_ctx, filename), "write_recover_data");
}
void read_recover_data(problem& pb, char* filename) {
  check(dns_read_recovery(g_ctx, filename), "read_recover_data");
  g_booted = true;
  mirror_host_state(pb);
  std::memcpy(pb.rhs_v_p, pb.rhs_v, pb.tSize);
  check(dns_get_history(g_ctx, pb.nonlinear_v, pb.nonlinear_omega_y, pb.tPitch, DNS_HOST), "history");
  std::memcpy(pb.lambx0, pb.nonlinear_v, pb.nz * sizeof(cuRPCF::complex));
  std::memcpy(pb.lambz0, pb.nonlinear_omega_y, pb.nz * sizeof(cuRPCF::complex));
  ensure_spectral_fields(pb);
  mirror_device_fields(pb);
}
