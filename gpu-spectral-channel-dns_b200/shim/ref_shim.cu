// The reference's hot-path entry points defined over libdnsb200's C ABI.
// Compiled against the reference's own include/ directory, so each
// definition must match the reference's declaration exactly, and linked with
// -ldnsb200 in place of source/transform.cu, transpose.cu, velocity.cu,
// nonlinear.cu, rhs.cpp, linear.cpp, solver.cpp and matrix_op.cpp.  Not
// part of libdnsb200 (it needs the reference's headers); tests compile it.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "data.h"
#include "nonlinear.cuh"
#include "output.h"
#include "RPCFKernels.cuh"
#include "rhs.cuh"
#include "solver.h"
#include "transform.cuh"
#include "transpose.cuh"
#include "velocity.h"

#include "dns_b200.h"

static dns_ctx* g_ctx = nullptr;

static void check(dns_status s) {
  if (s != DNS_OK) {
    std::fprintf(stderr, "dns_b200: %s\n", dns_last_error());
    std::exit((int)s);
  }
}

static int dir_of(DIRECTION d) { return d == FORWARD ? DNS_FORWARD : DNS_BACKWARD; }
static int pad_of(Padding_mode p) { return p == Padding ? DNS_PADDING : DNS_NO_PADDING; }

// source/transform.cu:18: one library context holds the plans, tables and
// state of the problem
__host__ int initFFT(problem& pb) {
  dns_params p;
  check(dns_params_default(&p));
  p.mx = pb.mx;
  p.my = pb.my;
  p.mz = pb.mz;
  p.n_pi_x = pb.para.numPara.n_pi_x;
  p.n_pi_y = pb.para.numPara.n_pi_y;
  p.Re = pb.Re;
  p.Ro = pb.Ro;
  p.dt = pb.dt;
  check(dns_create(&p, &g_ctx));
  return 0;
}

// source/transform.cu:95
__host__ int transform_3d_one(DIRECTION dir, cudaPitchedPtr& Ptr, cudaPitchedPtr& tPtr, int* dim,
                              int* tDim, Padding_mode pd, bool isOutput) {
  check(dns_transform_3d_one(g_ctx, dir_of(dir), Ptr.ptr, Ptr.pitch, tPtr.ptr, tPtr.pitch, pad_of(pd)));
  check(dns_synchronize(g_ctx));
  return 0;
}

// source/transform.cu:321: six fields backward, three forward
__host__ int transform(DIRECTION dir, problem& pb) {
  if (dir == BACKWARD) {
    void* phys[6] = {pb.dptr_u.ptr, pb.dptr_v.ptr, pb.dptr_w.ptr,
                     pb.dptr_omega_x.ptr, pb.dptr_omega_y.ptr, pb.dptr_omega_z.ptr};
    void* spec[6] = {pb.dptr_tu.ptr, pb.dptr_tv.ptr, pb.dptr_tw.ptr,
                     pb.dptr_tomega_x.ptr, pb.dptr_tomega_y.ptr, pb.dptr_tomega_z.ptr};
    check(dns_transform(g_ctx, DNS_BACKWARD, 6, phys, pb.pitch, spec, pb.tPitch));
  } else {
    void* phys[3] = {pb.dptr_lamb_x.ptr, pb.dptr_lamb_y.ptr, pb.dptr_lamb_z.ptr};
    void* spec[3] = {pb.dptr_tLamb_x.ptr, pb.dptr_tLamb_y.ptr, pb.dptr_tLamb_z.ptr};
    check(dns_transform(g_ctx, DNS_FORWARD, 3, phys, pb.pitch, spec, pb.tPitch));
  }
  check(dns_synchronize(g_ctx));
  return 0;
}

// source/transpose.cu:115
__host__ int cuda_transpose(DIRECTION dir, cudaPitchedPtr& input, cudaPitchedPtr& tPtr, int* dim,
                            int* tDim) {
  check(dns_cuda_transpose(g_ctx, dir_of(dir), input.ptr, input.pitch, tPtr.ptr, tPtr.pitch));
  return 0;
}

// source/transform.cu:538-748
__host__ void cheby_s2p(cudaPitchedPtr tPtr, int mx, int my, int mz, Padding_mode padding) {
  check(dns_cheby_s2p(g_ctx, tPtr.ptr, tPtr.pitch, pad_of(padding)));
}
__host__ void cheby_p2s(cudaPitchedPtr tPtr, int mx, int my, int mz, Padding_mode padding) {
  check(dns_cheby_p2s(g_ctx, tPtr.ptr, tPtr.pitch, pad_of(padding)));
}

// source/velocity.cu:22
int getUVW(problem& pb) {
  void* f[6] = {pb.dptr_tu.ptr, pb.dptr_tv.ptr, pb.dptr_tw.ptr,
                pb.dptr_tomega_x.ptr, pb.dptr_tomega_y.ptr, pb.dptr_tomega_z.ptr};
  check(dns_get_uvw(g_ctx, f, pb.tPitch));
  return 0;
}

// source/nonlinear.cu:307: lambda over u, v, w storage, as the reference does
__host__ int computeLambVector(problem& pb) {
  void* in[6] = {pb.dptr_u.ptr, pb.dptr_v.ptr, pb.dptr_w.ptr,
                 pb.dptr_omega_x.ptr, pb.dptr_omega_y.ptr, pb.dptr_omega_z.ptr};
  pb.dptr_lamb_x = pb.dptr_u;
  pb.dptr_lamb_y = pb.dptr_v;
  pb.dptr_lamb_z = pb.dptr_w;
  void* out[3] = {pb.dptr_lamb_x.ptr, pb.dptr_lamb_y.ptr, pb.dptr_lamb_z.ptr};
  check(dns_compute_lamb(g_ctx, in, out, pb.pitch));
  return 0;
}

// source/nonlinear.cu:130
__host__ int rhsNonlinear(problem& pb) {
  check(dns_rhs_nonlinear(g_ctx, pb.dptr_tLamb_x.ptr, pb.dptr_tLamb_y.ptr, pb.dptr_tLamb_z.ptr,
                          pb.tPitch));
  return 0;
}

// source/solver.cpp:107 (inv and rhs on the device)
int solveEq(cuRPCF::complex* inv_coef, cuRPCF::complex* rhs, int N, size_t pitch, int nx, int ny) {
  check(dns_solve_eq(g_ctx, inv_coef, rhs, N, pitch));
  return 0;
}

// source/solver.cpp:260: inverses for callers that still use solveEq
int initAuxMatrix(problem& pb, bool inversed) {
  check(dns_init_aux_matrix(g_ctx, pb.matrix_coeff_v, pb.matrix_coeff_omega, DNS_HOST));
  return 0;
}

// source/solver.cpp:35: the whole step on the device; the host state is
// mirrored for callers that read it
int nextStep(problem& pb) {
  check(dns_step(g_ctx, 1));
  check(dns_get_state(g_ctx, pb.rhs_v, pb.rhs_omega_y, pb.tPitch, DNS_HOST));
  return 0;  // the caller's loop advances pb.currenStep, as in the reference
}

// source/RPCFKernels.cu:358
__host__ int initFlow(problem& pb) {
  check(dns_init_flow(g_ctx));  // state only; dns_bootstrap replaces the extra previous step
  check(dns_get_state(g_ctx, pb.rhs_v, pb.rhs_omega_y, pb.tPitch, DNS_HOST));
  return 0;
}

// source/output.cpp:19
void output_velocity(problem& pb) {
  const std::string s = std::to_string(pb.currenStep);
  const std::string pre = pb.para.ioPara.output_file_prefix;
  check(dns_write_fields(g_ctx, (pre + "_velocity." + s + ".dat").c_str(),
                         (pre + "_vortricity." + s + ".dat").c_str()));
}

// source/output.cpp:105-178: state and the full AB2 history
void write_recover_data(problem& pb, char* filename) { check(dns_write_recovery(g_ctx, filename)); }
void read_recover_data(problem& pb, char* filename) {
  check(dns_read_recovery(g_ctx, filename));
  check(dns_get_state(g_ctx, pb.rhs_v, pb.rhs_omega_y, pb.tPitch, DNS_HOST));
}

// source/rhs.cpp:15-54: one stream, no worker thread
void launch_subthread(problem& pb) {}
void synchronizeGPUsolver() { check(dns_synchronize(g_ctx)); }
