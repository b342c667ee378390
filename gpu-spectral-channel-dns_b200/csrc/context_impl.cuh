// Internal layout of dns_ctx, shared by the translation units that implement
// the C ABI (context.cu, noalloc.cu).  Not part of the public interface.
#pragma once
#include <string>
#include <vector>

#include "../../include/dns_b200.h"
#include "kernels.cuh"
#include "wallsolve_dev.cuh"

template <typename C> struct DevFft {
  FftPlan plan;
  C* tw = nullptr;
  short* drev = nullptr;
  C* wt[3] = {nullptr, nullptr, nullptr};
  FftTab<C> tab() const {
    FftTab<C> t;
    t.plan = plan;
    t.tw = tw;
    t.drev = drev;
    for (int i = 0; i < 3; ++i) t.wt[i] = wt[i];
    return t;
  }
};

// One rank of a slab-decomposed step (dns_slab_create): the runs of its
// pencils (in local row order), its planes and the segments of the two
// exchanges in both roles, with the bytes per peer.
struct SlabRun {
  int kz0, nkz;
  long long row0;  // first local pencil row of the run
};
struct SlabState {
  int R = 1, r = 0;
  int s0 = 0, s1 = 0;          // operator slots kz' in [s0, s1)
  int y0 = 0, ny = 0, nyS = 0;  // planes [y0, y0 + ny), their pencil pitch nyS
  long long np = 0;            // pencils owned
  int nruns = 0;
  SlabRun run[2];
  std::vector<dns_slab_segment> segP, segY;  // as pencil owner / as plane owner
  std::vector<size_t> sendB[2], recvB[2];     // bytes per peer: [0] backward (6 fields), [1] forward (3)
  void* A = nullptr;                          // plane-local pencils (6 fields), then rows (3 fields)
};

struct dns_ctx {
  dns_params P;
  DnsGeom g;
  PhysParams ph;
  cudaStream_t st = nullptr;
  size_t bytes = 0;
  long long PyS = 0, KxS = 0, RS = 0;
  // tables
  DevFft<double2> fz_d, fx_d, fyP_d, fy0_d;
  DevFft<float2> fz_f, fx_f, fyP_f;
  double *T0 = nullptr, *T2 = nullptr, *T4 = nullptr;
  double *Ut = nullptr, *dUt = nullptr, *ddUt = nullptr, *Uy = nullptr;
  // state
  double2 *V = nullptr, *O = nullptr, *Nvp = nullptr, *Nop = nullptr, *rv = nullptr, *ro = nullptr;
  // banded wall-normal solve: packed factors, tilting table, dimensions
  double2* wfac = nullptr;
  double* wQ = nullptr;
  WallDims wd{};
  double* rtab = nullptr;  // y1 tables: B^4 C_m (4 x nv), B^2 C_m (2 x no), cos(k pi/N)
  void* F6 = nullptr;  // also the wall solve's scratch (free while it runs)
  void* G6 = nullptr;
  size_t F6_bytes = 0;
  double2* scratch = nullptr;
  double2* solve_io = nullptr;  // solve-only entry: both systems' vectors + wall polynomials
  double2* rhs_io = nullptr;    // right-hand-side drop-ins: host staging (6 H Ny)
  double2* nl_io = nullptr;     // dns_nonlinear: state in, nonlinear terms out (4 H Ny)
  unsigned char* eq_io = nullptr;  // dns_solve_eq on host buffers: inverse and rhs staging
  size_t eq_io_bytes = 0;
  int* probe = nullptr;         // dns_check_state: set when the state holds NaN or Inf
  int* status = nullptr;
  bool have_state = false, booted = false, wall_ready = false;
  int variant[DNS_NUM_PASSES] = {};  // kernel variant of each tunable pass
  uint32_t* y3tc_tab = nullptr;      // Chebyshev table of the tensor-core y3 pass
  cudaGraphExec_t graph = nullptr;
  cudaGraphExec_t solve_graph = nullptr;  // dns_solve_wall on device pencils
  const void* solve_key[2] = {nullptr, nullptr};
  size_t solve_pitch = 0;
  SlabState* slab = nullptr;  // set on the contexts of dns_slab_create
  std::vector<double> runs_h;  // a batch (g.nrun > 1): per-member (Re, Ro, dt)
  double* runs_d = nullptr;    // the same on the device (ph.runs)

  template <typename T> cudaError_t alloc(T** p, size_t n) {
    bytes += n * sizeof(T);
    return cudaMalloc((void**)p, n * sizeof(T));
  }
};


// record an error message for dns_last_error() and return the status
dns_status dns_internal_fail(dns_status s, const char* msg);

// context.cu internals used by the slab-decomposed step (slabstep.cu)
// nrun > 1: a batch of nrun runs of p's grid with per-member (Re, Ro, dt)
// in runs (3 each)
extern "C" dns_status ctx_create(const dns_params* p, SlabState* slab, dns_ctx** out, int nrun = 1,
                                 const double* runs = nullptr);
dns_status ctx_check_status(dns_ctx* c);
dns_status ctx_build_wall_solver(dns_ctx* c);
// slab.cpp: the runs of pencils of a rank (their count, or -1)
int slab_runs(int mx, int my, int mz, int nranks, int rank, int kz0[2], int nkz[2], long long row0[2]);
