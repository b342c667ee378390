// dns_ctx: device buffers, FFT tables, wall-normal solver factors and the C ABI of
// libdnsb200.so (include/dns_b200.h).
//
// One context = one problem on one device, one CUDA stream, no host threads.
// The reference splits a step over two host threads, the GPU and PCIe
// (source/solver.cpp:35-101, source/rhs.cpp:15-183); here the whole step is
// six kernels on one stream, captured once into a CUDA graph:
//
//   y3  state (v, omega_y) -> getUVW -> padded s2p -> six pencil fields
//   zb  spanwise inverse FFT with padding, transpose to streamwise rows
//   x   streamwise C2R -> Lamb vector + rotation -> R2C
//   zf  spanwise forward FFT with truncation, transpose back to pencils
//   y1  p2s -> rhsNonlinear -> collocation values -> CN/AB2 right-hand sides
//       -> integrated right-hand sides of the banded systems
//   y2  banded v solve, tilting term, banded omega solve (factors streamed)
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dns_b200.h"
#include "context_impl.cuh"
#include "wfft.cuh"
#include "kernels.cuh"
#include "setup.cuh"
#include "wallsolve.h"
#include "ypass.cuh"
#include "zxpass.cuh"

namespace {
thread_local std::string g_err;

dns_status fail(dns_status s, const std::string& m) {
  g_err = m;
  return s;
}

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) return fail(DNS_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename C> cudaError_t make_fft(int L, DevFft<C>& f) {
  if (!fft_make_plan(L, &f.plan)) return cudaErrorInvalidValue;
  std::vector<C> tw(L);
  std::vector<short> dr(L);
  const long double PI = 3.141592653589793238462643383279502884L;
  for (int j = 0; j < L; ++j) {
    const long double a = -2.0L * PI * (long double)j / (long double)L;
    tw[j] = cmk<C>((double)cosl(a), (double)sinl(a));
    dr[j] = (short)fft_digitrev(f.plan, j);
  }
  cudaError_t e = cudaMalloc(&f.tw, sizeof(C) * L);
  if (e) return e;
  e = cudaMalloc(&f.drev, sizeof(short) * L);
  if (e) return e;
  e = cudaMemcpy(f.tw, tw.data(), sizeof(C) * L, cudaMemcpyHostToDevice);
  if (e) return e;
  e = cudaMemcpy(f.drev, dr.data(), sizeof(short) * L, cudaMemcpyHostToDevice);
  if (e) return e;
  // FP32 warp-FFT tables (1, 2, 4 lines per warp) where the length has a plan
  if (std::is_same<C, float2>::value) {
    for (int i = 0; i < 3; ++i) {
      std::vector<C> t;
      const int n = i == 0 ? wtw_table_any<C, 1>(L, t) : (i == 1 ? wtw_table_any<C, 2>(L, t) : wtw_table_any<C, 4>(L, t));
      if (n <= 0) continue;
      if ((e = cudaMalloc(&f.wt[i], sizeof(C) * n))) return e;
      if ((e = cudaMemcpy(f.wt[i], t.data(), sizeof(C) * n, cudaMemcpyHostToDevice))) return e;
    }
  }
  return cudaSuccess;
}
template <typename C> void free_fft(DevFft<C>& f) {
  cudaFree(f.tw);
  cudaFree(f.drev);
  f.tw = nullptr;
  f.drev = nullptr;
  for (int i = 0; i < 3; ++i) {
    cudaFree(f.wt[i]);
    f.wt[i] = nullptr;
  }
}

bool fft_len_ok(int L) {
  FftPlan p;
  return L >= 2 && L <= 16384 && fft_make_plan(L, &p);
}

long long roundup(long long a, long long b) { return (a + b - 1) / b * b; }
}  // namespace

dns_status ctx_check_status(dns_ctx* c);
dns_status ctx_build_wall_solver(dns_ctx* c);
namespace {
dns_status check_status(dns_ctx* c) { return ctx_check_status(c); }
dns_status build_wall_solver(dns_ctx* c) { return ctx_build_wall_solver(c); }
}  // namespace

dns_status ctx_check_status(dns_ctx* c) {
  int s = 0;
  CK(cudaMemcpyAsync(&s, c->status, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (s) {
    // reported once: the flag is cleared, so that the context is usable again
    CK(cudaMemsetAsync(c->status, 0, sizeof(int), c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  if (s & 1) return fail(DNS_ERR_TIMEOUT, "a device wait ran past its iteration limit");
  if (s & 2) return fail(DNS_ERR_SINGULAR, "an operator matrix had a zero pivot");
  return DNS_OK;
}

// Factor the banded wall-normal systems of every operator slot (a slab
// rank: of its slots) on the host threads and upload them (once per
// context, before the first step).
dns_status ctx_build_wall_solver(dns_ctx* c) {
  if (c->wall_ready) return DNS_OK;
  const DnsGeom& g = c->g;
  const int N = g.Ny - 1;
  if (N < 8) return fail(DNS_ERR_ARG, "the time step needs Ny >= 9 (mz >= 32)");
  WallDims& wd = c->wd;
  int klv, kuv, klo, kuo;
  if (!wall_band_of(wd.delta, &klv, &kuv, &klo, &kuo)) return fail(DNS_ERR_ARG, "base flow degree");
  const wall::Shape sv{wd.nv, klv, kuv, 2}, so{wd.no, klo, kuo, 0};
  const wall::Packing pk = wall::make_packing(sv, so);
  wall::Grid gr{N, g.Kx, g.Nz, g.Kh, c->ph.aphi, c->ph.beta, c->ph.Re, c->ph.dt,
                c->ph.U0, c->ph.U1, c->ph.U2};
  const SlabState* sl = c->slab;
  if (sl) {
    gr.kz0 = sl->s0;
    gr.nkz = sl->s1 - sl->s0;
    // run 0 holds kz = kz' in [s0, s1) in slot order; run 1 the mirrored
    // pencils kz = Nz - kz'
    wd.kzs0 = sl->s0;
    wd.kza = sl->run[0].kz0;
    wd.rowa = sl->run[0].row0;
    wd.kzb = sl->nruns > 1 ? sl->run[1].kz0 : 0;
    wd.rowb = sl->nruns > 1 ? sl->run[1].row0 : 0;
  }
  std::vector<wall::cx> fac;
  unsigned nt = std::thread::hardware_concurrency();
  // a batch: each member's factors (its Re, dt), one after another
  for (int r = 0; r < g.nrun; ++r) {
    std::vector<wall::cx> f1;
    if (g.nrun > 1) {
      gr.Re = c->runs_h[3 * (size_t)r];
      gr.dt = c->runs_h[3 * (size_t)r + 2];
    }
    const std::string err = wall::pack_grid(gr, sv, so, g.nrun > 1 ? f1 : fac, (int)std::min(32u, std::max(1u, nt)));
    if (!err.empty()) return fail(DNS_ERR_SINGULAR, err);
    if (g.nrun > 1) fac.insert(fac.end(), f1.begin(), f1.end());
  }
  std::vector<double> Q((size_t)7 * wd.no);
  if (!wall::tilting_table(N, wd.no, c->ph.U1, c->ph.U2, Q.data()))
    return fail(DNS_ERR_ARG, "tilting table outside its band");
  wd.group_complex = pk.group_complex;
  wd.nslots = (long long)g.Kx * (sl ? sl->s1 - sl->s0 : g.Kh);
  wd.ngroups = (wd.nslots + 15) / 16;
  if (g.nrun > 1) {
    wd.groups_per_run = wd.ngroups;
    wd.ngroups *= g.nrun;
  }
  if (wall_smem_bytes(wd, DNS_Y2_RING2_8K_EF) > 227 * 1024) return fail(DNS_ERR_ARG, "Ny too large for the wall solve");
  if (wall_scratch_complex(wd) * 16 > c->F6_bytes)
    return fail(DNS_ERR_ARG, "wall solve scratch does not fit the transform buffer");
  CK(c->alloc(&c->wfac, fac.size()));
  CK(c->alloc(&c->wQ, Q.size()));
  CK(cudaMemcpy(c->wfac, fac.data(), fac.size() * 16, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->wQ, Q.data(), Q.size() * 8, cudaMemcpyHostToDevice));
  c->wall_ready = true;
  return DNS_OK;
}

namespace {
// the state and AB2 history a pass sequence reads and writes
struct StepBufs {
  double2 *V, *O, *Nvp, *Nop;
};

// Enqueue one step (boot = 0) or the history bootstrap (boot = 1).  With
// `ev` (7 events) an event is recorded before the first and after every
// kernel, for per-kernel timing on the launching stream.
template <typename C>
cudaError_t enqueue_pipeline(dns_ctx* c, int boot, const DevFft<C>& fz, const DevFft<C>& fx,
                             const DevFft<C>& fyP, cudaEvent_t* ev, StepBufs b) {
  const DnsGeom& g = c->g;  // one member's grid (g.nrun members in a batch)
  const long long H = g.H, NR = g.nrun, PR = (long long)g.Py * g.Pz * c->KxS;
  // a batch keeps every field field-major, then member-major: the
  // wall-normal passes see NR H pencils (gb), the spanwise passes 6 NR or
  // 3 NR fields, the streamwise pass NR Py Pz rows
  DnsGeom gb = g;
  gb.H = NR * H;
  PencilArr F6p{c->F6, c->PyS, NR * H * c->PyS};  // y3 out
  PencilArr F6z{c->F6, c->PyS, H * c->PyS};       // zb in
  RowArr G6r{c->G6, c->KxS, PR};                  // zb out
  RowArr G6x{c->G6, c->KxS, NR * PR};             // x in
  RowArr G3x{c->F6, c->KxS, NR * PR};             // x out
  RowArr G3r{c->F6, c->KxS, PR};                  // zf in
  PencilArr F3p{c->G6, c->PyS, H * c->PyS};       // zf out
  PencilArr F3y{c->G6, c->PyS, NR * H * c->PyS};  // y1 in
  cudaError_t e;
  int k = 0;
  auto mark = [&]() { if (ev) cudaEventRecord(ev[k++], c->st); };
  mark();
  // the context's variant of each tunable pass; a variant these buffers do
  // not allow (cudaErrorNotSupported, nothing launched) falls back to the
  // automatic choice
  auto var = [&](int pass, auto&& launch) {
    cudaError_t r = launch(c->variant[pass]);
    return r == cudaErrorNotSupported ? launch(VAR_AUTO) : r;
  };
  if (std::is_same<C, float2>::value && c->variant[DNS_PASS_Y3] == DNS_Y3_TENSOR)
    e = launch_y3tc(b.V, b.O, F6p, gb, c->ph, c->y3tc_tab, c->status, c->st);
  else
    e = var(DNS_PASS_Y3, [&](int v) { return launch_y3<C>(b.V, b.O, F6p, gb, c->ph, fyP.tab(), c->status, c->st, v); });
  if (e) return e;
  mark();
  if ((e = var(DNS_PASS_ZB, [&](int v) { return launch_zb<C>(F6z, G6r, 6 * (int)NR, g, fz.tab(), c->st, c->status, v); })))
    return e;
  mark();
  if ((e = var(DNS_PASS_X, [&](int v) {
         return launch_x_fused<C>(G6x, G3x, g, fx.tab(), c->Uy, c->ph.Ro, c->status, c->st, v, false, c->ph.runs);
       })))
    return e;
  mark();
  if ((e = var(DNS_PASS_ZF, [&](int v) { return launch_zf<C>(G3r, F3p, 3 * (int)NR, g, fz.tab(), c->st, c->status, v); })))
    return e;
  mark();
  const RhsDims rd{c->wd.nv, c->wd.no, c->wd.gp};
  const size_t nv = c->wd.nv, no = c->wd.no;
  const double* t0 = c->rtab;
  const RhsTabs tb{t0, t0 + 4 * nv, t0 + 4 * nv + 2 * no, t0 + 4 * nv + 2 * no + g.Ny,
                   t0 + 4 * nv + 2 * no + g.Ny + 5 * nv};
  if ((e = var(DNS_PASS_Y1, [&](int v) {
         return launch_y1<C>(F3y, b.V, b.O, b.Nvp, b.Nop, c->rv, c->ro, rd, tb, gb, c->ph, fyP.tab(), boot,
                             c->status, c->st, v);
       })))
    return e;
  mark();
  if (!boot)
    if ((e = var(DNS_PASS_Y2, [&](int v) {
           return launch_wall_solve(c->wfac, b.V, b.O, c->rv, c->ro, c->wQ, (double2*)c->F6, c->wd, g, c->ph,
                                    c->status, c->st, v == VAR_AUTO ? DNS_Y2_RING2_8K_EF : v);
         })))
      return e;
  mark();
  return cudaSuccess;
}

cudaError_t enqueue(dns_ctx* c, int boot, cudaEvent_t* ev = nullptr, const StepBufs* bufs = nullptr) {
  const StepBufs b = bufs ? *bufs : StepBufs{c->V, c->O, c->Nvp, c->Nop};
  if (c->P.precision == DNS_PREC_MIXED)
    return enqueue_pipeline<float2>(c, boot, c->fz_f, c->fx_f, c->fyP_f, ev, b);
  return enqueue_pipeline<double2>(c, boot, c->fz_d, c->fx_d, c->fyP_d, ev, b);
}

// Whether variant v of a tunable pass runs as itself on this context's
// step buffers (the launchers' probe: nothing is launched).
template <typename C>
bool probe_pass(const dns_ctx* c, int pass, int v, const DevFft<C>& fz, const DevFft<C>& fyP) {
  const DnsGeom& g = c->g;
  const long long H = g.H, NR = g.nrun, PR = (long long)g.Py * g.Pz * c->KxS;
  DnsGeom gb = g;
  gb.H = NR * H;
  PencilArr F6p{c->F6, c->PyS, NR * H * c->PyS};
  PencilArr F6z{c->F6, c->PyS, H * c->PyS};
  RowArr G6r{c->G6, c->KxS, PR};
  RowArr G6x{c->G6, c->KxS, NR * PR};
  RowArr G3x{c->F6, c->KxS, NR * PR};
  RowArr G3r{c->F6, c->KxS, PR};
  PencilArr F3p{c->G6, c->PyS, H * c->PyS};
  PencilArr F3y{c->G6, c->PyS, NR * H * c->PyS};
  switch (pass) {
    case DNS_PASS_Y3:
      if (v == DNS_Y3_TENSOR)
        return std::is_same<C, float2>::value && g.Ny == 129 && g.Py == 257;
      return launch_y3<C>(c->V, c->O, F6p, gb, c->ph, fyP.tab(), c->status, c->st, v, true) == cudaSuccess;
    case DNS_PASS_Y1: {
      const RhsDims rd{c->wd.nv, c->wd.no, c->wd.gp};
      const RhsTabs tb{};
      return launch_y1<C>(F3y, c->V, c->O, c->Nvp, c->Nop, c->rv, c->ro, rd, tb, gb, c->ph, fyP.tab(), 0,
                          c->status, c->st, v, true) == cudaSuccess;
    }
    case DNS_PASS_ZB:
      return launch_zb<C>(F6z, G6r, 6 * (int)NR, g, fz.tab(), c->st, c->status, v, true) == cudaSuccess;
    case DNS_PASS_ZF:
      return launch_zf<C>(G3r, F3p, 3 * (int)NR, g, fz.tab(), c->st, c->status, v, true) == cudaSuccess;
    case DNS_PASS_Y2:
      return v < DNS_WALL_VARIANTS && wall_smem_bytes(c->wd, v) <= 227 * 1024;
    case DNS_PASS_X: {
      const DevFft<C>& fx = *(const DevFft<C>*)(std::is_same<C, float2>::value ? (const void*)&c->fx_f
                                                                               : (const void*)&c->fx_d);
      return launch_x_fused<C>(G6x, G3x, g, fx.tab(), c->Uy, c->ph.Ro, c->status, c->st, v, true, c->ph.runs) ==
             cudaSuccess;
    }
  }
  return false;
}
bool variant_available(const dns_ctx* c, int pass, int v) {
  if (pass < 0 || pass >= DNS_NUM_PASSES || v < 0 || v >= DNS_MAX_VARIANTS) return false;
  if (c->P.precision == DNS_PREC_MIXED) return probe_pass<float2>(c, pass, v, c->fz_f, c->fyP_f);
  return probe_pass<double2>(c, pass, v, c->fz_d, c->fyP_d);
}
// starting variants: the first each precision's order allows
void default_variants(dns_ctx* c) {
  const bool mixed = c->P.precision == DNS_PREC_MIXED;
  static const int order_mixed[DNS_NUM_PASSES][3] = {
      {DNS_Y3_FFT, DNS_Y3_BLOCK, -1}, {DNS_Y1_WARP, DNS_Y1_BLOCK, -1},
      {DNS_Z_TENSOR_COPY, DNS_Z_WARP, DNS_Z_BLOCK}, {DNS_Z_TENSOR_COPY, DNS_Z_WARP, DNS_Z_BLOCK},
      {DNS_Y2_RING3_12K_EF, DNS_Y2_RING2_8K_EF, -1}, {DNS_X_WARP3, DNS_X_BLOCK, -1}};
  static const int order_fp64[DNS_NUM_PASSES][3] = {
      {DNS_Y3_FFT, DNS_Y3_BLOCK, -1}, {DNS_Y1_WARP, DNS_Y1_BLOCK, -1},
      {DNS_Z_WARP, DNS_Z_BLOCK, -1}, {DNS_Z_WARP, DNS_Z_BLOCK, -1},
      {DNS_Y2_RING3_12K_EF, DNS_Y2_RING2_8K_EF, -1}, {DNS_X_WARP3, DNS_X_BLOCK, -1}};
  for (int p = 0; p < DNS_NUM_PASSES; ++p) {
    const int* ord = mixed ? order_mixed[p] : order_fp64[p];
    c->variant[p] = ord[0];
    for (int i = 0; i < 3 && ord[i] >= 0; ++i)
      if (variant_available(c, p, ord[i])) { c->variant[p] = ord[i]; break; }
  }
}
// the spanwise variant of the FP64 per-function entries: the context's own
// in the FP64 form, else the block form
int zvar64(const dns_ctx* c, int pass) {
  return c->P.precision == DNS_PREC_FP64 ? c->variant[pass] : DNS_Z_BLOCK;
}

dns_status need_scratch(dns_ctx* c) {
  if (c->scratch) return DNS_OK;
  CK(c->alloc(&c->scratch, (size_t)c->g.Py * c->g.Pz * c->RS));
  return DNS_OK;
}

cudaMemcpyKind kind_of(int where, bool to_device) {
  if (where == DNS_DEVICE) return cudaMemcpyDeviceToDevice;
  return to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
}
}  // namespace

dns_status dns_internal_fail(dns_status s, const char* msg) { return fail(s, msg); }

extern "C" {

const char* dns_status_string(dns_status s) {
  switch (s) {
    case DNS_OK: return "ok";
    case DNS_ERR_ARG: return "invalid argument";
    case DNS_ERR_CUDA: return "CUDA error";
    case DNS_ERR_STATE: return "call out of order";
    case DNS_ERR_TIMEOUT: return "device wait timed out";
    case DNS_ERR_SINGULAR: return "singular operator";
    case DNS_ERR_IO: return "file error";
    case DNS_ERR_NONFINITE: return "non-finite state";
  }
  return "unknown";
}

const char* dns_last_error(void) { return g_err.c_str(); }
int dns_abi_version(void) { return DNS_B200_ABI_VERSION; }

dns_status dns_params_default(dns_params* p) {
  if (!p) return fail(DNS_ERR_ARG, "null params");
  std::memset(p, 0, sizeof(*p));
  p->mx = 128; p->my = 128; p->mz = 128;
  p->n_pi_x = 4.0; p->n_pi_y = 2.0;
  p->Re = 2600; p->Ro = 0.015; p->dt = 0.005;
  p->U0 = 0.5; p->U1 = 0.5; p->U2 = 0.0;
  p->precision = DNS_PREC_FP64;
  p->device = 0;
  return DNS_OK;
}

dns_status dns_read_parameter_file(const char* path, dns_params* p, dns_run_params* rp) {
  if (!path || !p) return fail(DNS_ERR_ARG, "null argument");
  std::ifstream in(path);
  if (!in.is_open()) return fail(DNS_ERR_IO, std::string("cannot open ") + path);
  dns_params q;
  dns_params_default(&q);
  dns_run_params r;
  std::memset(&r, 0, sizeof(r));
  std::string outp, recp;
  if (!(in >> q.mx >> q.my >> q.mz >> q.n_pi_x >> q.n_pi_y >> q.Re >> q.Ro >> q.dt))
    return fail(DNS_ERR_IO, "parameter file: numerical records missing or malformed");
  if (!(in >> r.start_type >> r.start_step >> r.end_step >> r.save_internal >> r.save_recovery_internal))
    return fail(DNS_ERR_IO, "parameter file: step record missing or malformed");
  if (!(in >> outp >> recp)) return fail(DNS_ERR_IO, "parameter file: output prefixes missing");
  if (outp.size() >= sizeof(r.output_file_prefix) || recp.size() >= sizeof(r.recovery_file_prefix))
    return fail(DNS_ERR_IO, "parameter file: prefix too long");
  std::strcpy(r.output_file_prefix, outp.c_str());
  std::strcpy(r.recovery_file_prefix, recp.c_str());
  *p = q;
  if (rp) *rp = r;
  return DNS_OK;
}

dns_status dns_create(const dns_params* p, dns_ctx** out) { return ctx_create(p, nullptr, out); }

dns_status dns_create_batch(const dns_params* runs, int nruns, dns_ctx** out) {
  if (!runs || !out || nruns < 1) return fail(DNS_ERR_ARG, "null argument or no runs");
  if (nruns > DNS_MAX_BATCH) return fail(DNS_ERR_ARG, "too many runs in one batch");
  std::vector<double> t(3 * (size_t)nruns);
  const dns_params& a = runs[0];
  for (int r = 0; r < nruns; ++r) {
    const dns_params& b = runs[r];
    if (b.mx != a.mx || b.my != a.my || b.mz != a.mz || b.n_pi_x != a.n_pi_x || b.n_pi_y != a.n_pi_y ||
        b.U0 != a.U0 || b.U1 != a.U1 || b.U2 != a.U2 || b.precision != a.precision || b.device != a.device)
      return fail(DNS_ERR_ARG, "the runs of a batch share grid, box, base flow, precision and device");
    if (!(b.Re > 0) || !(b.dt > 0)) return fail(DNS_ERR_ARG, "Re and dt must be positive");
    t[3 * (size_t)r] = b.Re;
    t[3 * (size_t)r + 1] = b.Ro;
    t[3 * (size_t)r + 2] = b.dt;
  }
  return ctx_create(&a, nullptr, out, nruns, t.data());
}

// A context of the whole grid (slab == NULL) or of one slab rank: then the
// pencil arrays hold the rank's pencils only and the transform buffers its
// pencils (all planes) and its planes (all pencils); the context takes
// ownership of slab.
dns_status ctx_create(const dns_params* p, SlabState* slab, dns_ctx** out, int nrun, const double* runs) {
  std::unique_ptr<SlabState> own(slab);
  if (nrun < 1 || (nrun > 1 && (!runs || slab))) return fail(DNS_ERR_ARG, "bad batch");
  if (!p || !out) return fail(DNS_ERR_ARG, "null argument");
  *out = nullptr;
  if (p->mx <= 0 || p->my <= 0 || p->mz <= 0 || p->mz % 4 != 0)
    return fail(DNS_ERR_ARG, "mx, my, mz must be positive and mz a multiple of 4");
  if (!(p->Re > 0) || !(p->dt > 0) || !(p->n_pi_x > 0) || !(p->n_pi_y > 0))
    return fail(DNS_ERR_ARG, "Re, dt and box lengths must be positive");
  if (p->precision != DNS_PREC_FP64 && p->precision != DNS_PREC_MIXED)
    return fail(DNS_ERR_ARG, "unknown precision");
  DnsGeom g = dns_make_geom(p->mx, p->my, p->mz);
  g.nrun = nrun;
  if ((double)g.H * nrun >= 2147483648.0) return fail(DNS_ERR_ARG, "too many pencils (2^31 or more in one launch)");
  if (g.Nx < 2 || g.Nz < 2 || g.Nx % 2 || g.Nz % 2 || g.Ny < 5)
    return fail(DNS_ERR_ARG, "need even Nx, Nz >= 2 and Ny >= 5");
  if (!fft_len_ok(g.Px) || !fft_len_ok(g.Pz) || !fft_len_ok(p->mz) || !fft_len_ok(p->mz / 2))
    return fail(DNS_ERR_ARG, "mx, my, mz and mz/2 must be products of 2 and 3 (2^a 3^b)");
  if (g.Px < g.Nx || g.Pz < g.Nz) return fail(DNS_ERR_ARG, "padded sizes below mode counts");

  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (p->device < 0 || p->device >= ndev) return fail(DNS_ERR_ARG, "no such CUDA device");
  CK(cudaSetDevice(p->device));

  dns_ctx* c = new dns_ctx();
  c->slab = own.release();
  c->P = *p;
  c->g = g;
  c->ph.aphi = p->n_pi_x / 2;
  c->ph.beta = p->n_pi_y / 2;
  c->ph.Re = p->Re;
  c->ph.Ro = p->Ro;
  c->ph.dt = p->dt;
  c->ph.U0 = p->U0;
  c->ph.U1 = p->U1;
  c->ph.U2 = p->U2;
  c->PyS = roundup(g.Py, 8);
  c->KxS = roundup(g.Kx, 8);
  c->RS = roundup(g.Px / 2 + 1, 8);
  auto bail = [&](dns_status s) { dns_destroy(c); return s; };
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking)) return bail(fail(DNS_ERR_CUDA, "stream"));
  cudaError_t e = cudaSuccess;
  e = e ? e : make_fft(g.Pz, c->fz_d);
  e = e ? e : make_fft(g.Px, c->fx_d);
  e = e ? e : make_fft(p->mz, c->fyP_d);
  e = e ? e : make_fft(p->mz / 2, c->fy0_d);
  e = e ? e : make_fft(g.Pz, c->fz_f);
  e = e ? e : make_fft(g.Px, c->fx_f);
  e = e ? e : make_fft(p->mz, c->fyP_f);
  if (e) return bail(fail(DNS_ERR_CUDA, std::string("fft tables: ") + cudaGetErrorString(e)));

  const int Ny = g.Ny;
  std::vector<double> T0((size_t)Ny * Ny), T2((size_t)Ny * Ny), T4((size_t)Ny * Ny);
  host_T_matrix(Ny - 1, T0.data(), T2.data(), T4.data());
  std::vector<double> U(Ny), dU(Ny), ddU(Ny), Uy(g.Py);
  host_base_flow(Ny, p->U0, p->U1, p->U2, U.data(), dU.data(), ddU.data());
  host_base_flow(g.Py, p->U0, p->U1, p->U2, Uy.data(), nullptr, nullptr);
  const size_t NN = (size_t)Ny * Ny;
  const size_t csz = p->precision == DNS_PREC_MIXED ? 8 : 16;
  SlabState* sl = c->slab;
  // whole grid: F6 = the six pencil fields, then the three Lamb rows; G6 =
  // the six rows, then the three pencil fields.  Slab rank: F6 = its
  // pencils' fields (all planes), G6 and sl->A = its planes' rows and
  // pencils (all pencils)
  size_t f6 = std::max((size_t)6 * g.H * c->PyS, (size_t)3 * g.Py * g.Pz * c->KxS);
  size_t g6 = std::max((size_t)6 * g.Py * g.Pz * c->KxS, (size_t)3 * g.H * c->PyS);
  if (sl) {
    f6 = (size_t)6 * sl->np * c->PyS;
    g6 = std::max((size_t)6 * sl->ny * g.Pz * c->KxS, (size_t)3 * g.H * sl->nyS);
  }
  f6 *= (size_t)nrun;  // a batch: every member's fields
  g6 *= (size_t)nrun;
  const size_t hn = (size_t)(sl ? sl->np : g.H * nrun) * Ny;
  // integrated right-hand sides: N + deg(U) + 1 rows per pencil
  c->wd.delta = wall::base_degree(p->U1, p->U2);
  c->wd.nv = c->wd.no = Ny + c->wd.delta;
  c->wd.gp = c->wd.nv;
  c->wd.qbytes = (int)((7 * (size_t)c->wd.no * 8 + 15) & ~(size_t)15);
  const size_t gn = (size_t)(sl ? sl->np : g.H * nrun) * c->wd.gp;
  if ((e = c->alloc(&c->T0, NN)) || (e = c->alloc(&c->T2, NN)) || (e = c->alloc(&c->T4, NN)) ||
      (e = c->alloc(&c->Ut, Ny)) || (e = c->alloc(&c->dUt, Ny)) || (e = c->alloc(&c->ddUt, Ny)) ||
      (e = c->alloc(&c->Uy, g.Py)) || (e = c->alloc(&c->V, hn)) || (e = c->alloc(&c->O, hn)) ||
      (e = c->alloc(&c->Nvp, hn)) || (e = c->alloc(&c->Nop, hn)) || (e = c->alloc(&c->rv, gn)) ||
      (e = c->alloc(&c->ro, gn)) || (e = c->alloc(&c->status, 1)) ||
      (e = c->alloc((unsigned char**)&c->F6, c->F6_bytes = f6 * csz)) ||
      (e = c->alloc((unsigned char**)&c->G6, g6 * csz)) ||
      (e = c->alloc(&c->rtab, 4 * (size_t)c->wd.nv + 2 * (size_t)c->wd.no + Ny + 8 * (size_t)c->wd.nv)) ||
      (sl && (e = c->alloc((unsigned char**)&sl->A,
                           std::max((size_t)6 * g.H * sl->nyS, (size_t)3 * sl->ny * g.Pz * c->KxS) * csz))))
    return bail(fail(DNS_ERR_CUDA, std::string("device allocation: ") + cudaGetErrorString(e)));
  cudaMemcpy(c->T0, T0.data(), NN * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->T2, T2.data(), NN * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->T4, T4.data(), NN * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->Ut, U.data(), Ny * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->dUt, dU.data(), Ny * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->ddUt, ddU.data(), Ny * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->Uy, Uy.data(), g.Py * 8, cudaMemcpyHostToDevice);
  {
    // y1 tables (integrated cardinal corrections, cos(k pi/N))
    const int N = Ny - 1, nv = c->wd.nv, no = c->wd.no;
    std::vector<double> tab(4 * (size_t)nv + 2 * (size_t)no + Ny + 8 * (size_t)nv);
    const int mv[4] = {0, 1, N - 1, N};
    for (int m = 0; m < 4; ++m) wall::cardinal_rows(N, mv[m], 4, nv, &tab[(size_t)m * nv]);
    wall::cardinal_rows(N, 0, 2, no, &tab[4 * (size_t)nv]);
    wall::cardinal_rows(N, N, 2, no, &tab[4 * (size_t)nv + no]);
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int k = 0; k <= N; ++k) tab[4 * (size_t)nv + 2 * (size_t)no + k] = (double)cosl(PI * k / N);
    // rows of B^4 (from row 4) and B^2 (from row 2) as 5- and 3-point
    // stencils, stored weight-major ([d][r]: a warp's rows read consecutive
    // entries)
    std::vector<double> s4((size_t)5 * nv), s2((size_t)3 * nv);
    wall::integration_stencils(N, nv, s4.data(), s2.data());
    double* b4 = &tab[4 * (size_t)nv + 2 * (size_t)no + Ny];
    double* b2 = b4 + 5 * (size_t)nv;
    for (int r = 0; r < nv; ++r) {
      for (int d = 0; d < 5; ++d) b4[(size_t)d * nv + r] = s4[(size_t)5 * r + d];
      for (int d = 0; d < 3; ++d) b2[(size_t)d * nv + r] = s2[(size_t)3 * r + d];
    }
    cudaMemcpy(c->rtab, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice);
  }
  if (nrun > 1) {
    c->runs_h.assign(runs, runs + 3 * (size_t)nrun);
    if ((e = c->alloc(&c->runs_d, 3 * (size_t)nrun)) ||
        (e = cudaMemcpy(c->runs_d, runs, 3 * (size_t)nrun * 8, cudaMemcpyHostToDevice)))
      return bail(fail(DNS_ERR_CUDA, std::string("device allocation: ") + cudaGetErrorString(e)));
    c->ph.runs = c->runs_d;
  }
  cudaMemset(c->status, 0, sizeof(int));
  cudaMemset(c->Nvp, 0, hn * 16);
  cudaMemset(c->Nop, 0, hn * 16);
  if ((e = cudaDeviceSynchronize())) return bail(fail(DNS_ERR_CUDA, cudaGetErrorString(e)));
  default_variants(c);
  *out = c;
  return DNS_OK;
}

dns_status dns_destroy(dns_ctx* c) {
  if (!c) return DNS_OK;
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  if (c->solve_graph) cudaGraphExecDestroy(c->solve_graph);
  free_fft(c->fz_d); free_fft(c->fx_d); free_fft(c->fyP_d); free_fft(c->fy0_d);
  free_fft(c->fz_f); free_fft(c->fx_f); free_fft(c->fyP_f);
  void* ptrs[] = {c->T0, c->T2, c->T4, c->Ut, c->dUt, c->ddUt, c->Uy, c->V, c->O, c->Nvp,
                  c->Nop, c->rv, c->ro, c->wfac, c->wQ, c->rtab, c->F6, c->G6, c->scratch, c->solve_io, c->rhs_io, c->nl_io, c->eq_io, c->probe, c->status,
                  c->y3tc_tab};
  for (void* q : ptrs) cudaFree(q);
  if (c->slab) cudaFree(c->slab->A);
  cudaFree(c->runs_d);
  delete c->slab;
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return DNS_OK;
}

dns_status dns_geometry(const dns_ctx* c, int out[8]) {
  if (!c || !out) return fail(DNS_ERR_ARG, "null argument");
  out[0] = c->g.Nx; out[1] = c->g.Ny; out[2] = c->g.Nz; out[3] = c->g.Kx;
  out[4] = c->g.Px; out[5] = c->g.Py; out[6] = c->g.Pz; out[7] = (int)c->g.H;
  return DNS_OK;
}

dns_status dns_get_stream(dns_ctx* c, void** s) {
  if (!c || !s) return fail(DNS_ERR_ARG, "null argument");
  *s = (void*)c->st;
  return DNS_OK;
}

dns_status dns_synchronize(dns_ctx* c) {
  if (!c) return fail(DNS_ERR_ARG, "null context");
  CK(cudaSetDevice(c->P.device));
  CK(cudaStreamSynchronize(c->st));
  return check_status(c);
}

dns_status dns_memory_bytes(const dns_ctx* c, size_t* b) {
  if (!c || !b) return fail(DNS_ERR_ARG, "null argument");
  *b = c->bytes;
  return DNS_OK;
}

// enqueue one field's copy between the caller's pencils (pitch) and the
// library's (Ny complex, unpadded); one linear copy when the pitches agree
static dns_status copy_pencils(dns_ctx* c, double2* dev, const void* src, void* dst, size_t pitch,
                               int where, bool to_dev) {
  const size_t w = (size_t)c->g.Ny * 16;
  const long long nH = c->g.H * c->g.nrun;  // every member of a batch
  if (pitch < w || pitch % 16) return fail(DNS_ERR_ARG, "pencil pitch must be >= Ny*16 and a multiple of 16");
  if (where != DNS_HOST && where != DNS_DEVICE) return fail(DNS_ERR_ARG, "where must be DNS_HOST or DNS_DEVICE");
  const cudaMemcpyKind k = kind_of(where, to_dev);
  if (pitch == w) {
    if (to_dev) CK(cudaMemcpyAsync(dev, src, w * (size_t)nH, k, c->st));
    else CK(cudaMemcpyAsync(dst, dev, w * (size_t)nH, k, c->st));
  } else if (to_dev) {
    CK(cudaMemcpy2DAsync(dev, w, src, pitch, w, (size_t)nH, k, c->st));
  } else {
    CK(cudaMemcpy2DAsync(dst, pitch, dev, w, w, (size_t)nH, k, c->st));
  }
  return DNS_OK;
}

dns_status dns_set_state(dns_ctx* c, const void* v, const void* o, size_t pitch, int where) {
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c || !v || !o) return fail(DNS_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->P.device));
  dns_status s = copy_pencils(c, c->V, v, nullptr, pitch, where, true);
  if (s == DNS_OK) s = copy_pencils(c, c->O, o, nullptr, pitch, where, true);
  if (s == DNS_OK) CK(cudaStreamSynchronize(c->st));
  if (s == DNS_OK) c->have_state = true;
  return s;
}

dns_status dns_get_state(dns_ctx* c, void* v, void* o, size_t pitch, int where) {
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c || !v || !o) return fail(DNS_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->P.device));
  dns_status s = copy_pencils(c, c->V, nullptr, v, pitch, where, false);
  if (s == DNS_OK) s = copy_pencils(c, c->O, nullptr, o, pitch, where, false);
  if (s == DNS_OK) CK(cudaStreamSynchronize(c->st));
  return s;
}

// The AB2 history is held as Chebyshev coefficients; the ABI exchanges it
// as values at the Gauss-Lobatto points (the reference's rhs_v_p /
// rhs_omega_y_p), converted here with the no-pad s2p / p2s.
// (k_cheby_inplace writes whole FFT lines, so the scratch pencils have
// pitch mz/2 >= the no-pad FFT length.)
static dns_status history_out(dns_ctx* c, const double2* src, void* dst, size_t pitch, int where) {
  dns_status s = need_scratch(c);
  if (s) return s;
  const size_t w = (size_t)c->g.Ny * 16, ps = (size_t)(c->P.mz / 2);
  if (where != DNS_HOST && where != DNS_DEVICE) return fail(DNS_ERR_ARG, "where must be DNS_HOST or DNS_DEVICE");
  if (pitch < w || pitch % 16) return fail(DNS_ERR_ARG, "pencil pitch must be >= Ny*16 and a multiple of 16");
  const long long H = c->g.H;
  for (int r = 0; r < c->g.nrun; ++r) {  // a batch: member by member through the scratch
    CK(cudaMemcpy2DAsync(c->scratch, ps * 16, src + r * H * c->g.Ny, w, w, (size_t)H, cudaMemcpyDeviceToDevice,
                         c->st));
    PencilArr a{c->scratch, (long long)ps, 0};
    CK(launch_cheby_inplace<double2>(a, H, 1, c->g.Ny, c->fy0_d.tab(), c->st));
    CK(cudaMemcpy2DAsync((char*)dst + (size_t)r * H * pitch, pitch, c->scratch, ps * 16, w, (size_t)H,
                         kind_of(where, false), c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  return DNS_OK;
}
static dns_status history_in(dns_ctx* c, double2* dst, const void* src, size_t pitch, int where) {
  dns_status s = need_scratch(c);
  if (s) return s;
  const size_t w = (size_t)c->g.Ny * 16, ps = (size_t)(c->P.mz / 2);
  if (where != DNS_HOST && where != DNS_DEVICE) return fail(DNS_ERR_ARG, "where must be DNS_HOST or DNS_DEVICE");
  if (pitch < w || pitch % 16) return fail(DNS_ERR_ARG, "pencil pitch must be >= Ny*16 and a multiple of 16");
  const long long H = c->g.H;
  for (int r = 0; r < c->g.nrun; ++r) {
    CK(cudaMemcpy2DAsync(c->scratch, ps * 16, (const char*)src + (size_t)r * H * pitch, pitch, w, (size_t)H,
                         kind_of(where, true), c->st));
    PencilArr a{c->scratch, (long long)ps, 0};
    CK(launch_cheby_inplace<double2>(a, H, 3, c->g.Ny, c->fy0_d.tab(), c->st));
    CK(cudaMemcpy2DAsync(dst + r * H * c->g.Ny, w, c->scratch, ps * 16, w, (size_t)H, cudaMemcpyDeviceToDevice,
                         c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  return DNS_OK;
}

dns_status dns_get_history(dns_ctx* c, void* nv, void* no, size_t pitch, int where) {
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c || !nv || !no) return fail(DNS_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->P.device));
  dns_status s = history_out(c, c->Nvp, nv, pitch, where);
  if (s == DNS_OK) s = history_out(c, c->Nop, no, pitch, where);
  return s;
}

dns_status dns_set_history(dns_ctx* c, const void* nv, const void* no, size_t pitch, int where) {
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c || !nv || !no) return fail(DNS_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->P.device));
  dns_status s = history_in(c, c->Nvp, nv, pitch, where);
  if (s == DNS_OK) s = history_in(c, c->Nop, no, pitch, where);
  if (s == DNS_OK) c->booted = true;
  return s;
}

dns_status dns_bootstrap(dns_ctx* c) {
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c) return fail(DNS_ERR_ARG, "null context");
  if (!c->have_state) return fail(DNS_ERR_STATE, "dns_set_state must precede dns_bootstrap");
  CK(cudaSetDevice(c->P.device));
  CK(enqueue(c, 1));
  dns_status s = check_status(c);
  if (s == DNS_OK) c->booted = true;
  return s;
}

dns_status dns_nonlinear(dns_ctx* c, const void* v, const void* o, void* nv, void* no, size_t tpitch,
                         int where) {
  if (c && c->g.nrun > 1) return fail(DNS_ERR_STATE, "a batch context: this entry point takes one run");
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c || !v || !o || !nv || !no) return fail(DNS_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->P.device));
  const size_t hn = (size_t)c->g.H * c->g.Ny;
  if (!c->nl_io) CK(c->alloc(&c->nl_io, 4 * hn));
  // the pass sequence of the bootstrap on the caller's state, into the
  // context's own vectors: the state and history of the context are untouched
  StepBufs b{c->nl_io, c->nl_io + hn, c->nl_io + 2 * hn, c->nl_io + 3 * hn};
  dns_status s = copy_pencils(c, b.V, v, nullptr, tpitch, where, true);
  if (s == DNS_OK) s = copy_pencils(c, b.O, o, nullptr, tpitch, where, true);
  if (s != DNS_OK) return s;
  CK(enqueue(c, 1, nullptr, &b));
  s = check_status(c);
  if (s == DNS_OK) s = history_out(c, b.Nvp, nv, tpitch, where);
  if (s == DNS_OK) s = history_out(c, b.Nop, no, tpitch, where);
  return s;
}

namespace {
// checks, factors and the captured step graph of one context
dns_status step_ready(dns_ctx* c) {
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c) return fail(DNS_ERR_ARG, "null context");
  if (!c->have_state || !c->booted)
    return fail(DNS_ERR_STATE, "dns_set_state and dns_bootstrap must precede dns_step");
  CK(cudaSetDevice(c->P.device));
  dns_status s = build_wall_solver(c);
  if (s != DNS_OK) return s;
  if (!c->graph) {
    cudaGraph_t gr;
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue(c, 0);
    cudaError_t e2 = cudaStreamEndCapture(c->st, &gr);
    if (e) return fail(DNS_ERR_CUDA, std::string("step capture: ") + cudaGetErrorString(e));
    CK(e2);
    CK(cudaGraphInstantiate(&c->graph, gr, 0));
    cudaGraphDestroy(gr);
  }
  return DNS_OK;
}
}  // namespace

dns_status dns_step(dns_ctx* c, int nsteps) {
  if (nsteps < 0) return fail(DNS_ERR_ARG, "nsteps < 0");
  dns_status s = step_ready(c);
  if (s != DNS_OK) return s;
  for (int i = 0; i < nsteps; ++i) CK(cudaGraphLaunch(c->graph, c->st));
  return DNS_OK;
}

dns_status dns_set_wait_limit(dns_ctx* c, long long cycles) {
  if (!c) return fail(DNS_ERR_ARG, "null context");
  CK(cudaSetDevice(c->P.device));
  CK(cudaStreamSynchronize(c->st));
  c->ph.wait_limit = cycles;
  if (c->graph) {  // the step graph holds the kernel parameters: capture it again
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  return DNS_OK;
}

dns_status dns_set_variant(dns_ctx* c, int pass, int v) {
  if (!c) return fail(DNS_ERR_ARG, "null context");
  if (pass < 0 || pass >= DNS_NUM_PASSES) return fail(DNS_ERR_ARG, "unknown pass");
  if (!variant_available(c, pass, v)) return fail(DNS_ERR_ARG, "variant not available for this context");
  CK(cudaSetDevice(c->P.device));
  CK(cudaStreamSynchronize(c->st));
  if (pass == DNS_PASS_Y3 && v == DNS_Y3_TENSOR && !c->y3tc_tab) {
    std::vector<uint32_t> w(y3tc_table_words());
    y3tc_table(w.data());
    CK(c->alloc(&c->y3tc_tab, w.size()));
    CK(cudaMemcpy(c->y3tc_tab, w.data(), w.size() * 4, cudaMemcpyHostToDevice));
  }
  if (c->variant[pass] != v && c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  if (c->variant[pass] != v && c->solve_graph) {  // the solve-only sequence holds the wall solve
    cudaGraphExecDestroy(c->solve_graph);
    c->solve_graph = nullptr;
  }
  c->variant[pass] = v;
  return DNS_OK;
}

dns_status dns_get_variant(const dns_ctx* c, int pass, int* v) {
  if (!c || !v) return fail(DNS_ERR_ARG, "null argument");
  if (pass < 0 || pass >= DNS_NUM_PASSES) return fail(DNS_ERR_ARG, "unknown pass");
  *v = c->variant[pass];
  return DNS_OK;
}

dns_status dns_autotune(dns_ctx* c, double ms[DNS_NUM_PASSES * DNS_MAX_VARIANTS]) {
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c) return fail(DNS_ERR_ARG, "null context");
  if (!c->have_state) return fail(DNS_ERR_STATE, "dns_autotune needs a state");
  CK(cudaSetDevice(c->P.device));
  CK(cudaStreamSynchronize(c->st));
  dns_status st = build_wall_solver(c);
  if (st != DNS_OK) return st;
  double t[DNS_NUM_PASSES * DNS_MAX_VARIANTS];
  bool avail[DNS_NUM_PASSES][DNS_MAX_VARIANTS];
  for (int p = 0; p < DNS_NUM_PASSES; ++p)
    for (int v = 0; v < DNS_MAX_VARIANTS; ++v) {
      t[p * DNS_MAX_VARIANTS + v] = -1.0;
      avail[p][v] = variant_available(c, p, v);
    }
  if (avail[DNS_PASS_Y3][DNS_Y3_TENSOR] && !c->y3tc_tab) {
    const int keep = c->variant[DNS_PASS_Y3];
    if ((st = dns_set_variant(c, DNS_PASS_Y3, DNS_Y3_TENSOR)) != DNS_OK) return st;
    if ((st = dns_set_variant(c, DNS_PASS_Y3, keep)) != DNS_OK) return st;
  }
  // Every candidate is timed inside whole steps (its inputs as the step
  // leaves them, its neighbours running), one pass at a time: pass p's
  // variants run with every other pass at its best so far (the context's
  // variant for the passes not yet tuned), two warm-up steps and five timed
  // steps with events around each kernel; p then keeps its fastest.  The
  // state and the AB2 history are saved first and put back after.
  const size_t hn = (size_t)c->g.H * c->g.nrun * c->g.Ny;
  double2* save = nullptr;
  CK(cudaMalloc(&save, 4 * hn * 16));
  double2* const bufs[4] = {c->V, c->O, c->Nvp, c->Nop};
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 4 && !e; ++i) e = cudaMemcpyAsync(save + i * hn, bufs[i], hn * 16, cudaMemcpyDeviceToDevice, c->st);
  int keep[DNS_NUM_PASSES], best[DNS_NUM_PASSES];
  for (int p = 0; p < DNS_NUM_PASSES; ++p) keep[p] = best[p] = c->variant[p];
  // kernel slot of each pass in a step's events
  static const int slot[DNS_NUM_PASSES] = {0, 4, 1, 3, 5, 2};
  const int ne = DNS_NUM_KERNELS + 1, nt = 5;
  std::vector<cudaEvent_t> ev((size_t)ne * (nt + 1));
  for (auto& x : ev)
    if (!e) e = cudaEventCreate(&x);
  for (int p = 0; p < DNS_NUM_PASSES && !e && st == DNS_OK; ++p) {
    double bt = 1e300;
    for (int r = 0; r < DNS_MAX_VARIANTS && !e && st == DNS_OK; ++r) {
      if (!avail[p][r]) continue;
      for (int q = 0; q < DNS_NUM_PASSES; ++q) c->variant[q] = best[q];
      c->variant[p] = r;
      e = enqueue(c, 0);
      for (int i = 0; i <= nt && !e; ++i) e = enqueue(c, 0, &ev[(size_t)i * ne]);
      if (!e) e = cudaStreamSynchronize(c->st);
      if (!e) st = check_status(c);
      if (e || st != DNS_OK) break;
      double sum = 0.0;
      for (int i = 1; i <= nt; ++i) {
        float x = 0.f;
        cudaEventElapsedTime(&x, ev[(size_t)i * ne + slot[p]], ev[(size_t)i * ne + slot[p] + 1]);
        sum += x;
      }
      t[p * DNS_MAX_VARIANTS + r] = sum / nt;
      if (sum / nt < bt) {
        bt = sum / nt;
        best[p] = r;
      }
    }
  }
  for (auto& x : ev)
    if (x) cudaEventDestroy(x);
  for (int i = 0; i < 4; ++i) {
    cudaError_t e2 = cudaMemcpyAsync(bufs[i], save + i * hn, hn * 16, cudaMemcpyDeviceToDevice, c->st);
    if (!e) e = e2;
  }
  cudaError_t e3 = cudaStreamSynchronize(c->st);
  if (!e) e = e3;
  cudaFree(save);
  for (int p = 0; p < DNS_NUM_PASSES; ++p) c->variant[p] = keep[p];
  if (e) return fail(DNS_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
  if (st != DNS_OK) return st;
  for (int p = 0; p < DNS_NUM_PASSES && st == DNS_OK; ++p) st = dns_set_variant(c, p, best[p]);
  if (ms)
    for (int i = 0; i < DNS_NUM_PASSES * DNS_MAX_VARIANTS; ++i) ms[i] = t[i];
  return st;
}

dns_status dns_step_many(dns_ctx* const* ctxs, int n, int nsteps) {
  if (!ctxs || n < 1) return fail(DNS_ERR_ARG, "no contexts");
  if (nsteps < 0) return fail(DNS_ERR_ARG, "nsteps < 0");
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < j; ++i)
      if (ctxs[i] == ctxs[j]) return fail(DNS_ERR_ARG, "a context is listed twice");
    dns_status s = step_ready(ctxs[j]);
    if (s != DNS_OK) return s;
  }
  // step by step across the runs, each run on its own stream: the graphs of
  // different runs overlap on the GPU, one run's steps stay in order
  for (int i = 0; i < nsteps; ++i)
    for (int j = 0; j < n; ++j) {
      CK(cudaSetDevice(ctxs[j]->P.device));
      CK(cudaGraphLaunch(ctxs[j]->graph, ctxs[j]->st));
    }
  return DNS_OK;
}

dns_status dns_step_profiled(dns_ctx* c, int nsteps, double kernel_ms[DNS_NUM_KERNELS]) {
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c || !kernel_ms) return fail(DNS_ERR_ARG, "null argument");
  if (nsteps < 1) return fail(DNS_ERR_ARG, "nsteps < 1");
  if (!c->have_state || !c->booted)
    return fail(DNS_ERR_STATE, "dns_set_state and dns_bootstrap must precede dns_step_profiled");
  CK(cudaSetDevice(c->P.device));
  dns_status s = build_wall_solver(c);
  if (s != DNS_OK) return s;
  const int ne = DNS_NUM_KERNELS + 1;
  std::vector<cudaEvent_t> ev((size_t)ne * nsteps);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  cudaError_t err = cudaSuccess;
  for (int i = 0; i < nsteps && !err; ++i) err = enqueue(c, 0, &ev[(size_t)i * ne]);
  if (!err) err = cudaStreamSynchronize(c->st);
  for (int k = 0; k < DNS_NUM_KERNELS; ++k) kernel_ms[k] = 0.0;
  for (int i = 0; i < nsteps && !err; ++i)
    for (int k = 0; k < DNS_NUM_KERNELS; ++k) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[(size_t)i * ne + k], ev[(size_t)i * ne + k + 1]);
      kernel_ms[k] += ms / nsteps;
    }
  for (auto& e : ev) cudaEventDestroy(e);
  if (err) return fail(DNS_ERR_CUDA, cudaGetErrorString(err));
  return check_status(c);
}

const char* dns_kernel_name(int k) {
  static const char* names[DNS_NUM_KERNELS] = {
      "y3_uvw_s2p", "zb_span_inverse", "x_c2r_lamb_r2c", "zf_span_forward", "y1_p2s_rhs", "y2_solve"};
  return (k >= 0 && k < DNS_NUM_KERNELS) ? names[k] : "";
}

// ---- reference-layout entry points ----------------------------------------

static dns_status check_spec_pitch(dns_ctx* c, size_t tpitch) {
  if (tpitch % 16 || tpitch < (size_t)c->P.mz * 16)
    return fail(DNS_ERR_ARG, "tpitch must be a multiple of 16 and hold mz complex values");
  return DNS_OK;
}
static dns_status check_phys_pitch(dns_ctx* c, size_t pitch) {
  if (pitch % 16 || pitch < (size_t)(c->g.Px / 2 + 1) * 16)
    return fail(DNS_ERR_ARG, "pitch must be a multiple of 16 and hold mx/2+1 complex values");
  return DNS_OK;
}

dns_status dns_transform_3d_one(dns_ctx* c, int dir, void* phys, size_t pitch, void* spec,
                                size_t tpitch, int pad) {
  if (!c || !phys || !spec) return fail(DNS_ERR_ARG, "null argument");
  if ((dir != DNS_FORWARD && dir != DNS_BACKWARD) || (pad != DNS_PADDING && pad != DNS_NO_PADDING))
    return fail(DNS_ERR_ARG, "bad direction or padding mode");
  dns_status s;
  if ((s = check_spec_pitch(c, tpitch)) || (s = check_phys_pitch(c, pitch))) return s;
  if ((s = need_scratch(c))) return s;
  CK(cudaSetDevice(c->P.device));
  const DnsGeom& g = c->g;
  PencilArr sp{spec, (long long)(tpitch / 16), 0};
  RowArr sr{c->scratch, c->RS, 0};
  const long long nrows = (long long)g.Py * g.Pz;
  const long long rps = (long long)(pitch / 8);
  if (dir == DNS_BACKWARD) {
    if (pad == DNS_PADDING) CK(launch_cheby_inplace<double2>(sp, g.H, 0, g.Ny, c->fyP_d.tab(), c->st));
    else CK(launch_cheby_inplace<double2>(sp, g.H, 1, g.Ny, c->fy0_d.tab(), c->st));
    CK(launch_zb<double2>(sp, sr, 1, g, c->fz_d.tab(), c->st, nullptr, zvar64(c, DNS_PASS_ZB)));
    CK(launch_x_c2r<double2>(sr, (double*)phys, rps, nrows, g, c->fx_d.tab(), c->st));
  } else {
    CK(launch_x_r2c<double2>((const double*)phys, rps, sr, nrows, g, c->fx_d.tab(),
                             1.0 / g.Px / g.Pz, c->st));
    CK(launch_zf<double2>(sr, sp, 1, g, c->fz_d.tab(), c->st, nullptr, zvar64(c, DNS_PASS_ZF)));
    if (pad == DNS_PADDING) CK(launch_cheby_inplace<double2>(sp, g.H, 2, g.Ny, c->fyP_d.tab(), c->st));
    else CK(launch_cheby_inplace<double2>(sp, g.H, 3, g.Ny, c->fy0_d.tab(), c->st));
  }
  return DNS_OK;
}

dns_status dns_transform(dns_ctx* c, int dir, int nf, void* const* phys, size_t pitch,
                         void* const* spec, size_t tpitch) {
  if (!c || !phys || !spec || nf < 1 || nf > 6) return fail(DNS_ERR_ARG, "bad arguments");
  for (int i = 0; i < nf; ++i) {
    dns_status s = dns_transform_3d_one(c, dir, phys[i], pitch, spec[i], tpitch, DNS_PADDING);
    if (s) return s;
  }
  return DNS_OK;
}

dns_status dns_cuda_transpose(dns_ctx* c, int dir, void* xyz, size_t pitch, void* zxy, size_t tpitch) {
  if (!c || !xyz || !zxy) return fail(DNS_ERR_ARG, "null argument");
  if (dir != DNS_FORWARD && dir != DNS_BACKWARD) return fail(DNS_ERR_ARG, "bad direction");
  if (pitch % 16 || tpitch % 16 || tpitch < (size_t)c->g.Py * 16 || pitch < (size_t)c->g.Kx * 16)
    return fail(DNS_ERR_ARG, "bad pitch");
  CK(cudaSetDevice(c->P.device));
  CK(launch_transpose_ref(dir == DNS_FORWARD ? 0 : 1, (double2*)xyz, (long long)(pitch / 16),
                          (double2*)zxy, (long long)(tpitch / 16), c->g, c->st));
  return DNS_OK;
}

static dns_status cheby_call(dns_ctx* c, void* zxy, size_t tpitch, int pad, bool s2p) {
  if (!c || !zxy) return fail(DNS_ERR_ARG, "null argument");
  if (pad != DNS_PADDING && pad != DNS_NO_PADDING) return fail(DNS_ERR_ARG, "bad padding mode");
  dns_status s = check_spec_pitch(c, tpitch);
  if (s) return s;
  CK(cudaSetDevice(c->P.device));
  PencilArr sp{zxy, (long long)(tpitch / 16), 0};
  const int mode = (s2p ? 0 : 2) + (pad == DNS_PADDING ? 0 : 1);
  const DevFft<double2>& t = (pad == DNS_PADDING) ? c->fyP_d : c->fy0_d;
  CK(launch_cheby_inplace<double2>(sp, c->g.H, mode, c->g.Ny, t.tab(), c->st));
  return DNS_OK;
}
dns_status dns_cheby_s2p(dns_ctx* c, void* zxy, size_t tpitch, int pad) { return cheby_call(c, zxy, tpitch, pad, true); }
dns_status dns_cheby_p2s(dns_ctx* c, void* zxy, size_t tpitch, int pad) { return cheby_call(c, zxy, tpitch, pad, false); }

dns_status dns_get_uvw(dns_ctx* c, void* const f[6], size_t tpitch) {
  if (!c || !f) return fail(DNS_ERR_ARG, "null argument");
  for (int i = 0; i < 6; ++i) if (!f[i]) return fail(DNS_ERR_ARG, "null field");
  if (tpitch % 16 || tpitch < (size_t)c->g.Ny * 16) return fail(DNS_ERR_ARG, "bad tpitch");
  CK(cudaSetDevice(c->P.device));
  double2* ff[6];
  for (int i = 0; i < 6; ++i) ff[i] = (double2*)f[i];
  CK(launch_get_uvw(ff, (long long)(tpitch / 16), c->g, c->ph, c->st));
  return DNS_OK;
}

dns_status dns_compute_lamb(dns_ctx* c, void* const in[6], void* const out[3], size_t pitch) {
  if (!c || !in || !out) return fail(DNS_ERR_ARG, "null argument");
  for (int i = 0; i < 6; ++i) if (!in[i]) return fail(DNS_ERR_ARG, "null field");
  for (int i = 0; i < 3; ++i) if (!out[i]) return fail(DNS_ERR_ARG, "null field");
  if (pitch % 8 || pitch < (size_t)c->g.Px * 8) return fail(DNS_ERR_ARG, "bad pitch");
  CK(cudaSetDevice(c->P.device));
  const double* i6[6];
  double* o3[3];
  for (int i = 0; i < 6; ++i) i6[i] = (const double*)in[i];
  for (int i = 0; i < 3; ++i) o3[i] = (double*)out[i];
  CK(launch_lamb_rows(i6, o3, (long long)(pitch / 8), (long long)c->g.Py * c->g.Pz, c->g, c->Uy,
                      c->ph.Ro, c->st));
  return DNS_OK;
}

dns_status dns_rhs_nonlinear(dns_ctx* c, void* lx, void* ly, const void* lz, size_t tpitch) {
  if (!c || !lx || !ly || !lz) return fail(DNS_ERR_ARG, "null argument");
  if (tpitch % 16 || tpitch < (size_t)c->g.Ny * 16) return fail(DNS_ERR_ARG, "bad tpitch");
  CK(cudaSetDevice(c->P.device));
  CK(launch_rhs_nonlinear((double2*)lx, (double2*)ly, (const double2*)lz, (long long)(tpitch / 16),
                          c->g, c->ph, c->st));
  return DNS_OK;
}

dns_status dns_solve_eq(dns_ctx* c, const void* inv, void* rhs, int N, size_t tpitch, int where) {
  if (!c || !inv || !rhs) return fail(DNS_ERR_ARG, "null argument");
  if (N < 1 || N > 4096 || tpitch % 16 || tpitch < (size_t)N * 16) return fail(DNS_ERR_ARG, "bad N or tpitch");
  if (where != DNS_HOST && where != DNS_DEVICE) return fail(DNS_ERR_ARG, "bad where");
  CK(cudaSetDevice(c->P.device));
  const long long H = c->g.H;
  if (where == DNS_DEVICE) {
    CK(launch_solve_eq((const double2*)inv, (double2*)rhs, (long long)(tpitch / 16), N, H, c->st));
    return DNS_OK;
  }
  // host inverses and right-hand sides (the reference keeps both in host
  // memory, source/solver.cpp:216-257): streamed through a device staging
  // buffer in batches of pencils, at most ~512 MiB of inverses at a time
  const size_t NN16 = (size_t)N * N * 16, row = (size_t)N * 16;
  const long long batch = std::max(1LL, std::min<long long>(H, (512LL << 20) / (long long)NN16));
  const size_t need = (size_t)batch * (NN16 + row);
  if (c->eq_io_bytes < need) {
    if (c->eq_io) cudaFree(c->eq_io);
    c->eq_io = nullptr;
    c->eq_io_bytes = 0;
    CK(c->alloc(&c->eq_io, need));
    c->eq_io_bytes = need;
  }
  double2* dinv = (double2*)c->eq_io;
  double2* drhs = (double2*)(c->eq_io + (size_t)batch * NN16);
  for (long long p0 = 0; p0 < H; p0 += batch) {
    const long long np = std::min(batch, H - p0);
    CK(cudaMemcpyAsync(dinv, (const char*)inv + (size_t)p0 * NN16, (size_t)np * NN16,
                       cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpy2DAsync(drhs, row, (const char*)rhs + (size_t)p0 * tpitch, tpitch, row, (size_t)np,
                         cudaMemcpyHostToDevice, c->st));
    CK(launch_solve_eq(dinv, drhs, N, N, np, c->st));
    CK(cudaMemcpy2DAsync((char*)rhs + (size_t)p0 * tpitch, tpitch, drhs, row, row, (size_t)np,
                         cudaMemcpyDeviceToHost, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  return DNS_OK;
}

dns_status dns_operator_matrices(dns_ctx* c, void* a_v, void* a_o, int where) {
  if (!c || !a_v || !a_o) return fail(DNS_ERR_ARG, "null argument");
  if (where != DNS_HOST && where != DNS_DEVICE) return fail(DNS_ERR_ARG, "bad where");
  CK(cudaSetDevice(c->P.device));
  const long long NN = (long long)c->g.Ny * c->g.Ny, H = c->g.H;
  if (where == DNS_DEVICE) {
    CK(launch_operator_matrices(0, H, c->g, c->ph, c->T0, c->T2, c->T4, c->Ut, c->ddUt,
                                (double2*)a_v, (double2*)a_o, c->st));
    CK(cudaStreamSynchronize(c->st));
    return DNS_OK;
  }
  const long long batch = std::max(1LL, std::min<long long>(H, (1LL << 30) / (NN * 32)));
  double2 *dv = nullptr, *dO = nullptr;
  CK(cudaMalloc(&dv, (size_t)batch * NN * 16));
  if (cudaMalloc(&dO, (size_t)batch * NN * 16)) { cudaFree(dv); return fail(DNS_ERR_CUDA, "staging"); }
  cudaError_t e = cudaSuccess;
  for (long long p0 = 0; p0 < H && !e; p0 += batch) {
    const long long np = std::min(batch, H - p0);
    e = launch_operator_matrices(p0, np, c->g, c->ph, c->T0, c->T2, c->T4, c->Ut, c->ddUt, dv, dO, c->st);
    if (!e) e = cudaMemcpyAsync((double2*)a_v + p0 * NN, dv, (size_t)np * NN * 16, cudaMemcpyDeviceToHost, c->st);
    if (!e) e = cudaMemcpyAsync((double2*)a_o + p0 * NN, dO, (size_t)np * NN * 16, cudaMemcpyDeviceToHost, c->st);
    if (!e) e = cudaStreamSynchronize(c->st);
  }
  cudaFree(dv);
  cudaFree(dO);
  if (e) return fail(DNS_ERR_CUDA, cudaGetErrorString(e));
  return DNS_OK;
}

dns_status dns_check_state(dns_ctx* c) {
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c) return fail(DNS_ERR_ARG, "null context");
  if (!c->have_state) return fail(DNS_ERR_STATE, "no state to check");
  CK(cudaSetDevice(c->P.device));
  if (!c->probe) CK(c->alloc(&c->probe, 1));
  CK(cudaMemsetAsync(c->probe, 0, sizeof(int), c->st));
  CK(launch_nonfinite(c->V, c->O, c->g.H * c->g.nrun * c->g.Ny, c->probe, c->st));
  // the AB2 history too: it is written to recovery files, and a non-finite
  // nonlinear term reaches the state only one step later
  CK(launch_nonfinite(c->Nvp, c->Nop, c->g.H * c->g.nrun * c->g.Ny, c->probe, c->st));
  int bad = 0;
  CK(cudaMemcpyAsync(&bad, c->probe, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (bad) return fail(DNS_ERR_NONFINITE, "the state or the AB2 history holds NaN or Inf");
  return DNS_OK;
}

namespace {
// The solve-only sequence on the device: right-hand sides bv, bo (pitch bp,
// either may stand for a zero system) -> solutions into ov, oo (pitch op).
// Point values and their DCT-I go through the transform buffer F6, which the
// banded solve then takes as its scratch.
cudaError_t enqueue_solve_wall(dns_ctx* c, const double2* bv, const double2* bo, long long bp,
                               double2* Xv, double2* Xo, double2* pbc, double2* ov, double2* oo,
                               long long op) {
  const DnsGeom& g = c->g;
  const long long ls = c->P.mz / 2;  // no-padding DCT-I length 2N
  double2* sv = (double2*)c->F6;
  double2* so = sv + g.H * ls;
  const double* cosk = c->rtab + 4 * (size_t)c->wd.nv + 2 * (size_t)c->wd.no;
  // one kernel where the DCT length has a warp plan, else three
  cudaError_t e = launch_colloc_fused(bv, bo, bp, pbc, cosk, c->Ut, c->ddUt, c->rv, c->ro, c->wd, g, c->ph,
                                      c->fy0_d.tab(), c->status, c->st);
  if (e == cudaErrorNotSupported) {
    e = launch_colloc_prep(bv, bo, bp, sv, so, ls, pbc, cosk, c->Ut, c->ddUt, g, c->ph, c->st);
    if (!e) e = launch_cheby_inplace<double2>(PencilArr{sv, ls, 0}, 2 * g.H, 3, g.Ny, c->fy0_d.tab(), c->st);
    if (!e) e = launch_colloc_integrate(sv, so, ls, c->rv, c->ro, c->wd, g, c->st);
  }
  WallDims wd = c->wd;
  wd.tilt = 0;
  if (!e) e = launch_wall_solve(c->wfac, Xv, Xo, c->rv, c->ro, c->wQ, (double2*)c->F6, wd, g, c->ph,
                                c->status, c->st, c->variant[DNS_PASS_Y2]);
  if (e == cudaErrorNotSupported)
    e = launch_wall_solve(c->wfac, Xv, Xo, c->rv, c->ro, c->wQ, (double2*)c->F6, wd, g, c->ph, c->status, c->st,
                          DNS_Y2_RING2_8K_EF);
  if (!e) e = launch_colloc_finish(Xv, Xo, pbc, ov, oo, op, g, c->st);
  return e;
}
}  // namespace

dns_status dns_solve_wall(dns_ctx* c, void* v, void* omega, size_t tpitch, int where) {
  if (c && c->g.nrun > 1) return fail(DNS_ERR_STATE, "a batch context: this entry point takes one run");
  if (c && c->slab) return fail(DNS_ERR_STATE, "a slab rank's context: use dns_slab_local and dns_slab_part");
  if (!c || (!v && !omega)) return fail(DNS_ERR_ARG, "null argument");
  if (where != DNS_HOST && where != DNS_DEVICE) return fail(DNS_ERR_ARG, "bad where");
  const DnsGeom& g = c->g;
  const size_t row = (size_t)g.Ny * 16;
  if (tpitch % 16 || tpitch < row) return fail(DNS_ERR_ARG, "bad tpitch");
  CK(cudaSetDevice(c->P.device));
  dns_status s = build_wall_solver(c);
  if (s != DNS_OK) return s;
  if ((size_t)2 * g.H * (c->P.mz / 2) * 16 > c->F6_bytes)
    return fail(DNS_ERR_ARG, "solve-only DCT buffer does not fit the transform buffer");
  const size_t hn = (size_t)g.H * g.Ny;
  if (!c->solve_io) CK(c->alloc(&c->solve_io, 2 * hn + 6 * (size_t)g.H));
  double2* Xv = c->solve_io;
  double2* Xo = Xv + hn;
  double2* pbc = Xo + hn;
  if (where == DNS_DEVICE && v && omega) {
    // in place on the caller's device pencils: one captured graph per
    // (buffers, pitch), launched on every call
    if (!c->solve_graph || c->solve_key[0] != v || c->solve_key[1] != omega || c->solve_pitch != tpitch) {
      if (c->solve_graph) cudaGraphExecDestroy(c->solve_graph);
      c->solve_graph = nullptr;
      cudaGraph_t gr;
      CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
      cudaError_t e = enqueue_solve_wall(c, (const double2*)v, (const double2*)omega, (long long)(tpitch / 16),
                                         Xv, Xo, pbc, (double2*)v, (double2*)omega, (long long)(tpitch / 16));
      cudaError_t e2 = cudaStreamEndCapture(c->st, &gr);
      if (e) return fail(DNS_ERR_CUDA, std::string("solve capture: ") + cudaGetErrorString(e));
      CK(e2);
      CK(cudaGraphInstantiate(&c->solve_graph, gr, 0));
      cudaGraphDestroy(gr);
      c->solve_key[0] = v;
      c->solve_key[1] = omega;
      c->solve_pitch = tpitch;
    }
    CK(cudaGraphLaunch(c->solve_graph, c->st));
    return check_status(c);
  }
  // host buffers, or one system only: staged through Xv, Xo (pitch Ny); a
  // missing system is solved for a zero right-hand side and not written
  if (v) CK(cudaMemcpy2DAsync(Xv, row, v, tpitch, row, g.H, kind_of(where, true), c->st));
  else CK(cudaMemsetAsync(Xv, 0, hn * 16, c->st));
  if (omega) CK(cudaMemcpy2DAsync(Xo, row, omega, tpitch, row, g.H, kind_of(where, true), c->st));
  else CK(cudaMemsetAsync(Xo, 0, hn * 16, c->st));
  if (where == DNS_HOST) {
    CK(enqueue_solve_wall(c, Xv, Xo, g.Ny, Xv, Xo, pbc, Xv, Xo, g.Ny));
    if (v) CK(cudaMemcpy2DAsync(v, tpitch, Xv, row, row, g.H, cudaMemcpyDeviceToHost, c->st));
    if (omega) CK(cudaMemcpy2DAsync(omega, tpitch, Xo, row, row, g.H, cudaMemcpyDeviceToHost, c->st));
  } else {
    CK(enqueue_solve_wall(c, Xv, Xo, g.Ny, Xv, Xo, pbc, (double2*)v, (double2*)omega, (long long)(tpitch / 16)));
  }
  return check_status(c);
}

dns_status dns_solve_residual(dns_ctx* c, const void* bv, const void* bo, const void* xv, const void* xo,
                              size_t tpitch, int where, double out[6]) {
  if (!c || !bv || !bo || !xv || !xo || !out) return fail(DNS_ERR_ARG, "null argument");
  if (where != DNS_HOST && where != DNS_DEVICE) return fail(DNS_ERR_ARG, "bad where");
  const DnsGeom& g = c->g;
  const size_t row = (size_t)g.Ny * 16, hn = (size_t)g.H * g.Ny;
  if (tpitch % 16 || tpitch < row) return fail(DNS_ERR_ARG, "bad tpitch");
  CK(cudaSetDevice(c->P.device));
  double2* stage = nullptr;
  double* per = nullptr;
  const void* src[4] = {bv, bo, xv, xo};
  const double2* d[4];
  long long ps = (long long)(tpitch / 16);
  cudaError_t e = cudaMalloc(&per, (size_t)g.H * 6 * sizeof(double));
  if (!e && where == DNS_HOST) {
    e = cudaMalloc(&stage, 4 * hn * 16);
    for (int i = 0; i < 4 && !e; ++i) {
      e = cudaMemcpy2DAsync(stage + i * hn, row, src[i], tpitch, row, g.H, cudaMemcpyHostToDevice, c->st);
      d[i] = stage + i * hn;
    }
    ps = g.Ny;
  } else {
    for (int i = 0; i < 4; ++i) d[i] = (const double2*)src[i];
  }
  if (!e) e = launch_solve_residual(d[0], d[1], d[2], d[3], ps, g, c->ph, c->T0, c->T2, c->T4, c->Ut,
                                    c->ddUt, per, c->st);
  std::vector<double> h((size_t)g.H * 6);
  if (!e) e = cudaMemcpyAsync(h.data(), per, h.size() * 8, cudaMemcpyDeviceToHost, c->st);
  if (!e) e = cudaStreamSynchronize(c->st);
  cudaFree(per);
  cudaFree(stage);
  if (e) return fail(DNS_ERR_CUDA, cudaGetErrorString(e));
  // per pencil: |r_v|^2, |b_v|^2, |r_o|^2, |b_o|^2, backward error v, omega
  double rv = 0, bvn = 0, ro = 0, bon = 0, mv = 0, mo = 0, bwv = 0, bwo = 0;
  for (long long p = 0; p < g.H; ++p) {
    const double* q = &h[(size_t)p * 6];
    rv += q[0]; bvn += q[1]; ro += q[2]; bon += q[3];
    if (q[1] > 0) mv = std::max(mv, std::sqrt(q[0] / q[1]));
    if (q[3] > 0) mo = std::max(mo, std::sqrt(q[2] / q[3]));
    bwv = std::max(bwv, q[4]);
    bwo = std::max(bwo, q[5]);
  }
  out[0] = mv;
  out[1] = mo;
  out[2] = bvn > 0 ? std::sqrt(rv / bvn) : 0.0;
  out[3] = bon > 0 ? std::sqrt(ro / bon) : 0.0;
  out[4] = bwv;
  out[5] = bwo;
  return DNS_OK;
}

dns_status dns_init_aux_matrix(dns_ctx* c, void* inv_v, void* inv_o, int where) {
  if (!c || !inv_v || !inv_o) return fail(DNS_ERR_ARG, "null argument");
  if (where != DNS_HOST && where != DNS_DEVICE) return fail(DNS_ERR_ARG, "bad where");
  CK(cudaSetDevice(c->P.device));
  if (gj_cluster_size(c->g.Ny) < 0) return fail(DNS_ERR_ARG, "Ny too large for the operator inversion");
  const long long NN = (long long)c->g.Ny * c->g.Ny;
  if (where == DNS_DEVICE) {
    CK(launch_gj_invert(1, 0, c->g.H, c->g, c->ph, c->T0, c->T2, c->T4, c->Ut, c->ddUt, nullptr,
                        (double2*)inv_v, (double2*)inv_o, c->status, c->st));
    return check_status(c);
  }
  // host destination: invert in batches through a device staging buffer
  const long long batch = std::max(1LL, std::min<long long>(c->g.H, (1LL << 30) / (NN * 32)));
  double2 *dv = nullptr, *dO = nullptr;
  CK(cudaMalloc(&dv, (size_t)batch * NN * 16));
  if (cudaMalloc(&dO, (size_t)batch * NN * 16)) { cudaFree(dv); return fail(DNS_ERR_CUDA, "staging"); }
  dns_status s = DNS_OK;
  for (long long u0 = 0; u0 < c->g.H && s == DNS_OK; u0 += batch) {
    const long long nu = std::min(batch, c->g.H - u0);
    cudaError_t e = launch_gj_invert(1, u0, nu, c->g, c->ph, c->T0, c->T2, c->T4, c->Ut, c->ddUt,
                                     nullptr, dv, dO, c->status, c->st);
    if (!e) e = cudaMemcpyAsync((double2*)inv_v + u0 * NN, dv, (size_t)nu * NN * 16, cudaMemcpyDeviceToHost, c->st);
    if (!e) e = cudaMemcpyAsync((double2*)inv_o + u0 * NN, dO, (size_t)nu * NN * 16, cudaMemcpyDeviceToHost, c->st);
    if (e) s = fail(DNS_ERR_CUDA, cudaGetErrorString(e));
    else s = check_status(c);
  }
  cudaFree(dv);
  cudaFree(dO);
  return s;
}

}  // extern "C"
