// The slab-decomposed time step: one context per rank (dns_slab_create),
// each holding only the pencils of its operator slots and the wall-normal
// planes it transforms, and a step in three parts with the two exchanges of
// the slab plan (slab.cpp) between them:
//
//   part DNS_SLAB_Y3  y3 on the rank's pencil runs (all Py planes), then the
//                     six fields packed for the plane owners;
//   (exchange 0)      the caller moves the packed blocks: NCCL all-to-all
//                     over NVLink, or copies on one device;
//   part DNS_SLAB_XZ  unpack into plane-local pencils (every pencil, the
//                     rank's planes), zb, x (base flow of those planes), zf,
//                     the three Lamb fields packed back for the pencil owners;
//   (exchange 1)
//   part DNS_SLAB_Y1  unpack into the rank's pencils (all planes), y1 on its
//                     runs, the banded solve of its slots (factors of its
//                     slots only).
//
// The kernels are the whole-grid kernels launched on sub-ranges: the
// wall-normal passes per run of pencils (DnsGeom::kz0 gives the run's first
// spanwise index, the data pointers its first local row), the spanwise and
// streamwise passes on a geometry of ny planes.  Packed layout (the same at
// both ends): per peer, per field, the peer's segments in plan order, each
// a block [pencil][plane].  No counterpart in the reference, whose
// multi-GPU transform is dead code (source/transform_multi_gpu.cpp).
#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "context_impl.cuh"
#include "ypass.cuh"
#include "zxpass.cuh"

namespace {

dns_status sfail(dns_status s, const std::string& m) { return dns_internal_fail(s, m.c_str()); }
#define SCK(x)                                                                   \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess) return sfail(DNS_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

// nf x npen rows of `words` 8-byte words: row (f, i) from src + f s_fs + i s_ps
// to dst + f d_fs + i d_ps (strides in words); a warp per row
__global__ void __launch_bounds__(128) k_copy_rows(const unsigned long long* __restrict__ src, long long s_fs,
                                                   long long s_ps, unsigned long long* __restrict__ dst,
                                                   long long d_fs, long long d_ps, long long npen, int words) {
  const int f = blockIdx.y;
  const long long i = (long long)blockIdx.x * 4 + (threadIdx.x >> 5);
  if (i >= npen) return;
  const unsigned long long* a = src + f * s_fs + i * s_ps;
  unsigned long long* b = dst + f * d_fs + i * d_ps;
  for (int w = threadIdx.x & 31; w < words; w += 32) b[w] = a[w];
}

cudaError_t copy_rows(const void* src, long long s_fs, long long s_ps, void* dst, long long d_fs, long long d_ps,
                      int nf, long long npen, int words, cudaStream_t st) {
  if (nf <= 0 || npen <= 0 || words <= 0) return cudaSuccess;
  dim3 grid((unsigned)((npen + 3) / 4), (unsigned)nf);
  k_copy_rows<<<grid, 128, 0, st>>>((const unsigned long long*)src, s_fs, s_ps, (unsigned long long*)dst, d_fs,
                                     d_ps, npen, words);
  return cudaGetLastError();
}

size_t elem_bytes(const dns_ctx* c) { return c->P.precision == DNS_PREC_MIXED ? 8 : 16; }

// words of one field's blocks for a peer: sum over its segments of npen ny
long long field_words(const dns_ctx* c, const std::vector<dns_slab_segment>& segs, int peer) {
  long long w = 0;
  for (const auto& sg : segs)
    if (sg.peer == peer) w += (long long)sg.nkz * c->g.Kx * sg.ny;
  return w * (long long)(elem_bytes(c) / 8);
}

// Pack (to_buf) or unpack a set of segments between the packed buffer and
// the pencil arrays at `arr` [field][pencil][plane] (pitch aps, field stride
// afs, elements).  by_rows: the pencil rows of a segment are the pencil
// owner's local rows (local_row0 ..) and its planes start at the segment's
// y0; else they are the global pencils kz0 Kx .. and the planes start at 0.
cudaError_t move_segments(const dns_ctx* c, const std::vector<dns_slab_segment>& segs, int nf, void* buf,
                          void* arr, long long aps, long long afs, bool by_rows, bool to_buf) {
  const SlabState& S = *c->slab;
  const long long m = (long long)(elem_bytes(c) / 8);
  long long peer_off = 0;
  for (int peer = 0; peer < S.R; ++peer) {
    const long long fw = field_words(c, segs, peer);
    long long seg_off = 0;
    for (const auto& sg : segs) {
      if (sg.peer != peer) continue;
      const long long npen = (long long)sg.nkz * c->g.Kx;
      const long long row = by_rows ? sg.local_row0 : (long long)sg.kz0 * c->g.Kx;
      const long long y = by_rows ? sg.y0 : 0;
      unsigned long long* b = (unsigned long long*)buf + peer_off + seg_off;
      unsigned long long* a = (unsigned long long*)arr + (row * aps + y) * m;
      cudaError_t e = to_buf ? copy_rows(a, afs * m, aps * m, b, fw, sg.ny * m, nf, npen, (int)(sg.ny * m), c->st)
                             : copy_rows(b, fw, sg.ny * m, a, afs * m, aps * m, nf, npen, (int)(sg.ny * m), c->st);
      if (e) return e;
      seg_off += npen * sg.ny * m;
    }
    peer_off += nf * fw;
  }
  return cudaSuccess;
}

template <typename C>
cudaError_t part_y3(dns_ctx* c, void* send) {
  SlabState& S = *c->slab;
  const DnsGeom& g = c->g;
  const DevFft<C>& fyP = *(const DevFft<C>*)(std::is_same<C, float2>::value ? (const void*)&c->fyP_f
                                                                             : (const void*)&c->fyP_d);
  for (int k = 0; k < S.nruns; ++k) {
    const SlabRun& run = S.run[k];
    DnsGeom gs = g;
    gs.H = (long long)run.nkz * g.Kx;
    gs.kz0 = run.kz0;
    const double2* V = c->V + run.row0 * g.Ny;
    const double2* O = c->O + run.row0 * g.Ny;
    PencilArr out{(C*)c->F6 + run.row0 * c->PyS, c->PyS, S.np * c->PyS};
    cudaError_t e;
    if (std::is_same<C, float2>::value && c->variant[DNS_PASS_Y3] == DNS_Y3_TENSOR) {
      e = launch_y3tc(V, O, out, gs, c->ph, c->y3tc_tab, c->status, c->st);
    } else {
      e = launch_y3<C>(V, O, out, gs, c->ph, fyP.tab(), c->status, c->st, c->variant[DNS_PASS_Y3]);
      if (e == cudaErrorNotSupported) e = launch_y3<C>(V, O, out, gs, c->ph, fyP.tab(), c->status, c->st);
    }
    if (e) return e;
  }
  return move_segments(c, S.segP, 6, send, c->F6, c->PyS, S.np * c->PyS, true, true);
}

template <typename C>
cudaError_t part_xz(dns_ctx* c, const void* recv, void* send) {
  SlabState& S = *c->slab;
  const DnsGeom& g = c->g;
  const bool mixed = std::is_same<C, float2>::value;
  const DevFft<C>& fz = *(const DevFft<C>*)(mixed ? (const void*)&c->fz_f : (const void*)&c->fz_d);
  const DevFft<C>& fx = *(const DevFft<C>*)(mixed ? (const void*)&c->fx_f : (const void*)&c->fx_d);
  cudaError_t e = move_segments(c, S.segY, 6, (void*)recv, S.A, S.nyS, g.H * S.nyS, false, false);
  if (e) return e;
  DnsGeom gs = g;
  gs.Py = S.ny;
  const long long rows = (long long)S.ny * g.Pz * c->KxS;
  PencilArr Q6{S.A, S.nyS, g.H * S.nyS};
  RowArr R6{c->G6, c->KxS, rows};
  RowArr R3{S.A, c->KxS, rows};
  PencilArr Q3{c->G6, S.nyS, g.H * S.nyS};
  e = launch_zb<C>(Q6, R6, 6, gs, fz.tab(), c->st, c->status, c->variant[DNS_PASS_ZB]);
  if (e == cudaErrorNotSupported) e = launch_zb<C>(Q6, R6, 6, gs, fz.tab(), c->st, c->status);
  if (!e) {
    e = launch_x_fused<C>(R6, R3, gs, fx.tab(), c->Uy + S.y0, c->ph.Ro, c->status, c->st, c->variant[DNS_PASS_X]);
    if (e == cudaErrorNotSupported) e = launch_x_fused<C>(R6, R3, gs, fx.tab(), c->Uy + S.y0, c->ph.Ro, c->status, c->st);
  }
  if (!e) {
    e = launch_zf<C>(R3, Q3, 3, gs, fz.tab(), c->st, c->status, c->variant[DNS_PASS_ZF]);
    if (e == cudaErrorNotSupported) e = launch_zf<C>(R3, Q3, 3, gs, fz.tab(), c->st, c->status);
  }
  if (!e) e = move_segments(c, S.segY, 3, send, c->G6, S.nyS, g.H * S.nyS, false, true);
  return e;
}

template <typename C>
cudaError_t part_y1(dns_ctx* c, int boot, const void* recv) {
  SlabState& S = *c->slab;
  const DnsGeom& g = c->g;
  const DevFft<C>& fyP = *(const DevFft<C>*)(std::is_same<C, float2>::value ? (const void*)&c->fyP_f
                                                                             : (const void*)&c->fyP_d);
  cudaError_t e = move_segments(c, S.segP, 3, (void*)recv, c->F6, c->PyS, S.np * c->PyS, true, false);
  if (e) return e;
  const RhsDims rd{c->wd.nv, c->wd.no, c->wd.gp};
  const size_t nv = c->wd.nv, no = c->wd.no;
  const double* t0 = c->rtab;
  const RhsTabs tb{t0, t0 + 4 * nv, t0 + 4 * nv + 2 * no, t0 + 4 * nv + 2 * no + g.Ny,
                   t0 + 4 * nv + 2 * no + g.Ny + 5 * nv};
  for (int k = 0; k < S.nruns && !e; ++k) {
    const SlabRun& run = S.run[k];
    DnsGeom gs = g;
    gs.H = (long long)run.nkz * g.Kx;
    gs.kz0 = run.kz0;
    const long long o = run.row0 * g.Ny, og = run.row0 * c->wd.gp;
    PencilArr lam{(C*)c->F6 + run.row0 * c->PyS, c->PyS, S.np * c->PyS};
    auto go = [&](int v) {
      return launch_y1<C>(lam, c->V + o, c->O + o, c->Nvp + o, c->Nop + o, c->rv + og, c->ro + og, rd, tb, gs,
                          c->ph, fyP.tab(), boot, c->status, c->st, v);
    };
    e = go(c->variant[DNS_PASS_Y1]);
    if (e == cudaErrorNotSupported) e = go(VAR_AUTO);
  }
  if (!e && !boot) {
    e = launch_wall_solve(c->wfac, c->V, c->O, c->rv, c->ro, c->wQ, (double2*)c->F6, c->wd, g, c->ph, c->status,
                          c->st, c->variant[DNS_PASS_Y2]);
    if (e == cudaErrorNotSupported)
      e = launch_wall_solve(c->wfac, c->V, c->O, c->rv, c->ro, c->wQ, (double2*)c->F6, c->wd, g, c->ph,
                            c->status, c->st, DNS_Y2_RING2_8K_EF);
  }
  return e;
}

}  // namespace

extern "C" {

dns_status dns_slab_create(const dns_params* p, int nranks, int rank, dns_ctx** out) {
  if (!p || !out) return sfail(DNS_ERR_ARG, "null argument");
  *out = nullptr;
  int rg[5];
  dns_status s = dns_slab_ranges(p->mx, p->my, p->mz, nranks, rank, rg);
  if (s != DNS_OK) return s;
  std::unique_ptr<SlabState> S(new SlabState());
  S->R = nranks;
  S->r = rank;
  S->s0 = rg[0];
  S->s1 = rg[1];
  S->y0 = rg[2];
  S->ny = rg[3] - rg[2];
  S->nyS = (S->ny + 1) & ~1;  // even: 16-byte pencil pitch in the mixed form
  S->np = rg[4];
  int kz0[2], nkz[2];
  long long row0[2];
  S->nruns = slab_runs(p->mx, p->my, p->mz, nranks, rank, kz0, nkz, row0);
  if (S->nruns < 1 || S->ny < 1) return sfail(DNS_ERR_ARG, "slab rank without pencils or planes");
  for (int i = 0; i < S->nruns; ++i) S->run[i] = SlabRun{kz0[i], nkz[i], row0[i]};
  for (int role = 0; role < 2; ++role) {
    int n = 0;
    if ((s = dns_slab_segments(p->mx, p->my, p->mz, nranks, rank, role, nullptr, 0, &n)) != DNS_OK) return s;
    std::vector<dns_slab_segment>& v = role == DNS_SLAB_PENCILS ? S->segP : S->segY;
    v.resize(n);
    if ((s = dns_slab_segments(p->mx, p->my, p->mz, nranks, rank, role, v.data(), n, &n)) != DNS_OK) return s;
  }
  // bytes per peer: backward exchange 6 fields, forward 3, in the
  // transform precision
  const DnsGeom g = dns_make_geom(p->mx, p->my, p->mz);
  const size_t esz = p->precision == DNS_PREC_MIXED ? 8 : 16;
  for (int x = 0; x < 2; ++x) {
    S->sendB[x].assign(nranks, 0);
    S->recvB[x].assign(nranks, 0);
  }
  for (const auto& sg : S->segP) {
    const size_t b = (size_t)sg.nkz * g.Kx * sg.ny * esz;
    S->sendB[0][sg.peer] += 6 * b;
    S->recvB[1][sg.peer] += 3 * b;
  }
  for (const auto& sg : S->segY) {
    const size_t b = (size_t)sg.nkz * g.Kx * sg.ny * esz;
    S->recvB[0][sg.peer] += 6 * b;
    S->sendB[1][sg.peer] += 3 * b;
  }
  return ctx_create(p, S.release(), out);
}

dns_status dns_slab_exchange_bytes(const dns_ctx* c, int exchange, size_t* send, size_t* recv) {
  if (!c || !send || !recv) return sfail(DNS_ERR_ARG, "null argument");
  if (!c->slab) return sfail(DNS_ERR_ARG, "not a slab rank's context");
  if (exchange != 0 && exchange != 1) return sfail(DNS_ERR_ARG, "exchange must be 0 or 1");
  for (int i = 0; i < c->slab->R; ++i) {
    send[i] = c->slab->sendB[exchange][i];
    recv[i] = c->slab->recvB[exchange][i];
  }
  return DNS_OK;
}

dns_status dns_slab_local(dns_ctx* c, int which, void* buf, int where, int to_ctx) {
  if (!c || !buf) return sfail(DNS_ERR_ARG, "null argument");
  if (!c->slab) return sfail(DNS_ERR_ARG, "not a slab rank's context");
  if (which < DNS_SLAB_V || which > DNS_SLAB_NOMEGA) return sfail(DNS_ERR_ARG, "unknown array");
  if (where != DNS_HOST && where != DNS_DEVICE) return sfail(DNS_ERR_ARG, "bad where");
  SCK(cudaSetDevice(c->P.device));
  double2* arr[4] = {c->V, c->O, c->Nvp, c->Nop};
  const size_t bytes = (size_t)c->slab->np * c->g.Ny * 16;
  cudaMemcpyKind kind = where == DNS_DEVICE ? cudaMemcpyDeviceToDevice
                                            : (to_ctx ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost);
  if (to_ctx) SCK(cudaMemcpyAsync(arr[which], buf, bytes, kind, c->st));
  else SCK(cudaMemcpyAsync(buf, arr[which], bytes, kind, c->st));
  SCK(cudaStreamSynchronize(c->st));
  if (to_ctx && which <= DNS_SLAB_OMEGA) c->have_state = true;
  if (to_ctx && which >= DNS_SLAB_NV) c->booted = true;
  return DNS_OK;
}

dns_status dns_slab_part(dns_ctx* c, int part, int boot, void* send, const void* recv) {
  if (!c) return sfail(DNS_ERR_ARG, "null context");
  if (!c->slab) return sfail(DNS_ERR_ARG, "not a slab rank's context");
  if (part < DNS_SLAB_Y3 || part > DNS_SLAB_Y1) return sfail(DNS_ERR_ARG, "unknown part");
  if ((part != DNS_SLAB_Y1 && !send) || (part != DNS_SLAB_Y3 && !recv))
    return sfail(DNS_ERR_ARG, "missing exchange buffer");
  if (!c->have_state) return sfail(DNS_ERR_STATE, "the rank's state must be set first");
  if (part == DNS_SLAB_Y1 && !boot && !c->booted) return sfail(DNS_ERR_STATE, "bootstrap first (boot = 1)");
  SCK(cudaSetDevice(c->P.device));
  dns_status s = DNS_OK;
  if (part == DNS_SLAB_Y1 && !boot && (s = ctx_build_wall_solver(c)) != DNS_OK) return s;
  const bool mixed = c->P.precision == DNS_PREC_MIXED;
  cudaError_t e = cudaSuccess;
  switch (part) {
    case DNS_SLAB_Y3: e = mixed ? part_y3<float2>(c, send) : part_y3<double2>(c, send); break;
    case DNS_SLAB_XZ: e = mixed ? part_xz<float2>(c, recv, send) : part_xz<double2>(c, recv, send); break;
    case DNS_SLAB_Y1: e = mixed ? part_y1<float2>(c, boot, recv) : part_y1<double2>(c, boot, recv); break;
  }
  if (e) return sfail(DNS_ERR_CUDA, std::string("slab part: ") + cudaGetErrorString(e));
  if (part == DNS_SLAB_Y1 && boot) c->booted = true;
  return DNS_OK;
}

}  // extern "C"
