// Per-step wall-normal solves (the y2 kernel): v solve, tilting term,
// omega_y solve, for every Fourier mode, on the banded integrated systems of
// wallsolve.h.  Replaces the reference's explicit-inverse products
// (source/solver.cpp:107-123, matrix_op.cpp:68-78) and the tilting term of
// _get_linear_omega_y (source/linear.cpp:147-151).
//
// One CTA = one warp = a group of 16 operator slots; lane 2q + b handles
// pencil b (kz' or Nz - kz') of slot q, both pencils sharing the slot's
// factors.  The factors of a group are stored as one contiguous stream in
// the order the solve reads them (v forward rows, v backward rows, omega
// forward rows, omega backward rows; each row holds its entries for the 16
// slots side by side), and are streamed through a shared-memory ring with
// cp.async.bulk and mbarriers.  Each lane keeps its intermediate solution
// and tilting term in one column of a global scratch of the group (rows
// interleaved over the lanes, L2-resident, read two ring chunks ahead into
// registers), so that a CTA needs only the ring and two small tables in
// shared memory and several CTAs share an SM.
//
// Inputs from the y1 kernel: g_v, g_o (rows K.. of the integrated
// collocation right-hand sides, the v^n part of the tilting term included).
// Outputs: V, O (Chebyshev coefficients of v^{n+1}, omega_y^{n+1}).
#include "kernels.cuh"
#include "mbar.cuh"
#include "wallsolve_dev.cuh"

#define WALL_WAIT_LIMIT (1LL << 31)

namespace {

constexpr int WALL_HDR = 128;        // mbarriers

// Variants (the solve's tunable block shape): ring stages, bytes per stage,
// whether the tilting table sits in shared memory (else read through L1),
// and whether the factor stream is read with the L2 evict-first policy (the
// scratch vectors then stay in L2).  Smaller rings leave room for more CTAs
// per SM.
struct WallVar {
  int nst, stg;
  bool qsm, ef;
};
constexpr WallVar kWallVar[DNS_WALL_VARIANTS] = {
    {3, 12288, true, false}, {3, 12288, true, true}, {2, 8192, false, true}, {3, 8192, false, true}};

__host__ __device__ constexpr int rows_per_chunk(int stg, int entries, int cap) {
  return (stg / (entries * 256)) < cap ? (stg / (entries * 256)) : cap;
}

__device__ __forceinline__ double2 sel(bool p, double2 a) { return p ? a : make_double2(0.0, 0.0); }

template <int KLV, int KUV, int KLO, int KUO, int STG>
struct WallCfg {
  static constexpr int E0 = KLV, E1 = 1 + KUV + 2, E2 = KLO, E3 = 1 + KUO;
  // rows per ring chunk; the solve keeps two chunks of vector rows in registers
  static constexpr int R0 = rows_per_chunk(STG, E0, 12), R1 = rows_per_chunk(STG, E1, 12);
  static constexpr int R2 = rows_per_chunk(STG, E2, 8), R3 = rows_per_chunk(STG, E3, 12);
  static_assert(R0 > 0 && R1 > 0 && R2 > 0 && R3 > 0, "stage too small for a row");
};

// chunk c of a group's stream: byte count and offset (complex values)
template <class CF>
__device__ __forceinline__ void chunk_of(int c, const WallDims& wd, uint32_t& bytes, long long& off) {
  const int n0 = (wd.nv + CF::R0 - 1) / CF::R0, n1 = (wd.nv + CF::R1 - 1) / CF::R1;
  const int n2 = (wd.no + CF::R2 - 1) / CF::R2;
  long long base;
  int r0, rows, E;
  if (c < n0) {
    base = 0; E = CF::E0; r0 = c * CF::R0; rows = min(CF::R0, wd.nv - r0);
  } else if (c < n0 + n1) {
    base = 16LL * wd.nv * CF::E0; E = CF::E1; r0 = (c - n0) * CF::R1; rows = min(CF::R1, wd.nv - r0);
  } else if (c < n0 + n1 + n2) {
    base = 16LL * wd.nv * (CF::E0 + CF::E1); E = CF::E2; r0 = (c - n0 - n1) * CF::R2;
    rows = min(CF::R2, wd.no - r0);
  } else {
    base = 16LL * (wd.nv * (CF::E0 + CF::E1) + wd.no * CF::E2); E = CF::E3;
    r0 = (c - n0 - n1 - n2) * CF::R3; rows = min(CF::R3, wd.no - r0);
  }
  off = base + 16LL * r0 * E;
  bytes = (uint32_t)(rows * E * 256);
}

}  // namespace

template <int KLV, int KUV, int KLO, int KUO, int WALL_NST, int WALL_STG, bool QSM, bool EF>
__global__ void __launch_bounds__(32) k_wall_solve(const double2* __restrict__ fac, double2* V,
                                                   double2* O, const double2* __restrict__ gv,
                                                   const double2* __restrict__ go,
                                                   const double* __restrict__ Qg, double2* Sw,
                                                   WallDims wd, DnsGeom g, PhysParams ph, int* status) {
  typedef WallCfg<KLV, KUV, KLO, KUO, WALL_STG> CF;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* full = (uint64_t*)smem_raw;
  double2* ring = (double2*)(smem_raw + WALL_HDR);
  double* Qsm = (double*)(smem_raw + WALL_HDR + WALL_NST * WALL_STG);
  const double* Qs = QSM ? Qsm : Qg;  // tilting table: shared memory or through L1
  // recombination weights 2k/(k+1), (k-3)/(k-1) of the clamped basis, k <= N
  double* rc2 = Qsm + (QSM ? wd.qbytes / 8 : 0);
  double* rc4 = rc2 + g.Ny;

  const int lane = threadIdx.x;
  const int q = lane >> 1, b = lane & 1;
  // member of a batch (its groups are consecutive CTAs)
  const long long gpr = wd.groups_per_run > 0 ? wd.groups_per_run : (long long)gridDim.x;
  const int run = (int)(blockIdx.x / gpr);
  const long long slot = ((long long)blockIdx.x - run * gpr) * 16 + q;
  const bool valid = slot < wd.nslots;
  const int kx = valid ? (int)(slot % g.Kx) : 0;
  const int kzs = valid ? wd.kzs0 + (int)(slot / g.Kx) : 0;
  const int npen = (kzs == 0 || kzs == g.Nz / 2) ? 1 : 2;
  const bool active = valid && b < npen;
  const int kz = (b == 0) ? kzs : g.Nz - kzs;
  const long long pen = (long long)run * g.Hrun +
                        ((b == 0) ? wd.rowa + (long long)(kz - wd.kza) * g.Kx + kx
                                  : wd.rowb + (long long)(kz - wd.kzb) * g.Kx + kx);
  const bool zero = valid && kzs == 0 && kx == 0;
  double ia, ib;
  wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
  const double kap = (zero || !wd.tilt) ? 0.0 : -0.5 * ib * run_dt(ph, run);  // tilting weight of this pencil
  const int N = g.Ny - 1, Ny = g.Ny;
  // this lane's vector (right-hand side, intermediate solution, tilting
  // term) in the group's scratch, rows interleaved over the 32 lanes: a
  // row of the warp is one contiguous 512-byte access
  double2* S = Sw + (long long)blockIdx.x * 32 * wd.nv + lane;
  const double2 z2 = make_double2(0.0, 0.0);
  const double2* gfac = fac + (long long)blockIdx.x * wd.group_complex;
  const int nch0 = (wd.nv + CF::R0 - 1) / CF::R0, nch1 = (wd.nv + CF::R1 - 1) / CF::R1;
  const int nch2 = (wd.no + CF::R2 - 1) / CF::R2, nch3 = (wd.no + CF::R3 - 1) / CF::R3;
  const int total = nch0 + nch1 + nch2 + nch3;

  const uint64_t pol = EF ? l2_evict_first() : 0;
  auto issue = [&](int c) {
    uint32_t bytes;
    long long off;
    chunk_of<CF>(c, wd, bytes, off);
    uint64_t* bar = &full[c % WALL_NST];
    mbar_expect_tx(bar, bytes);
    if (EF) bulk_g2s_hint(ring + (size_t)(c % WALL_NST) * (WALL_STG / 16), gfac + off, bytes, bar, pol);
    else bulk_g2s(ring + (size_t)(c % WALL_NST) * (WALL_STG / 16), gfac + off, bytes, bar);
  };
  // on a timed-out wait: report, let the copies in flight land, leave
  auto abort_at = [&](int c) {
    if (lane == 0) {
      atomicOr(status, 1);
      for (int cc = c; cc < min(c + WALL_NST, total); ++cc)
        mbar_wait_bounded(&full[cc % WALL_NST], (uint32_t)((cc / WALL_NST) & 1), WALL_WAIT_LIMIT, nullptr);
    }
  };
  auto wait_chunk = [&](int c) {
    const bool ok = mbar_wait_bounded(&full[c % WALL_NST], (uint32_t)((c / WALL_NST) & 1),
                                      WALL_WAIT_LIMIT, status);
    return __all_sync(0xffffffffu, ok);
  };
  auto release = [&](int c) {
    __syncwarp();
    if (lane == 0 && c + WALL_NST < total) {
      fence_proxy_async();
      issue(c + WALL_NST);
    }
  };
  // scratch rows (plain loads: the kernel writes them) and right-hand sides
  auto lds = [&](int i) { return (i >= 0 && i < wd.nv) ? S[32 * i] : z2; };
  const double2* gvp = gv + pen * wd.gp;
  const double2* gop = go + pen * wd.gp;

  // ---- start: barriers, ring prefetch, tables ----------------------------
  if (lane == 0) {
    for (int s = 0; s < WALL_NST; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  __syncwarp();
  if (QSM)
    for (int k = lane; k < 7 * wd.no; k += 32) Qsm[k] = Qg[k];
  for (int k = lane; k < g.Ny; k += 32) {
    rc2[k] = 2.0 * k / (k + 1);
    rc4[k] = (k >= 4) ? (double)(k - 3) / (double)(k - 1) : 0.0;
  }
  if (lane == 0)
    for (int c = 0; c < min(WALL_NST, total); ++c) issue(c);
  __syncwarp();

  int c = 0;
  // ---- v: forward substitution (unit lower band) -------------------------
  // the right-hand side rows of each chunk are loaded one chunk ahead
  {
    constexpr int R = CF::R0;
    double2 yw[KLV];
#pragma unroll
    for (int e = 0; e < KLV; ++e) yw[e] = z2;
    double2 nxt[R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) nxt[rr] = (active && rr < wd.nv) ? __ldg(gvp + rr) : z2;
    for (int r0 = 0; r0 < wd.nv; r0 += R, ++c) {
      double2 cur[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        cur[rr] = nxt[rr];
        const int i = r0 + R + rr;
        nxt[rr] = (active && i < wd.nv) ? __ldg(gvp + i) : z2;
      }
      if (!wait_chunk(c)) { abort_at(c); return; }
      const double2* ch = ring + (size_t)(c % WALL_NST) * (WALL_STG / 16) + q;
      const int rows = min(R, wd.nv - r0);
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        if (rr < rows) {
          const int i = r0 + rr;
          const double2* Lr = ch + rr * CF::E0 * 16;
          // the older entries in independent partial sums; the newest
          // (y_{i-1}) last, so only it is on the row-to-row critical path
          double2 a0 = cur[rr], a1 = z2;
#pragma unroll
          for (int e = 0; e < KLV - 1; ++e) {
            if (e & 1) a1 = a1 + cmul(Lr[e * 16], yw[e]);
            else a0 = a0 - cmul(Lr[e * 16], yw[e]);
          }
          const double2 acc = (a0 - a1) - cmul(Lr[(KLV - 1) * 16], yw[KLV - 1]);
          S[32 * i] = acc;
#pragma unroll
          for (int e = 0; e < KLV - 1; ++e) yw[e] = yw[e + 1];
          yw[KLV - 1] = acc;
        }
      }
      release(c);
    }
  }
  // ---- v: back substitution, recombination, tilting term -----------------
  // rows descend; a chunk's rows are loaded one chunk ahead.  The tilting
  // term of row k+1 is written over rows already consumed (k + 1 > i).
  {
    constexpr int R = CF::R1;
    double2 xw[KUV];
#pragma unroll
    for (int e = 0; e < KUV; ++e) xw[e] = z2;
    double2 xd0 = z2, xd1 = z2;
    double2 P[7];  // P[j]: partial tilting sum of row k+1-j, k = next coefficient emitted
#pragma unroll
    for (int j = 0; j < 7; ++j) P[j] = z2;
    const int nbv = zero ? N - 1 : N - 3;
    // base-flow degree (KLV = deg U + 4): U' = U1 (degree 1) makes the
    // tilting operator B^2 U1, three diagonals; U' = 0 (degree 0) none
    constexpr int DEG = KLV - 4;
    auto emit = [&](int k, double2 a) {
      if (active) V[pen * Ny + k] = a;
#pragma unroll
      for (int j = 0; j < 7; ++j) {
        if (DEG == 0 || (DEG == 1 && (j & 1) == 0)) continue;
        const int r = k + 1 - j;
        if (r >= 0 && r < wd.no) P[j] = P[j] + a * (QSM ? Qs[7 * r + j] : __ldg(Qs + 7 * r + j));
      }
      if (k + 1 < wd.no) S[32 * (k + 1)] = muli(P[0] * kap);
#pragma unroll
      for (int j = 0; j < 6; ++j) P[j] = P[j + 1];
      P[6] = z2;
    };
    double2 nxt[R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) nxt[rr] = lds(wd.nv - 1 - rr);
    for (int r0 = 0; r0 < wd.nv; r0 += R, ++c) {
      double2 cur[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        cur[rr] = nxt[rr];
        nxt[rr] = lds(wd.nv - 1 - (r0 + R + rr));
      }
      if (!wait_chunk(c)) { abort_at(c); return; }
      const double2* ch = ring + (size_t)(c % WALL_NST) * (WALL_STG / 16) + q;
      const int rows = min(R, wd.nv - r0);
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        if (rr < rows) {
          const int i = wd.nv - 1 - (r0 + rr);
          const double2* Ur = ch + rr * CF::E1 * 16;
          const double2 a0 = cur[rr];
          if (i >= N + 2) S[32 * i] = z2;  // no tilting term above row N+1
          // independent partial sums; x_{i+1} enters last
          double2 a1 = cmul(Ur[(KUV + 1) * 16], xd0) + cmul(Ur[(KUV + 2) * 16], xd1);
          double2 a2 = z2;
#pragma unroll
          for (int e = KUV; e >= 2; --e) {
            if (e & 1) a1 = a1 + cmul(Ur[e * 16], xw[e - 1]);
            else a2 = a2 + cmul(Ur[e * 16], xw[e - 1]);
          }
          const double2 acc = (a0 - (a1 + a2)) - cmul(Ur[16], xw[0]);
          const double2 x = cmul(Ur[0], acc);
          if (i == wd.nv - 1) xd1 = x;
          if (i == wd.nv - 2) xd0 = x;
#pragma unroll
          for (int e = KUV - 1; e >= 1; --e) xw[e] = xw[e - 1];
          xw[0] = x;
          if (i < nbv) {
            if (!zero) {
              const int k = i + 4;
              emit(k, sel(i + 4 < nbv, xw[4]) - sel(i + 2 < nbv, xw[2]) * rc2[k] + x * rc4[k]);
            } else {
              emit(i + 2, x - sel(i + 2 < nbv, xw[2]));
            }
          }
        }
      }
      release(c);
    }
    if (!zero) {
      emit(3, xw[3] - xw[1] * 1.5);
      emit(2, xw[2] - xw[0] * (4.0 / 3.0));
      emit(1, xw[1]);
      emit(0, xw[0]);
    } else {
      emit(1, make_double2(-xw[1].x, -xw[1].y));
      emit(0, make_double2(-xw[0].x, -xw[0].y));
    }
    S[0] = muli(P[0] * kap);
  }
  // ---- omega: forward substitution (adds g_o to the tilting term) --------
  {
    constexpr int R = CF::R2;
    double2 ow[KLO];
#pragma unroll
    for (int e = 0; e < KLO; ++e) ow[e] = z2;
    double2 gnext[R], snext[R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      gnext[rr] = (active && rr < wd.no) ? __ldg(gop + rr) : z2;
      snext[rr] = (rr < wd.no) ? lds(rr) : z2;
    }
    for (int r0 = 0; r0 < wd.no; r0 += R, ++c) {
      double2 gcur[R], scur[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        gcur[rr] = gnext[rr];
        scur[rr] = snext[rr];
        const int i = r0 + R + rr;
        gnext[rr] = (active && i < wd.no) ? __ldg(gop + i) : z2;
        snext[rr] = (i < wd.no) ? lds(i) : z2;
      }
      if (!wait_chunk(c)) { abort_at(c); return; }
      const double2* ch = ring + (size_t)(c % WALL_NST) * (WALL_STG / 16) + q;
      const int rows = min(R, wd.no - r0);
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        if (rr < rows) {
          const int i = r0 + rr;
          const double2* Lr = ch + rr * CF::E2 * 16;
          double2 a0 = scur[rr] + gcur[rr], a1 = z2;
#pragma unroll
          for (int e = 0; e < KLO - 1; ++e) {
            if (e & 1) a1 = a1 + cmul(Lr[e * 16], ow[e]);
            else a0 = a0 - cmul(Lr[e * 16], ow[e]);
          }
          const double2 acc = (a0 - a1) - cmul(Lr[(KLO - 1) * 16], ow[KLO - 1]);
          S[32 * i] = acc;
#pragma unroll
          for (int e = 0; e < KLO - 1; ++e) ow[e] = ow[e + 1];
          ow[KLO - 1] = acc;
        }
      }
      release(c);
    }
  }
  // ---- omega: back substitution and recombination ------------------------
  {
    constexpr int R = CF::R3;
    double2 zw[KUO];
#pragma unroll
    for (int e = 0; e < KUO; ++e) zw[e] = z2;
    const int nbo = N - 1;
    double2 nxt[R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) nxt[rr] = (rr < wd.no) ? lds(wd.no - 1 - rr) : z2;
    for (int r0 = 0; r0 < wd.no; r0 += R, ++c) {
      double2 cur[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        cur[rr] = nxt[rr];
        nxt[rr] = lds(wd.no - 1 - (r0 + R + rr));
      }
      if (!wait_chunk(c)) { abort_at(c); return; }
      const double2* ch = ring + (size_t)(c % WALL_NST) * (WALL_STG / 16) + q;
      const int rows = min(R, wd.no - r0);
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        if (rr < rows) {
          const int i = wd.no - 1 - (r0 + rr);
          const double2* Ur = ch + rr * CF::E3 * 16;
          double2 a1 = z2, a2 = z2;
#pragma unroll
          for (int e = KUO; e >= 2; --e) {
            if (e & 1) a1 = a1 + cmul(Ur[e * 16], zw[e - 1]);
            else a2 = a2 + cmul(Ur[e * 16], zw[e - 1]);
          }
          const double2 acc = (cur[rr] - (a1 + a2)) - cmul(Ur[16], zw[0]);
          const double2 x = cmul(Ur[0], acc);
#pragma unroll
          for (int e = KUO - 1; e >= 1; --e) zw[e] = zw[e - 1];
          zw[0] = x;
          if (i < nbo && active) O[pen * Ny + i + 2] = x - sel(i + 2 < nbo, zw[2]);
        }
      }
      release(c);
    }
    if (active) {
      O[pen * Ny + 1] = make_double2(-zw[1].x, -zw[1].y);
      O[pen * Ny + 0] = make_double2(-zw[0].x, -zw[0].y);
    }
  }
}

size_t wall_smem_bytes(const WallDims& wd, int variant) {
  const WallVar& v = kWallVar[variant];
  return (size_t)WALL_HDR + (size_t)v.nst * v.stg + (v.qsm ? wd.qbytes : 0) + (size_t)2 * (wd.nv + 2) * 8;
}
size_t wall_scratch_complex(const WallDims& wd) { return (size_t)wd.ngroups * 32 * wd.nv; }

// band instances: base-flow degree 0, 1, 2
bool wall_band_of(int delta, int* klv, int* kuv, int* klo, int* kuo) {
  static const int tab[3][4] = {{4, 8, 2, 4}, {5, 9, 3, 6}, {6, 10, 4, 8}};
  if (delta < 0 || delta > 2) return false;
  *klv = tab[delta][0]; *kuv = tab[delta][1]; *klo = tab[delta][2]; *kuo = tab[delta][3];
  return true;
}

template <int A, int B, int C, int D, int VAR>
static cudaError_t launch_inst(const double2* fac, double2* V, double2* O, const double2* gv,
                               const double2* go, const double* Q, double2* Sw, const WallDims& wd,
                               const DnsGeom& g, const PhysParams& ph, int* status, cudaStream_t st) {
  constexpr WallVar v = kWallVar[VAR];
  auto k = k_wall_solve<A, B, C, D, v.nst, v.stg, v.qsm, v.ef>;
  const size_t sm = wall_smem_bytes(wd, VAR);
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e) return e;
  k<<<(unsigned)wd.ngroups, 32, sm, st>>>(fac, V, O, gv, go, Q, Sw, wd, g, ph, status);
  return cudaGetLastError();
}

template <int A, int B, int C, int D>
static cudaError_t launch_var(int variant, const double2* fac, double2* V, double2* O, const double2* gv,
                              const double2* go, const double* Q, double2* Sw, const WallDims& wd,
                              const DnsGeom& g, const PhysParams& ph, int* status, cudaStream_t st) {
  switch (variant) {
    case 0: return launch_inst<A, B, C, D, 0>(fac, V, O, gv, go, Q, Sw, wd, g, ph, status, st);
    case 1: return launch_inst<A, B, C, D, 1>(fac, V, O, gv, go, Q, Sw, wd, g, ph, status, st);
    case 2: return launch_inst<A, B, C, D, 2>(fac, V, O, gv, go, Q, Sw, wd, g, ph, status, st);
    case 3: return launch_inst<A, B, C, D, 3>(fac, V, O, gv, go, Q, Sw, wd, g, ph, status, st);
  }
  return cudaErrorNotSupported;
}

cudaError_t launch_wall_solve(const double2* fac, double2* V, double2* O, const double2* gv,
                              const double2* go, const double* Q, double2* Sw, const WallDims& wd,
                              const DnsGeom& g, const PhysParams& ph, int* status, cudaStream_t st,
                              int variant) {
  if (variant < 0 || variant >= DNS_WALL_VARIANTS) return cudaErrorNotSupported;
  if (wall_smem_bytes(wd, variant) > 227 * 1024) return cudaErrorNotSupported;
  switch (wd.delta) {
    case 0: return launch_var<4, 8, 2, 4>(variant, fac, V, O, gv, go, Q, Sw, wd, g, ph, status, st);
    case 1: return launch_var<5, 9, 3, 6>(variant, fac, V, O, gv, go, Q, Sw, wd, g, ph, status, st);
    case 2: return launch_var<6, 10, 4, 8>(variant, fac, V, O, gv, go, Q, Sw, wd, g, ph, status, st);
  }
  return cudaErrorInvalidValue;
}
