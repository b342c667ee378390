// Kernel parameter blocks and launch helpers shared by the pass kernels.
//
// Layouts (element = complex of the pass precision unless stated):
//   pencil arrays  [field][pencil][n]     pencil p = kz*Kx + kx, wall-normal
//                                         index n contiguous (pitch ps); this
//                                         is the reference's ZXY layout
//                                         (include/data.h:265-284) when ps is
//                                         tPitch/16 and the field stride is 0
//   row arrays     [field][y][zp][kx]     streamwise index contiguous (row
//                                         pitch rs, Pz rows per wall-normal
//                                         plane); the reference's XYZ complex
//                                         layout before its 2D C2R
//   state arrays   [pencil][n] FP64 complex, n < Ny, pitch Ny
#pragma once
#include "../../include/dns_b200.h"
#include "dns_common.cuh"
#include "fft.cuh"

template <typename C> struct FftTab {
  FftPlan plan;
  const C* tw;          // W_L^j, j < L
  const short* drev;    // digit-reversed position of natural index n
  const C* wt[3];       // FP32 warp-FFT twiddle tables of the plans with 1, 2, 4 lines per warp
};

// twiddles of a warp-FFT plan: FP32, the plan's own table (lines per warp
// 1, 2, 4 -> i = 0, 1, 2); FP64, W_L^j and product recurrences
template <typename C> DNS_HD const C* wtw_of(const FftTab<C>& t, int i) {
  return sizeof(C) == 16 ? t.tw : t.wt[i];
}

// Pass launchers take a variant (the DNS_Y3_*, DNS_Y1_*, DNS_Z_* values of
// the public header) or VAR_AUTO, the first form the arguments allow in the
// order tensor copies, warp FFTs, block FFT.  With a variant they launch
// exactly that form or return cudaErrorNotSupported; with probe = true they
// only report which of the two it would be.
#define VAR_AUTO (-1)

struct PencilArr {      // generic pencil-major array
  void* base;
  long long ps;         // pencil pitch (elements)
  long long fs;         // field stride (elements)
};

struct RowArr {         // generic row-major [field][y][zp][kx] array
  void* base;
  long long rs;         // row pitch (elements)
  long long fs;         // field stride (elements)
};

// default bound of a device wait, in SM clock cycles (~1 s at 2 GHz)
#define DNS_WAIT_LIMIT (1LL << 31)

struct PhysParams {
  double aphi, beta;    // box: alpha_k = kx/aphi, beta_k = kz/beta
  double Re, Ro, dt;
  double U0, U1, U2;    // base flow U(y) = U0 + U1 y + U2 y^2
  long long wait_limit = DNS_WAIT_LIMIT;  // staging waits of the wall-normal warp passes
  const double* runs = nullptr;  // a batch's per-member (Re, Ro, dt), 3 each; null: one run
};
// a batch member's parameters (the context's own for one run)
DNS_HD double run_Re(const PhysParams& ph, int r) { return ph.runs ? ph.runs[3 * r] : ph.Re; }
DNS_HD double run_Ro(const PhysParams& ph, int r) { return ph.runs ? ph.runs[3 * r + 1] : ph.Ro; }
DNS_HD double run_dt(const PhysParams& ph, int r) { return ph.runs ? ph.runs[3 * r + 2] : ph.dt; }

// 16-byte alignment of a device pointer (bulk-copy sources)
inline bool aligned16(const void* p) { return ((unsigned long long)p & 15ull) == 0; }

#define DNS_CHECK_LAUNCH() do { cudaError_t e__ = cudaGetLastError(); if (e__ != cudaSuccess) return e__; } while (0)
