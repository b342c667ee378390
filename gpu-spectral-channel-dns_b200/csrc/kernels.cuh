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
#include "dns_common.cuh"
#include "fft.cuh"

template <typename C> struct FftTab {
  FftPlan plan;
  const C* tw;          // W_L^j, j < L
  const short* drev;    // digit-reversed position of natural index n
  const C* wt[3];       // FP32 warp-FFT twiddle tables of the plans with 1, 2, 4 lines per warp
};

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
};

// 16-byte alignment of a device pointer (bulk-copy sources)
inline bool aligned16(const void* p) { return ((unsigned long long)p & 15ull) == 0; }

#define DNS_CHECK_LAUNCH() do { cudaError_t e__ = cudaGetLastError(); if (e__ != cudaSuccess) return e__; } while (0)
