// Spanwise (z) and streamwise (x) pass kernels.
//
// Reference counterparts:
//   transpose_forward / transpose_backward ... source/transpose.cu:223-257, 358-382
//   setZerosKernel ........................... source/transform.cu:355-377
//   2D cuFFT Z2D / D2Z + normalizeKernel ..... source/transform.cu:176, 240, 388-412
//   computeLambVectorKernel / computeLambDevice source/nonlinear.cu:366-428
//
// Spanwise pass: a CTA owns a tile of TX streamwise modes x TY wall-normal
// points and transforms those TX*TY lines along the span in shared memory.
// It reads one layout (pencil-major, wall-normal index contiguous) and
// writes the other (row-major, streamwise index contiguous) with TX- or
// TY-element contiguous runs, so the x-y-z transpose, the span remap
// ky' = ky or ky + Pz - Nz, the zero padding Nz -> Pz (and truncation), and
// the zeroing of both Nyquist modes are folded into the one pass.
//
// Streamwise pass: two real rows share one complex FFT (a + i b).
#include "fftline.cuh"
#include "kernels.cuh"
#include <cuda.h>
#include <cudaTypedefs.h>
#include <type_traits>

#include "mbar.cuh"
#include "wfft.cuh"
#include "zxpass.cuh"

namespace {
template <typename C>
__device__ __forceinline__ C* prow(const RowArr& a, int f, long long row) {
  return (C*)a.base + (long long)f * a.fs + row * a.rs;
}
template <typename C>
__device__ __forceinline__ C* ppen(const PencilArr& a, int f, long long p) {
  return (C*)a.base + (long long)f * a.fs + p * a.ps;
}
}  // namespace

// ---------------------------------------------------------------------------
// spanwise backward: pencils [f][kz*Kx+kx][y] -> rows [f][y][zp][kx]
// ---------------------------------------------------------------------------
template <typename C, int TX, int TY, int L>
__global__ void __launch_bounds__(256, 3) k_zb(PencilArr in, RowArr out, DnsGeom g, FftTab<C> tab) {
  typedef FLine<C, L> FL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* lines = (C*)smem_raw;
  const int Pz = L > 0 ? L : g.Pz;
  const int Nz = g.Nz, Kx = g.Kx, Py = g.Py;
  const int ls = FL::stride(Pz);
  const int kx0 = blockIdx.x * TX;
  const int y0 = blockIdx.y * TY;
  const int f = blockIdx.z;
  const int NL = TX * TY;
  const int hz = Nz / 2;
  // zero band [Nz/2, Pz - Nz/2] (Nyquist and padding)
  const int nzero = Pz - Nz + 1;
  for (int t = threadIdx.x; t < NL * nzero; t += blockDim.x) {
    const int li = t / nzero;
    const int n = hz + (t - li * nzero);
    lines[(size_t)li * ls + FL::in_pos(tab, n)] = cmk<C>(0.0, 0.0);
  }
  for (int t = threadIdx.x; t < Nz * NL; t += blockDim.x) {
    const int yl = t % TY;
    const int kxl = (t / TY) % TX;
    const int kz = t / NL;
    if (kz == hz) continue;
    const int n = (kz < hz) ? kz : kz + (Pz - Nz);
    const int kx = kx0 + kxl;
    const int y = y0 + yl;
    C v = cmk<C>(0.0, 0.0);
    if (kx < Kx - 1 && y < Py) v = ppen<C>(in, f, (long long)kz * Kx + kx)[y];
    lines[(size_t)(kxl * TY + yl) * ls + FL::in_pos(tab, n)] = v;
  }
  FL::template fft<true>(lines, NL, ls, tab);
  for (int t = threadIdx.x; t < TY * Pz * TX; t += blockDim.x) {
    const int kxl = t % TX;
    const int zp = (t / TX) % Pz;
    const int yl = t / (TX * Pz);
    const int kx = kx0 + kxl;
    const int y = y0 + yl;
    if (kx < Kx && y < Py)
      prow<C>(out, f, (long long)y * Pz + zp)[kx] = lines[(size_t)(kxl * TY + yl) * ls + FL::out_pos(zp)];
  }
}

// ---------------------------------------------------------------------------
// spanwise forward: rows [f][y][zp][kx] -> pencils [f][kz*Kx+kx][y]
// ---------------------------------------------------------------------------
template <typename C, int TX, int TY, int L>
__global__ void __launch_bounds__(256, 3) k_zf(RowArr in, PencilArr out, DnsGeom g, FftTab<C> tab) {
  typedef FLine<C, L> FL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* lines = (C*)smem_raw;
  const int Pz = L > 0 ? L : g.Pz;
  const int Nz = g.Nz, Kx = g.Kx, Py = g.Py;
  const int ls = FL::stride(Pz);
  const int kx0 = blockIdx.x * TX;
  const int y0 = blockIdx.y * TY;
  const int f = blockIdx.z;
  const int NL = TX * TY;
  for (int t = threadIdx.x; t < TY * Pz * TX; t += blockDim.x) {
    const int kxl = t % TX;
    const int zp = (t / TX) % Pz;
    const int yl = t / (TX * Pz);
    const int kx = kx0 + kxl;
    const int y = y0 + yl;
    C v = cmk<C>(0.0, 0.0);
    if (kx < Kx && y < Py) v = prow<C>(in, f, (long long)y * Pz + zp)[kx];
    lines[(size_t)(kxl * TY + yl) * ls + FL::in_pos(tab, zp)] = v;
  }
  FL::template fft<false>(lines, NL, ls, tab);
  const int hz = Nz / 2;
  for (int t = threadIdx.x; t < Nz * NL; t += blockDim.x) {
    const int yl = t % TY;
    const int kxl = (t / TY) % TX;
    const int kz = t / NL;
    const int kx = kx0 + kxl;
    const int y = y0 + yl;
    const int n = (kz <= hz) ? kz : kz + (Pz - Nz);
    if (kx < Kx && y < Py)
      ppen<C>(out, f, (long long)kz * Kx + kx)[y] = lines[(size_t)(kxl * TY + yl) * ls + FL::out_pos(n)];
  }
}

// Same spanwise passes with warp FFTs: a TX x TY tile of 16 lines
// (streamwise modes x wall-normal points), NW warps with 16/NW lines each,
// no block barrier inside the transforms.  The kernels below that read
// through L1 (k_zbw, k_zfw) use 4 x 4 tiles: 32-byte runs, whole sectors, on
// both sides; the tensor-staged ones (k_zbt 8 x 2, k_zft 4 x 4) are chosen
// for their row side.
//
// Index arithmetic: on the pencil side a thread keeps one line (its kx and
// y) and walks the spanwise wavenumbers kz = t/16 + 16 m; on the row side it
// keeps one kx and walks the flat (y, zp) index of the tile's rows, whose
// global offset is i * rs from the tile's first row.  Both walks are strided
// by a constant, so an element costs one multiply-add of its address.
namespace {
template <typename C, int L, int TX, int TY, int NT>
struct SpanTile {
  static constexpr int NL = TX * TY;
  static constexpr int LS = wlen<C>(L) + 1;  // odd line stride: the 16 lines of a position fall in distinct banks
  static constexpr int KS = NT / NL;         // kz stride of the pencil-side walk
  static constexpr int IS = NT / TX;         // (y, zp) stride of the row-side walk
  static_assert(NT % NL == 0 && NT % TX == 0, "tile does not divide the block");
};
}  // namespace

template <typename C, int L, int NW, int TX, int TY>
__global__ void __launch_bounds__(32 * NW) k_zbw(PencilArr in, RowArr out, DnsGeom g, FftTab<C> tab) {
  typedef SpanTile<C, L, TX, TY, 32 * NW> ST;
  constexpr int NL = ST::NL, LS = ST::LS, Pz = L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* lines = (C*)smem_raw;
  constexpr int Nz = L / 3 * 2;  // my / 3 * 2 (the launcher checks g.Nz)
  const int Kx = g.Kx, Py = g.Py;
  const int kx0 = blockIdx.x * TX;
  const int y0 = blockIdx.y * TY;
  const int f = blockIdx.z;
  constexpr int hz = Nz / 2;
  // pencil side: line li = (kxl, yl) of this thread
  {
    const int li = threadIdx.x % NL;
    const int kx = kx0 + li / TY, y = y0 + li % TY;
    C* dst = lines + li * LS;
    // zero band [Nz/2, Pz - Nz/2] (Nyquist and padding)
    for (int n = hz + threadIdx.x / NL; n <= Pz - hz; n += ST::KS) dst[wsw<C>(n)] = cmk<C>(0.0, 0.0);
    // the streamwise Nyquist column (kx = Kx - 1) and rows beyond Py stay zero
    const bool ok = kx < Kx - 1 && y < Py;
    const C* src = ppen<C>(in, f, ok ? kx : 0) + (ok ? y : 0);
    const long long kzs = (long long)Kx * in.ps;
    // loads in batches of ZB independent requests per thread before their stores
    constexpr int ZB = 8;
    for (int kz0 = threadIdx.x / NL; kz0 < Nz; kz0 += ZB * ST::KS) {
      C v[ZB];
#pragma unroll
      for (int u = 0; u < ZB; ++u) {
        const int kz = kz0 + u * ST::KS;
        v[u] = (ok && kz < Nz && kz != hz) ? src[kz * kzs] : cmk<C>(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < ZB; ++u) {
        const int kz = kz0 + u * ST::KS;
        if (kz < Nz && kz != hz) dst[wsw<C>(kz < hz ? kz : kz + (Pz - Nz))] = v[u];
      }
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  constexpr int NLW = NL / NW;  // lines per warp
  wfft<C, L, NLW, true>(lines + (size_t)NLW * warp * LS, wtw_of(tab, 1), LS);
  __syncthreads();
  // row side: this thread's kx, flat index i = yl * Pz + zp
  const int kxl = threadIdx.x % TX;
  const int kx = kx0 + kxl;
  if (kx >= Kx || y0 >= Py) return;
  const int ni = min(TY, Py - y0) * Pz;
  C* rowb = prow<C>(out, f, (long long)y0 * Pz) + kx;
  const C* lb = lines + kxl * TY * LS;
  constexpr int ZB = 8;
  for (int i0 = threadIdx.x / TX; i0 < ni; i0 += ZB * ST::IS) {
    C v[ZB];
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int i = i0 + u * ST::IS;
      const int yl = i / Pz, zp = i - yl * Pz;
      v[u] = (i < ni) ? lb[yl * LS + wsw<C>(zp)] : cmk<C>(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int i = i0 + u * ST::IS;
      if (i < ni) rowb[(long long)i * out.rs] = v[u];
    }
  }
}

// The same inverse pass with the pencils staged by the tensor-memory
// accelerator: warp w owns lines 2w, 2w+1 (one kx, two consecutive y) and
// loads their Nz spanwise values with one tiled 4-D copy (box y 2 x kx 1 x
// kz Nz x field 1, 4 KB at Nz = 256) into its own line buffer; the first FFT
// pass reads them there (padding, Nyquist and streamwise-Nyquist zeros
// applied in the read) before it writes the lines.  Rows beyond Py and
// columns beyond Kx read as the copy's zero fill.  No per-element global
// loads, no L1 dependence.
template <typename C, int L, int NW, int TX, int TY>
__global__ void __launch_bounds__(32 * NW, 3) k_zbt(const __grid_constant__ CUtensorMap tin, RowArr out,
                                                 DnsGeom g, FftTab<C> tab, int* status) {
  typedef SpanTile<C, L, TX, TY, 32 * NW> ST;
  constexpr int NL = ST::NL, LS = ST::LS, Pz = L;
  static_assert(NL == 2 * NW && TY % 2 == 0 && ST::KS > 0, "two lines per warp, a y pair each");
  extern __shared__ __align__(16) unsigned char smem_raw[];  // the tile is rounded up to 128 bytes
  __shared__ uint64_t bars[NW];
  C* lines = (C*)smem_raw;
  constexpr int Nz = L / 3 * 2;  // my / 3 * 2 (the launcher checks g.Nz)
  constexpr int hz = Nz / 2;
  const int Kx = g.Kx, Py = g.Py;
  const int kx0 = blockIdx.x * TX;
  const int y0 = blockIdx.y * TY;
  const int f = blockIdx.z;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int li0 = 2 * warp;                       // lines (kxl, yl0), (kxl, yl0 + 1)
  const int kxl = li0 / TY, yl0 = li0 % TY;
  C* wl = lines + (size_t)li0 * LS;
  // the staged values [kz][y pair] at the first 128-byte boundary of the warp's lines
  C* tile = (C*)(((uintptr_t)wl + 127) & ~(uintptr_t)127);
  uint64_t* bar = bars + warp;
  if (lane == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    mbar_expect_tx(bar, (uint32_t)(2 * Nz * sizeof(C)));
    tma_load_4d(tile, &tin, y0 + yl0, kx0 + kxl, 0, f, bar);
  }
  __syncwarp();
  // a wait that runs out is reported and waited once more (bounded); the
  // warp then goes on, so that every warp reaches the block barriers
  if (!__all_sync(0xffffffffu, mbar_wait_bounded(bar, 0, 1LL << 31, status))) {
    if (lane == 0) {
      atomicOr(status, 1);
      mbar_wait_bounded(bar, 0, 1LL << 31, nullptr);
    }
    __syncwarp();
  }
  // the streamwise Nyquist column (kx = Kx - 1) stays zero
  const bool kxok = kx0 + kxl < Kx - 1;
  auto ld = [&](int l, int n) -> C {
    const int kz = (n < hz) ? n : (n > Pz - hz ? n - (Pz - Nz) : -1);
    return (kxok && kz >= 0) ? tile[2 * kz + l] : cmk<C>(0.0, 0.0);
  };
  auto st = [&](int l, int k, C v) { wl[(size_t)l * LS + wsw<C>(k)] = v; };
  wfft_io<C, L, 2, true>(wl, tab.wt[1], ld, st, LS);
  __syncthreads();
  // row side: this thread's kx, flat index i = yl * Pz + zp
  const int kxr = threadIdx.x % TX;
  const int kx = kx0 + kxr;
  if (kx >= Kx || y0 >= Py) return;
  const int ni = min(TY, Py - y0) * Pz;
  C* rowb = prow<C>(out, f, (long long)y0 * Pz) + kx;
  const C* lb = lines + kxr * TY * LS;
  constexpr int ZB = 8;
  for (int i0 = threadIdx.x / TX; i0 < ni; i0 += ZB * ST::IS) {
    C v[ZB];
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int i = i0 + u * ST::IS;
      const int yl = i / Pz, zp = i - yl * Pz;
      v[u] = (i < ni) ? lb[yl * LS + wsw<C>(zp)] : cmk<C>(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int i = i0 + u * ST::IS;
      if (i < ni) rowb[(long long)i * out.rs] = v[u];
    }
  }
}

template <typename C, int L, int NW, int TX, int TY>
__global__ void __launch_bounds__(32 * NW) k_zfw(RowArr in, PencilArr out, DnsGeom g, FftTab<C> tab) {
  typedef SpanTile<C, L, TX, TY, 32 * NW> ST;
  constexpr int NL = ST::NL, LS = ST::LS, Pz = L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* lines = (C*)smem_raw;
  constexpr int Nz = L / 3 * 2;  // my / 3 * 2 (the launcher checks g.Nz)
  const int Kx = g.Kx, Py = g.Py;
  const int kx0 = blockIdx.x * TX;
  const int y0 = blockIdx.y * TY;
  const int f = blockIdx.z;
  constexpr int ZB = 8;
  // row side: this thread's kx, flat index i = yl * Pz + zp; rows beyond
  // Py and columns beyond Kx read as zero
  {
    const int kxl = threadIdx.x % TX;
    const int kx = kx0 + kxl;
    const int ni = TY * Pz;
    const int nv = (kx < Kx && y0 < Py) ? min(TY, Py - y0) * Pz : 0;
    const C* rowb = prow<C>(in, f, (long long)y0 * Pz) + kx;
    C* lb = lines + kxl * TY * LS;
    for (int i0 = threadIdx.x / TX; i0 < ni; i0 += ZB * ST::IS) {
      C v[ZB];
#pragma unroll
      for (int u = 0; u < ZB; ++u) {
        const int i = i0 + u * ST::IS;
        v[u] = (i < nv) ? rowb[(long long)i * in.rs] : cmk<C>(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < ZB; ++u) {
        const int i = i0 + u * ST::IS;
        const int yl = i / Pz, zp = i - yl * Pz;
        if (i < ni) lb[yl * LS + wsw<C>(zp)] = v[u];
      }
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  constexpr int NLW = NL / NW;  // lines per warp
  wfft<C, L, NLW, false>(lines + (size_t)NLW * warp * LS, wtw_of(tab, 1), LS);
  __syncthreads();
  // pencil side: line li = (kxl, yl) of this thread, wavenumbers kz
  constexpr int hz = Nz / 2;
  const int li = threadIdx.x % NL;
  const int kx = kx0 + li / TY, y = y0 + li % TY;
  if (kx >= Kx || y >= Py) return;
  const C* lsrc = lines + li * LS;
  C* dst = ppen<C>(out, f, kx) + y;
  const long long kzs = (long long)Kx * out.ps;
  for (int kz0 = threadIdx.x / NL; kz0 < Nz; kz0 += ZB * ST::KS) {
    C v[ZB];
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int kz = kz0 + u * ST::KS;
      v[u] = (kz < Nz) ? lsrc[wsw<C>(kz <= hz ? kz : kz + (Pz - Nz))] : cmk<C>(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int kz = kz0 + u * ST::KS;
      if (kz < Nz) dst[kz * kzs] = v[u];
    }
  }
}

// The same forward pass with the rows staged by tensor copies: lines are
// numbered y-major (li = yl * 4 + kxl), warp w owns lines 2w, 2w+1 (one y,
// a kx pair) and loads their Pz values with two tiled 4-D copies (box kx 2
// x zp Pz/2 x y 1 x field 1) into its own line buffer, [zp][kx pair]; the
// first FFT pass reads them there.  Rows beyond Py and columns beyond Kx
// read as the copy's zero fill.
template <typename C, int L, int NW>
__global__ void __launch_bounds__(32 * NW, 3) k_zft(const __grid_constant__ CUtensorMap tin, PencilArr out,
                                                    DnsGeom g, FftTab<C> tab, int* status) {
  constexpr int TX = 4, TY = 4;
  typedef SpanTile<C, L, TX, TY, 32 * NW> ST;
  constexpr int NL = ST::NL, LS = ST::LS, Pz = L;
  static_assert(NL == 2 * NW && Pz % 2 == 0, "two lines per warp, a kx pair each");
  extern __shared__ __align__(16) unsigned char smem_raw[];  // the tile is rounded up to 128 bytes
  __shared__ uint64_t bars[NW];
  C* lines = (C*)smem_raw;
  constexpr int Nz = L / 3 * 2;  // my / 3 * 2 (the launcher checks g.Nz)
  constexpr int hz = Nz / 2;
  const int Kx = g.Kx, Py = g.Py;
  const int kx0 = blockIdx.x * TX;
  const int y0 = blockIdx.y * TY;
  const int f = blockIdx.z;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int li0 = 2 * warp;
  const int yl = li0 / TX, kxl0 = li0 % TX;
  C* wl = lines + (size_t)li0 * LS;
  C* tile = (C*)(((uintptr_t)wl + 127) & ~(uintptr_t)127);
  uint64_t* bar = bars + warp;
  if (lane == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    mbar_expect_tx(bar, (uint32_t)(2 * Pz * sizeof(C)));
    tma_load_4d(tile, &tin, kx0 + kxl0, 0, y0 + yl, f, bar);
    tma_load_4d(tile + Pz, &tin, kx0 + kxl0, Pz / 2, y0 + yl, f, bar);
  }
  __syncwarp();
  // a wait that runs out is reported and waited once more (bounded); the
  // warp then goes on, so that every warp reaches the block barriers
  if (!__all_sync(0xffffffffu, mbar_wait_bounded(bar, 0, 1LL << 31, status))) {
    if (lane == 0) {
      atomicOr(status, 1);
      mbar_wait_bounded(bar, 0, 1LL << 31, nullptr);
    }
    __syncwarp();
  }
  auto ld = [&](int l, int n) -> C { return tile[2 * n + l]; };
  auto st = [&](int l, int k, C v) { wl[(size_t)l * LS + wsw<C>(k)] = v; };
  wfft_io<C, L, 2, false>(wl, tab.wt[1], ld, st, LS);
  __syncthreads();
  // pencil side: line li = (yl, kxl) of this thread, wavenumbers kz
  constexpr int ZB = 8;
  const int li = threadIdx.x % NL;
  const int kx = kx0 + li % TX, y = y0 + li / TX;
  if (kx >= Kx || y >= Py) return;
  const C* lsrc = lines + li * LS;
  C* dst = ppen<C>(out, f, kx) + y;
  const long long kzs = (long long)Kx * out.ps;
  for (int kz0 = threadIdx.x / NL; kz0 < Nz; kz0 += ZB * ST::KS) {
    C v[ZB];
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int kz = kz0 + u * ST::KS;
      v[u] = (kz < Nz) ? lsrc[wsw<C>(kz <= hz ? kz : kz + (Pz - Nz))] : cmk<C>(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int kz = kz0 + u * ST::KS;
      if (kz < Nz) dst[kz * kzs] = v[u];
    }
  }
}

namespace {
// Hermitian half-spectra a, b (bins 0..Kx-1, Nyquist and padding zero) packed
// as Z = A + iB over the full length Px, so that IFFT(Z) = a(x) + i b(x).
// The imaginary parts of the DC bins are dropped (C2R convention).
template <typename C>
__device__ __forceinline__ C pack_c2r(const C* a, const C* b, int n, int Px, int hx) {
  if (n == 0) return cmk<C>((double)a[0].x, (double)b[0].x);
  if (n < hx) {
    const C av = a[n], bv = b[n];
    C z; z.x = av.x - bv.y; z.y = av.y + bv.x; return z;
  }
  if (n > Px - hx) {
    const int k = Px - n;
    const C av = a[k], bv = b[k];
    C z; z.x = av.x + bv.y; z.y = bv.x - av.y; return z;  // conj(a) + i conj(b)
  }
  return cmk<C>(0.0, 0.0);
}
// unpack the spectra of the real and imaginary parts of a complex signal
template <typename C>
__device__ __forceinline__ C unpack_r2c(const C* Z, int k, int Px, bool imag_part) {
  const C zk = Z[k];
  const C zm = Z[(Px - k) % Px];
  C r;
  if (!imag_part) { r.x = (zk.x + zm.x); r.y = (zk.y - zm.y); }   // Zk + conj(Zm)
  else { r.x = (zk.y + zm.y); r.y = (zm.x - zk.x); }              // -i (Zk - conj(Zm))
  return r;
}
}  // namespace

// ---------------------------------------------------------------------------
// fused streamwise pass: 6 half-spectra rows -> physical -> Lamb vector with
// the rotation term -> 3 half-spectra rows, x 1/(Px Pz).
// Input fields u, v(span), w(wall), omega_x, omega_y, omega_z; output
// lambda_x, lambda_y(span), lambda_z(wall).  RB rows per CTA (even, rows of
// one wall-normal plane).
// ---------------------------------------------------------------------------
template <typename C, int L>
__global__ void __launch_bounds__(256, 3) k_x_fused(RowArr in, RowArr out, DnsGeom g, FftTab<C> tab,
                                                   const double* __restrict__ Uy, double Ro,
                                                   const double* __restrict__ runs) {
  // two rows per CTA: lines 0-2 hold row 0's packed fields (u,v) (ox,oy)
  // (w,oz), lines 3-5 row 1's; after the inverse transform a thread owning
  // point j of both rows writes lambda_x + i lambda_y of row 0 / row 1 into
  // lines 0 / 1 and lambda_z(row 0) + i lambda_z(row 1) into line 2 at the
  // same position, then lines 0-2 are transformed forward.
  typedef FLine<C, L> FL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  typedef T_of<C> T;
  const int Px = L > 0 ? L : g.Px;
  const int hx = g.Nx / 2;
  const int ls = FL::stride(Px);
  C* z = (C*)smem_raw;  // 6 lines (9 for the runtime-length FFT)
  const long long r0 = (long long)blockIdx.x * 2;
  const long long nrows = (long long)g.Py * g.Pz * g.nrun;  // a batch: members' rows one after another
  for (int t = threadIdx.x; t < 2 * 3 * Px; t += blockDim.x) {
    const int rl = t / (3 * Px);
    const int rem = t - rl * 3 * Px;
    const int q = rem / Px;
    const int n = rem - q * Px;
    const long long row = r0 + rl;
    C zz = cmk<C>(0.0, 0.0);
    if (row < nrows) {
      // fields of similar magnitude share a transform (the smaller one's
      // rounding error is relative to the larger): (u, v), (ox, oy), (w, oz)
      const int fa = (q == 0) ? 0 : (q == 1 ? 3 : 2);
      const int fb = (q == 0) ? 1 : (q == 1 ? 4 : 5);
      zz = pack_c2r<C>(prow<C>(in, fa, row), prow<C>(in, fb, row), n, Px, hx);
    }
    z[(size_t)(rl * 3 + q) * ls + FL::in_pos(tab, n)] = zz;
  }
  FL::template fft<true>(z, 6, ls, tab);
  // both rows lie in one wall-normal plane of one member
  const long long pr = (long long)g.Py * g.Pz;
  const int run = (int)(r0 / pr);
  const T ro = (T)(runs ? runs[3 * run + 1] : Ro);
  const int y = (int)((r0 - run * pr) / g.Pz);
  const T Ub = (T)Uy[y < g.Py ? y : 0];
  for (int j = threadIdx.x; j < Px; j += blockDim.x) {
    const int op = FL::out_pos(j);
    T lz[2];
    C A[2];
#pragma unroll
    for (int rl = 0; rl < 2; ++rl) {
      const C z0 = z[(size_t)(rl * 3 + 0) * ls + op];
      const C z1 = z[(size_t)(rl * 3 + 1) * ls + op];
      const C z2 = z[(size_t)(rl * 3 + 2) * ls + op];
      const T u = z0.x, v = z0.y, ox = z1.x, oy = z1.y, w = z2.x, oz = z2.y;
      A[rl].x = oz * v - oy * w - ro * w;
      A[rl].y = ox * w - oz * u;
      lz[rl] = oy * u - ox * v + ro * (u + Ub);
    }
    if (L > 0) {  // natural order: write in place
      z[(size_t)0 * ls + op] = A[0];
      z[(size_t)1 * ls + op] = A[1];
      C B; B.x = lz[0]; B.y = lz[1];
      z[(size_t)2 * ls + op] = B;
    } else {      // digit-reversed input order: separate lines 6-8
      const int pos = FL::in_pos(tab, j);
      z[(size_t)6 * ls + pos] = A[0];
      z[(size_t)7 * ls + pos] = A[1];
      C B; B.x = lz[0]; B.y = lz[1];
      z[(size_t)8 * ls + pos] = B;
    }
  }
  C* zf = (L > 0) ? z : z + (size_t)6 * ls;
  FL::template fft<false>(zf, 3, ls, tab);
  const int Kx = g.Kx;
  const T sc = (T)(0.5 / ((double)g.Px * (double)g.Pz));
  for (int t = threadIdx.x; t < 2 * 3 * Kx; t += blockDim.x) {
    const int k = t % Kx;
    const int fl = (t / Kx) % 3;
    const int rl = t / (3 * Kx);
    const long long row = r0 + rl;
    if (row >= nrows) continue;
    const C* Z = (fl < 2) ? zf + (size_t)rl * ls : zf + (size_t)2 * ls;
    const bool im = (fl < 2) ? (fl == 1) : (rl == 1);
    const C zk = Z[FL::out_pos(k)];
    const C zm = Z[FL::out_pos((Px - k) % Px)];
    C v;
    if (!im) { v.x = zk.x + zm.x; v.y = zk.y - zm.y; }
    else { v.x = zk.y + zm.y; v.y = zm.x - zk.x; }
    prow<C>(out, fl, row)[k] = v * sc;
  }
}

// Same pass with warp FFTs: a CTA of NW warps (3 or 6) owns four rows of
// one wall-normal plane.  Warp w inverse-transforms lines LPW w .. LPW w +
// LPW - 1, LPW = 12 / NW (line 3r+q holds row r's packed pair q), reading
// the half spectra straight from the row arrays in the first FFT pass;
// after a block barrier the Lamb vector of the four rows is formed
// pointwise into lines 0-5 (lines r < 4: lambda_x + i lambda_y of row r;
// lines 4, 5: lambda_z of rows (0, 1), (2, 3)); each warp forward-transforms
// 6 / NW of them, and the half spectra are unpacked to the output rows.
// Six warps hold half the lines each: half the registers per thread, twice
// the warps per SM.
template <typename C, int L, int NW>
__global__ void __launch_bounds__(32 * NW, sizeof(C) == 8 ? 5 : 2) k_xw(RowArr in, RowArr out, DnsGeom g,
                                                                      FftTab<C> tab, const double* __restrict__ Uy,
                                                                      double Ro, const double* __restrict__ runs,
                                                                      int* status) {
  static_assert(NW == 3 || NW == 6, "three or six warps");
  constexpr int LPW = 12 / NW;  // inverse lines per warp
  constexpr int FPW = 6 / NW;   // forward lines per warp
  extern __shared__ __align__(16) unsigned char smem_raw[];
  typedef T_of<C> T;
  constexpr int Px = L;
  constexpr int hx = L / 3;  // Nx / 2 = mx / 3 (the launcher checks it): branches of the packing resolve at compile time
  constexpr int LW = wlen<C>(L);                        // line stride
  C* z = (C*)smem_raw;                                  // 12 lines
  uint64_t* bars = (uint64_t*)(z + (size_t)12 * LW);     // one per warp
  const long long r0 = (long long)blockIdx.x * 4;
  const long long nrows = (long long)g.Py * g.Pz * g.nrun;  // a batch: members' rows one after another
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* zw = z + (size_t)LPW * warp * LW;
  // stage this warp's 2 LPW half-spectrum rows (bins 0..hx-1, 16 B aligned)
  // at the start of its own lines: the first FFT pass reads them all before
  // it writes its output over them
  constexpr int SR = (hx + 15) / 16 * 16;  // staged bins per row (>= hx; 128 at L = 384)
  uint64_t* bar = bars + warp;
  if (lane == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    mbar_expect_tx(bar, 2 * LPW * SR * sizeof(C));
  }
  __syncwarp();
  if (lane < 2 * LPW) {
    const int line = LPW * warp + (lane >> 1);
    const int rl = line / 3, q = line - 3 * (line / 3);
    long long row = r0 + rl;
    if (row >= nrows) row = nrows - 1;  // duplicate work, not stored
    // fields of similar magnitude share a transform: (u, v), (ox, oy), (w, oz)
    const int fa = q == 0 ? 0 : (q == 1 ? 3 : 2), fb = q == 0 ? 1 : (q == 1 ? 4 : 5);
    bulk_g2s(zw + (size_t)lane * SR, prow<C>(in, (lane & 1) ? fb : fa, row), SR * sizeof(C), bar);
  }
  // a wait that runs out is reported and waited once more (bounded); the
  // warp then goes on, so that every warp reaches the block barriers
  if (!__all_sync(0xffffffffu, mbar_wait_bounded(bar, 0, 1LL << 31, status))) {
    if (lane == 0) {
      atomicOr(status, 1);
      mbar_wait_bounded(bar, 0, 1LL << 31, nullptr);
    }
    __syncwarp();
  }
  __syncthreads();
  {
    const C* stg = zw;
    auto ld = [&](int l, int n) -> C { return pack_c2r<C>(stg + (size_t)(2 * l) * SR, stg + (size_t)(2 * l + 1) * SR, n, Px, hx); };
    auto st = [&](int l, int k, C v) { zw[(size_t)l * LW + wsw<C>(k)] = v; };
    wfft_io<C, L, LPW, true>(zw, wtw_of(tab, LPW == 4 ? 2 : 1), ld, st);
  }
  __syncthreads();
  // the four rows lie in one wall-normal plane of one member
  const long long pr = (long long)g.Py * g.Pz;
  const int run = (int)(r0 / pr);
  const T ro = (T)(runs ? runs[3 * run + 1] : Ro);
  const int y = (int)((r0 - run * pr) / g.Pz);
  const T Ub = (T)Uy[y < g.Py ? y : 0];
  for (int j = threadIdx.x; j < Px; j += blockDim.x) {
    const int op = wsw<C>(j);
    C A[4];
    T lz[4];
#pragma unroll
    for (int rl = 0; rl < 4; ++rl) {
      const C z0 = z[(size_t)(3 * rl + 0) * LW + op];
      const C z1 = z[(size_t)(3 * rl + 1) * LW + op];
      const C z2 = z[(size_t)(3 * rl + 2) * LW + op];
      const T u = z0.x, v = z0.y, ox = z1.x, oy = z1.y, w = z2.x, oz = z2.y;
      A[rl].x = oz * v - oy * w - ro * w;
      A[rl].y = ox * w - oz * u;
      lz[rl] = oy * u - ox * v + ro * (u + Ub);
    }
#pragma unroll
    for (int rl = 0; rl < 4; ++rl) z[(size_t)rl * LW + op] = A[rl];
    C B0, B1;
    B0.x = lz[0]; B0.y = lz[1];
    B1.x = lz[2]; B1.y = lz[3];
    z[(size_t)4 * LW + op] = B0;
    z[(size_t)5 * LW + op] = B1;
  }
  __syncthreads();
  wfft<C, L, FPW, false>(z + (size_t)FPW * warp * LW, wtw_of(tab, FPW - 1));
  __syncthreads();
  // unpack: output row o = 3 rl + fl (field fl of row rl) by warp o mod 3,
  // lanes over the bins k; shared loads of a batch before its stores
  const int Kx = g.Kx;
  const T sc = (T)(0.5 / ((double)g.Px * (double)g.Pz));
  constexpr int XB = 5;
  for (int o = warp; o < 12; o += NW) {
    const int rl = o / 3, fl = o - 3 * rl;
    const long long row = r0 + rl;
    if (row >= nrows) continue;
    const C* Z = (fl < 2) ? z + (size_t)rl * LW : z + (size_t)(4 + rl / 2) * LW;
    const bool im = (fl < 2) ? (fl == 1) : (rl & 1);
    C* dst = prow<C>(out, fl, row);
    for (int k0 = lane; k0 < Kx; k0 += 32 * XB) {
      C zk[XB], zm[XB];
#pragma unroll
      for (int u = 0; u < XB; ++u) {
        const int k = min(k0 + 32 * u, Kx - 1);
        zk[u] = Z[wsw<C>(k)];
        zm[u] = Z[wsw<C>(k ? Px - k : 0)];
      }
#pragma unroll
      for (int u = 0; u < XB; ++u) {
        const int k = k0 + 32 * u;
        if (k >= Kx) continue;
        C v;
        if (!im) { v.x = zk[u].x + zm[u].x; v.y = zk[u].y - zm[u].y; }
        else { v.x = zk[u].y + zm[u].y; v.y = zm[u].x - zk[u].x; }
        dst[k] = v * sc;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// standalone streamwise C2R / R2C (drop-in transform_3d_one pieces)
// complex rows in [row][kx] (pitch rs) <-> real rows [row][x] (pitch rps)
// ---------------------------------------------------------------------------
template <typename C>
__global__ void k_x_c2r(RowArr in, T_of<C>* outr, long long rps, long long nrows, DnsGeom g,
                        FftTab<C> tab, int RB) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* z = (C*)smem_raw;  // RB/2 lines
  const int Px = g.Px;
  const int hx = g.Nx / 2;
  const long long r0 = (long long)blockIdx.x * RB;
  const int NP = RB / 2;
  for (int t = threadIdx.x; t < NP * Px; t += blockDim.x) {
    const int q = t / Px;
    const int n = t - q * Px;
    const long long ra = r0 + 2 * q, rb = ra + 1;
    C v = cmk<C>(0.0, 0.0);
    if (ra < nrows) {
      const C* a = prow<C>(in, 0, ra);
      const C* b = (rb < nrows) ? prow<C>(in, 0, rb) : a;
      v = pack_c2r<C>(a, b, n, Px, hx);
      if (rb >= nrows) v.y = 0;
    }
    z[(size_t)q * Px + tab.drev[n]] = v;
  }
  fft_batch<C, true>(z, NP, Px, tab.plan, tab.tw);
  for (int t = threadIdx.x; t < RB * Px; t += blockDim.x) {
    const int rl = t / Px;
    const int j = t - rl * Px;
    const long long row = r0 + rl;
    if (row >= nrows) continue;
    const C v = z[(size_t)(rl / 2) * Px + j];
    outr[row * rps + j] = (rl & 1) ? v.y : v.x;
  }
}

template <typename C>
__global__ void k_x_r2c(const T_of<C>* inr, long long rps, RowArr out, long long nrows,
                        DnsGeom g, FftTab<C> tab, int RB, double scale) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  typedef T_of<C> T;
  C* z = (C*)smem_raw;
  const int Px = g.Px;
  const long long r0 = (long long)blockIdx.x * RB;
  const int NP = RB / 2;
  for (int t = threadIdx.x; t < NP * Px; t += blockDim.x) {
    const int q = t / Px;
    const int j = t - q * Px;
    const long long ra = r0 + 2 * q, rb = ra + 1;
    C v = cmk<C>(0.0, 0.0);
    if (ra < nrows) v.x = inr[ra * rps + j];
    if (rb < nrows) v.y = inr[rb * rps + j];
    z[(size_t)q * Px + tab.drev[j]] = v;
  }
  fft_batch<C, false>(z, NP, Px, tab.plan, tab.tw);
  const int nk = Px / 2 + 1;  // the reference keeps all mx/2+1 bins
  const T sc = (T)(0.5 * scale);
  for (int t = threadIdx.x; t < RB * nk; t += blockDim.x) {
    const int rl = t / nk;
    const int k = t - rl * nk;
    const long long row = r0 + rl;
    if (row >= nrows) continue;
    const C v = unpack_r2c<C>(z + (size_t)(rl / 2) * Px, k, Px, (rl & 1) != 0);
    prow<C>(out, 0, row)[k] = v * sc;
  }
}

// pointwise Lamb vector on physical rows (drop-in computeLambVector):
// lambda may alias (u, v, w) as in the reference.
__global__ void k_lamb_rows(const double* u, const double* v, const double* w,
                            const double* ox, const double* oy, const double* oz,
                            double* lx, double* ly, double* lz, long long rps, int Px,
                            int Pz, long long nrows, const double* __restrict__ Uy, double Ro) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long row = idx / Px;
  const int j = (int)(idx - row * Px);
  if (row >= nrows) return;
  const long long o = row * rps + j;
  const double U = Uy[row / Pz];
  const double uu = u[o], vv = v[o], ww = w[o], a = ox[o], b = oy[o], c = oz[o];
  lx[o] = c * vv - b * ww - Ro * ww;
  ly[o] = a * ww - c * uu;
  lz[o] = b * uu - a * vv + Ro * (uu + U);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <typename C> struct ZTile;
// TX x TY lines per CTA: TX runs of the streamwise index (64 B) on the row
// side, TY runs of the wall-normal index on the pencil side; small enough
// for three CTAs per SM.
template <> struct ZTile<double2> { enum { TX = 4, TY = 2 }; };
template <> struct ZTile<float2> { enum { TX = 8, TY = 2 }; };

namespace {
// cuTensorMapEncodeTiled from the driver, looked up once (no -lcuda)
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return (PFN_cuTensorMapEncodeTiled_v12000)p;
  }();
  return fn;
}
// 4-D map (y, kx, kz, field) over 8-byte pencil elements, box 2 x 1 x Nz x 1
bool pencil_tmap(const PencilArr& in, int nf, const DnsGeom& g, size_t esz, CUtensorMap* m) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc || esz != 8 || !aligned16(in.base) || (in.ps * esz) % 16 || (in.fs * esz) % 16 || g.Nz > 256)
    return false;
  const cuuint64_t dims[4] = {(cuuint64_t)g.Py, (cuuint64_t)g.Kx, (cuuint64_t)g.Nz, (cuuint64_t)nf};
  const cuuint64_t strides[3] = {(cuuint64_t)(in.ps * esz), (cuuint64_t)((long long)g.Kx * in.ps * esz),
                                 (cuuint64_t)(in.fs * esz)};
  const cuuint32_t box[4] = {2, 1, (cuuint32_t)g.Nz, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, in.base, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
// 4-D map (kx, zp, y, field) over 8-byte row elements, box 2 x Pz/2 x 1 x 1
bool row_tmap(const RowArr& in, int nf, const DnsGeom& g, size_t esz, CUtensorMap* m) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc || esz != 8 || !aligned16(in.base) || (in.rs * esz) % 16 || (in.fs * esz) % 16 || g.Pz % 2 ||
      g.Pz / 2 > 256)
    return false;
  const cuuint64_t dims[4] = {(cuuint64_t)g.Kx, (cuuint64_t)g.Pz, (cuuint64_t)g.Py, (cuuint64_t)nf};
  const cuuint64_t strides[3] = {(cuuint64_t)(in.rs * esz), (cuuint64_t)((long long)g.Pz * in.rs * esz),
                                 (cuuint64_t)(in.fs * esz)};
  const cuuint32_t box[4] = {2, (cuuint32_t)(g.Pz / 2), 1, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, in.base, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

// warp-FFT tiles gathered through L1: FP32 4 x 4 lines on 8 warps (whole
// 32-byte sectors on both sides, three CTAs per SM); FP64 4 x 2 lines on 4
// warps (64-byte runs on the row side, 32-byte runs of y pairs on the
// pencil side, four CTAs per SM)
template <typename C> struct ZWarpTile;
template <> struct ZWarpTile<float2> { enum { NW = 8, TX = 4, TY = 4 }; };
template <> struct ZWarpTile<double2> { enum { NW = 4, TX = 4, TY = 2 }; };

template <typename C>
cudaError_t launch_zb(PencilArr in, RowArr out, int nf, DnsGeom g, FftTab<C> tab, cudaStream_t st,
                      int* status, int variant, bool probe) {
  const int TX = ZTile<C>::TX, TY = ZTile<C>::TY;
  const bool any = variant == VAR_AUTO;
  return with_len_xz(g.Pz, [&](auto LL) -> cudaError_t {
    constexpr int L = decltype(LL)::value;
    if constexpr (L > 0 && WPlan<L, 2, FftMaxRadix<C>::v>::ok) {
     const C* tw = wtw_of(tab, 1);
     constexpr int LS = wlen<C>(L) + 1;
     if constexpr (sizeof(C) == 8) {
      CUtensorMap tm;
      if ((any || variant == DNS_Z_TENSOR_COPY) && status && g.Nz == L / 3 * 2 && tw &&
          (size_t)g.Nz * 16 + 128 <= (size_t)2 * LS * sizeof(C) && pencil_tmap(in, nf, g, sizeof(C), &tm)) {
       if (probe) return cudaSuccess;
       // pencils staged by tensor copies (a y pair per line pair), 8 x 2
       // tile: 64-byte runs on the row side
       const size_t sm = ((size_t)16 * LS) * sizeof(C);
       cudaFuncSetAttribute(k_zbt<C, L, 8, 8, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
       dim3 grid((g.Kx + 7) / 8, (g.Py + 1) / 2, nf);
       k_zbt<C, L, 8, 8, 2><<<grid, 256, sm, st>>>(tm, out, g, tab, status);
       return cudaGetLastError();
      }
     }
     if ((any || variant == DNS_Z_WARP) && g.Nz == L / 3 * 2 && tw) {
      if (probe) return cudaSuccess;
      typedef ZWarpTile<C> WT;
      const size_t sm = ((size_t)WT::TX * WT::TY * LS) * sizeof(C);
      // the rest of the SM's memory as L1: the pencil-side gathers of
      // neighbouring threads share sectors (measured in FP32: a quarter
      // faster than four CTAs with a small L1)
      auto k = k_zbw<C, L, WT::NW, WT::TX, WT::TY>;
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 75);
      dim3 grid((g.Kx + WT::TX - 1) / WT::TX, (g.Py + WT::TY - 1) / WT::TY, nf);
      k<<<grid, 32 * WT::NW, sm, st>>>(in, out, g, tab);
      return cudaGetLastError();
     }
    }
    if (!any && variant != DNS_Z_BLOCK) return cudaErrorNotSupported;
    if (probe) return cudaSuccess;
    const size_t sm = (size_t)TX * TY * FLine<C, L>::stride(g.Pz) * sizeof(C);
    cudaFuncSetAttribute(k_zb<C, TX, TY, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    dim3 grid((g.Kx + TX - 1) / TX, (g.Py + TY - 1) / TY, nf);
    k_zb<C, TX, TY, L><<<grid, 256, sm, st>>>(in, out, g, tab);
    return cudaGetLastError();
  });
}
template <typename C>
cudaError_t launch_zf(RowArr in, PencilArr out, int nf, DnsGeom g, FftTab<C> tab, cudaStream_t st,
                      int* status, int variant, bool probe) {
  const int TX = ZTile<C>::TX, TY = ZTile<C>::TY;
  const bool any = variant == VAR_AUTO;
  return with_len_xz(g.Pz, [&](auto LL) -> cudaError_t {
    constexpr int L = decltype(LL)::value;
    if constexpr (L > 0 && WPlan<L, 2, FftMaxRadix<C>::v>::ok) {
     const C* tw = wtw_of(tab, 1);
     constexpr int LS = wlen<C>(L) + 1;
     if constexpr (sizeof(C) == 8) {
      CUtensorMap tm;
      if ((any || variant == DNS_Z_TENSOR_COPY) && status && g.Nz == L / 3 * 2 && tw &&
          (size_t)L * 16 + 128 <= (size_t)2 * LS * sizeof(C) && row_tmap(in, nf, g, sizeof(C), &tm)) {
       if (probe) return cudaSuccess;
       // rows staged by tensor copies, 4 x 4 tile
       const size_t sm = ((size_t)16 * LS) * sizeof(C);
       cudaFuncSetAttribute(k_zft<C, L, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
       dim3 grid((g.Kx + 3) / 4, (g.Py + 3) / 4, nf);
       k_zft<C, L, 8><<<grid, 256, sm, st>>>(tm, out, g, tab, status);
       return cudaGetLastError();
      }
     }
     if ((any || variant == DNS_Z_WARP) && g.Nz == L / 3 * 2 && tw) {
      if (probe) return cudaSuccess;
      typedef ZWarpTile<C> WT;
      const size_t sm = ((size_t)WT::TX * WT::TY * LS) * sizeof(C);
      auto k = k_zfw<C, L, WT::NW, WT::TX, WT::TY>;
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 75);
      dim3 grid((g.Kx + WT::TX - 1) / WT::TX, (g.Py + WT::TY - 1) / WT::TY, nf);
      k<<<grid, 32 * WT::NW, sm, st>>>(in, out, g, tab);
      return cudaGetLastError();
     }
    }
    if (!any && variant != DNS_Z_BLOCK) return cudaErrorNotSupported;
    if (probe) return cudaSuccess;
    const size_t sm = (size_t)TX * TY * FLine<C, L>::stride(g.Pz) * sizeof(C);
    cudaFuncSetAttribute(k_zf<C, TX, TY, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    dim3 grid((g.Kx + TX - 1) / TX, (g.Py + TY - 1) / TY, nf);
    k_zf<C, TX, TY, L><<<grid, 256, sm, st>>>(in, out, g, tab);
    return cudaGetLastError();
  });
}
template <typename C>
cudaError_t launch_x_fused(RowArr in, RowArr out, DnsGeom g, FftTab<C> tab, const double* Uy,
                           double Ro, int* status, cudaStream_t st, int variant, bool probe,
                           const double* runs) {
  const bool any = variant == VAR_AUTO;
  return with_len_xz(g.Px, [&](auto LL) -> cudaError_t {
    constexpr int L = decltype(LL)::value;
    if constexpr (L > 0) {
      const long long nrows = (long long)g.Py * g.Pz * g.nrun;
      // four rows per CTA within one wall-normal plane; a warp's staged
      // rows of SR >= Nx/2 bins (2 SR <= a line) fit in its lines
      constexpr int SR = (L / 3 + 15) / 16 * 16;
      const bool ok = g.Pz % 4 == 0 && g.Nx / 2 == L / 3 && 2 * SR <= wlen<C>(L) && in.rs >= SR &&
                      (in.rs * sizeof(C)) % 16 == 0 && (in.fs * sizeof(C)) % 16 == 0;
      const size_t sm = ((size_t)12 * wlen<C>(L)) * sizeof(C) + 64;
      // FP32: the plans' twiddle tables; FP64: W^j with product recurrences
      if constexpr (WPlan<L, 4, FftMaxRadix<C>::v>::ok && WPlan<L, 2, FftMaxRadix<C>::v>::ok) {
        if (ok && wtw_of(tab, 1) && wtw_of(tab, 2) && (any || variant == DNS_X_WARP3)) {
          if (probe) return cudaSuccess;
          cudaFuncSetAttribute(k_xw<C, L, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
          k_xw<C, L, 3><<<(unsigned)((nrows + 3) / 4), 96, sm, st>>>(in, out, g, tab, Uy, Ro, runs, status);
          return cudaGetLastError();
        }
      }
      if constexpr (WPlan<L, 2, FftMaxRadix<C>::v>::ok && WPlan<L, 1, FftMaxRadix<C>::v>::ok) {
        if (ok && wtw_of(tab, 0) && wtw_of(tab, 1) && variant == DNS_X_WARP6) {
          if (probe) return cudaSuccess;
          cudaFuncSetAttribute(k_xw<C, L, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
          k_xw<C, L, 6><<<(unsigned)((nrows + 3) / 4), 192, sm, st>>>(in, out, g, tab, Uy, Ro, runs, status);
          return cudaGetLastError();
        }
      }
    }
    if (!any && variant != DNS_X_BLOCK) return cudaErrorNotSupported;
    if (probe) return cudaSuccess;
    const size_t sm = (size_t)(L > 0 ? 6 : 9) * FLine<C, L>::stride(g.Px) * sizeof(C);
    cudaFuncSetAttribute(k_x_fused<C, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    const long long nrows = (long long)g.Py * g.Pz * g.nrun;  // Pz is even: row pairs share a plane
    k_x_fused<C, L><<<(unsigned)((nrows + 1) / 2), 256, sm, st>>>(in, out, g, tab, Uy, Ro, runs);
    return cudaGetLastError();
  });
}
template <typename C>
cudaError_t launch_x_c2r(RowArr in, T_of<C>* outr, long long rps, long long nrows, DnsGeom g,
                         FftTab<C> tab, cudaStream_t st) {
  const int RB = 4;
  const size_t sm = (size_t)(RB / 2) * g.Px * sizeof(C);
  cudaFuncSetAttribute(k_x_c2r<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_x_c2r<C><<<(unsigned)((nrows + RB - 1) / RB), 256, sm, st>>>(in, outr, rps, nrows, g, tab, RB);
  return cudaGetLastError();
}
template <typename C>
cudaError_t launch_x_r2c(const T_of<C>* inr, long long rps, RowArr out, long long nrows,
                         DnsGeom g, FftTab<C> tab, double scale, cudaStream_t st) {
  const int RB = 4;
  const size_t sm = (size_t)(RB / 2) * g.Px * sizeof(C);
  cudaFuncSetAttribute(k_x_r2c<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_x_r2c<C><<<(unsigned)((nrows + RB - 1) / RB), 256, sm, st>>>(inr, rps, out, nrows, g, tab, RB, scale);
  return cudaGetLastError();
}
cudaError_t launch_lamb_rows(const double* const in6[6], double* const out3[3], long long rps,
                             long long nrows, DnsGeom g, const double* Uy, double Ro,
                             cudaStream_t st) {
  const long long n = nrows * g.Px;
  const int th = 256;
  k_lamb_rows<<<(unsigned)((n + th - 1) / th), th, 0, st>>>(
      in6[0], in6[1], in6[2], in6[3], in6[4], in6[5], out3[0], out3[1], out3[2], rps, g.Px, g.Pz,
      nrows, Uy, Ro);
  return cudaGetLastError();
}

#define INST_Z(C)                                                                                  \
  template cudaError_t launch_zb<C>(PencilArr, RowArr, int, DnsGeom, FftTab<C>, cudaStream_t, int*, int, bool); \
  template cudaError_t launch_zf<C>(RowArr, PencilArr, int, DnsGeom, FftTab<C>, cudaStream_t, int*, int, bool); \
  template cudaError_t launch_x_fused<C>(RowArr, RowArr, DnsGeom, FftTab<C>, const double*,       \
                                         double, int*, cudaStream_t, int, bool, const double*);   \
  template cudaError_t launch_x_c2r<C>(RowArr, T_of<C>*, long long, long long, DnsGeom,           \
                                       FftTab<C>, cudaStream_t);                                  \
  template cudaError_t launch_x_r2c<C>(const T_of<C>*, long long, RowArr, long long, DnsGeom,     \
                                       FftTab<C>, double, cudaStream_t);
INST_Z(double2)
INST_Z(float2)
