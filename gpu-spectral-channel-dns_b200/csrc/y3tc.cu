// Backward wall-normal pass (y3) on the tensor cores: getUVW and the padded
// Chebyshev synthesis (source/velocity.cu:90-170, source/transform.cu:
// 416-453,679-697) of the six velocity / vorticity fields as batched dense
// 3xTF32 products with FP32 accumulation, for Ny = 129 (mz = 512) in the
// mixed form.
//
// The padded s2p of a pencil is f(y_m) = sum_k c_k T_k(y_m) at the Py = 257
// Gauss-Lobatto points y_m = cos(pi m / 256).  With T_k(-y) = (-1)^k T_k(y)
// it splits into the even and odd halves
//   E(m) = sum_j c_2j T_2j(y_m),  O(m) = sum_j c_2j+1 T_2j+1(y_m),  m < 128,
//   f(y_m) = E + O,  f(y_256-m) = E - O,
// two 128 x 64 real matrices T_E, T_O (the coefficient c_128 of the even half
// is added in the epilogue: T_128(y_m) = cos(pi m / 2)), and the centre point
// y_128 = 0 is a weighted sum done on the CUDA cores.  The derivatives that
// getUVW needs are taken in coefficient space first (the ddz recurrence,
// source/RPCFKernels.cu:439-520, in FP64), so every output is a combination
// of T applied to five coefficient vectors per pencil: v, Dv, D^2 v, omega,
// D omega.  Per tile of 8 pencils the B operand has 8 x 5 x 2 (re, im) = 80
// columns; D = T_par * B for par = E, O is 2 x 80 FP32 accumulator columns.
//
// Precision (3xTF32): each operand x is split into TF32 hi + lo (x = hi + lo
// to 2^-22 relative) and D += A_hi B_hi + A_hi B_lo + A_lo B_hi, accumulated
// in FP32 in tensor memory.
//
// CTA layout (one per SM, persistent over tiles; 224 threads):
//   warps 0-3  epilogue: TMEM lanes 32w..32w+31 = points m; the T matrices
//              are written into TMEM by these warps at the start
//   warp 4     MMA issue (one thread)
//   warps 5-6  producers, one tile each in turn: the FP64 state of 8
//              pencils (bulk-copied into shared memory one tile ahead) ->
//              derivative recurrences -> TF32 hi/lo -> B (smem), with the
//              c_128 and centre-point values handed to the epilogue through
//              four rotating side slots
// Tensor memory (512 columns): A = T_E hi | T_E lo | T_O hi | T_O lo (4 x 64
// columns), D_E (80), D_O (80).  Shared memory: B double-buffered (2 x 80
// KB), the state staging of each producer (2 x 32 KB), side slots, barriers.
// Every mbarrier wait is bounded; a CTA that gives up records the timeout in
// *status, lets its tensor-core work finish and frees its tensor memory.
#include <cmath>
#include <cstring>

#include "kernels.cuh"
#include "tc05.cuh"

namespace {

constexpr int TC_NY = 129;                 // Chebyshev modes
constexpr int TC_PY = 257;                 // padded points
constexpr int TC_NH = 128;                 // points per half (M of the MMA)
constexpr int TC_KP = 64;                  // coefficients per parity (K)
constexpr int TC_NP = 8;                   // pencils per tile
constexpr int TC_NV = 5;                   // coefficient vectors per pencil
constexpr int TC_N = TC_NP * TC_NV * 2;    // B columns (N of the MMA) = 80
constexpr uint32_t TC_KC_BYTES = (TC_N / 8) * 128;            // one 16-byte K chunk of all N rows
constexpr uint32_t TC_PART_BYTES = (TC_KP / 4) * TC_KC_BYTES; // one (parity, hi|lo) operand: 20 KB
constexpr uint32_t TC_BUF_BYTES = 4 * TC_PART_BYTES;          // one tile: E hi, E lo, O hi, O lo
constexpr uint32_t TC_STAGE_BYTES = 2 * TC_NP * TC_NY * 16;   // the FP64 state (v, omega) of a tile
constexpr int TC_NSIDE = 4;                                   // rotating side-data slots
constexpr uint32_t TC_TMEM_COLS = 512;
constexpr uint32_t TC_COL_A = 0;           // A: [par][hi|lo][64]
constexpr uint32_t TC_COL_D = 256;         // D: [par][80]
constexpr int TC_THREADS = 224;

static_assert(TC_N % 16 == 0 && TC_N <= 256, "N of an M = 128 MMA");
static_assert(TC_COL_D + 2 * TC_N <= TC_TMEM_COLS, "tensor memory");

// per tile, from the producer to the epilogue: c_128 of v and omega (the
// T_128 term of the even half) and the values at the centre point y = 0 of
// the five coefficient vectors, per B column (j, q, re|im)
struct Side {
  float a128[TC_NP][2][2];  // [pencil][v | omega][re | im]
  float centre[TC_N];
};

struct Bars {
  uint64_t full_b[2], empty_b[2], stage[2], side[TC_NSIDE], full_d, empty_d, done;
  uint32_t tmem_base;
  int abort;
};

constexpr size_t TC_SMEM = 2 * (size_t)TC_BUF_BYTES + 2 * (size_t)TC_STAGE_BYTES +
                           TC_NSIDE * sizeof(Side) + ((sizeof(Bars) + 127) / 128) * 128;
static_assert(TC_SMEM <= 232448, "shared memory of one CTA");

__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity, Bars* bs, int* status) {
  if (*(volatile int*)&bs->abort) return false;
  if (mbar_wait_bounded(bar, parity, DNS_WAIT_LIMIT, status)) return true;
  atomicOr(status, 1);
  *(volatile int*)&bs->abort = 1;
  return false;
}

// byte offset of element (row n, K chunk kc) of one operand part: core
// matrices of 8 rows x 4 K values, 8-row groups 128 B apart, K chunks
// TC_KC_BYTES apart
__device__ __forceinline__ uint32_t b_off(int n, int kc) {
  return (uint32_t)kc * TC_KC_BYTES + (uint32_t)(n >> 3) * 128u + (uint32_t)(n & 7) * 16u;
}

// FP32 bits -> TF32 bits, round to nearest with ties away from zero (the
// rounding of cvt.rna.tf32.f32) on the integer pipe: add half an ulp of the
// 10-bit mantissa, clear the 13 low bits
__device__ __forceinline__ uint32_t tf32_bits(uint32_t u) { return (u + 0x1000u) & ~0x1FFFu; }

// x = hi + lo: hi rounded to TF32, lo the exact FP32 remainder passed as
// it is (the tensor core reads the top 19 bits of a TF32 operand, so lo
// enters truncated: error < 2^-10 |lo| <= 2^-21 |x|)
__device__ __forceinline__ void split_f(float x, uint32_t& hi, uint32_t& lo) {
  hi = tf32_bits(__float_as_uint(x));
  lo = __float_as_uint(x - __uint_as_float(hi));
}

__device__ __forceinline__ float2 cmul_i(float2 a, float s) { return make_float2(-a.y * s, a.x * s); }  // i s a

// the six fields at one point from the five coefficient-vector values x
// (v, Dv, D^2 v, omega, D omega), getUVW's combination
// (source/velocity.cu:106-169); the mean pencil carries u0, w0
__device__ __forceinline__ void uvw_point(const float2 (&x)[5], bool zero, float fa, float fb, float fia,
                                          float fib, float2 (&f)[6]) {
  if (zero) {
    f[0] = x[0];
    f[1] = x[3];
    f[2] = make_float2(0.f, 0.f);
    f[3] = x[4];
    f[4] = make_float2(-x[1].x, -x[1].y);
    f[5] = make_float2(0.f, 0.f);
  } else {
    const float2 du = cmul_i(x[2], fa) - cmul_i(x[4], fb);
    const float2 dv = cmul_i(x[2], fb) + cmul_i(x[4], fa);
    f[0] = cmul_i(x[1], fa) - cmul_i(x[3], fb);
    f[1] = cmul_i(x[1], fb) + cmul_i(x[3], fa);
    f[2] = x[0];
    f[3] = dv - cmul_i(x[0], fib);
    f[4] = cmul_i(x[0], fia) - du;
    f[5] = x[3];
  }
}

}  // namespace

__global__ void __launch_bounds__(TC_THREADS, 1)
    k_y3tc(const double2* __restrict__ V, const double2* __restrict__ O, PencilArr out, DnsGeom g,
           PhysParams ph, const uint32_t* __restrict__ atab, long long ntiles, int* status) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* bbuf = smem_raw;                               // [2][par][hl] operand parts
  double* stage = (double*)(smem_raw + 2 * TC_BUF_BYTES);       // [producer][v|omega][pencil][k][re|im]
  Side* side = (Side*)(smem_raw + 2 * TC_BUF_BYTES + 2 * TC_STAGE_BYTES);
  Bars* bs = (Bars*)(smem_raw + 2 * TC_BUF_BYTES + 2 * TC_STAGE_BYTES + TC_NSIDE * sizeof(Side));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long H = g.H;

  if (threadIdx.x == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&bs->full_b[i], 1);
      mbar_init(&bs->empty_b[i], 1);
      mbar_init(&bs->stage[i], 1);
    }
    for (int i = 0; i < TC_NSIDE; ++i) mbar_init(&bs->side[i], 1);
    mbar_init(&bs->full_d, 1);
    mbar_init(&bs->empty_d, 4);
    mbar_init(&bs->done, 1);
    bs->abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) {
    tmem_alloc(&bs->tmem_base, TC_TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = bs->tmem_base;

  // the producers start their first copies now, under the A set-up
  auto issue_stage = [&](int b, long long t) {
    const long long p0 = t * TC_NP;
    const long long np = (H - p0) < TC_NP ? (H - p0) : TC_NP;
    const uint32_t bytes = (uint32_t)(np * TC_NY * 16);
    double* st = stage + (size_t)b * (TC_STAGE_BYTES / 8);
    mbar_expect_tx(&bs->stage[b], 2 * bytes);
    bulk_g2s(st, V + p0 * TC_NY, bytes, &bs->stage[b]);
    bulk_g2s(st + TC_NP * TC_NY * 2, O + p0 * TC_NY, bytes, &bs->stage[b]);
  };
  if (warp >= 5 && lane == 0) {
    const int b = warp - 5;
    const long long t = blockIdx.x + (long long)b * gridDim.x;
    if (t < ntiles) issue_stage(b, t);
  }

  // A operand: row m of T_E, T_O (hi, lo) into TMEM lane m, from the
  // table [column][m] (consecutive lanes read consecutive words)
  if (warp < 4) {
    const int m = warp * 32 + lane;
    const uint32_t lane_addr = tbase + ((uint32_t)(warp * 32) << 16);
    // 32 loads in flight per thread
    for (int c0 = 0; c0 < 4 * TC_KP; c0 += 32) {
      uint32_t w[4][8];
#pragma unroll
      for (int i = 0; i < 32; ++i) w[i >> 3][i & 7] = __ldg(&atab[(size_t)(c0 + i) * TC_NH + m]);
#pragma unroll
      for (int q = 0; q < 4; ++q) tmem_st_x8(lane_addr + TC_COL_A + (uint32_t)(c0 + 8 * q), w[q]);
    }
    tmem_wait_st();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  if (warp == 4) {
    // ---- MMA issue ---------------------------------------------------------
    if (lane == 0) {
      const uint32_t idesc = tc_idesc_tf32(TC_NH, TC_N);
      const uint32_t bbase = smem_u32(bbuf);
      // descriptors of the K steps of buffer 0 (buffer 1: + TC_BUF_BYTES >> 4
      // in the start-address field, which stays below 2^14)
      uint64_t dsc[2][2][TC_KP / 8];  // [par][hi|lo][s]
#pragma unroll
      for (int par = 0; par < 2; ++par)
#pragma unroll
        for (int hl = 0; hl < 2; ++hl)
#pragma unroll
          for (int s = 0; s < TC_KP / 8; ++s)
            dsc[par][hl][s] = tc_sdesc(bbase + (uint32_t)(par * 2 + hl) * TC_PART_BYTES +
                                           (uint32_t)(2 * s) * TC_KC_BYTES,
                                       TC_KC_BYTES, 128);
      long long it = 0;
      for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int b = (int)(it & 1);
        const uint32_t use = (uint32_t)(it >> 1);
        if (!tc_wait(&bs->full_b[b], use & 1u, bs, status)) break;
        if (!tc_wait(&bs->empty_d, ((uint32_t)it & 1u) ^ 1u, bs, status)) break;
        tc_fence_after();
        // the even and odd products alternate, so that consecutive MMAs
        // accumulate into different tensor-memory tiles
        const uint64_t boff = (uint64_t)(b * (TC_BUF_BYTES >> 4));
#pragma unroll
        for (int s = 0; s < TC_KP / 8; ++s)
#pragma unroll
          for (int k3 = 0; k3 < 3; ++k3)
#pragma unroll
            for (int par = 0; par < 2; ++par) {
              const uint32_t d = tbase + TC_COL_D + (uint32_t)(par * TC_N);
              const uint32_t a = tbase + TC_COL_A + (uint32_t)(par * 128 + 8 * s + (k3 == 2 ? 64 : 0));
              const uint64_t bd = dsc[par][k3 == 1 ? 1 : 0][s] + boff;
              mma_tf32_ts(d, a, bd, idesc, (s > 0 || k3 > 0) ? 1u : 0u);
            }
        umma_commit(&bs->empty_b[b]);
        umma_commit(&bs->full_d);
      }
      // every tensor-core operation issued here has completed before the
      // tensor memory is freed
      umma_commit(&bs->done);
      mbar_wait_bounded(&bs->done, 0, DNS_WAIT_LIMIT, nullptr);
    }
  } else if (warp >= 5) {
    // ---- producers: tiles it = warp - 5, warp - 5 + 2, ... ------------------
    const int b = warp - 5;
    const int j = lane >> 2, fld = (lane >> 1) & 1, r = lane & 1;
    const int q0 = fld ? 3 : 0;  // first coefficient vector of this thread
    const int nv = fld ? 2 : 3;  // v, Dv, D^2v  |  omega, D omega
    unsigned char* buf = bbuf + (size_t)b * TC_BUF_BYTES;
    const double* src = stage + (size_t)b * (TC_STAGE_BYTES / 8) + (size_t)fld * TC_NP * TC_NY * 2 +
                        (size_t)j * TC_NY * 2 + r;  // element k at src[2k]
    long long it = b;
    for (long long t = blockIdx.x + (long long)b * gridDim.x; t < ntiles; t += 2LL * gridDim.x, it += 2) {
      const uint32_t use = (uint32_t)(it >> 1);
      if (!tc_wait(&bs->stage[b], use & 1u, bs, status)) break;
      if (!tc_wait(&bs->empty_b[b], (use & 1u) ^ 1u, bs, status)) break;
      const bool ok = t * TC_NP + j < H;
      // backward sweep k = 127 .. 0: b_k = b_k+2 + 2(k+1) a_k+1 (D),
      // c_k = c_k+2 + 2(k+1) b_k+1 (D^2), b_0 and c_0 halved; the centre
      // values sum_k x_k T_k(0) on the way.  In FP32: the products are
      // FP32-accurate (3xTF32) and feed FP32 transforms only.
      const float a128 = ok ? (float)src[2 * 128] : 0.f;
      float a_next = a128;
      float b1 = 0.f, b2 = 0.f, c1 = 0.f, c2 = 0.f;
      float z0 = a128, z1 = 0.f, z2 = 0.f;  // T_128(0) = 1
      for (int kc = TC_KP / 4 - 1; kc >= 0; --kc) {
        uint32_t h[3][2][4], l[3][2][4];  // [vector][parity][slot]
#pragma unroll
        for (int i = 7; i >= 0; --i) {
          const int k = 8 * kc + i;
          const float ak = ok ? (float)src[2 * k] : 0.f;
          const float f = (float)(2 * (k + 1));
          float bk = b2 + f * a_next;
          float ck = c2 + f * b1;
          if (k == 0) {
            bk *= 0.5f;
            ck *= 0.5f;
          }
          if (!(i & 1)) {  // T_k(0) = (-1)^(k/2) for even k, 0 for odd k
            const float w = (i & 2) ? -1.f : 1.f;
            z0 += w * ak;
            z1 += w * bk;
            z2 += w * ck;
          }
          const int par = i & 1, slot = i >> 1;
          split_f(ak, h[0][par][slot], l[0][par][slot]);
          split_f(bk, h[1][par][slot], l[1][par][slot]);
          split_f(ck, h[2][par][slot], l[2][par][slot]);
          b2 = b1;
          b1 = bk;
          c2 = c1;
          c1 = ck;
          a_next = ak;
        }
#pragma unroll
        for (int v = 0; v < 3; ++v) {
          if (v >= nv) break;
          const int n = j * 10 + (q0 + v) * 2 + r;
#pragma unroll
          for (int par = 0; par < 2; ++par) {
            const uint32_t o = b_off(n, kc);
            *(uint4*)(buf + (size_t)(par * 2) * TC_PART_BYTES + o) =
                make_uint4(h[v][par][0], h[v][par][1], h[v][par][2], h[v][par][3]);
            *(uint4*)(buf + (size_t)(par * 2 + 1) * TC_PART_BYTES + o) =
                make_uint4(l[v][par][0], l[v][par][1], l[v][par][2], l[v][par][3]);
          }
        }
      }
      // side data of this tile (slot it % 4)
      Side& sd = side[it & (TC_NSIDE - 1)];
      sd.a128[j][fld][r] = a128;
      sd.centre[j * 10 + q0 * 2 + r] = z0;
      sd.centre[j * 10 + (q0 + 1) * 2 + r] = z1;
      if (!fld) sd.centre[j * 10 + 4 + r] = z2;
      // the staging buffer is free: fetch this warp's next tile under the
      // other producer's and the epilogue's work
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) {
        const long long tn = t + 2LL * gridDim.x;
        if (tn < ntiles) issue_stage(b, tn);
        mbar_arrive(&bs->side[it & (TC_NSIDE - 1)]);
        mbar_arrive(&bs->full_b[b]);
      }
    }
  } else {
    // ---- epilogue (warps 0-3): point m = 32 warp + lane ---------------------
    const int m = warp * 32 + lane;
    const uint32_t lane_addr = tbase + ((uint32_t)(warp * 32) << 16) + TC_COL_D;
    const float cs = (m & 3) == 0 ? 1.f : ((m & 3) == 2 ? -1.f : 0.f);  // T_128(y_m)
    long long it = 0;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
      // per-pencil factors while the tensor cores work: lane j < 8 forms
      // pencil j's (FP64 divisions, once per warp), the warp shares them
      float lfa = 0.f, lfb = 0.f, lfia = 0.f, lfib = 0.f;
      bool lzero = false;
      if (lane < TC_NP) {
        const long long p = t * TC_NP + lane;
        int run, kx, kz;
        pencil_modes(g, p, run, kx, kz);
        double ia, ib;
        wavenumbers(kx, kz, g.Nz, ph.aphi, ph.beta, ia, ib);
        lzero = kx == 0 && kz == 0;
        const double kmn1 = lzero ? 0.0 : 1.0 / kmn_of(ia, ib);
        lfa = (float)(ia * kmn1);
        lfb = (float)(ib * kmn1);
        lfia = (float)ia;
        lfib = (float)ib;
      }
      float fa[TC_NP], fb[TC_NP], fia[TC_NP], fib[TC_NP];
      const unsigned zero_mask = __ballot_sync(0xffffffffu, lzero) & ((1u << TC_NP) - 1u);
#pragma unroll
      for (int j = 0; j < TC_NP; ++j) {
        fa[j] = __shfl_sync(0xffffffffu, lfa, j);
        fb[j] = __shfl_sync(0xffffffffu, lfb, j);
        fia[j] = __shfl_sync(0xffffffffu, lfia, j);
        fib[j] = __shfl_sync(0xffffffffu, lfib, j);
      }
      const int sl = (int)(it & (TC_NSIDE - 1));
      if (!tc_wait(&bs->side[sl], (uint32_t)(it >> 2) & 1u, bs, status)) break;
      const Side& sd = side[sl];
      if (!tc_wait(&bs->full_d, (uint32_t)it & 1u, bs, status)) break;
      tc_fence_after();
      // the whole tile's accumulators into registers (E: columns 0-79, O:
      // 80-159), then the tensor memory is released for the next tile's
      // products while this tile is combined and stored
      uint32_t acc[2 * TC_N];
#pragma unroll
      for (int c = 0; c < 2 * TC_N; c += 16) tmem_ld_x16(lane_addr + (uint32_t)c, &acc[c]);
      tmem_wait_ld();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bs->empty_d);
#pragma unroll
      for (int j = 0; j < TC_NP; ++j) {
        const long long p = t * TC_NP + j;
        if (p >= H) continue;
        float2 E[5], Od[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          E[q] = make_float2(__uint_as_float(acc[j * 10 + 2 * q]), __uint_as_float(acc[j * 10 + 2 * q + 1]));
          Od[q] = make_float2(__uint_as_float(acc[TC_N + j * 10 + 2 * q]),
                              __uint_as_float(acc[TC_N + j * 10 + 2 * q + 1]));
        }
        E[0].x += sd.a128[j][0][0] * cs;
        E[0].y += sd.a128[j][0][1] * cs;
        E[3].x += sd.a128[j][1][0] * cs;
        E[3].y += sd.a128[j][1][1] * cs;
        float2* base = (float2*)out.base + p * out.ps;
#pragma unroll
        for (int sideb = 0; sideb < 2; ++sideb) {
          float2 x[5];
          const float sg = sideb ? -1.f : 1.f;
#pragma unroll
          for (int q = 0; q < 5; ++q) x[q] = make_float2(E[q].x + sg * Od[q].x, E[q].y + sg * Od[q].y);
          float2 f[6];
          uvw_point(x, (zero_mask >> j) & 1u, fa[j], fb[j], fia[j], fib[j], f);
          const int pt = sideb ? TC_PY - 1 - m : m;
#pragma unroll
          for (int fi = 0; fi < 6; ++fi) base[fi * out.fs + pt] = f[fi];
        }
      }
      // the centre point y = 0 (m = 128) of the tile's pencils, lanes 0-7 of warp 0
      if (warp == 0 && lane < TC_NP) {
        const int j = lane;
        const long long p = t * TC_NP + j;
        if (p < H) {
          float2 x[5];
          for (int q = 0; q < 5; ++q) x[q] = make_float2(sd.centre[j * 10 + 2 * q], sd.centre[j * 10 + 2 * q + 1]);
          float2 f[6];
          uvw_point(x, lzero, lfa, lfb, lfia, lfib, f);  // this lane's own pencil j
          float2* base = (float2*)out.base + p * out.ps;
          for (int fi = 0; fi < 6; ++fi) base[fi * out.fs + TC_NH] = f[fi];
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, TC_TMEM_COLS);
  }
}

// The tensor-core y3 pass: Ny = 129 (mz = 512), FP32 output pencils of
// pitch >= 257; V, O the FP64 state.  Returns cudaErrorNotSupported for
// other sizes (the caller keeps the FFT pass).
cudaError_t launch_y3tc(const double2* V, const double2* O, PencilArr out, DnsGeom g, PhysParams ph,
                        const uint32_t* atab, int* status, cudaStream_t st) {
  if (g.Ny != TC_NY || g.Py != TC_PY || out.ps < TC_PY || !atab) return cudaErrorNotSupported;
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (!e) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e) return e;
  e = cudaFuncSetAttribute(k_y3tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
  if (e) return e;
  if (!aligned16(V) || !aligned16(O)) return cudaErrorNotSupported;
  const long long ntiles = (g.H + TC_NP - 1) / TC_NP;
  const unsigned grid = (unsigned)(ntiles < nsm ? ntiles : nsm);
  k_y3tc<<<grid, TC_THREADS, TC_SMEM, st>>>(V, O, out, g, ph, atab, ntiles, status);
  return cudaGetLastError();
}

// The A table of the tensor-core y3 pass: word [c][m] for TMEM column c and
// point m < 128; columns 0-63 T_2j(y_m) TF32 hi, 64-127 its lo part,
// 128-191 T_2j+1(y_m) hi, 192-255 lo (y_m = cos(pi m / 256)); hi is the value
// rounded to TF32 (nearest, ties away), lo the rounded remainder.
size_t y3tc_table_words() { return (size_t)4 * TC_KP * TC_NH; }

static uint32_t host_tf32(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u = (u + 0x1000u) & ~0x1FFFu;  // 10 mantissa bits, ties away from zero
  return u;
}

void y3tc_table(uint32_t* w) {
  const long double PI = 3.141592653589793238462643383279502884L;
  for (int par = 0; par < 2; ++par)
    for (int j = 0; j < TC_KP; ++j)
      for (int m = 0; m < TC_NH; ++m) {
        const int num = ((2 * j + par) * m) % 512;  // angle num * pi / 256, exact reduction
        const double x = (double)cosl(PI * (long double)num / 256.0L);
        const uint32_t hi = host_tf32((float)x);
        float hf;
        std::memcpy(&hf, &hi, 4);
        const uint32_t lo = host_tf32((float)(x - (double)hf));
        w[(size_t)(par * 128 + j) * TC_NH + m] = hi;
        w[(size_t)(par * 128 + 64 + j) * TC_NH + m] = lo;
      }
}
