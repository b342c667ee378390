// Slab decomposition plan (host only): which pencils and which wall-normal
// planes each of R ranks owns, and the blocks the two exchanges of a step
// move between them.  No counterpart in the reference (its multi-GPU
// transform is dead code); the partition follows the structure of the step:
//
//   * the wall-normal passes (y3, y1) and the solve work per pencil, and the
//     solve pairs the pencils kz' and Nz - kz' on one operator slot, so a
//     rank owns a contiguous range of slots kz' in [k0, k1) and both pencils
//     of each: two runs of spanwise indices, [k0, k1) and
//     [Nz - k1 + 1, Nz - k0] minus kz' in {0, Nz/2}, pencils p = kz Kx + kx
//     contiguous within a run;
//   * the spanwise and streamwise passes (zb, x, zf) work per wall-normal
//     plane, so a rank owns a contiguous range of the Py planes.
//
// Backward exchange (after y3, 6 fields): the pencil owner r sends, for
// every plane owner s, its pencils restricted to s's planes; forward (after
// zf, 3 fields) the same blocks travel back.  A segment is one run of
// pencils x one range of planes; the pencil owner lists, per peer, the runs
// in increasing kz, and the plane owner lists the same segments per peer in
// the same order, so packed buffers agree field by field.
#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

#include "../../include/dns_b200.h"

// records the message for dns_last_error() (context.cu)
dns_status dns_internal_fail(dns_status s, const char* msg);

namespace {

struct Part {
  int Nz, Kx, Kh, Py;
  std::vector<int> s0, s1, y0, y1;  // slot and plane ranges per rank
};

int pencils_of_slot(int kzs, int Nz) { return (kzs == 0 || kzs == Nz / 2) ? 1 : 2; }

bool make_part(int mx, int my, int mz, int R, Part& P) {
  if (mx <= 0 || my <= 0 || mz <= 0 || mz % 4 || R < 1) return false;
  // the step's sizes (dns_make_geom): Nx = mx/3*2, Nz = my/3*2, Py = mz/2 + 1
  const int Nx = mx / 3 * 2;
  P.Nz = my / 3 * 2;
  P.Kx = Nx / 2 + 1;
  P.Kh = P.Nz / 2 + 1;
  P.Py = mz / 2 + 1;
  if (Nx < 2 || P.Nz < 2 || P.Nz % 2 || R > P.Kh || R > P.Py) return false;
  // slot ranges: boundaries nearest to equal pencil counts, one slot at least each
  std::vector<int> cum(P.Kh + 1, 0);
  for (int k = 0; k < P.Kh; ++k) cum[k + 1] = cum[k] + pencils_of_slot(k, P.Nz);
  P.s0.assign(R, 0);
  P.s1.assign(R, P.Kh);
  for (int r = 1; r < R; ++r) {
    const double target = (double)P.Nz * r / R;
    const int lo = P.s0[r - 1] + 1, hi = P.Kh - (R - r);
    int best = lo;
    for (int k = lo; k <= hi; ++k)
      if (std::fabs(cum[k] - target) < std::fabs(cum[best] - target)) best = k;
    P.s1[r - 1] = P.s0[r] = best;
  }
  P.y0.assign(R, 0);
  P.y1.assign(R, 0);
  for (int r = 0; r < R; ++r) {
    P.y0[r] = (int)((long long)P.Py * r / R);
    P.y1[r] = (int)((long long)P.Py * (r + 1) / R);
  }
  return true;
}

// the spanwise runs of rank r: (kz0, nkz, first local pencil row)
std::vector<std::array<int, 3>> runs_of(const Part& P, int r) {
  std::vector<std::array<int, 3>> out;
  const int a = P.s0[r], b = P.s1[r];
  int row = 0;
  if (b > a) {
    out.push_back({a, b - a, row});
    row += (b - a) * P.Kx;
  }
  // mirrored pencils Nz - kz' for kz' in [a, b), kz' not 0 or Nz/2
  const int lo = std::max(a, 1), hi = std::min(b, P.Nz / 2);  // kz' in [lo, hi)
  if (hi > lo) out.push_back({P.Nz - hi + 1, hi - lo, row});
  return out;
}

}  // namespace

// the runs of rank r (kz0, nkz, first local row) for the slab step
int slab_runs(int mx, int my, int mz, int nranks, int rank, int kz0[2], int nkz[2], long long row0[2]) {
  Part P;
  if (rank < 0 || rank >= nranks || !make_part(mx, my, mz, nranks, P)) return -1;
  const auto runs = runs_of(P, rank);
  for (size_t i = 0; i < runs.size() && i < 2; ++i) {
    kz0[i] = runs[i][0];
    nkz[i] = runs[i][1];
    row0[i] = (long long)runs[i][2];
  }
  return (int)runs.size();
}

extern "C" {

dns_status dns_slab_ranges(int mx, int my, int mz, int nranks, int rank, int out[5]) {
  Part P;
  if (!out || rank < 0 || rank >= nranks || !make_part(mx, my, mz, nranks, P))
    return dns_internal_fail(DNS_ERR_ARG, "slab plan: bad grid, rank count or rank");
  int np = 0;
  for (const auto& run : runs_of(P, rank)) np += run[1] * P.Kx;
  out[0] = P.s0[rank];
  out[1] = P.s1[rank];
  out[2] = P.y0[rank];
  out[3] = P.y1[rank];
  out[4] = np;
  return DNS_OK;
}

dns_status dns_slab_segments(int mx, int my, int mz, int nranks, int rank, int role,
                             dns_slab_segment* seg, int cap, int* count) {
  Part P;
  if (!count || rank < 0 || rank >= nranks || !make_part(mx, my, mz, nranks, P) ||
      (role != DNS_SLAB_PENCILS && role != DNS_SLAB_PLANES))
    return dns_internal_fail(DNS_ERR_ARG, "slab plan: bad grid, rank count, rank or role");
  std::vector<dns_slab_segment> v;
  for (int peer = 0; peer < nranks; ++peer) {
    const int po = role == DNS_SLAB_PENCILS ? rank : peer;  // pencil owner
    const int yo = role == DNS_SLAB_PENCILS ? peer : rank;  // plane owner
    if (P.y1[yo] <= P.y0[yo]) continue;
    for (const auto& run : runs_of(P, po)) {
      dns_slab_segment s;
      s.peer = peer;
      s.kz0 = run[0];
      s.nkz = run[1];
      s.local_row0 = run[2];
      s.y0 = P.y0[yo];
      s.ny = P.y1[yo] - P.y0[yo];
      v.push_back(s);
    }
  }
  *count = (int)v.size();
  if (seg) {
    if (cap < (int)v.size()) return dns_internal_fail(DNS_ERR_ARG, "slab plan: segment array too small");
    std::copy(v.begin(), v.end(), seg);
  }
  return DNS_OK;
}

}  // extern "C"
