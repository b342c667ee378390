// Device side of the banded wall-normal solve (wallsolve.cu): dimensions and
// launcher.
#pragma once
#include "kernels.cuh"

struct WallDims {
  int nv, no;              // rows of the packed v and omega systems (N + deg U + 1)
  int delta;               // base-flow degree: selects the band instance
  int qbytes;              // bytes of the tilting table in shared memory (16-aligned)
  long long gp;            // pitch (complex) of the integrated right-hand sides
  long long nslots;        // operator slots Kx * (Nz/2 + 1)
  long long ngroups;       // groups of 16 slots = CTAs
  long long group_complex; // packed factor values per group
  int tilt = 1;            // 0: no tilting term (the solve-only entry)
  // a slab's slots: operator slots kz' = kzs0 + s / Kx (local slot s); the
  // pencil of (kx, kz) with kz = kz' sits at row rowa + (kz - kza) Kx + kx of
  // the data arrays, with kz = Nz - kz' at rowb + (kz - kzb) Kx + kx (the
  // whole grid: all zero, row kz Kx + kx)
  int kzs0 = 0, kza = 0, kzb = 0;
  long long rowa = 0, rowb = 0;
  // a batch of runs: groups per member (its factors, then the next
  // member's); 0 for one run
  long long groups_per_run = 0;
};

// band instance (v lower/upper, omega lower/upper) for base-flow degree delta
bool wall_band_of(int delta, int* klv, int* kuv, int* klo, int* kuo);
#define DNS_WALL_VARIANTS 4
// block shapes of the solve (ring stages x stage bytes, tilting table
// placement): variant 0 .. DNS_WALL_VARIANTS - 1
size_t wall_smem_bytes(const WallDims& wd, int variant);
// complex values of the solve's global scratch (Sw of the launcher)
size_t wall_scratch_complex(const WallDims& wd);
cudaError_t launch_wall_solve(const double2* fac, double2* V, double2* O, const double2* gv,
                              const double2* go, const double* Q, double2* Sw, const WallDims& wd,
                              const DnsGeom& g, const PhysParams& ph, int* status, cudaStream_t st,
                              int variant = 0);

// Solve-only entry (wallentry.cu): collocation right-hand sides in the
// reference's pencil layout -> integrated right-hand sides of the banded
// systems plus the wall polynomial (6 complex per pencil); and the solution
// plus that polynomial back into pencils of pitch op (complex).
// prep: wall polynomial (pbc) and the point values (pitch sp) of the interior
// right-hand side minus A p; integrate: the K-fold integrals of the
// interpolant coefficients (pitch cp) into the banded systems' right-hand sides
cudaError_t launch_colloc_prep(const double2* bv, const double2* bo, long long bp, double2* sv,
                               double2* so, long long sp, double2* pbc, const double* cosk,
                               const double* Ut, const double* ddUt, const DnsGeom& g,
                               const PhysParams& ph, cudaStream_t st);
cudaError_t launch_colloc_integrate(const double2* cv, const double2* co, long long cp, double2* gv,
                                    double2* go, const WallDims& wd, const DnsGeom& g, cudaStream_t st);
// prep, DCT-I and integration in one kernel (warp FFTs over L = 2 (Ny - 1)
// with the no-padding plan tab); cudaErrorNotSupported, nothing launched,
// for lengths without a warp plan
cudaError_t launch_colloc_fused(const double2* bv, const double2* bo, long long bp, double2* pbc,
                                const double* cosk, const double* Ut, const double* ddUt, double2* gv,
                                double2* go, const WallDims& wd, const DnsGeom& g, const PhysParams& ph,
                                FftTab<double2> tab, int* status, cudaStream_t st);
cudaError_t launch_colloc_finish(const double2* Xv, const double2* Xo, const double2* pbc,
                                 double2* ov, double2* oo, long long op, const DnsGeom& g,
                                 cudaStream_t st);
// *flag |= 1 if any of the n complex values of a or b is not finite
cudaError_t launch_nonfinite(const double2* a, const double2* b, long long n, int* flag,
                             cudaStream_t st);
