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
};

// band instance (v lower/upper, omega lower/upper) for base-flow degree delta
bool wall_band_of(int delta, int* klv, int* kuv, int* klo, int* kuo);
size_t wall_smem_bytes(const WallDims& wd);
// complex values of the solve's global scratch (Sw of the launcher)
size_t wall_scratch_complex(const WallDims& wd);
cudaError_t launch_wall_solve(const double2* fac, double2* V, double2* O, const double2* gv,
                              const double2* go, const double* Q, double2* Sw, const WallDims& wd,
                              const DnsGeom& g, const PhysParams& ph, int* status, cudaStream_t st);
