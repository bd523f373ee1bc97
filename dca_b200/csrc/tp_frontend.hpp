// Launch interface of the two-particle front-end kernels (tp_frontend.cu).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "tp_layout.hpp"

namespace dcaacc {

struct FrontendArgs {
  TpDims dims;
  const SectorDesc* sectors;  // [n_sectors], device
  int n_sectors;
  int n_max;                  // largest expansion order among the sectors
  const double* tau;          // packed per-vertex tau, original order (device)
  const int* perm_r;          // packed row-sorted -> original vertex index (device)
  const int* perm_c;          // packed column-sorted -> original vertex index (device)
  const int* row_start;       // packed orbital starts, row order ((n_orb + 1) per sector)
  const int* col_start;       // packed orbital starts, column order
  double2* Tr;                // packed twiddles, row-sorted order (n x NwExt per sector)
  double2* Tc;                // packed twiddles, column-sorted order (== Tr when rows == cols)
  const double2* Fb;          // (r, k, b): e^{i k (r + a_b)}, nb * Nc * Nc
  const double2* G0;          // (b1, b2, k, w, s) over the extended mesh
};

void launchTwiddles(const FrontendArgs& a, cudaStream_t stream);

// Row transform: M -> X' for every sector.
template <typename Real>
void launchRowTransform(const FrontendArgs& a, cplx_t<Real>* Xp, cudaStream_t stream);

// Column transform + G epilogue: X' -> G, one D x D block-layout matrix per (slot, spin) at
// offset g_sector_stride * (2 * slot + spin).
template <typename Real>
void launchColTransform(const FrontendArgs& a, const cplx_t<Real>* Xp, cplx_t<Real>* G,
                        long g_sector_stride, cudaStream_t stream);

size_t frontendSmemRequirement(const TpDims& d, int n_max, bool fp64);

}  // namespace dcaacc
