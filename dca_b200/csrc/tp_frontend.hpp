// Launch interface of the two-particle front-end kernels (tp_frontend.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch_tuner.hpp"
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
  LaunchTuner* tuner;         // launch-shape tuner (null: the built-in shapes)
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

// ---- Tensor-core front-end of the mixed path (tp_frontend_tc.cu) ----
// Workspace: split-BF16 operand planes for a batch of n_sectors sectors of order <= max_order.
struct FrontTcShape {
  int D;    // R * NwExt, rows and columns of G
  int Dp;   // D rounded up to 128 (GEMM row tiles)
  int Dq;   // D rounded up to 128 (GEMM complex column tiles)
  int Kr;   // max_order rounded up to 64 (vertex extent of each real / imaginary half of a plane row)
  int n_sectors;
  size_t pr_elems, mb_elems, ac_elems, bq_elems;  // FP16 elements of P, M, X' and Q planes
};
// The cluster transform of an L x L square cluster (L = 4 or 6) as a 2D FFT: grid point g = a + L b
// is site rmap[g] (coordinates (a, b)) and momentum kmap[g] (2 pi (a, b) / L); r0 is the site at
// the origin.  Set up on the host when the cluster's phase table has exactly that structure.
struct ColFft {
  int on;
  int r0;
  int L;
  unsigned char rmap[36], kmap[36];
};

struct FrontTcWorkspace {
  FrontTcShape shape;
  void* pr = nullptr;
  void* mb = nullptr;
  void* ac = nullptr;
  void* bq = nullptr;
  int* eP = nullptr;       // [spin][Dp] power-of-two exponents of P's rows
  int* eQ = nullptr;       // [spin][Dp] ... of Q's rows
  float* mInv = nullptr;   // [sector][Kr] inverse scales of M's rows j
  float* xInv = nullptr;   // [sector][Dp][Kr / 32] inverse scales of X' row chunks
  int n_sm = 0;            // SMs of the device (persistent GEMM grids)
  bool factored_col = false;  // the column step runs factored by orbital (tp_colfactor.cu), not as a GEMM
  ColFft fft{};               // ... with its cluster transform as an L x L FFT (when fft.on)
  void* tp = nullptr;         // ... FFT form: FP16 planes of the column twiddles (colTwiddlePlaneBytes)
  bool col_tc = false;        // ... FFT form with the per-site sums in tensor memory (tp_colfactor_tc.cu)
  CUtensorMap tm_pr, tm_mb, tm_ac, tm_bq;  // TMA descriptors of the four plane arrays
};
FrontTcShape frontTcShape(const TpDims& d, int n_sectors, int max_order);
size_t frontTcBytes(const FrontTcShape& s);
// Carves `mem` (frontTcBytes, zero-filled by the caller), encodes the tensor maps and computes the
// P / Q row scales from the device G0 slice (one launch on `stream`).
void frontTcInit(FrontTcWorkspace& w, const FrontTcShape& s, void* mem, const TpDims& d, const double2* G0,
                 cudaStream_t stream);
// Twiddles in (w, vertex) order into a.Tr / a.Tc and the P, M and Q planes; returns the number of
// kernels launched.  orb_r / orb_c: orbital (band + nb site) of each vertex in row / column order.
int launchFrontendTcPrep(const FrontendArgs& a, const FrontTcWorkspace& w, const int* orb_r, const int* orb_c,
                         cudaStream_t stream);
// X' = P M (one launch).
void launchFrontendTcRow(const FrontendArgs& a, const FrontTcWorkspace& w, int* err, cudaStream_t stream);
// G = X' Q^H + beta G0 delta into the block-layout G; returns the number of kernels launched.
// gmax (or null): [2 slot + spin] set to each sector's largest |G| (float bits).
int launchFrontendTcCol(const FrontendArgs& a, const FrontTcWorkspace& w, float2* G, long g_sector_stride,
                         int* gmax, int* err, cudaStream_t stream);
// The same G through the orbital-factored column step (tp_colfactor.cu): one band, Nc = 16.
// With the FFT cluster transform it runs on the tensor cores and needs colTwiddlePlaneBytes of
// workspace (FrontTcWorkspace::tp); otherwise on the CUDA cores.
bool colFactorApplies(const TpDims& d);
// One band on a 36-site cluster: the factored column step with the 6 x 6 FFT (when ColFft has L = 6).
bool colFactorWideApplies(const TpDims& d);
size_t colTwiddlePlaneBytes(const TpDims& d, int n_sectors, int Kr);
// The tensor-memory form (tp_colfactor_tc.cu): one band, 4 x 4 cluster, rows in whole 128-row tiles.
bool colFactorTcApplies(const TpDims& d, int D, int row0, int max_order);
int launchColFactorTc(const FrontendArgs& a, const FrontTcWorkspace& w, float2* G, long g_sector_stride, int* gmax,
                      int* err, cudaStream_t stream);
int launchColFactor(const FrontendArgs& a, const FrontTcWorkspace& w, float2* G, long g_sector_stride, int* gmax,
                     cudaStream_t stream);

}  // namespace dcaacc
