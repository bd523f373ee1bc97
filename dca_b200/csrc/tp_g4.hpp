// Launch interface of the G4 update kernel (tp_g4.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "common.cuh"
#include "launch_tuner.hpp"
#include "tp_layout.hpp"

namespace dcaacc {

struct G4Args {
  TpDims dims;
  const int* signs;     // [n_slots] measurement signs (device)
  int n_slots;          // measurements summed by this launch
  const int* k_add;     // [Nc * Nc] (device)
  const int* k_sub;     // [Nc * Nc] (device)
  const int* q_list;    // [nq] momentum-transfer indices (device)
  const int* wex_list;  // [nwq] frequency transfers (device)
  double2* const* G4;   // [n_channels] device pointers to each channel's running sum (device array)
  bool atomic;          // several accumulators share G4
  int* err;             // device error word (async_copy.cuh kErr* bits)
  bool q_all = false;             // q_list is a permutation of all Nc cluster momenta
  const struct DiscWorkspace* disc = nullptr;  // tensor-core disconnected-term workspace (or null)
  const int* gmax = nullptr;  // [2 slot + spin] largest |G| of each sector as float bits (or null)
  int n_sm = 0;               // multiprocessors (persistent grids)
  const unsigned* tile_order = nullptr;  // half_g4: the (w1 | w2 << 16) tiles to update, mirror pairs adjacent
  LaunchTuner* tuner = nullptr;          // launch-shape tuner (null: the built-in shapes)
  // Error-path tests: polls of a bounded device wait before it gives up (0: the built-in limit),
  // and the pipeline step before which the tensor-core direct term's first CTA stops feeding its
  // consumers (-1: never).
  uint32_t wait_limit = 0;
  int fault_stop_step = -1;
};

// Workspace of the tensor-core disconnected-term GEMM (tp_g4_disc.cu): U / V operand planes, their
// row scales, the FP32 result and the TMA descriptors, for batches of up to max_batch measurements.
struct DiscWorkspace {
  void* U = nullptr;
  void* V = nullptr;
  int* eU = nullptr;
  int* eV = nullptr;
  float2* out = nullptr;
  int max_batch = 0;
  int n_sm = 0;
  CUtensorMap tm_u, tm_v;
};

// dst += src; src = 0 (sumTo of two accumulators on the same device).
void launchAddAndClear(double2* dst, double2* src, size_t n, cudaStream_t stream);

// Batched FP32 single-band PH update (tp_g4_batched.cu): one band, Nc in {4, 8, 16}, channels
// PH-magnetic / PH-charge only.
bool singlebandBatchedApplies(const TpDims& d);
// Returns the number of kernels launched, 0 when the configuration is not covered (then
// launchUpdateG4 uses the general kernels).  With a.disc_scratch large enough, the disconnected
// terms run on the tensor cores (launchDiscGemm) and the update kernel only adds the direct term.
int launchUpdateG4SinglebandBatched(const G4Args& a, const float2* G, long g_sector_stride,
                                    cudaStream_t stream);

// Multiband particle-particle up-down update, mixed path (tp_g4_pp.cu): three bands, that channel
// alone, full G and G4.  Returns false (nothing launched) when the configuration is not covered.
bool launchUpdateG4PPMultiband(const G4Args& a, const float2* G, long g_sector_stride, cudaStream_t stream);

// Tensor-core disconnected terms (tp_g4_disc.cu): one band, PH channels, batches of at most 256.
// discInit carves `mem` (discScratchBytes) and builds the descriptors; launchDiscGemm returns the
// device result (per problem an M x M FP32 matrix), or null without a workspace.
bool discGemmApplies(const TpDims& d, int max_batch);
size_t discScratchBytes(const TpDims& d, int max_batch);
void discInit(DiscWorkspace& w, const TpDims& d, int max_batch, void* mem, size_t bytes);
const float2* launchDiscGemm(const G4Args& a, const float2* G, long g_sector_stride, cudaStream_t stream);

// Tensor-core direct term (tp_g4_mma.cu): one band, Nc = 16, all momentum transfers, with the
// disconnected terms precomputed (disc) and the per-sector maxima of G recorded by the column step.
bool directTcApplies(const G4Args& a);
void launchDirectTc(const G4Args& a, const float2* G, long g_sector_stride, const float2* disc, int n_sm,
                    cudaStream_t stream);

// half_g4: G4 entries with w1 < Nw / 2 := conj of their mirror (-k1 w1', -k2 w2', -q, -wq);
// q_mirror[iq] / wq_mirror[iwq] are the positions of -q / -wq in the transfer lists.
void launchG4Mirror(double2* G4, const TpDims& d, const int* q_mirror, const int* wq_mirror, cudaStream_t stream);
// Entries [offset, offset + count) of G4 with the mirror applied (half_g4) into out (device).
void launchG4Window(const double2* G4, const TpDims& d, const int* q_mirror, const int* wq_mirror, size_t offset,
                    size_t count, double2* out, cudaStream_t stream);

// G: block-layout G of n_slots measurements, sector (slot, spin) at g_sector_stride * (2 slot + spin).
// Returns the number of kernels launched.
template <typename GT>
int launchUpdateG4(const G4Args& a, const GT* G, long g_sector_stride, cudaStream_t stream);

}  // namespace dcaacc
