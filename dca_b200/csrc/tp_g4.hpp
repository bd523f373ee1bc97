// Launch interface of the G4 update kernel (tp_g4.cu).
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "common.cuh"
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
};

// dst += src; src = 0 (sumTo of two accumulators on the same device).
void launchAddAndClear(double2* dst, double2* src, size_t n, cudaStream_t stream);

// Batched FP32 single-band PH update (tp_g4_batched.cu); false when the configuration is not
// covered (then launchUpdateG4 uses the general kernels).
bool launchUpdateG4SinglebandBatched(const G4Args& a, const float2* G, long g_sector_stride,
                                     cudaStream_t stream);

// G: block-layout G of n_slots measurements, sector (slot, spin) at g_sector_stride * (2 slot + spin).
template <typename GT>
void launchUpdateG4(const G4Args& a, const GT* G, long g_sector_stride, cudaStream_t stream);

}  // namespace dcaacc
