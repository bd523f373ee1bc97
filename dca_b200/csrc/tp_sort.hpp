// Device-side vertex sort of the two-particle accumulator (tp_sort.cu).
#pragma once

#include <cuda_runtime.h>

#include "tp_layout.hpp"

namespace dcaacc {

// For each of n_sectors sectors (descriptors on the device): sorts its vertices by orbital =
// band[v] + nb * site[v] (packed per-vertex arrays at the sector's vtx_off), stably.
//   perm[vtx_off + i]  original index of the vertex at sorted position i
//   start[orb_off + o] first sorted position of orbital o (n_orb + 1 entries, the last is n)
//   orb[vtx_off + i]   orbital of sorted position i (orb may be null)
// n_orb <= 1024 (two n_orb-int tables in shared memory).
void launchSortVertices(const SectorDesc* sectors, int n_sectors, const int* band, const int* site, int nb,
                        int n_orb, int* perm, int* start, int* orb, cudaStream_t stream);

}  // namespace dcaacc
