// Vertex sort of one side of each sector on the device: CachedNdftBase::sortConfiguration
// (cached_ndft_base.hpp:89-129) orders the vertices by (orbital, index) with orbital = band +
// nb * site of that side (the right band / site for the rows, the left ones for the columns of
// non-density-density models, :97-103), and records where each orbital's run starts.  Here one
// CTA per sector runs a stable counting sort: a shared-memory histogram of the orbitals, a warp
// scan into the run starts, and one warp that places the vertices 32 at a time in index order
// (lanes with equal orbitals take consecutive places in lane order), so equal orbitals keep their
// original order as the reference's (orbital, idx) comparison does.
#include <cuda_runtime.h>

#include "common.cuh"
#include "tp_layout.hpp"
#include "tp_sort.hpp"

namespace dcaacc {

namespace {

__global__ void __launch_bounds__(256)
sortVerticesKernel(const SectorDesc* __restrict__ sectors, const int* __restrict__ band,
                   const int* __restrict__ site, int nb, int n_orb, int* __restrict__ perm,
                   int* __restrict__ start, int* __restrict__ orb) {
  extern __shared__ int sh[];
  int* count = sh;           // [n_orb]
  int* fill = sh + n_orb;    // [n_orb] next free place per orbital
  const SectorDesc sd = sectors[blockIdx.x];
  const int n = sd.n, off = sd.vtx_off;
  const int t = threadIdx.x, lane = t & 31;
  for (int o = t; o < n_orb; o += blockDim.x)
    count[o] = 0;
  __syncthreads();
  for (int v = t; v < n; v += blockDim.x)
    atomicAdd(&count[band[off + v] + nb * site[off + v]], 1);
  __syncthreads();
  if (t < 32) {
    // Exclusive scan: lane l owns orbitals [l c, (l + 1) c).
    const int c = (n_orb + 31) / 32, o0 = min(lane * c, n_orb), o1 = min(o0 + c, n_orb);
    int local = 0;
    for (int o = o0; o < o1; ++o)
      local += count[o];
    int incl = local;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d)
        incl += y;
    }
    int run = incl - local;
    for (int o = o0; o < o1; ++o) {
      start[sd.orb_off + o] = run;
      fill[o] = run;
      run += count[o];
    }
    if (lane == 31)
      start[sd.orb_off + n_orb] = incl;
    __syncwarp();
    // Stable placement, 32 vertices at a time in index order.
    const unsigned lt = (1u << lane) - 1;
    for (int v0 = 0; v0 < n; v0 += 32) {
      const int v = v0 + lane;
      const int o = v < n ? band[off + v] + nb * site[off + v] : -1;
      const unsigned same = __match_any_sync(0xffffffffu, o);
      int pos = 0;
      if (o >= 0) {
        pos = fill[o] + __popc(same & lt);
        perm[off + pos] = v;
        if (orb)
          orb[off + pos] = o;
      }
      __syncwarp();
      if (o >= 0 && (same & lt) == 0)  // the group's first lane advances its orbital
        fill[o] += __popc(same);
      __syncwarp();
    }
  }
}

}  // namespace

void launchSortVertices(const SectorDesc* sectors, int n_sectors, const int* band, const int* site, int nb,
                        int n_orb, int* perm, int* start, int* orb, cudaStream_t stream) {
  const size_t smem = 2 * sizeof(int) * size_t(n_orb);
  sortVerticesKernel<<<n_sectors, 256, smem, stream>>>(sectors, band, site, nb, n_orb, perm, start, orb);
  DCAACC_LAUNCH_CHECK();
}

}  // namespace dcaacc
