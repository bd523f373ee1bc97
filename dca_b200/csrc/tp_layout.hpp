// Device-side description of one two-particle accumulation problem and of the per-sector work
// items that the kernels read.  Shared by the front-end (NDFT + cluster transform + G) and the
// G4 update kernels.
#pragma once

#include <cstdint>

namespace dcaacc {

constexpr int kMaxChannels = 4;

// Static sizes.  Index conventions (all "first index fastest"):
//   G0   (b1, b2, k, w_ext, s)                      nb^2 Nc NwExt 2
//   X'   per sector: (row, jj, w1_ext) with row = b1 + nb k1 and jj the column of M in
//        column-sorted order
//   G    per sector, frequency-block layout: (c, r, w_c, w_r) with r = b_r + nb k_r and
//        c = b_c + nb k_c, i.e. one R x R block (row-major inside the block) per pair of
//        extended frequencies (w_r, w_c).  G(r, w_r; c, w_c) is the reference's
//        G_(b_r, b_c, s, k_r, k_c, w_r, w_c) (tp_accumulator_base.hpp:79-80).
//   G4   (b1, b2, b3, b4, k1, w1, k2, w2, q, wq)      dca_data.hpp:108-112
struct TpDims {
  int nb, nc, nw, nw_ext, ext;
  int n_orb;  // nb * nc
  int R;      // rows per extended frequency = nb * nc
  int nq, nwq;
  int n_channels;
  int channels[kMaxChannels];
  double beta;
};

// One spin sector of one measurement, as the kernels see it after host-side sorting.
struct SectorDesc {
  const double* M;  // device pointer, column major
  long x_off;       // offset (complex elements) of this sector's X' in the workspace
  int ldm;
  int n;            // expansion order
  int vtx_off;      // offset of this sector in the packed per-vertex arrays
  int orb_off;      // offset of this sector in the packed orbital-start arrays ((n_orb + 1) each)
  int spin;         // 0 or 1
  int slot;         // measurement slot inside the batch
};

}  // namespace dcaacc
