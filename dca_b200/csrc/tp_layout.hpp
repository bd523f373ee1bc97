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
  // Mixed path, one band, Nc <= kMaxMirrorNc: G rows of the lower frequency half (w1 < nw_ext / 2)
  // are not computed; G(k1 w1; k2 w2) = conj G(-k1 w1'; -k2 w2') with w' = nw_ext - 1 - w (real M
  // and G0(-k, -w) = conj G0(k, w)), and the consumers read that mirror instead.
  int half_g;
  unsigned char kneg[64];  // index of -k (half_g only; Nc <= kMaxKneg)
  // With half_g, and momentum and frequency transfers closed under negation, G4 itself obeys
  // G4(-k1 w1', -k2 w2', -q, -wq) = conj G4(k1 w1, k2 w2, q, wq) (w' = Nw - 1 - w): the update
  // accumulates the frequency tiles with w1 >= Nw / 2 only and the rest is filled from them when
  // G4 is read (finalize, peek).
  int half_g4;
};
constexpr int kMaxMirrorNc = 16;  // cluster of the tensor-core direct G4 term
constexpr int kMaxKneg = 64;      // clusters whose -k table TpDims carries

// Index of element (k1 w1; k2 w2) of a one-band block-layout G (R = Nc) and whether it is stored
// conjugated there (half_g: the lower-half rows are read from their mirror).
__host__ __device__ inline long gIndexMirrored(const TpDims& d, int w1, int w2, int k1, int k2, bool& conj) {
  conj = d.half_g && 2 * w1 < d.nw_ext;
  if (conj) {
    w1 = d.nw_ext - 1 - w1;
    w2 = d.nw_ext - 1 - w2;
    k1 = d.kneg[k1];
    k2 = d.kneg[k2];
  }
  return ((static_cast<long>(w1) * d.nw_ext + w2) * d.R + k1) * d.R + k2;
}

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
  int m_f32;        // 1: M holds float elements (the reference's SpScalar = float), else double
};

// Element (i, j) of a sector's M, read in its stored precision.
__host__ __device__ inline double loadM(const SectorDesc& sd, long idx) {
  return sd.m_f32 ? static_cast<double>(reinterpret_cast<const float*>(sd.M)[idx]) : sd.M[idx];
}

}  // namespace dcaacc
