// Tensor-core front-end of the mixed-precision path: M(tau, tau') -> G(k1, w1; k2, w2) for every
// sector of a batch, as two dense complex contractions on tcgen05.
//
// The reference computes the NDFT per orbital pair (CachedNdft<GPU>::execute,
// cached_ndft_gpu.hpp:131-252), the cluster transform (SpaceTransform2DGpu::execute,
// space_transform_2D_gpu.hpp:116-171) and G = -G0 G~ G0 + beta G0 delta (computeGSingleband /
// computeGMultiband, tp_accumulator_kernels.cu:73-217) as separate passes.  Here the phases and
// G0 are folded into two operand matrices.  With rho = r + R w (r = b + nb k, R = nb Nc), the row
// vertices i in row-sorted order and the column vertices j in column-sorted order:
//   P(rho1, i) = G0_s(b1, b_i; k1, w1) e^{i k1 (x_i + a_{b_i})} e^{i w1 tau_i}
//   Q(rho2, j) = -(1/Nc) e^{i k2 (x_j + a_{b_j})} e^{i w2 tau_j} conj(G0_s(b_j, b2; k2, w2))
//   X' = P M          (row step)
//   G  = X' Q^H + beta G0_s(b1, b2; k1, w1) delta_{k1 k2} delta_{w1 w2}     (column step)
// where x_i, b_i are vertex i's site and band.  This is the reference's G exactly (the band sums
// of -G0 G~ G0 become the G0 factors inside P and Q).
//
// Precision.  Every operand is split into two FP16 planes, x ~ hi + lo (22 significant bits), and
// the three plane products lo*hi, hi*lo, hi*hi are accumulated in FP32 tensor memory (the dropped
// lo*lo is below 2^-22).  FP16's exponent range is handled with exact power-of-two scales chosen so
// that the largest magnitude of each scaled row (or row chunk) lies in [2^13, 2^15): then nothing
// overflows, and every entry down to 2^-17 of that maximum keeps a normal lo part.  P and Q rows
// are scaled by a bound from |G0| (which fixes the magnitude of every entry); M columns by their
// maximum; X' per (row, 32-wide K chunk, real and imaginary parts together) by the maximum the row
// step's epilogue sees, and the column step undoes that scale chunk by chunk.  Against the FP64 G,
// the split's own error is about 3e-8 relative (Frobenius) on the 4x4-cluster workload, the same
// order as rounding G to FP32; the FP32 accumulation that follows dominates.  The tensor core's
// FP32 accumulation does not round to nearest and its error grows with the number of MMAs that
// feed one accumulator, and the diagonal blocks of G are coherent sums over the vertices; so every
// 32-wide K chunk goes to a fresh accumulator pair (small products first), which the epilogue
// warps read and add into FP32 registers in round-to-nearest while the next chunk runs.
//
// Both steps are complex-pair GEMMs.  A stage holds one 32-wide K chunk of the real and the
// imaginary part of A (and of B in the column step), 2 FP16 planes each, as 64-byte-swizzled
// 128-row tiles; per 16-wide K step and plane product the MMAs are
//   row step:    Re += Ar Mt,   Im += Ai Mt                         (M real)
//   column step: Re += Ar Br^T + Ai Bi^T,  Im += Ai Br^T - Ar Bi^T  (negate-A for the last)
// into 128 x 128 FP32 accumulators Re and Im (columns 0-127 and 128-255 of a 256-column buffer;
// two buffers, chunk parity, = all 512 tensor-memory columns).  So the column step's B operand is
// Q itself, not the doubled real form [Qr | Qi; -Qi | Qr], and each staged byte feeds twice the
// MMAs of a real-form 128 x 64-complex tile.
//
// GEMM kernel: persistent, one CTA per SM (shared memory), 576 threads (18 warps: five share one
// SM sub-partition's 16K registers, so at most 96 registers per thread), tiles of 128 rows x 128
// (complex) columns taken round-robin over (sector, row tile, column tile).
//   warp 0      TMA producer: 3-stage ring over the chunks of all of the CTA's tiles;
//   warp 1      allocates tensor memory; one thread issues a chunk's MMAs and commits them to the
//               stage's "empty" barrier and the accumulator buffer's "full" barrier;
//   warps 2-17  promote each finished accumulator buffer into registers (warp w: lanes
//               32 (w % 4) .. + 31, complex columns 32 ((w - 2) / 4) .. + 31), then run the tile's
//               epilogue while the next tile's chunks load and multiply (row step: rescale and
//               split X' into the column step's planes; column step: unscale and store G).
// Every wait is bounded (kWaitLimit polls, then the error word is set and the roles stop).
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/dcaacc.h"
#include "async_copy.cuh"
#include "common.cuh"
#include "tc_gemm.cuh"
#include "tcgen05.cuh"
#include "tp_frontend.hpp"

namespace dcaacc {

namespace {

using namespace tcg;

// Matsubara frequency of extended index w (vertex_frequency_domain.hpp, EXTENDED).
__device__ inline double extFreq(int w, int nw_ext, double beta) {
  const int half = nw_ext / 2;
  if (w >= half)
    return M_PI / beta * (1 + 2 * (w - half));
  return -M_PI / beta * (1 + 2 * (half - 1 - w));
}

// Row scales of P and Q per (spin, rho) from |G0|: P row rho1 holds G0_s(b1, b; k1, w1) times unit
// phases, Q row rho2 holds G0_s(b, b2; k2, w2) / Nc.  Stored as exponents; rows >= D get 0.
__global__ void operandScalesKernel(const TpDims dims, const double2* __restrict__ G0, int D, int Dp,
                                    int* __restrict__ eP, int* __restrict__ eQ) {
  const int nb = dims.nb, nc = dims.nc, R = dims.R, nw_ext = dims.nw_ext;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < 2 * Dp; idx += gridDim.x * blockDim.x) {
    const int s = idx / Dp, rho = idx % Dp;
    int ep = 0, eq = 0;
    if (rho < D) {
      const int r = rho % R, w = rho / R, b = r % nb, k = r / nb;
      const double2* g0s = G0 + static_cast<long>(s) * nw_ext * nc * nb * nb;
      double mp = 0, mq = 0;
      for (int c = 0; c < nb; ++c) {
        const double2 gp = g0s[b + nb * (c + nb * (k + nc * w))];
        const double2 gq = g0s[c + nb * (b + nb * (k + nc * w))];
        mp = fmax(mp, hypot(gp.x, gp.y));
        mq = fmax(mq, hypot(gq.x, gq.y));
      }
      // hypot and the phase products round; one binade of margin keeps the maxima below 2^15.
      ep = scaleExp(mp) - 1;
      eq = scaleExp(mq / nc) - 1;
    }
    eP[idx] = ep;
    eQ[idx] = eq;
  }
}

// T(w, i) = e^{i w tau_{perm[i]}}, per sector in (w, i) order: T[vtx_off * NwExt + w * n + i].
// grid (NwExt, n_sectors).
__global__ void twiddleWiKernel(const SectorDesc* __restrict__ sectors, const double* __restrict__ tau,
                                const int* __restrict__ perm, double2* __restrict__ T, int nw_ext, double beta) {
  const SectorDesc sd = sectors[blockIdx.y];
  const int w = blockIdx.x;
  const double om = extFreq(w, nw_ext, beta);
  double2* out = T + static_cast<long>(sd.vtx_off) * nw_ext + static_cast<long>(w) * sd.n;
  for (int i = threadIdx.x; i < sd.n; i += blockDim.x) {
    // x = tau * w as in CachedNdft<CPU>::computeT (cached_ndft_cpu.hpp:151-156).
    const double x = tau[sd.vtx_off + perm[sd.vtx_off + i]] * om;
    double s, c;
    sincos(x, &s, &c);
    out[i] = make_double2(c, s);
  }
}

// Phase operand (P for the rows, Q for the columns), planes [sector][plane][rows][2 Kr]: real part
// at column v, imaginary part at column Kr + v, for vertices v < roundup(n, 32) (zero for v >= n);
// rows rho = r + R w < D.  One thread per (w, 8 vertices): it loads the 8 twiddles and orbitals once
// and walks the R rows of frequency w, writing 16 bytes per plane and part per row (consecutive
// threads: consecutive vertex groups of one row).
//   ROW = true:  P(rho, i) 2^eP  = G0_s(b1, b_i; k1, w) Fb(b_i, k1, x_i) T(w, i) 2^eP
//   ROW = false: Q(rho, j) 2^eQ  = -(1/Nc) Fb(b_j, k2, x_j) T(w, j) conj(G0_s(b_j, b2; k2, w)) 2^eQ
template <bool ROW>
__global__ void __launch_bounds__(256)
buildPhaseOperandKernel(const TpDims dims, const SectorDesc* __restrict__ sectors, const double2* __restrict__ T,
                        const int* __restrict__ orb, const double2* __restrict__ Fb, const double2* __restrict__ G0,
                        const int* __restrict__ eRow, int D, int Dp, int rows, int Kr, __half* __restrict__ out) {
  const SectorDesc sd = sectors[blockIdx.y];
  const int n = sd.n;
  const int groups = (n + kBK - 1) / kBK * (kBK / 8);
  const int nb = dims.nb, nc = dims.nc, R = dims.R, nw_ext = dims.nw_ext;
  const long kp = 2L * Kr;
  const long plane = static_cast<long>(rows) * kp;
  __half* o = out + static_cast<long>(blockIdx.y) * kPl * plane;
  const double2* g0s = G0 + static_cast<long>(sd.spin) * nw_ext * nc * nb * nb;
  const double2* Ts = T + static_cast<long>(sd.vtx_off) * nw_ext;
  const int* es = eRow + sd.spin * Dp;
  const double qscale = -1.0 / nc;
  const int w_lo = ROW && dims.half_g ? nw_ext / 2 : 0;  // half G: P rows of the upper half only
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < long(groups) * (nw_ext - w_lo);
       idx += long(gridDim.x) * blockDim.x) {
    const int grp = static_cast<int>(idx % groups);
    const int w = w_lo + static_cast<int>(idx / groups);
    double2 tv[8];
    int bv[8], xv[8];
#pragma unroll
    for (int x = 0; x < 8; ++x) {
      const int v = grp * 8 + x;
      const bool in = v < n;
      tv[x] = in ? Ts[static_cast<long>(w) * n + v] : make_double2(0., 0.);
      const int ov = in ? orb[sd.vtx_off + v] : 0;
      bv[x] = ov % nb;
      xv[x] = ov / nb;
    }
    for (int r = 0; r < R; ++r) {
      const int b = r % nb, k = r / nb;
      const int rho = r + R * w;
      const double sc = pow2d(es[rho]);
      Pack8 re[kPl], im[kPl];
      float yr[8], yi[8];  // the FP64 products, scaled, rounded once to FP32 and then split
#pragma unroll
      for (int x = 0; x < 8; ++x) {
        const double2 ph = zmul(Fb[(bv[x] * nc + k) * nc + xv[x]], tv[x]);
        double2 z;
        if (ROW) {
          z = zmul(g0s[b + nb * (bv[x] + nb * (k + nc * w))], ph);
        }
        else {
          const double2 g = g0s[bv[x] + nb * (b + nb * (k + nc * w))];
          z = zmul(ph, make_double2(g.x * qscale, -g.y * qscale));
        }
        yr[x] = static_cast<float>(z.x * sc);
        yi[x] = static_cast<float>(z.y * sc);
      }
      split8(yr, re[0], re[1]);
      split8(yi, im[0], im[1]);
#pragma unroll
      for (int pl = 0; pl < kPl; ++pl) {
        __half* op = o + pl * plane + static_cast<long>(rho) * kp + grp * 8;
        store8(op, re[pl]);
        store8(op + Kr, im[pl]);
      }
    }
  }
}

// Density-density models (the same vertex order on both sides): P and Q from one pass, sharing
// the phase product Fb(b_i, k, x_i) T(w, i).  Thread per (w, 4 vertices) (4 rather than 8 keeps the
// FP64 state small enough for 4 blocks per SM); Q for every row, P for the rows the row step reads
// (half G: the upper frequency half).  NB1: one band, where G0 depends on (k, w) only and the
// row scales fold into it once per row.
template <bool NB1>
__global__ void __launch_bounds__(256)
buildPhasePairKernel(const TpDims dims, const SectorDesc* __restrict__ sectors, const double2* __restrict__ T,
                     const int* __restrict__ orb, const double2* __restrict__ Fb, const double2* __restrict__ G0,
                     const int* __restrict__ eP, const int* __restrict__ eQ, int Dp, int Dq, int Kr,
                     __half* __restrict__ outP, __half* __restrict__ outQ) {
  const SectorDesc sd = sectors[blockIdx.y];
  const int n = sd.n;
  const int groups = (n + kBK - 1) / kBK * (kBK / 4);
  const int nb = dims.nb, nc = dims.nc, R = dims.R, nw_ext = dims.nw_ext;
  const long kp = 2L * Kr;
  const long planeP = static_cast<long>(Dp) * kp, planeQ = static_cast<long>(Dq) * kp;
  __half* oP = outP + static_cast<long>(blockIdx.y) * kPl * planeP;
  __half* oQ = outQ + static_cast<long>(blockIdx.y) * kPl * planeQ;
  const double2* g0s = G0 + static_cast<long>(sd.spin) * nw_ext * nc * nb * nb;
  const double2* Ts = T + static_cast<long>(sd.vtx_off) * nw_ext;
  const int* esP = eP + sd.spin * Dp;
  const int* esQ = eQ + sd.spin * Dp;
  const double qscale = -1.0 / nc;
  const int w_lo = dims.half_g ? nw_ext / 2 : 0;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < long(groups) * nw_ext;
       idx += long(gridDim.x) * blockDim.x) {
    const int grp = static_cast<int>(idx % groups);
    const int w = static_cast<int>(idx / groups);
    const bool doP = w >= w_lo;
    double2 tv[4];
    int bv[4], xv[4];
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      const int v = grp * 4 + x;
      const bool in = v < n;
      tv[x] = in ? Ts[static_cast<long>(w) * n + v] : make_double2(0., 0.);
      const int ov = in ? orb[sd.vtx_off + v] : 0;
      bv[x] = ov % nb;
      xv[x] = ov / nb;
    }
    for (int r = 0; r < R; ++r) {
      const int b = r % nb, k = r / nb;
      const int rho = r + R * w;
      const double scQ = pow2d(esQ[rho]) * qscale, scP = pow2d(esP[rho]);
      float qr[4], qi[4], pr[4], pi[4];
      if (NB1) {
        const double2 g = g0s[k + nc * w];
        const double2 gq = make_double2(g.x * scQ, -g.y * scQ), gp = make_double2(g.x * scP, g.y * scP);
        const double2* fbk = Fb + k * nc;
#pragma unroll
        for (int x = 0; x < 4; ++x) {
          const double2 ph = zmul(fbk[xv[x]], tv[x]);
          const double2 zq = zmul(ph, gq), zp = zmul(gp, ph);
          qr[x] = static_cast<float>(zq.x);
          qi[x] = static_cast<float>(zq.y);
          pr[x] = static_cast<float>(zp.x);
          pi[x] = static_cast<float>(zp.y);
        }
      }
      else {
#pragma unroll
        for (int x = 0; x < 4; ++x) {
          const double2 ph = zmul(Fb[(bv[x] * nc + k) * nc + xv[x]], tv[x]);
          const double2 gq = g0s[bv[x] + nb * (b + nb * (k + nc * w))];  // G0(b_j, b2; k2, w2), conjugated
          const double2 zq = zmul(ph, make_double2(gq.x, -gq.y));
          qr[x] = static_cast<float>(zq.x * scQ);
          qi[x] = static_cast<float>(zq.y * scQ);
          const double2 zp = zmul(g0s[b + nb * (bv[x] + nb * (k + nc * w))], ph);  // G0(b1, b_i; k1, w1)
          pr[x] = static_cast<float>(zp.x * scP);
          pi[x] = static_cast<float>(zp.y * scP);
        }
      }
      uint2 h, l;
      __half* q = oQ + static_cast<long>(rho) * kp + grp * 4;
      split4(qr, h, l);
      *reinterpret_cast<uint2*>(q) = h;
      *reinterpret_cast<uint2*>(q + planeQ) = l;
      split4(qi, h, l);
      *reinterpret_cast<uint2*>(q + Kr) = h;
      *reinterpret_cast<uint2*>(q + planeQ + Kr) = l;
      if (doP) {
        __half* pp = oP + static_cast<long>(rho) * kp + grp * 4;
        split4(pr, h, l);
        *reinterpret_cast<uint2*>(pp) = h;
        *reinterpret_cast<uint2*>(pp + planeP) = l;
        split4(pi, h, l);
        *reinterpret_cast<uint2*>(pp + Kr) = h;
        *reinterpret_cast<uint2*>(pp + planeP + Kr) = l;
      }
    }
  }
}

// M operand, planes [sector][plane][Kr rows j][Kr columns i]: M(perm_r[i], perm_c[j]) * 2^{e_j}
// for i, j < n, zero up to i < roundup(n, 32) and j < min(roundup(n, 128), Kr).  One warp per
// row j: the column perm_c[j] of M is read contiguously into the warp's shared-memory row (its
// maximum on the way), then the permuted entries come from there; 2^{-e_j} goes to
// mInv[sector][j].  Dynamic shared memory: Kr doubles per warp.
__global__ void __launch_bounds__(256)
buildMOperandKernel(const SectorDesc* __restrict__ sectors, const int* __restrict__ perm_r,
                    const int* __restrict__ perm_c, int Kr, __half* __restrict__ out, float* __restrict__ mInv) {
  extern __shared__ double mrow_all[];
  const SectorDesc sd = sectors[blockIdx.y];
  const int n = sd.n;
  const int groups = (n + kBK - 1) / kBK * (kBK / 8);
  const int rows = min((n + kBN - 1) / kBN * kBN, Kr);
  const long plane = static_cast<long>(Kr) * Kr;
  __half* o = out + static_cast<long>(blockIdx.y) * kPl * plane;
  const int lane = threadIdx.x % 32;
  double* mrow = mrow_all + static_cast<long>(threadIdx.x / 32) * Kr;
  const int* pr = perm_r + sd.vtx_off;
  const int warps = gridDim.x * (blockDim.x / 32);
  for (int j = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; j < rows; j += warps) {
    const long col0 = j < n ? static_cast<long>(sd.ldm) * perm_c[sd.vtx_off + j] : -1;
    double mx = 0;
    __syncwarp();  // the previous row's reads of mrow are done
    for (int i0 = 0; i0 < n; i0 += 128) {  // four loads in flight per lane
      double m[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + 32 * u + lane;
        m[u] = (col0 >= 0 && i < n) ? loadM(sd, col0 + i) : 0.;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + 32 * u + lane;
        if (i < n)
          mrow[i] = m[u];
        mx = fmax(mx, fabs(m[u]));
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    __syncwarp();
    const int e = scaleExp(mx);
    const double sc = pow2d(e);
    for (int grp = lane; grp < groups; grp += 32) {
      Pack8 v[kPl];
      float y[8];
#pragma unroll
      for (int x = 0; x < 8; ++x) {
        const int i = grp * 8 + x;
        y[x] = static_cast<float>((i < n ? mrow[pr[i]] : 0.) * sc);
      }
      split8(y, v[0], v[1]);
#pragma unroll
      for (int pl = 0; pl < kPl; ++pl)
        store8(o + pl * plane + static_cast<long>(j) * Kr + grp * 8, v[pl]);
    }
    if (lane == 0)
      mInv[static_cast<long>(blockIdx.y) * Kr + j] = pow2f(-e);
  }
}

unsigned gridX(long work) {
  return static_cast<unsigned>(std::max(1L, std::min(4096L, (work + 255) / 256)));
}

size_t align256(size_t b) {
  return (b + 255) / 256 * 256;
}

GemmParams gemmParams(const FrontendArgs& a, const FrontTcWorkspace& w, int* err) {
  const FrontTcShape& s = w.shape;
  GemmParams p{};
  p.dims = a.dims;
  p.sectors = a.sectors;
  p.n_sectors = a.n_sectors;
  p.D = s.D;
  p.Dp = s.Dp;
  p.Kr = s.Kr;
  p.eP = w.eP;
  p.eQ = w.eQ;
  p.mInv = w.mInv;
  p.xInv = w.xInv;
  p.ac = static_cast<__half*>(w.ac);
  p.G0 = a.G0;
  p.err = err;
  return p;
}

}  // namespace

FrontTcShape frontTcShape(const TpDims& d, int n_sectors, int max_order) {
  FrontTcShape s;
  s.D = d.R * d.nw_ext;
  s.Dp = (s.D + kBM - 1) / kBM * kBM;
  s.Dq = (s.D + kBN - 1) / kBN * kBN;
  s.Kr = (std::max(max_order, 1) + 63) / 64 * 64;
  s.n_sectors = n_sectors;
  s.pr_elems = size_t(n_sectors) * kPl * s.Dp * 2 * s.Kr;
  s.mb_elems = size_t(n_sectors) * kPl * s.Kr * s.Kr;
  s.ac_elems = size_t(n_sectors) * kPl * s.Dp * 2 * s.Kr;
  s.bq_elems = size_t(n_sectors) * kPl * s.Dq * 2 * s.Kr;
  return s;
}

size_t frontTcBytes(const FrontTcShape& s) {
  const size_t planes = align256((s.pr_elems + s.mb_elems + s.ac_elems + s.bq_elems) * sizeof(__half));
  const size_t scales = align256(2 * sizeof(int) * 2 * s.Dp) + align256(sizeof(float) * s.n_sectors * s.Kr) +
                        align256(sizeof(float) * s.n_sectors * size_t(s.Dp / kBM) * (s.Kr / kBK));
  return planes + scales;
}

void frontTcInit(FrontTcWorkspace& w, const FrontTcShape& s, void* mem, const TpDims& d, const double2* G0,
                 cudaStream_t stream) {
  w.shape = s;
  unsigned char* b = static_cast<unsigned char*>(mem);
  __half* h = reinterpret_cast<__half*>(b);
  w.pr = h;
  w.mb = h + s.pr_elems;
  w.ac = h + s.pr_elems + s.mb_elems;
  w.bq = h + s.pr_elems + s.mb_elems + s.ac_elems;
  size_t off = align256((s.pr_elems + s.mb_elems + s.ac_elems + s.bq_elems) * sizeof(__half));
  w.eP = reinterpret_cast<int*>(b + off);
  w.eQ = w.eP + 2 * s.Dp;
  off += align256(2 * sizeof(int) * 2 * s.Dp);
  w.mInv = reinterpret_cast<float*>(b + off);
  off += align256(sizeof(float) * s.n_sectors * s.Kr);
  w.xInv = reinterpret_cast<float*>(b + off);
  const long depth = long(s.n_sectors) * kPl;
  makePlaneMap(&w.tm_pr, w.pr, 2L * s.Kr, s.Dp, depth);
  makePlaneMap(&w.tm_mb, w.mb, s.Kr, s.Kr, depth);
  makePlaneMap(&w.tm_ac, w.ac, 2L * s.Kr, s.Dp, depth);
  makePlaneMap(&w.tm_bq, w.bq, 2L * s.Kr, s.Dq, depth);
  int dev = 0;
  DCAACC_CUDA_CHECK(cudaGetDevice(&dev));
  DCAACC_CUDA_CHECK(cudaDeviceGetAttribute(&w.n_sm, cudaDevAttrMultiProcessorCount, dev));
  operandScalesKernel<<<gridX(2L * s.Dp), 256, 0, stream>>>(d, G0, s.D, s.Dp, w.eP, w.eQ);
  DCAACC_LAUNCH_CHECK();
}

int launchFrontendTcPrep(const FrontendArgs& a, const FrontTcWorkspace& w, const int* orb_r, const int* orb_c,
                         cudaStream_t stream) {
  const TpDims& d = a.dims;
  const FrontTcShape& s = w.shape;
  if (a.n_max == 0)
    return 0;
  int launches = 0;
  twiddleWiKernel<<<dim3(d.nw_ext, a.n_sectors), 128, 0, stream>>>(a.sectors, a.tau, a.perm_r, a.Tr, d.nw_ext,
                                                                   d.beta);
  DCAACC_LAUNCH_CHECK();
  ++launches;
  if (a.Tc != a.Tr) {
    twiddleWiKernel<<<dim3(d.nw_ext, a.n_sectors), 128, 0, stream>>>(a.sectors, a.tau, a.perm_c, a.Tc,
                                                                     d.nw_ext, d.beta);
    DCAACC_LAUNCH_CHECK();
    ++launches;
  }
  const long mrows = std::min<long>((a.n_max + kBN - 1) / kBN * kBN, s.Kr);
  // Up to 8 warps per block, as many as their Kr-double rows fit in 200 KB of shared memory; the
  // tuner may halve it (each row is one warp's work whatever the block).
  const int mwarps_max = static_cast<int>(std::max<long>(1, std::min<long>(8, 200L * 1024 / (8L * s.Kr))));
  const auto pm = tunePick(a.tuner, tuneKey("tc_m", d.nb, d.nc, d.nw_ext, a.n_max, a.n_sectors, 2),
                           mwarps_max >= 2 ? 2 : 1, stream);
  const int mwarps = mwarps_max >> pm.choice;
  const size_t msmem = sizeof(double) * mwarps * size_t(s.Kr);
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(buildMOperandKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(msmem)));
  buildMOperandKernel<<<dim3(static_cast<unsigned>((mrows + mwarps - 1) / mwarps), a.n_sectors), 32 * mwarps, msmem,
                        stream>>>(a.sectors, a.perm_r, a.perm_c, s.Kr, static_cast<__half*>(w.mb), w.mInv);
  DCAACC_LAUNCH_CHECK();
  tuneEnd(a.tuner, pm, stream);
  if (w.factored_col) {  // the factored column step reads X' and the twiddles, not Q: P only
    const long groups = (a.n_max + kBK - 1) / kBK * (kBK / 8);
    buildPhaseOperandKernel<true><<<dim3(gridX(groups * d.nw_ext), a.n_sectors), 256, 0, stream>>>(
        d, a.sectors, a.Tr, orb_r, a.Fb, a.G0, w.eP, s.D, s.Dp, s.Dp, s.Kr, static_cast<__half*>(w.pr));
    DCAACC_LAUNCH_CHECK();
    return launches + 2;
  }
  if (a.Tc == a.Tr && orb_c == orb_r) {  // density-density: one pass for P and Q
    // 256 or 128 threads per block (grid-stride loop over independent elements).
    const long groups4 = (a.n_max + kBK - 1) / kBK * (kBK / 4);
    const auto pp = tunePick(a.tuner, tuneKey("tc_pq", d.nb, d.nc, d.nw_ext, a.n_max, a.n_sectors, 2), 2, stream);
    const int threads = pp.choice == 0 ? 256 : 128;
    const unsigned gx = static_cast<unsigned>(std::max(1L, std::min(8192L, (groups4 * d.nw_ext + threads - 1) / threads)));
    auto k = d.nb == 1 ? buildPhasePairKernel<true> : buildPhasePairKernel<false>;
    k<<<dim3(gx, a.n_sectors), threads, 0, stream>>>(
        d, a.sectors, a.Tr, orb_r, a.Fb, a.G0, w.eP, w.eQ, s.Dp, s.Dq, s.Kr, static_cast<__half*>(w.pr),
        static_cast<__half*>(w.bq));
    DCAACC_LAUNCH_CHECK();
    tuneEnd(a.tuner, pp, stream);
    return launches + 2;
  }
  const long groups = (a.n_max + kBK - 1) / kBK * (kBK / 8);
  buildPhaseOperandKernel<true><<<dim3(gridX(groups * d.nw_ext), a.n_sectors), 256, 0, stream>>>(
      d, a.sectors, a.Tr, orb_r, a.Fb, a.G0, w.eP, s.D, s.Dp, s.Dp, s.Kr, static_cast<__half*>(w.pr));
  DCAACC_LAUNCH_CHECK();
  buildPhaseOperandKernel<false><<<dim3(gridX(groups * d.nw_ext), a.n_sectors), 256, 0, stream>>>(
      d, a.sectors, a.Tc, orb_c, a.Fb, a.G0, w.eQ, s.D, s.Dp, s.Dq, s.Kr, static_cast<__half*>(w.bq));
  DCAACC_LAUNCH_CHECK();
  return launches + 3;
}

void launchFrontendTcRow(const FrontendArgs& a, const FrontTcWorkspace& w, int* err, cudaStream_t stream) {
  const FrontTcShape& s = w.shape;
  if (a.n_max == 0)
    return;
  GemmParams p = gemmParams(a, w, err);
  p.mt0 = a.dims.half_g ? s.D / 2 / kBM : 0;  // half G: X' rows of the upper frequency half only
  p.mt = s.Dp / kBM - p.mt0;
  p.nt = (a.n_max + kBN - 1) / kBN;
  const TpDims& d = a.dims;
  const auto pk = tunePick(a.tuner, tuneKey("tc_row_order", d.nb, d.nc, d.nw_ext, a.n_max, a.n_sectors, 2), 2,
                           stream);
  p.order = pk.choice;
  launchGemm<0>(p, w.tm_pr, w.tm_mb, w.n_sm, stream);
  tuneEnd(a.tuner, pk, stream);
}

int launchFrontendTcCol(const FrontendArgs& a, const FrontTcWorkspace& w, float2* G, long g_sector_stride,
                        int* gmax, int* err, cudaStream_t stream) {
  const FrontTcShape& s = w.shape;
  if (w.factored_col && w.col_tc)  // one band, 4 x 4: factored, the site sums in tensor memory
    return launchColFactorTc(a, w, G, g_sector_stride, gmax, err, stream);
  if (w.factored_col)  // one band: the orbital-factored column step (tp_colfactor.cu)
    return launchColFactor(a, w, G, g_sector_stride, gmax, stream);
  GemmParams p = gemmParams(a, w, err);
  p.G = G;
  p.g_sector_stride = g_sector_stride;
  p.gmax = gmax;
  if (gmax)
    DCAACC_CUDA_CHECK(cudaMemsetAsync(gmax, 0, sizeof(int) * size_t(a.n_sectors), stream));
  p.mt = s.Dq / kBM;                          // rows of G^T: rho2
  p.nt0 = a.dims.half_g ? s.D / 2 / kBN : 0;  // columns of G^T: rho1 (half G: the upper half)
  p.nt = s.Dp / kBN - p.nt0;
  const TpDims& d = a.dims;
  const auto pk = tunePick(a.tuner, tuneKey("tc_col_order", d.nb, d.nc, d.nw_ext, a.n_max, a.n_sectors, 2), 2,
                           stream);
  p.order = pk.choice;
  launchGemm<1>(p, w.tm_bq, w.tm_ac, w.n_sm, stream);
  tuneEnd(a.tuner, pk, stream);
  return 1;
}

}  // namespace dcaacc
