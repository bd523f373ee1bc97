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
#include "tcgen05.cuh"
#include "tp_frontend.hpp"

namespace dcaacc {

namespace {

constexpr int kPl = 2;                            // FP16 planes per operand
constexpr int kBM = 128;                          // rows per tile
constexpr int kBN = 128;                          // (complex) columns per tile
constexpr int kBK = 32;                           // K per chunk: one 64-byte swizzle row
constexpr uint32_t kBox = kBM * kBK * 2;          // one 128 x 32 FP16 box: 8 KB
constexpr uint32_t kStageStride = 4 * kPl * kBox; // A re, A im, B re, B im (x planes): 64 KB
constexpr int kStages = 3;
constexpr size_t kGemmSmem = 1024 + kStages * kStageStride + 256;
constexpr int kEpiWarps = 16;
constexpr int kGemmThreads = 32 * (2 + kEpiWarps);  // 576
constexpr int kScaleTop = 14;  // scaled maxima land in [2^14, 2^15) (one binade lower for bounds)

// Offsets inside a stage.
__host__ __device__ constexpr uint32_t boxOff(int part, int plane) {
  return static_cast<uint32_t>(part * kPl + plane) * kBox;  // part: 0 A re, 1 A im, 2 B re, 3 B im
}

// Matsubara frequency of extended index w (vertex_frequency_domain.hpp, EXTENDED).
__device__ inline double extFreq(int w, int nw_ext, double beta) {
  const int half = nw_ext / 2;
  if (w >= half)
    return M_PI / beta * (1 + 2 * (w - half));
  return -M_PI / beta * (1 + 2 * (half - 1 - w));
}

// Exponent e with mx * 2^e in [2^14, 2^15) (0 for mx = 0).
__device__ inline int scaleExp(double mx) {
  return mx > 0 ? kScaleTop - ilogb(mx) : 0;
}

struct Split2 {
  __half h, l;
};
// x * 2^e = h + l with |x 2^e - h - l| <= 2^-22 |x 2^e| (both parts rounded to nearest).
__device__ inline Split2 split2d(double x, int e) {
  const double y = ldexp(x, e);
  const __half h = __double2half(y);
  return {h, __double2half(y - static_cast<double>(__half2float(h)))};
}
__device__ inline Split2 split2f(float x, int e) {
  const float y = ldexpf(x, e);
  const __half h = __float2half_rn(y);
  return {h, __float2half_rn(y - __half2float(h))};
}

struct Pack8 {
  __half v[8];
};
__device__ inline void store8(__half* dst, const Pack8& p) {
  *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(&p);
}

__device__ inline double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
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
// rows rho < D.  One thread per (rho, 8 vertices).
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
  const double qscale = -1.0 / nc;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < long(groups) * D;
       idx += long(gridDim.x) * blockDim.x) {
    const int grp = static_cast<int>(idx % groups);
    const int rho = static_cast<int>(idx / groups);
    const int r = rho % R, w = rho / R, b = r % nb, k = r / nb;
    const int e = eRow[sd.spin * Dp + rho];
    Pack8 re[kPl], im[kPl];
#pragma unroll
    for (int x = 0; x < 8; ++x) {
      const int v = grp * 8 + x;
      double2 z = make_double2(0., 0.);
      if (v < n) {
        const int ov = orb[sd.vtx_off + v];
        const int bv = ov % nb, xv = ov / nb;
        const double2 ph = zmul(Fb[(bv * nc + k) * nc + xv], Ts[static_cast<long>(w) * n + v]);
        if (ROW) {
          z = zmul(g0s[b + nb * (bv + nb * (k + nc * w))], ph);
        }
        else {
          const double2 g = g0s[bv + nb * (b + nb * (k + nc * w))];
          z = zmul(ph, make_double2(g.x, -g.y));
          z.x *= qscale;
          z.y *= qscale;
        }
      }
      const Split2 a = split2d(z.x, e), c = split2d(z.y, e);
      re[0].v[x] = a.h, re[1].v[x] = a.l;
      im[0].v[x] = c.h, im[1].v[x] = c.l;
    }
#pragma unroll
    for (int pl = 0; pl < kPl; ++pl) {
      __half* op = o + pl * plane + static_cast<long>(rho) * kp + grp * 8;
      store8(op, re[pl]);
      store8(op + Kr, im[pl]);
    }
  }
}

// M operand, planes [sector][plane][Kr rows j][Kr columns i]: M(perm_r[i], perm_c[j]) * 2^{e_j}
// for i, j < n, zero up to i < roundup(n, 32) and j < min(roundup(n, 128), Kr).  One warp per
// row j: the first pass finds the row's maximum, the second writes the scaled planes; 2^{-e_j}
// goes to mInv[sector][j].
__global__ void __launch_bounds__(256)
buildMOperandKernel(const SectorDesc* __restrict__ sectors, const int* __restrict__ perm_r,
                    const int* __restrict__ perm_c, int Kr, __half* __restrict__ out, float* __restrict__ mInv) {
  const SectorDesc sd = sectors[blockIdx.y];
  const int n = sd.n;
  const int groups = (n + kBK - 1) / kBK * (kBK / 8);
  const int rows = min((n + kBN - 1) / kBN * kBN, Kr);
  const long plane = static_cast<long>(Kr) * Kr;
  __half* o = out + static_cast<long>(blockIdx.y) * kPl * plane;
  const int lane = threadIdx.x % 32;
  const int warps = gridDim.x * (blockDim.x / 32);
  for (int j = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; j < rows; j += warps) {
    const double* col = j < n ? sd.M + static_cast<long>(sd.ldm) * perm_c[sd.vtx_off + j] : nullptr;
    double mx = 0;
    if (col)
      for (int i = lane; i < n; i += 32)
        mx = fmax(mx, fabs(col[perm_r[sd.vtx_off + i]]));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    const int e = scaleExp(mx);
    for (int grp = lane; grp < groups; grp += 32) {
      Pack8 v[kPl];
#pragma unroll
      for (int x = 0; x < 8; ++x) {
        const int i = grp * 8 + x;
        const double m = (col && i < n) ? col[perm_r[sd.vtx_off + i]] : 0.;
        const Split2 s = split2d(m, e);
        v[0].v[x] = s.h, v[1].v[x] = s.l;
      }
#pragma unroll
      for (int pl = 0; pl < kPl; ++pl)
        store8(o + pl * plane + static_cast<long>(j) * Kr + grp * 8, v[pl]);
    }
    if (lane == 0)
      mInv[static_cast<long>(blockIdx.y) * Kr + j] = ldexpf(1.f, -e);
  }
}

struct GemmParams {
  TpDims dims;
  const SectorDesc* sectors;
  int n_sectors;
  int D, Dp, Kr;
  int mt, nt;           // row and column tiles per sector
  const int* eP;        // [spin][Dp] row exponents of P
  const int* eQ;        // [spin][Dp] row exponents of Q
  const float* mInv;    // [sector][Kr] 2^-e of M's rows j (row step's output columns)
  float* xInv;          // [sector][Dp / 128][Kr / 32] 2^-e of X' per (128-row tile, 32-wide chunk)
  __half* ac;           // row step: X' planes out
  float2* G;            // column step: G out
  long g_sector_stride;
  const double2* G0;
  int* err;
};

// Tile t of the persistent schedule -> (sector, row tile, column tile, K chunks); chunks < 0 when
// the tile has no work (row step: columns j beyond the sector's order).
template <int MODE>
__device__ inline void tileOf(const GemmParams& p, int t, int& sec, int& mt, int& nt, int& chunks) {
  const int per = p.mt * p.nt;
  sec = t / per;
  const int rem = t % per;
  mt = rem / p.nt;
  nt = rem % p.nt;
  const int n = p.sectors[sec].n;
  chunks = (n + kBK - 1) / kBK;
  if (MODE == 0 && nt * kBN >= n)
    chunks = -1;
}

// MODE 0: row step, A = P planes, B = M planes (rows j), output X' planes and their chunk scales.
// MODE 1: column step on the transpose, A = Q planes (rows rho2), B = X' planes (rows rho1):
//   tensor-memory lane = rho2, so consecutive lanes store consecutive columns of a G block row
//   (two full 128-byte lines per store instruction); output G.
template <int MODE>
__global__ void __launch_bounds__(kGemmThreads, 1)
frontGemmKernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const GemmParams p) {
  constexpr uint32_t stage_bytes = (MODE == 0 ? 3 : 4) * kPl * kBox;
  const int n_tiles = p.n_sectors * p.mt * p.nt;
  const int kxc = p.Kr / kBK;  // X' chunks per row (scale table stride)
  const int xtiles = p.Dp / kBM;

  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kStages * kStageStride);
  uint64_t* full = bars;                     // [kStages] TMA -> MMA
  uint64_t* empty = bars + kStages;          // [kStages] MMA -> TMA
  uint64_t* acc_full = bars + 2 * kStages;   // [2] MMA -> epilogue
  uint64_t* acc_empty = acc_full + 2;        // [2] epilogue -> MMA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  uint64_t* red_bar = bars + 12;                     // epilogue warps exchanged their chunk maxima
  float* red = reinterpret_cast<float*>(bars + 16);  // [2][4 quarters][4 column groups] chunk maxima

  const int t = threadIdx.x, warp = t / 32, lane = t % 32;
  int* err = p.err;
  if (warp == 1) {
    tc::tmemAlloc(tmem_slot, 512);
    tc::tmemRelinquish();
  }
  if (t == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbarInit(&full[s], 1);
      mbarInit(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbarInit(&acc_full[b], 1);
      mbarInit(&acc_empty[b], kEpiWarps);  // one arrival per epilogue warp
    }
    mbarInit(red_bar, kEpiWarps);
    fenceBarrierInit();
    tc::prefetchTensorMap(&tmA);
    tc::prefetchTensorMap(&tmB);
  }
  tc::fenceBeforeThreadSync();
  __syncthreads();
  tc::fenceAfterThreadSync();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int g = 0;  // chunks issued (global over the CTA's tiles)
      bool ok = true;
      for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        int sec, mt, nt, chunks;
        tileOf<MODE>(p, tile, sec, mt, nt, chunks);
        for (int c = 0; c < chunks; ++c, ++g) {
          const int s = g % kStages, use = g / kStages;
          if (use > 0 && !mbarWait(&empty[s], (use - 1) & 1, err)) {
            ok = false;
            break;
          }
          unsigned char* st = base + s * kStageStride;
          mbarArriveExpectTx(&full[s], stage_bytes);
          const int xr = c * kBK, xi = p.Kr + c * kBK;
#pragma unroll
          for (int pl = 0; pl < kPl; ++pl) {
            const int z = sec * kPl + pl;
            tc::tmaLoad3d(st + boxOff(0, pl), &tmA, xr, mt * kBM, z, &full[s]);
            tc::tmaLoad3d(st + boxOff(1, pl), &tmA, xi, mt * kBM, z, &full[s]);
            tc::tmaLoad3d(st + boxOff(2, pl), &tmB, xr, nt * kBN, z, &full[s]);
            if (MODE == 1)
              tc::tmaLoad3d(st + boxOff(3, pl), &tmB, xi, nt * kBN, z, &full[s]);
          }
        }
      }
      // Loads still in flight are waited for (bounded) before the CTA can exit; on the normal
      // path every issued stage has been consumed already.
      for (int c = max(0, g - kStages); c < g; ++c)
        mbarWait(&full[c % kStages], (c / kStages) & 1, err);
    }
  }
  else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = tc::instrDescF16F32(kBM, kBN);
      // (A plane, B plane) products kept by the two-way split, smallest first: lo*hi, hi*lo, hi*hi.
      const int pa[3] = {1, 0, 0};
      const int pb[3] = {0, 1, 0};
      int g = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        int sec, mt, nt, chunks;
        tileOf<MODE>(p, tile, sec, mt, nt, chunks);
        for (int c = 0; c < chunks; ++c, ++g) {
          const int s = g % kStages, buf = g & 1;
          if (!mbarWait(&full[s], (g / kStages) & 1, err) ||
              (g >= 2 && !mbarWait(&acc_empty[buf], ((g >> 1) - 1) & 1, err))) {
            ok = false;
            break;
          }
          tc::fenceAfterThreadSync();
          unsigned char* st = base + s * kStageStride;
          const uint32_t re = tmem + buf * 256, im = re + 128;
#pragma unroll
          for (int pp = 0; pp < 3; ++pp) {
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {  // 2 x K16 per 32-wide chunk: 32 bytes each
              const uint32_t first = (pp | kk) != 0;
              const uint64_t ar = tc::descAdvance(tc::smemDescSw64(st + boxOff(0, pa[pp])), kk * 32);
              const uint64_t ai = tc::descAdvance(tc::smemDescSw64(st + boxOff(1, pa[pp])), kk * 32);
              const uint64_t br = tc::descAdvance(tc::smemDescSw64(st + boxOff(2, pb[pp])), kk * 32);
              if (MODE == 0) {
                tc::mmaBf16(re, ar, br, idesc, first);
                tc::mmaBf16(im, ai, br, idesc, first);
              }
              else {
                const uint64_t bi = tc::descAdvance(tc::smemDescSw64(st + boxOff(3, pb[pp])), kk * 32);
                // G^T: Re = Qr Xr^T + Qi Xi^T, Im = Qr Xi^T - Qi Xr^T.
                tc::mmaBf16(re, ar, br, idesc, first);
                tc::mmaBf16(re, ai, bi, idesc, 1);
                tc::mmaBf16(im, ar, bi, idesc, first);
                tc::mmaBf16(im, ai, br, idesc | tc::kNegateA, 1);
              }
            }
          }
          tc::commitTo(&empty[s]);
          tc::commitTo(&acc_full[buf]);
        }
      }
    }
  }
  else {
    // Epilogue warps 2..17: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (rows of the tile)
    // and complex columns 32 cg .. + 31, cg = (w - 2) / 4.
    const int quarter = warp & 3;
    const int cg = (warp - 2) >> 2;
    const int row = quarter * 32 + lane;
    const uint32_t lane_addr = static_cast<uint32_t>(quarter * 32) << 16;
    int g = 0, tiles_done = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
      int sec, mt, nt, chunks;
      tileOf<MODE>(p, tile, sec, mt, nt, chunks);
      if (chunks < 0)
        continue;
      ++tiles_done;
      const SectorDesc sd = p.sectors[sec];
      float ar[32], ai[32];
#pragma unroll
      for (int i = 0; i < 32; ++i)
        ar[i] = ai[i] = 0.f;
      const int rho = mt * kBM + row;
      const float* xinv = p.xInv + (static_cast<long>(sec) * xtiles + nt) * kxc;
      for (int c = 0; c < chunks; ++c, ++g) {
        const int buf = g & 1;
        // Column step: the A rows of chunk c carry the scale 2^e of that X' row chunk; undo it.
        const float f = MODE == 1 ? xinv[c] : 1.f;
        ok = __all_sync(0xffffffffu, mbarWait(&acc_full[buf], (g >> 1) & 1, err));
        if (!ok)
          break;
        tc::fenceAfterThreadSync();
        const uint32_t col = tmem + lane_addr + buf * 256 + cg * 32;
#pragma unroll
        for (int piece = 0; piece < 2; ++piece) {
          float v[16];
          tc::ld32x32bx16(col + piece * 16, v);
          tc::waitLd();
#pragma unroll
          for (int i = 0; i < 16; ++i)
            ar[piece * 16 + i] = fmaf(v[i], f, ar[piece * 16 + i]);
          tc::ld32x32bx16(col + 128 + piece * 16, v);
          tc::waitLd();
#pragma unroll
          for (int i = 0; i < 16; ++i)
            ai[piece * 16 + i] = fmaf(v[i], f, ai[piece * 16 + i]);
        }
        tc::fenceBeforeThreadSync();
        __syncwarp();
        if (lane == 0)
          mbarArrive(&acc_empty[buf]);
      }
      if (!ok)
        break;
      if (MODE == 0) {
        // X'(rho, j) = acc 2^{-eP(rho)} 2^{-e_j}, j = 128 nt + 32 cg + i: one 32-wide K chunk of the
        // column step, whose B tile (128 rows rho of this tile) needs one scale for the whole
        // chunk: the maximum over the four warps with this column group, exchanged through `red`
        // (double-buffered by tile parity) at a barrier of the 16 epilogue warps.  The chunk is
        // written only if the column step reads it (j0 < roundup(n, 32)).
        const int j0 = nt * kBN + cg * 32;
        const bool live = j0 < chunks * kBK;
        float mx = 0.f;
        if (live) {
          const float pinv = ldexpf(1.f, -p.eP[sd.spin * p.Dp + rho]);
          const float* minv = p.mInv + static_cast<long>(sec) * p.Kr + j0;
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const float sc = pinv * minv[i];
            ar[i] *= sc;
            ai[i] *= sc;
            mx = fmaxf(mx, fmaxf(fabsf(ar[i]), fabsf(ai[i])));
          }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
          mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        float* rb = red + (tiles_done & 1) * 16;
        __syncwarp();
        if (lane == 0) {
          rb[quarter * 4 + cg] = mx;
          mbarArrive(red_bar);  // release: this warp's maximum is visible to the waiters
        }
        ok = __all_sync(0xffffffffu, mbarWait(red_bar, (tiles_done - 1) & 1, err));
        if (!ok)
          break;
        mx = fmaxf(fmaxf(rb[cg], rb[4 + cg]), fmaxf(rb[8 + cg], rb[12 + cg]));
        if (live) {
          const int e = mx > 0.f ? kScaleTop - ilogbf(mx) : 0;
          const long kp = 2L * p.Kr;
          const long plane = static_cast<long>(p.Dp) * kp;
          __half* o = p.ac + static_cast<long>(sec) * kPl * plane + static_cast<long>(rho) * kp + j0;
#pragma unroll
          for (int g8 = 0; g8 < 4; ++g8) {
            Pack8 hr, lr, hi, li;
#pragma unroll
            for (int x = 0; x < 8; ++x) {
              const Split2 a = split2f(ar[g8 * 8 + x], e), b = split2f(ai[g8 * 8 + x], e);
              hr.v[x] = a.h, lr.v[x] = a.l, hi.v[x] = b.h, li.v[x] = b.l;
            }
            store8(o + g8 * 8, hr);
            store8(o + plane + g8 * 8, lr);
            store8(o + p.Kr + g8 * 8, hi);
            store8(o + plane + p.Kr + g8 * 8, li);
          }
          if (quarter == 0 && lane == 0)
            p.xInv[(static_cast<long>(sec) * xtiles + mt) * kxc + j0 / kBK] = ldexpf(1.f, -e);
        }
      }
      else if (rho < p.D) {
        // Lane row rho = rho2 (a column of G), columns i -> rho1 = 128 nt + 32 cg + i (rows of G):
        // G(rho1, rho2) = acc 2^{-eQ(rho2)} + beta G0 delta.
        const TpDims& d = p.dims;
        const int R = d.R, nb = d.nb, nc = d.nc, nw_ext = d.nw_ext;
        const int r2 = rho % R, w2 = rho / R, b2 = r2 % nb, k2 = r2 / nb;
        float2* gout = p.G + p.g_sector_stride * (2 * sd.slot + sd.spin) + static_cast<long>(w2) * R * R + r2;
        const double2* g0s = p.G0 + static_cast<long>(sd.spin) * nw_ext * nc * nb * nb;
        const float qinv = ldexpf(1.f, -p.eQ[sd.spin * p.Dp + rho]);
        const float beta = static_cast<float>(d.beta);
        const int rho0 = nt * kBN + cg * 32;
        int r1 = rho0 % R, w1 = rho0 / R;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          if (rho0 + i < p.D) {
            float2 v = make_float2(ar[i] * qinv, ai[i] * qinv);
            if (w1 == w2 && r1 / nb == k2) {
              const double2 g0 = g0s[r1 % nb + nb * (b2 + nb * (k2 + nc * w2))];
              v.x += beta * static_cast<float>(g0.x);
              v.y += beta * static_cast<float>(g0.y);
            }
            gout[static_cast<long>(w1) * nw_ext * R * R + static_cast<long>(r1) * R] = v;
          }
          if (++r1 == R) {
            r1 = 0;
            ++w1;
          }
        }
      }
    }
  }
  tc::fenceBeforeThreadSync();
  __syncthreads();
  if (warp == 1) {
    tc::fenceAfterThreadSync();
    tc::tmemDealloc(tmem, 512);
  }
}

// ---- tensor maps ----
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encodeTiledFn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    DCAACC_CUDA_CHECK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p)
      throw Error(DCAACC_CUDA_ERR, "cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// FP16 planes [depth][rows][cols] (cols fastest), 32 x 128 x 1 boxes, 64-byte swizzle; rows or
// columns beyond the extents read as zero.
void makePlaneMap(CUtensorMap* map, void* base, long cols, long rows, long depth) {
  const cuuint64_t dims[3] = {cuuint64_t(cols), cuuint64_t(rows), cuuint64_t(depth)};
  const cuuint64_t strides[2] = {cuuint64_t(cols) * 2, cuuint64_t(cols) * rows * 2};
  const cuuint32_t box[3] = {kBK, kBM, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encodeTiledFn()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, base, dims, strides, box, estr,
                                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    throw Error(DCAACC_CUDA_ERR, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
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

template <int MODE>
void launchGemm(const GemmParams& p, const CUtensorMap& ta, const CUtensorMap& tb, int n_sm, cudaStream_t stream) {
  auto k = frontGemmKernel<MODE>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGemmSmem)));
  const long tiles = long(p.n_sectors) * p.mt * p.nt;
  const unsigned grid = static_cast<unsigned>(std::max(1L, std::min<long>(tiles, n_sm)));
  k<<<grid, kGemmThreads, kGemmSmem, stream>>>(ta, tb, p);
  DCAACC_LAUNCH_CHECK();
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
  const long groups = (a.n_max + kBK - 1) / kBK * (kBK / 8);
  buildPhaseOperandKernel<true><<<dim3(gridX(groups * s.D), a.n_sectors), 256, 0, stream>>>(
      d, a.sectors, a.Tr, orb_r, a.Fb, a.G0, w.eP, s.D, s.Dp, s.Dp, s.Kr, static_cast<__half*>(w.pr));
  DCAACC_LAUNCH_CHECK();
  const long mrows = std::min<long>((a.n_max + kBN - 1) / kBN * kBN, s.Kr);
  buildMOperandKernel<<<dim3(static_cast<unsigned>((mrows + 7) / 8), a.n_sectors), 256, 0, stream>>>(
      a.sectors, a.perm_r, a.perm_c, s.Kr, static_cast<__half*>(w.mb), w.mInv);
  DCAACC_LAUNCH_CHECK();
  buildPhaseOperandKernel<false><<<dim3(gridX(groups * s.D), a.n_sectors), 256, 0, stream>>>(
      d, a.sectors, a.Tc, orb_c, a.Fb, a.G0, w.eQ, s.D, s.Dp, s.Dq, s.Kr, static_cast<__half*>(w.bq));
  DCAACC_LAUNCH_CHECK();
  return launches + 3;
}

void launchFrontendTcRow(const FrontendArgs& a, const FrontTcWorkspace& w, int* err, cudaStream_t stream) {
  const FrontTcShape& s = w.shape;
  if (a.n_max == 0)
    return;
  GemmParams p = gemmParams(a, w, err);
  p.mt = s.Dp / kBM;
  p.nt = (a.n_max + kBN - 1) / kBN;
  launchGemm<0>(p, w.tm_pr, w.tm_mb, w.n_sm, stream);
}

void launchFrontendTcCol(const FrontendArgs& a, const FrontTcWorkspace& w, float2* G, long g_sector_stride,
                         int* err, cudaStream_t stream) {
  const FrontTcShape& s = w.shape;
  GemmParams p = gemmParams(a, w, err);
  p.G = G;
  p.g_sector_stride = g_sector_stride;
  p.mt = s.Dq / kBM;  // rows of G^T: rho2
  p.nt = s.Dp / kBN;  // columns of G^T: rho1
  launchGemm<1>(p, w.tm_bq, w.tm_ac, w.n_sm, stream);
}

}  // namespace dcaacc
