// Persistent, warp-specialised tcgen05 GEMM over split-FP16 operand planes, shared by the
// tensor-core front-end (tp_frontend_tc.cu: MODE 0 row step, MODE 1 column step) and the
// disconnected G4 terms (tp_g4_disc.cu: MODE 2).  The design notes are at the top of
// tp_frontend_tc.cu; MODE 2 computes, per (q, wq, channel) problem, D = U V^T over the batch
// (Re = Ur Vr^T - Ui Vi^T, Im = Ur Vi^T + Ui Vr^T) with U, V scaled per row by powers of two.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/dcaacc.h"
#include "async_copy.cuh"
#include "common.cuh"
#include "tcgen05.cuh"
#include "tp_layout.hpp"

namespace dcaacc {
namespace tcg {

constexpr int kPl = 2;                            // FP16 planes per operand
constexpr int kBM = 128;                          // rows per tile
constexpr int kBN = 128;                          // (complex) columns per tile
constexpr int kBK = 32;                           // K per chunk: one 64-byte swizzle row
constexpr uint32_t kBox = kBM * kBK * 2;          // one 128 x 32 FP16 box: 8 KB
constexpr uint32_t kStageStride = 4 * kPl * kBox; // A re, A im, B re, B im (x planes): 64 KB
constexpr int kStages = 3;
constexpr int kEpiWarps = 16;
constexpr uint32_t kBarBytes = 256;  // barriers, tensor-memory slot, chunk maxima
// Dynamic shared memory: alignment slack, operand stages, barriers.
template <int MODE>
__host__ __device__ constexpr size_t gemmSmem() {
  return 1024 + kStages * kStageStride + kBarBytes;
}
constexpr int kGemmThreads = 32 * (2 + kEpiWarps);  // 576
constexpr int kScaleTop = 14;  // scaled maxima land in [2^14, 2^15) (one binade lower for bounds)
constexpr int kMaxDeltaBands = 1;  // bands whose delta-term G0 values the epilogue preloads (registers)

// Offsets inside a stage.
__host__ __device__ constexpr uint32_t boxOff(int part, int plane) {
  return static_cast<uint32_t>(part * kPl + plane) * kBox;  // part: 0 A re, 1 A im, 2 B re, 3 B im
}

// Exponent e with mx * 2^e in [2^14, 2^15) (0 for mx = 0), clamped to [-100, 100] so that both
// 2^e and 2^-e are exact in FP32 (values that far out are zero for all purposes here).
__device__ inline int scaleExp(double mx) {
  return mx > 0 ? max(-100, min(100, kScaleTop - ilogb(mx))) : 0;
}

// Exact powers of two built from their exponent bits (e clamped to the normal range, where the
// scaled values that matter live; anything scaled by a clamped exponent is far below FP16's range).
__device__ inline double pow2d(int e) {
  e = max(-1022, min(1023, e));
  return __hiloint2double((1023 + e) << 20, 0);
}
__device__ inline float pow2f(int e) {
  e = max(-126, min(127, e));
  return __int_as_float((127 + e) << 23);
}

struct Split2 {
  __half h, l;
};
// y = x * 2^e (scale given as the exact power of two) = h + l with |y - h - l| <= 2^-22 |y|,
// both parts rounded to nearest.
__device__ inline Split2 split2f(float x, float scale) {
  const float y = x * scale;
  const __half h = __float2half_rn(y);
  return {h, __float2half_rn(y - __half2float(h))};
}

struct alignas(16) Pack8 {
  __half v[8];
};
__device__ inline void store8(__half* dst, const Pack8& p) {
  *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(&p);
}

// Four values already scaled into FP16 range, y = hi + lo (as split8), packed as 4 halves each.
__device__ inline void split4(const float (&y)[4], uint2& hi, uint2& lo) {
  __half2 h[2], l[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    h[q] = __floats2half2_rn(y[2 * q], y[2 * q + 1]);
    const float2 f = __half22float2(h[q]);
    l[q] = __floats2half2_rn(y[2 * q] - f.x, y[2 * q + 1] - f.y);
  }
  hi = make_uint2(*reinterpret_cast<uint32_t*>(&h[0]), *reinterpret_cast<uint32_t*>(&h[1]));
  lo = make_uint2(*reinterpret_cast<uint32_t*>(&l[0]), *reinterpret_cast<uint32_t*>(&l[1]));
}

// Eight values already scaled into FP16 range, y = hi + lo with both parts rounded to nearest
// (|y - hi - lo| <= 2^-22 |y|): one packed conversion per pair for hi, one for lo.
__device__ inline void split8(const float (&y)[8], Pack8& hi, Pack8& lo) {
  __half2* h = reinterpret_cast<__half2*>(hi.v);
  __half2* l = reinterpret_cast<__half2*>(lo.v);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    h[q] = __floats2half2_rn(y[2 * q], y[2 * q + 1]);
    const float2 f = __half22float2(h[q]);
    l[q] = __floats2half2_rn(y[2 * q] - f.x, y[2 * q + 1] - f.y);
  }
}

__device__ inline double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

struct GemmParams {
  TpDims dims;
  const SectorDesc* sectors;
  int n_sectors;
  int D, Dp, Kr;
  int mt, nt;           // row and column tiles per sector
  int mt0, nt0;         // index of the first row / column tile
  const int* eP;        // [spin][Dp] row exponents of P
  const int* eQ;        // [spin][Dp] row exponents of Q
  const float* mInv;    // [sector][Kr] 2^-e of M's rows j (row step's output columns)
  float* xInv;          // [sector][Dp / 128][Kr / 32] 2^-e of X' per (128-row tile, 32-wide chunk)
  __half* ac;           // row step: X' planes out
  float2* G;            // column step: G out
  long g_sector_stride;
  const double2* G0;
  int* err;
  // MODE 2 (disconnected terms): problems in place of sectors, M x M outputs.
  int n_slots;          // measurements in the batch (K = n_slots per part)
  int Md;               // M = Nc Nw
  const int* eU;        // [problem][Dp] row exponents of U
  const int* eV;        // [problem][Dp] row exponents of V
  float2* disc;         // [problem][n][m] FP32 result
  int* gmax;            // column step: [2 slot + spin] largest |G| of the sector (float bits), or null
  int order;            // persistent tile order within a sector: 0 the built-in one, 1 the two tile
                        // indices swapped (chosen by the launch-shape tuner; results are identical)
};

// Column step, bands beyond those preloaded: adds beta G0_s(b1, b2; k2, w2) to v when column rho1
// of G is a delta column of row rho2 = rho (rho < D).
__device__ inline float2 addDeltaInPlace(const GemmParams& p, const SectorDesc& sd, int rho, int rho1, float2 v) {
  const TpDims& d = p.dims;
  const int r2 = rho % d.R, w2 = rho / d.R;
  const int b1 = rho1 - (d.R * w2 + d.nb * (r2 / d.nb));
  if (b1 >= 0 && b1 < d.nb) {
    const double2 g0 = p.G0[static_cast<long>(sd.spin) * d.nw_ext * d.nc * d.nb * d.nb + b1 +
                            d.nb * (r2 % d.nb + d.nb * (r2 / d.nb + d.nc * w2))];
    v.x += static_cast<float>(d.beta) * static_cast<float>(g0.x);
    v.y += static_cast<float>(d.beta) * static_cast<float>(g0.y);
  }
  return v;
}

// Tile t of the persistent schedule -> (sector, row tile, column tile, K chunks); chunks < 0 when
// the tile has no work (row step: columns j beyond the sector's order).
template <int MODE>
__device__ inline void tileOf(const GemmParams& p, int t, int& sec, int& mt, int& nt, int& chunks) {
  // Within a sector the tiles go either row-tile fastest or column-tile fastest; which one reuses
  // L2 better depends on the shape, so both are launch-shape tuner candidates (order 0 is the
  // built-in one per mode).  Every output tile is computed the same way in either order.
  const int per = p.mt * p.nt;
  sec = t / per;
  const int rem = t % per;
  const bool rows_fastest = (MODE == 0) != (p.order != 0);
  if (rows_fastest) {
    // Row step default: (sector, column tile, row tile).  The eight row tiles that share an M tile
    // run at once, and the few column tiles of a sector, which re-read its P row tiles, follow each
    // other closely enough for those reads to hit L2.  Tiles with j beyond a sector's order are
    // skipped; a CTA's tiles (stride = grid) still visit every column tile.
    nt = p.nt0 + rem / p.mt;
    mt = p.mt0 + rem % p.mt;
  }
  else {
    mt = p.mt0 + rem / p.nt;
    nt = p.nt0 + rem % p.nt;
  }
  if (MODE == 2) {
    chunks = (p.n_slots + kBK - 1) / kBK;
    return;
  }
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
  uint64_t* empty = bars + kStages;          // [kStages] MMA -> TMA, and MMA -> epilogue
  uint64_t* acc_empty = bars + 2 * kStages;  // [2] epilogue -> MMA
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
    for (int b = 0; b < 2; ++b)
      mbarInit(&acc_empty[b], kEpiWarps);  // one arrival per epilogue warp
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
            if (MODE != 0)
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
              else if (MODE == 1) {
                const uint64_t bi = tc::descAdvance(tc::smemDescSw64(st + boxOff(3, pb[pp])), kk * 32);
                // G^T: Re = Qr Xr^T + Qi Xi^T, Im = Qr Xi^T - Qi Xr^T.
                tc::mmaBf16(re, ar, br, idesc, first);
                tc::mmaBf16(re, ai, bi, idesc, 1);
                tc::mmaBf16(im, ar, bi, idesc, first);
                tc::mmaBf16(im, ai, br, idesc | tc::kNegateA, 1);
              }
              else {
                const uint64_t bi = tc::descAdvance(tc::smemDescSw64(st + boxOff(3, pb[pp])), kk * 32);
                // U V^T: Re = Ur Vr^T - Ui Vi^T, Im = Ur Vi^T + Ui Vr^T.
                tc::mmaBf16(re, ar, br, idesc, first);
                tc::mmaBf16(re, ai, bi, idesc | tc::kNegateA, 1);
                tc::mmaBf16(im, ar, bi, idesc, first);
                tc::mmaBf16(im, ai, br, idesc, 1);
              }
            }
          }
          // One commit per chunk: its arrival on the stage's empty barrier both frees the stage for
          // the producer and tells the epilogue that the chunk's sums are in tensor memory.
          tc::commitTo(&empty[s]);
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
      const SectorDesc sd = MODE == 2 ? SectorDesc{} : p.sectors[sec];
      float ar[32], ai[32];
#pragma unroll
      for (int i = 0; i < 32; ++i)
        ar[i] = ai[i] = 0.f;
      const int rho = mt * kBM + row;
      const float* xinv = MODE == 1 ? p.xInv + (static_cast<long>(sec) * xtiles + nt) * kxc : nullptr;
      // Column scales of this warp's 32 columns, one per lane, loaded now (their latency hides
      // behind the chunk loop) and broadcast with shuffles in the epilogue.
      float col_scale = 1.f;
      if (MODE == 0) {
        const int jl = nt * kBN + cg * 32 + lane;
        col_scale = jl < p.Kr ? p.mInv[static_cast<long>(sec) * p.Kr + jl] : 1.f;
      }
      else if (MODE == 2) {
        const int nl = nt * kBN + cg * 32 + lane;
        col_scale = nl < p.Dp ? pow2f(-p.eV[static_cast<long>(sec) * p.Dp + nl]) : 1.f;
      }
      // Row scale of this thread's row, and (column step) the beta G0 values of the row's delta
      // columns when they fall in this warp's 32 columns: all loaded before the chunk loop.
      float row_scale = 1.f;
      float2 dterm[kMaxDeltaBands];
      int dcol = -1;  // first delta column relative to this warp's columns, -1 if none here
      if (MODE == 0)
        row_scale = pow2f(-p.eP[sd.spin * p.Dp + rho]);
      else if (MODE == 2)
        row_scale = rho < p.Md ? pow2f(-p.eU[static_cast<long>(sec) * p.Dp + rho]) : 0.f;
      else if (rho < p.D) {
        row_scale = pow2f(-p.eQ[sd.spin * p.Dp + rho]);
        const TpDims& d = p.dims;
        const int r2 = rho % d.R, w2 = rho / d.R, b2 = r2 % d.nb, k2 = r2 / d.nb;
        const int delta0 = d.R * w2 + d.nb * k2 - (nt * kBN + cg * 32);
        if (delta0 + d.nb > 0 && delta0 < 32 && d.nb <= kMaxDeltaBands) {
          dcol = delta0;
          const double2* g0d = p.G0 + static_cast<long>(sd.spin) * d.nw_ext * d.nc * d.nb * d.nb +
                               d.nb * (b2 + d.nb * (k2 + d.nc * w2));  // + b1 -> G0_s(b1, b2; k2, w2)
          const float beta = static_cast<float>(d.beta);
#pragma unroll
          for (int b = 0; b < kMaxDeltaBands; ++b) {
            const double2 g0 = b < d.nb ? g0d[b] : make_double2(0., 0.);
            dterm[b] = make_float2(beta * static_cast<float>(g0.x), beta * static_cast<float>(g0.y));
          }
        }
      }
      for (int c = 0; c < chunks; ++c, ++g) {
        const int buf = g & 1;
        // Column step: the A rows of chunk c carry the scale 2^e of that X' row chunk; undo it.
        const float f = MODE == 1 ? xinv[c] : 1.f;
        // Chunk g's MMAs are complete when their commit arrives on empty[g % kStages] (its
        // (g / kStages)-th phase).  That barrier cannot run a phase further ahead meanwhile: chunk
        // g + kStages reuses the tensor-memory buffer of chunk g + 1, which this warp releases
        // only after this wait.
        ok = __all_sync(0xffffffffu, mbarWait(&empty[g % kStages], (g / kStages) & 1, err));
        if (!ok)
          break;
        tc::fenceAfterThreadSync();
        const uint32_t col = tmem + lane_addr + buf * 256 + cg * 32;
#pragma unroll
        for (int piece = 0; piece < 2; ++piece) {  // real and imaginary loads share one wait
          float vr[16], vi[16];
          tc::ld32x32bx16(col + piece * 16, vr);
          tc::ld32x32bx16(col + 128 + piece * 16, vi);
          tc::waitLd();
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            ar[piece * 16 + i] = fmaf(vr[i], f, ar[piece * 16 + i]);
            ai[piece * 16 + i] = fmaf(vi[i], f, ai[piece * 16 + i]);
          }
        }
        tc::fenceBeforeThreadSync();
        __syncwarp();
        if (lane == 0)
          mbarArrive(&acc_empty[buf]);
      }
      if (!ok)
        break;
      float gabs = 0.f;  // column step: largest |Re|, |Im| this thread stores
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
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const float sc = row_scale * __shfl_sync(0xffffffffu, col_scale, i);
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
          // The warp's 32 rows x 32 columns go out per part (re hi, re lo, im hi, im lo) through
          // 2 KB of shared memory: lane = row writes its 64-byte row segment (16-byte chunk c at
          // c ^ ((row >> 1) & 3), conflict-free), then each store instruction writes eight whole
          // row segments (lane: row 8 pass + lane / 4, chunk lane % 4).  The staging lies in the
          // B-imaginary part of stages 0 and 1, which the row step's loads never fill.
          const int e = scaleExp(mx);
          const float sc = pow2f(e);
          const long kp = 2L * p.Kr;
          const long plane = static_cast<long>(p.Dp) * kp;
          const int ew = warp - 2;
          unsigned char* stg = base + (ew >> 3) * kStageStride + boxOff(3, 0) + (ew & 7) * 2048;
          __half* o = p.ac + static_cast<long>(sec) * kPl * plane + static_cast<long>(mt * kBM + quarter * 32) * kp + j0;
#pragma unroll
          for (int part = 0; part < 4; ++part) {
            __syncwarp();  // the previous part's reads of the staging are done
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              Pack8 h;
#pragma unroll
              for (int x = 0; x < 8; ++x) {
                const Split2 s2 = split2f(part < 2 ? ar[c * 8 + x] : ai[c * 8 + x], sc);
                h.v[x] = (part & 1) ? s2.l : s2.h;
              }
              store8(reinterpret_cast<__half*>(stg + lane * 64 + ((c ^ ((lane >> 1) & 3)) * 16)), h);
            }
            __syncwarp();
            __half* op = o + (part & 1) * plane + (part >> 1) * p.Kr;
#pragma unroll
            for (int pass = 0; pass < 4; ++pass) {
              const int r = pass * 8 + lane / 4, ch = lane & 3;
              const uint4 w = *reinterpret_cast<const uint4*>(stg + r * 64 + ((ch ^ ((r >> 1) & 3)) * 16));
              *reinterpret_cast<uint4*>(op + static_cast<long>(r) * kp + ch * 8) = w;
            }
          }
          if (quarter == 0 && lane == 0)
            p.xInv[(static_cast<long>(sec) * xtiles + mt) * kxc + j0 / kBK] = pow2f(-e);
        }
      }
      else if (MODE == 2) {
        // Lane row rho = m, columns n = 128 nt + 32 cg + i: disc[(problem M + n) M + m] =
        // acc 2^{-eU(m)} 2^{-eV(n)}; consecutive lanes store consecutive m.
        const int n0 = nt * kBN + cg * 32;
        float2* o = p.disc + static_cast<long>(sec) * p.Md * p.Md + rho;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const float sc = row_scale * __shfl_sync(0xffffffffu, col_scale, i);  // all lanes take part
          if (rho < p.Md && n0 + i < p.Md)
            o[static_cast<long>(n0 + i) * p.Md] = make_float2(ar[i] * sc, ai[i] * sc);
        }
      }
      else if (rho < p.D) {
        // Lane row rho = rho2 (a column of G), columns i -> rho1 = 128 nt + 32 cg + i (rows of G):
        // G(rho1, rho2) = acc 2^{-eQ(rho2)} + beta G0 delta (preloaded: dterm at i = dcol + b1).
        // The G offset of rho1 advances incrementally.
        const TpDims& d = p.dims;
        const int R = d.R, nw_ext = d.nw_ext;
        const int r2 = rho % R, w2 = rho / R;
        float2* gout = p.G + p.g_sector_stride * (2 * sd.slot + sd.spin) + static_cast<long>(w2) * R * R + r2;
        const int rho0 = nt * kBN + cg * 32;
        const int row_step = R, wrap_step = nw_ext * R * R - (R - 1) * R;
        int r1 = rho0 % R;
        int off = (rho0 / R) * nw_ext * R * R + r1 * R;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          if (rho0 + i < p.D) {
            float2 v = make_float2(ar[i] * row_scale, ai[i] * row_scale);
#pragma unroll
            for (int b = 0; b < kMaxDeltaBands; ++b)
              if (i == dcol + b && b < d.nb) {
                v.x += dterm[b].x;
                v.y += dterm[b].y;
              }
            if (d.nb > kMaxDeltaBands)  // more bands than preloaded: load in place
              v = addDeltaInPlace(p, sd, rho, rho0 + i, v);
            gout[off] = v;
            gabs = fmaxf(gabs, fmaxf(fabsf(v.x), fabsf(v.y)));
          }
          if (++r1 == R) {
            r1 = 0;
            off += wrap_step;
          }
          else {
            off += row_step;
          }
        }
      }
      if (MODE == 1 && p.gmax) {
        // The sector's largest |G| (the G4 kernel scales its FP16 operands with it): warp maximum,
        // then one atomic per warp and tile (non-negative floats order like their bit patterns).
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
          gabs = fmaxf(gabs, __shfl_xor_sync(0xffffffffu, gabs, off));
        if (lane == 0 && gabs > 0.f)
          atomicMax(p.gmax + 2 * sd.slot + sd.spin, __float_as_int(gabs));
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

inline EncodeTiledFn encodeTiledFn() {
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
inline void makePlaneMap(CUtensorMap* map, void* base, long cols, long rows, long depth) {
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

template <int MODE>
void launchGemm(const GemmParams& p, const CUtensorMap& ta, const CUtensorMap& tb, int n_sm, cudaStream_t stream) {
  auto k = frontGemmKernel<MODE>;
  constexpr size_t smem = gemmSmem<MODE>();
  static_assert(smem <= 227 * 1024, "shared memory per CTA");
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const long tiles = long(p.n_sectors) * p.mt * p.nt;
  const unsigned grid = static_cast<unsigned>(std::max(1L, std::min<long>(tiles, n_sm)));
  k<<<grid, kGemmThreads, smem, stream>>>(ta, tb, p);
  DCAACC_LAUNCH_CHECK();
}

}  // namespace tcg
}  // namespace dcaacc
