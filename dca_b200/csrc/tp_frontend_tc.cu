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
//   X' = P M          (row step,    real GEMM [Pr; Pi] x M)
//   G  = X' Q^H + beta G0_s(b1, b2; k1, w1) delta_{k1 k2} delta_{w1 w2}
//                     (column step, real GEMM [X'r | X'i] x rows [Qr | Qi] and [-Qi | Qr])
// where x_i, b_i are vertex i's site and band.  This is the reference's G exactly (the band sums
// of -G0 G~ G0 become the G0 factors inside P and Q).
//
// Precision: every operand is split into three BF16 planes (x = hi + mid + lo to 2^-24), and the
// six plane products above 2^-24 (lh, mm, hl, mh, hm, hh, smallest first) are accumulated in FP32
// tensor memory.  The tensor core's accumulation does not round to nearest and its error grows with
// the number of MMAs that feed one accumulator, and the diagonal blocks of G are coherent sums over
// the vertices; so each 64-wide K chunk goes to a fresh pair of accumulators, which the epilogue
// warps read and add into FP32 registers in round-to-nearest while the next chunk runs
// (double-buffered tensor memory: 2 chunks x 2 accumulators x 128 columns = all 512 columns).
//
// GEMM kernel: CTA = 128 rows x 128 real columns, 320 threads, one CTA per SM (shared memory).
//   warp 0      TMA producer: per K chunk, 3 A planes + 3 B planes (64 x 128 boxes, 128-byte
//               swizzle) into one of two shared-memory stages;
//   warp 1      allocates tensor memory; one thread issues the 24 MMAs of a chunk and commits
//               them to the stage's "empty" barrier and the accumulator pair's "full" barrier;
//   warps 2-9   promote each finished accumulator pair into registers, then run the epilogue
//               (row step: split X' into the column step's planes; column step: store G).
// Every wait is bounded (kWaitLimit polls, then the error word is set and the roles stop).
#include <cuda.h>
#include <cuda_bf16.h>
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

constexpr int kPl = 3;                                  // BF16 planes per operand
constexpr int kBM = 128;                                // rows per CTA
constexpr int kBN = 128;                                // real accumulator columns per CTA
constexpr int kBK = 64;                                 // K per stage: one 128-byte swizzle atom
constexpr uint32_t kTileBytes = kBM * kBK * 2;          // one plane of A or B: 16 KB
constexpr uint32_t kStageBytes = 2 * kPl * kTileBytes;  // 96 KB
constexpr int kStages = 2;
constexpr size_t kGemmSmem = 1024 + kStages * kStageBytes + 128;
constexpr int kGemmThreads = 320;

// Matsubara frequency of extended index w (vertex_frequency_domain.hpp, EXTENDED).
__device__ inline double extFreq(int w, int nw_ext, double beta) {
  const int half = nw_ext / 2;
  if (w >= half)
    return M_PI / beta * (1 + 2 * (w - half));
  return -M_PI / beta * (1 + 2 * (half - 1 - w));
}

struct Split3d {
  __nv_bfloat16 h, m, l;
};
// x = h + m + l to about 2^-24 |x|, each part rounded to nearest from the exact remainder.
__device__ inline Split3d split3d(double x) {
  const __nv_bfloat16 h = __double2bfloat16(x);
  const double r1 = x - static_cast<double>(__bfloat162float(h));
  const __nv_bfloat16 m = __double2bfloat16(r1);
  const double r2 = r1 - static_cast<double>(__bfloat162float(m));
  return {h, m, __double2bfloat16(r2)};
}
__device__ inline Split3d split3f(float x) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(h);
  const __nv_bfloat16 m = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(m);
  return {h, m, __float2bfloat16_rn(r2)};
}

struct Pack8 {
  __nv_bfloat16 v[8];
};
__device__ inline void store8(__nv_bfloat16* dst, const Pack8& p) {
  *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(&p);
}

__device__ inline double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
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

// Row operand P, planes [sector][plane][2 Dp rows][Kr]: rows 0..Dp-1 real part, Dp..2Dp-1
// imaginary part; columns i < roundup(n, 64) (zero for i >= n).  One thread per (rho, 8 columns).
__global__ void __launch_bounds__(256)
buildRowOperandKernel(const TpDims dims, const SectorDesc* __restrict__ sectors, const double2* __restrict__ T,
                      const int* __restrict__ orb, const double2* __restrict__ Fb, const double2* __restrict__ G0,
                      int D, int Dp, int Kr, __nv_bfloat16* __restrict__ out) {
  const SectorDesc sd = sectors[blockIdx.y];
  const int n = sd.n;
  const int groups = (n + kBK - 1) / kBK * (kBK / 8);
  const int nb = dims.nb, nc = dims.nc, R = dims.R, nw_ext = dims.nw_ext;
  const long plane = 2L * Dp * Kr;
  __nv_bfloat16* o = out + static_cast<long>(blockIdx.y) * kPl * plane;
  const double2* g0s = G0 + static_cast<long>(sd.spin) * nw_ext * nc * nb * nb;
  const double2* Ts = T + static_cast<long>(sd.vtx_off) * nw_ext;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < long(groups) * D;
       idx += long(gridDim.x) * blockDim.x) {
    const int grp = static_cast<int>(idx % groups);
    const int rho = static_cast<int>(idx / groups);
    const int r = rho % R, w = rho / R, b1 = r % nb, k1 = r / nb;
    Pack8 re[kPl], im[kPl];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int i = grp * 8 + e;
      double2 v = make_double2(0., 0.);
      if (i < n) {
        const int oi = orb[sd.vtx_off + i];
        const int bi = oi % nb, xi = oi / nb;
        v = zmul(zmul(g0s[b1 + nb * (bi + nb * (k1 + nc * w))], Fb[(bi * nc + k1) * nc + xi]),
                 Ts[static_cast<long>(w) * n + i]);
      }
      const Split3d a = split3d(v.x), b = split3d(v.y);
      re[0].v[e] = a.h, re[1].v[e] = a.m, re[2].v[e] = a.l;
      im[0].v[e] = b.h, im[1].v[e] = b.m, im[2].v[e] = b.l;
    }
#pragma unroll
    for (int pl = 0; pl < kPl; ++pl) {
      store8(o + pl * plane + static_cast<long>(rho) * Kr + grp * 8, re[pl]);
      store8(o + pl * plane + static_cast<long>(Dp + rho) * Kr + grp * 8, im[pl]);
    }
  }
}

// M operand, planes [sector][plane][Kr rows j][Kr columns i]: M(perm_r[i], perm_c[j]) for
// i, j < n, zero up to i < roundup(n, 64) and j < min(roundup(n, 128), Kr).
__global__ void __launch_bounds__(256)
buildMOperandKernel(const SectorDesc* __restrict__ sectors, const int* __restrict__ perm_r,
                    const int* __restrict__ perm_c, int Kr, __nv_bfloat16* __restrict__ out) {
  const SectorDesc sd = sectors[blockIdx.y];
  const int n = sd.n;
  const int groups = (n + kBK - 1) / kBK * (kBK / 8);
  const int rows = min((n + kBN - 1) / kBN * kBN, Kr);
  const long plane = static_cast<long>(Kr) * Kr;
  __nv_bfloat16* o = out + static_cast<long>(blockIdx.y) * kPl * plane;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < long(groups) * rows;
       idx += long(gridDim.x) * blockDim.x) {
    const int grp = static_cast<int>(idx % groups);
    const int j = static_cast<int>(idx / groups);
    const double* col = j < n ? sd.M + static_cast<long>(sd.ldm) * perm_c[sd.vtx_off + j] : nullptr;
    Pack8 v[kPl];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int i = grp * 8 + e;
      const double m = (col && i < n) ? col[perm_r[sd.vtx_off + i]] : 0.;
      const Split3d s = split3d(m);
      v[0].v[e] = s.h, v[1].v[e] = s.m, v[2].v[e] = s.l;
    }
#pragma unroll
    for (int pl = 0; pl < kPl; ++pl)
      store8(o + pl * plane + static_cast<long>(j) * Kr + grp * 8, v[pl]);
  }
}

// Column operand Q, planes [sector][plane][2 Dq rows][2 Kr]: for rho2 = 64 cb + c, row 128 cb + c
// holds [Qr | Qi] and row 128 cb + 64 + c holds [-Qi | Qr] (imaginary parts at column Kr + j).
__global__ void __launch_bounds__(256)
buildColOperandKernel(const TpDims dims, const SectorDesc* __restrict__ sectors, const double2* __restrict__ T,
                      const int* __restrict__ orb, const double2* __restrict__ Fb, const double2* __restrict__ G0,
                      int D, int Dq, int Kr, __nv_bfloat16* __restrict__ out) {
  const SectorDesc sd = sectors[blockIdx.y];
  const int n = sd.n;
  const int groups = (n + kBK - 1) / kBK * (kBK / 8);
  const int nb = dims.nb, nc = dims.nc, R = dims.R, nw_ext = dims.nw_ext;
  const long kp = 2L * Kr;
  const long plane = 2L * Dq * kp;
  __nv_bfloat16* o = out + static_cast<long>(blockIdx.y) * kPl * plane;
  const double2* g0s = G0 + static_cast<long>(sd.spin) * nw_ext * nc * nb * nb;
  const double2* Ts = T + static_cast<long>(sd.vtx_off) * nw_ext;
  const double scale = -1.0 / nc;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < long(groups) * D;
       idx += long(gridDim.x) * blockDim.x) {
    const int grp = static_cast<int>(idx % groups);
    const int rho = static_cast<int>(idx / groups);
    const int r = rho % R, w = rho / R, b2 = r % nb, k2 = r / nb;
    Pack8 qr[kPl], qi[kPl], mqi[kPl];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int j = grp * 8 + e;
      double2 v = make_double2(0., 0.);
      if (j < n) {
        const int oj = orb[sd.vtx_off + j];
        const int bj = oj % nb, xj = oj / nb;
        const double2 g = g0s[bj + nb * (b2 + nb * (k2 + nc * w))];
        v = zmul(zmul(Fb[(bj * nc + k2) * nc + xj], Ts[static_cast<long>(w) * n + j]), make_double2(g.x, -g.y));
        v.x *= scale;
        v.y *= scale;
      }
      const Split3d a = split3d(v.x), b = split3d(v.y), c = split3d(-v.y);
      qr[0].v[e] = a.h, qr[1].v[e] = a.m, qr[2].v[e] = a.l;
      qi[0].v[e] = b.h, qi[1].v[e] = b.m, qi[2].v[e] = b.l;
      mqi[0].v[e] = c.h, mqi[1].v[e] = c.m, mqi[2].v[e] = c.l;
    }
    const long rre = static_cast<long>(rho / 64) * 128 + rho % 64, rim = rre + 64;
#pragma unroll
    for (int pl = 0; pl < kPl; ++pl) {
      __nv_bfloat16* op = o + pl * plane;
      store8(op + rre * kp + grp * 8, qr[pl]);
      store8(op + rre * kp + Kr + grp * 8, qi[pl]);
      store8(op + rim * kp + grp * 8, mqi[pl]);
      store8(op + rim * kp + Kr + grp * 8, qr[pl]);
    }
  }
}

struct GemmParams {
  TpDims dims;
  const SectorDesc* sectors;
  int D, Dp, Kr;
  __nv_bfloat16* ac;  // row step: X' planes out
  float2* G;          // column step: G out
  long g_sector_stride;
  const double2* G0;
  int* err;
};

// MODE 0: row step, A = P planes (2 Dp rows), B = M planes (rows j), output X' planes.
// MODE 1: column step, A = X' planes (Dp rows), B = Q planes (interleaved rows), output G.
// grid (A rows / 128, column tiles, n_sectors).
template <int MODE>
__global__ void __launch_bounds__(kGemmThreads, 1)
frontGemmKernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const GemmParams p) {
  const int sec = blockIdx.z;
  const SectorDesc sd = p.sectors[sec];
  const int n = sd.n;
  const int m0 = blockIdx.x * kBM;
  const int nt = blockIdx.y;
  const int nc1 = (n + kBK - 1) / kBK;  // K chunks over the vertices
  if (MODE == 0 && nt * kBN >= n)
    return;  // whole CTA: no columns j of this sector in this tile
  const int n_chunks = MODE == 0 ? nc1 : 2 * nc1;

  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kStages * kStageBytes);
  uint64_t* full = bars;          // [kStages] TMA -> MMA
  uint64_t* empty = bars + 2;     // [kStages] MMA -> TMA
  uint64_t* acc_full = bars + 4;  // [2] MMA -> epilogue
  uint64_t* acc_empty = bars + 6; // [2] epilogue -> MMA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 8);

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
      mbarInit(&acc_empty[b], 8);  // one arrival per epilogue warp
    }
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
      int issued = 0;
      for (int c = 0; c < n_chunks; ++c) {
        const int s = c & 1;
        if (c >= 2 && !mbarWait(&empty[s], ((c >> 1) - 1) & 1, err))
          break;
        const int kx = (MODE == 0 || c < nc1) ? c * kBK : p.Kr + (c - nc1) * kBK;
        unsigned char* st = base + s * kStageBytes;
        mbarArriveExpectTx(&full[s], kStageBytes);
#pragma unroll
        for (int pl = 0; pl < kPl; ++pl)
          tc::tmaLoad3d(st + pl * kTileBytes, &tmA, kx, m0, sec * kPl + pl, &full[s]);
#pragma unroll
        for (int pl = 0; pl < kPl; ++pl)
          tc::tmaLoad3d(st + (kPl + pl) * kTileBytes, &tmB, kx, nt * kBN, sec * kPl + pl, &full[s]);
        ++issued;
      }
      // Loads still in flight are waited for (bounded) before the CTA can exit; on the normal
      // path every issued stage has been consumed already.
      for (int c = max(0, issued - 2); c < issued; ++c)
        mbarWait(&full[c & 1], (c >> 1) & 1, err);
    }
  }
  else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = tc::instrDescBf16F32(kBM, kBN);
      // (A plane, B plane) pairs kept by the three-way split, smallest first.
      const int pa[6] = {2, 1, 0, 1, 0, 0};
      const int pb[6] = {0, 1, 2, 0, 1, 0};
      for (int c = 0; c < n_chunks; ++c) {
        const int s = c & 1, pb2 = c & 1;
        if (!mbarWait(&full[s], (c >> 1) & 1, err))
          break;
        if (c >= 2 && !mbarWait(&acc_empty[pb2], ((c >> 1) - 1) & 1, err))
          break;
        tc::fenceAfterThreadSync();
        unsigned char* st = base + s * kStageBytes;
#pragma unroll
        for (int pp = 0; pp < 6; ++pp) {
          const uint64_t da = tc::smemDescSw128(st + pa[pp] * kTileBytes);
          const uint64_t db = tc::smemDescSw128(st + (kPl + pb[pp]) * kTileBytes);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint32_t col = static_cast<uint32_t>(2 * pb2 + (kk >> 1)) * 128;
            tc::mmaBf16(tmem + col, tc::descAdvance(da, kk * 32), tc::descAdvance(db, kk * 32), idesc,
                        (pp | (kk & 1)) != 0);
          }
        }
        tc::commitTo(&empty[s]);
        tc::commitTo(&acc_full[pb2]);
      }
    }
  }
  else {
    // Epilogue warps 2..9: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (rows of the tile);
    // warps 2-5 take the first half of this thread's columns, warps 6-9 the second half.
    const int quarter = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = quarter * 32 + lane;
    const uint32_t lane_addr = static_cast<uint32_t>(quarter * 32) << 16;
    // MODE 0: acc[i] = column h*64 + i.  MODE 1: acc[i] = Re, acc[32 + i] = Im of complex
    // column h*32 + i (tensor-memory columns h*32 + i and 64 + h*32 + i).
    float acc[64];
#pragma unroll
    for (int i = 0; i < 64; ++i)
      acc[i] = 0.f;
    bool ok = true;
    for (int c = 0; c < n_chunks; ++c) {
      const int pb2 = c & 1;
      ok = __all_sync(0xffffffffu, mbarWait(&acc_full[pb2], (c >> 1) & 1, err));
      if (!ok)
        break;
      tc::fenceAfterThreadSync();
#pragma unroll
      for (int part = 0; part < 2; ++part) {
        const uint32_t col = MODE == 0 ? half * 64 + part * 32 : part * 64 + half * 32;
        float v0[32], v1[32];
        tc::ld32x32bx32(tmem + lane_addr + (2 * pb2) * 128 + col, v0);
        tc::ld32x32bx32(tmem + lane_addr + (2 * pb2 + 1) * 128 + col, v1);
        tc::waitLd();
#pragma unroll
        for (int i = 0; i < 32; ++i)
          acc[part * 32 + i] += v0[i] + v1[i];
      }
      tc::fenceBeforeThreadSync();
      __syncwarp();
      if (lane == 0)
        mbarArrive(&acc_empty[pb2]);
    }
    if (ok) {
      if (MODE == 0) {
        // X'(rho', j) -> column-step planes: rho' < Dp real part at column j, else imaginary part
        // of row rho' - Dp at column Kr + j; only j < roundup(n, 64) (the range the column step
        // reads).
        const int rho = m0 + row;
        const int dst = rho < p.Dp ? rho : rho - p.Dp;
        const int koff = rho < p.Dp ? 0 : p.Kr;
        const int n_pad = nc1 * kBK;
        const long kp = 2L * p.Kr;
        const long plane = static_cast<long>(p.Dp) * kp;
        __nv_bfloat16* o = p.ac + static_cast<long>(sec) * kPl * plane + static_cast<long>(dst) * kp + koff;
#pragma unroll
        for (int g = 0; g < 8; ++g) {
          const int j0 = nt * kBN + half * 64 + g * 8;
          if (j0 < n_pad) {
            Pack8 hi, mid, lo;
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const Split3d s = split3f(acc[g * 8 + e]);
              hi.v[e] = s.h, mid.v[e] = s.m, lo.v[e] = s.l;
            }
            store8(o + j0, hi);
            store8(o + plane + j0, mid);
            store8(o + 2 * plane + j0, lo);
          }
        }
      }
      else {
        const TpDims& d = p.dims;
        const int rho1 = m0 + row;
        if (rho1 < p.D) {
          const int R = d.R, nb = d.nb, nc = d.nc, nw_ext = d.nw_ext;
          const int r1 = rho1 % R, w1 = rho1 / R, b1 = r1 % nb, k1 = r1 / nb;
          float2* gout = p.G + p.g_sector_stride * (2 * sd.slot + sd.spin);
          const double2* g0s = p.G0 + static_cast<long>(sd.spin) * nw_ext * nc * nb * nb;
          const float beta = static_cast<float>(d.beta);
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const int rho2 = nt * 64 + half * 32 + i;
            if (rho2 < p.D) {
              const int r2 = rho2 % R, w2 = rho2 / R;
              float2 v = make_float2(acc[i], acc[32 + i]);
              if (w2 == w1 && r2 / nb == k1) {
                const double2 g = g0s[b1 + nb * (r2 % nb + nb * (k1 + nc * w1))];
                v.x += beta * static_cast<float>(g.x);
                v.y += beta * static_cast<float>(g.y);
              }
              gout[(static_cast<long>(w1) * nw_ext + w2) * R * R + static_cast<long>(r1) * R + r2] = v;
            }
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

// BF16 planes [depth][rows][cols] (cols fastest), 64 x 128 x 1 boxes, 128-byte swizzle; rows or
// columns beyond the extents read as zero.
void makePlaneMap(CUtensorMap* map, void* base, long cols, long rows, long depth) {
  const cuuint64_t dims[3] = {cuuint64_t(cols), cuuint64_t(rows), cuuint64_t(depth)};
  const cuuint64_t strides[2] = {cuuint64_t(cols) * 2, cuuint64_t(cols) * rows * 2};
  const cuuint32_t box[3] = {kBK, kBM, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encodeTiledFn()(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, base, dims, strides, box, estr,
                                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    throw Error(DCAACC_CUDA_ERR, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
}

unsigned gridX(long work) {
  return static_cast<unsigned>(std::max(1L, std::min(4096L, (work + 255) / 256)));
}

}  // namespace

FrontTcShape frontTcShape(const TpDims& d, int n_sectors, int max_order) {
  FrontTcShape s;
  s.D = d.R * d.nw_ext;
  s.Dp = (s.D + kBM - 1) / kBM * kBM;
  s.Dq = (s.D + 63) / 64 * 64;
  s.Kr = (std::max(max_order, 1) + kBK - 1) / kBK * kBK;
  s.n_sectors = n_sectors;
  s.pr_elems = size_t(n_sectors) * kPl * 2 * s.Dp * s.Kr;
  s.mb_elems = size_t(n_sectors) * kPl * s.Kr * s.Kr;
  s.ac_elems = size_t(n_sectors) * kPl * s.Dp * 2 * s.Kr;
  s.bq_elems = size_t(n_sectors) * kPl * 2 * s.Dq * 2 * s.Kr;
  return s;
}

size_t frontTcBytes(const FrontTcShape& s) {
  return (s.pr_elems + s.mb_elems + s.ac_elems + s.bq_elems) * sizeof(__nv_bfloat16);
}

void frontTcInit(FrontTcWorkspace& w, const FrontTcShape& s, void* mem) {
  w.shape = s;
  __nv_bfloat16* b = static_cast<__nv_bfloat16*>(mem);
  w.pr = b;
  w.mb = b + s.pr_elems;
  w.ac = b + s.pr_elems + s.mb_elems;
  w.bq = b + s.pr_elems + s.mb_elems + s.ac_elems;
  const long depth = long(s.n_sectors) * kPl;
  makePlaneMap(&w.tm_pr, w.pr, s.Kr, 2L * s.Dp, depth);
  makePlaneMap(&w.tm_mb, w.mb, s.Kr, s.Kr, depth);
  makePlaneMap(&w.tm_ac, w.ac, 2L * s.Kr, s.Dp, depth);
  makePlaneMap(&w.tm_bq, w.bq, 2L * s.Kr, 2L * s.Dq, depth);
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
  buildRowOperandKernel<<<dim3(gridX(groups * s.D), a.n_sectors), 256, 0, stream>>>(
      d, a.sectors, a.Tr, orb_r, a.Fb, a.G0, s.D, s.Dp, s.Kr, static_cast<__nv_bfloat16*>(w.pr));
  DCAACC_LAUNCH_CHECK();
  const long mrows = std::min<long>((a.n_max + kBN - 1) / kBN * kBN, s.Kr);
  buildMOperandKernel<<<dim3(gridX(groups * mrows), a.n_sectors), 256, 0, stream>>>(a.sectors, a.perm_r,
                                                                                    a.perm_c, s.Kr, static_cast<__nv_bfloat16*>(w.mb));
  DCAACC_LAUNCH_CHECK();
  buildColOperandKernel<<<dim3(gridX(groups * s.D), a.n_sectors), 256, 0, stream>>>(
      d, a.sectors, a.Tc, orb_c, a.Fb, a.G0, s.D, s.Dq, s.Kr, static_cast<__nv_bfloat16*>(w.bq));
  DCAACC_LAUNCH_CHECK();
  return launches + 3;
}

void launchFrontendTcRow(const FrontendArgs& a, const FrontTcWorkspace& w, int* err, cudaStream_t stream) {
  const FrontTcShape& s = w.shape;
  if (a.n_max == 0)
    return;
  GemmParams p{};
  p.dims = a.dims;
  p.sectors = a.sectors;
  p.D = s.D;
  p.Dp = s.Dp;
  p.Kr = s.Kr;
  p.ac = static_cast<__nv_bfloat16*>(w.ac);
  p.G0 = a.G0;
  p.err = err;
  auto k = frontGemmKernel<0>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGemmSmem)));
  const dim3 grid(2 * s.Dp / kBM, (a.n_max + kBN - 1) / kBN, a.n_sectors);
  k<<<grid, kGemmThreads, kGemmSmem, stream>>>(w.tm_pr, w.tm_mb, p);
  DCAACC_LAUNCH_CHECK();
}

void launchFrontendTcCol(const FrontendArgs& a, const FrontTcWorkspace& w, float2* G, long g_sector_stride,
                         int* err, cudaStream_t stream) {
  const FrontTcShape& s = w.shape;
  GemmParams p{};
  p.dims = a.dims;
  p.sectors = a.sectors;
  p.D = s.D;
  p.Dp = s.Dp;
  p.Kr = s.Kr;
  p.G = G;
  p.g_sector_stride = g_sector_stride;
  p.G0 = a.G0;
  p.err = err;
  auto k = frontGemmKernel<1>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGemmSmem)));
  const dim3 grid(s.Dp / kBM, s.Dq / 64, a.n_sectors);
  k<<<grid, kGemmThreads, kGemmSmem, stream>>>(w.tm_ac, w.tm_bq, p);
  DCAACC_LAUNCH_CHECK();
}

}  // namespace dcaacc
