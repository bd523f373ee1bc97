// Disconnected (spin-difference / spin-sum) term of the batched PH-magnetic / PH-charge G4 update,
// as a tensor-core GEMM.
//
// For one band, PH-magnetic and PH-charge contain (tp_accumulator_cpu.hpp:491-575)
//   sum_m s_m/2 u_m(k1, w1; q) v_m(k2, w2; q),   u = G_0(k1 w1; k1+q w1+x) -+ G_1(...),
//                                                v = G_0(k2+q w2+x; k2 w2) -+ G_1(...),
// (- for magnetic, + for charge), i.e. for each (q, x, channel) the product U V^T of two
// (Nc Nw x B) complex matrices over the batch index m.  This file
//   * builds U (with s_m/2 folded in) and V from the diagonal G blocks of the batch and stores them
//     as three BF16 planes each (x = hi + mid + lo, |x - hi - mid - lo| <= 2^-24 |x|), K-major,
//     with the complex product written as a real one:
//       [Ur | Ui] (M x 2B)  times  rows [Vr | -Vi] (real part) and [Vi | Vr] (imaginary part);
//   * multiplies them with tcgen05.mma (BF16 x BF16 -> FP32 in tensor memory), keeping the six
//     plane products whose order is above 2^-24 (hh, hm, mh, hl, mm, lh).  The tensor core's FP32
//     accumulation does not round to nearest, so its error grows with the number of MMAs feeding
//     one accumulator and is biased where a sum is coherent (the charge channel's q = 0 entries
//     sum |G|^2-like terms over the whole batch).  So the MMAs are spread over four tensor-memory
//     accumulators (all 512 columns); each accumulator takes the small plane products first and
//     the hh products last, so only two MMAs per accumulator add to a large running sum; and every
//     K chunk (64 measurements) is read out and added to the result in round-to-nearest FP32;
//   * writes the FP32 result per problem as an M x M matrix, row index m = k1 + Nc w1 fastest,
//     which the direct-term kernel (tp_g4_batched.cu) adds to G4 at its flush.
// Rows are padded to a multiple of 128 and the batch to a multiple of 64 with zeros.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "async_copy.cuh"
#include "common.cuh"
#include "tcgen05.cuh"
#include "tp_g4.hpp"

namespace dcaacc {

namespace {

constexpr int kTileM = 128;   // rows (k1, w1) per CTA
constexpr int kTileNc = 64;   // complex columns (k2, w2) per CTA -> 128 real accumulator columns
constexpr int kPlanes = 3;
constexpr int kChunkK = 128;  // K columns staged per step (two 64-wide swizzle sub-tiles)
constexpr int kSub = kChunkK / 64;
constexpr uint32_t kSubBytes = kTileM * 128;  // one 64-wide sub-tile: 128 rows x 128 bytes
constexpr size_t kGemmSmem = 1024 + 2 * kPlanes * kSub * kSubBytes + 64;
constexpr int kAccs = 4;               // tensor-memory accumulators, 128 columns each
constexpr uint32_t kTmemCols = 128 * kAccs;

struct Split3 {
  __nv_bfloat16 h, m, l;
};
__device__ inline Split3 split3(float x) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(h);
  const __nv_bfloat16 m = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(m);
  return {h, m, __float2bfloat16_rn(r2)};
}

struct DiscShape {
  int M;      // Nc * Nw
  int P;      // M rounded up to kTileM
  int Bp;     // batch rounded up to 64
  long kp;    // 2 Bp
  long plane_a, plane_b;
  int probs;  // nq * nwq * n_channels
};

DiscShape discShape(const TpDims& d, int batch) {
  DiscShape s;
  s.M = d.nc * d.nw;
  s.P = (s.M + kTileM - 1) / kTileM * kTileM;
  s.Bp = (std::max(batch, 1) + 63) / 64 * 64;
  s.kp = 2L * s.Bp;
  s.plane_a = long(s.P) * s.kp;
  s.plane_b = 2L * s.P * s.kp;
  s.probs = d.nq * d.nwq * d.n_channels;
  return s;
}

// Eight BF16 values packed for one 16-byte store.
struct Pack8 {
  __nv_bfloat16 v[8];
};
__device__ inline void store8(__nv_bfloat16* dst, const Pack8& p) {
  *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(&p);
}

// One thread per (row, group of 8 measurements) of one problem (blockIdx.y = iwq * nq + iq,
// blockIdx.z = channel); the 8 groups of a row are adjacent threads, so each plane row is written
// with contiguous 16-byte stores.  A planes: [prob][plane][P rows][kp], B planes:
// [prob][plane][2P rows][kp], kp = 2 Bp.
__global__ void __launch_bounds__(256)
discPlanesKernel(const TpDims dims, const float2* __restrict__ G, long g_sector_stride,
                 const int* __restrict__ signs, int n_slots, int Bp, int P, const int* __restrict__ k_add,
                 const int* __restrict__ q_list, const int* __restrict__ wex_list,
                 __nv_bfloat16* __restrict__ Ap, __nv_bfloat16* __restrict__ Bpl) {
  const int nc = dims.nc, nw_ext = dims.nw_ext, ext = dims.ext, R = dims.R;
  const int M = nc * dims.nw;
  const int p = blockIdx.y;
  const int ch = blockIdx.z;
  const float sg = dims.channels[ch] == 2 ? -1.f : 1.f;  // magnetic: difference, charge: sum
  const int iq = p % dims.nq, iwq = p / dims.nq;
  const int q = q_list[iq], wex = wex_list[iwq];
  const long kp = 2L * Bp;
  const long plane_a = static_cast<long>(P) * kp;
  const long plane_b = 2L * P * kp;
  const long prob = static_cast<long>(p) * gridDim.z + ch;
  __nv_bfloat16* A = Ap + prob * kPlanes * plane_a;
  __nv_bfloat16* Bm = Bpl + prob * kPlanes * plane_b;
  const int groups = Bp / 8;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < long(groups) * P;
       idx += long(gridDim.x) * blockDim.x) {
    const int grp = static_cast<int>(idx % groups);
    const int row = static_cast<int>(idx / groups);
    const int slot0 = grp * 8;
    long bc = 0, be = 0;
    const bool in_row = row < M;
    if (in_row) {
      const int k = row % nc, w = row / nc;
      const int kq = k_add[k + nc * q];
      const int we = w + ext, wx = we + wex;
      bc = (static_cast<long>(we) * nw_ext + wx) * R * R + static_cast<long>(k) * R + kq;
      be = (static_cast<long>(wx) * nw_ext + we) * R * R + static_cast<long>(kq) * R + k;
    }
    Pack8 ur[kPlanes], ui[kPlanes], vr[kPlanes], vi[kPlanes], mvi[kPlanes];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int slot = slot0 + e;
      float2 u = make_float2(0.f, 0.f), v = make_float2(0.f, 0.f);
      if (in_row && slot < n_slots) {
        const float hs = 0.5f * static_cast<float>(signs[slot]);
        const float2* G0s = G + g_sector_stride * (2 * slot);
        const float2* G1s = G0s + g_sector_stride;
        const float2 c0 = G0s[bc], c1 = G1s[bc], e0 = G0s[be], e1 = G1s[be];
        u = make_float2(hs * (c0.x + sg * c1.x), hs * (c0.y + sg * c1.y));
        v = make_float2(e0.x + sg * e1.x, e0.y + sg * e1.y);
      }
      const Split3 a = split3(u.x), b = split3(u.y), c = split3(v.x), d = split3(v.y), f = split3(-v.y);
      ur[0].v[e] = a.h, ur[1].v[e] = a.m, ur[2].v[e] = a.l;
      ui[0].v[e] = b.h, ui[1].v[e] = b.m, ui[2].v[e] = b.l;
      vr[0].v[e] = c.h, vr[1].v[e] = c.m, vr[2].v[e] = c.l;
      vi[0].v[e] = d.h, vi[1].v[e] = d.m, vi[2].v[e] = d.l;
      mvi[0].v[e] = f.h, mvi[1].v[e] = f.m, mvi[2].v[e] = f.l;
    }
    // A: row m = k + nc w, columns slot (real) and Bp + slot (imaginary).
    // B: complex column n = row in block cb = n / 64; real-part row cb*128 + c holds
    // [Vr | -Vi], imaginary-part row cb*128 + 64 + c holds [Vi | Vr].
    const int cb = row / kTileNc, cc = row % kTileNc;
    const long rre = static_cast<long>(cb) * 2 * kTileNc + cc, rim = rre + kTileNc;
    const long a0 = static_cast<long>(row) * kp + slot0, a1 = a0 + Bp;
    const long bre0 = rre * kp + slot0, bre1 = bre0 + Bp, bim0 = rim * kp + slot0, bim1 = bim0 + Bp;
#pragma unroll
    for (int pl = 0; pl < kPlanes; ++pl) {
      store8(A + pl * plane_a + a0, ur[pl]);
      store8(A + pl * plane_a + a1, ui[pl]);
      store8(Bm + pl * plane_b + bre0, vr[pl]);
      store8(Bm + pl * plane_b + bre1, mvi[pl]);
      store8(Bm + pl * plane_b + bim0, vi[pl]);
      store8(Bm + pl * plane_b + bim1, vr[pl]);
    }
  }
}

// CTA = 128 rows x 64 complex columns of one problem; 128 threads, one CTA per SM (shared memory),
// which owns all 512 tensor-memory columns.  K is processed in chunks of 128 columns: the three
// planes of both operands are staged in shared memory (128-byte swizzle, K-major), one thread
// issues the 6 plane products x 8 MMAs (M = 128, N = 128, K = 16), K16 steps 2g and 2g + 1 into
// accumulator g, and commits them to an mbarrier, which every thread waits on (bounded); the
// epilogue then adds the four accumulators and stores (first chunk) or adds (later chunks) the
// chunk's result to `out`, before the next chunk overwrites the stage and the accumulators.
__global__ void __launch_bounds__(128, 1)
discGemmKernel(const __nv_bfloat16* __restrict__ Ap, const __nv_bfloat16* __restrict__ Bpl, int M, int P,
               int kp, float2* __restrict__ out, int* __restrict__ err) {
  const int m0 = blockIdx.x * kTileM;
  const int nb = blockIdx.y;  // complex column block
  const long prob = blockIdx.z;
  const long plane_a = static_cast<long>(P) * kp;
  const long plane_b = 2L * P * kp;
  const __nv_bfloat16* A = Ap + prob * kPlanes * plane_a;
  const __nv_bfloat16* B = Bpl + prob * kPlanes * plane_b;

  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1 KB alignment for the swizzle atoms.
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sA = base;                              // [plane][sub][kSubBytes]
  unsigned char* sB = base + kPlanes * kSub * kSubBytes;  // [plane][sub][kSubBytes]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sB + kPlanes * kSub * kSubBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);

  const int t = threadIdx.x, warp = t / 32;
  if (warp == 0) {
    tc::tmemAlloc(tmem_slot, kTmemCols);
    tc::tmemRelinquish();
  }
  if (t == 0) {
    mbarInit(bar, 1);
    fenceBarrierInit();
  }
  tc::fenceBeforeThreadSync();
  __syncthreads();
  tc::fenceAfterThreadSync();
  const uint32_t tmem = *tmem_slot;

  constexpr int chunks_per_row = kChunkK / 8;  // 16-byte pieces per staged row
  const int n_chunks = kp / kChunkK;
  const int row = m0 + warp * 32 + (t % 32);  // epilogue: warp w owns accumulator lanes 32w .. 32w + 31
  const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
  for (int kc = 0; kc < n_chunks; ++kc) {
    for (int idx = t; idx < kPlanes * kTileM * chunks_per_row; idx += blockDim.x) {
      const int pl = idx / (kTileM * chunks_per_row);
      const int rem = idx % (kTileM * chunks_per_row);
      const int r = rem / chunks_per_row, c = rem % chunks_per_row;
      const int ks = c / 8, kcol = c % 8;
      const long col = static_cast<long>(kc) * kChunkK + c * 8;
      tc::cpAsync16(sA + (pl * kSub + ks) * kSubBytes + tc::sw128Offset(r, kcol * 8),
                    A + pl * plane_a + static_cast<long>(m0 + r) * kp + col);
      tc::cpAsync16(sB + (pl * kSub + ks) * kSubBytes + tc::sw128Offset(r, kcol * 8),
                    B + pl * plane_b + static_cast<long>(nb * 2 * kTileNc + r) * kp + col);
    }
    tc::cpAsyncWaitAll();
    fenceProxyAsync();  // the staged tiles become visible to the tensor core's (async-proxy) reads
    tc::fenceBeforeThreadSync();
    __syncthreads();    // also: the previous chunk's accumulator reads are done
    tc::fenceAfterThreadSync();
    if (t == 0) {
      constexpr uint32_t idesc = tc::instrDescBf16F32(kTileM, 2 * kTileNc);
      // (A plane, B plane) pairs kept by the three-way split, smallest first: lh, mm, hl, mh, hm, hh.
      const int pa[6] = {2, 1, 0, 1, 0, 0};
      const int pb[6] = {0, 1, 2, 0, 1, 0};
      for (int pp = 0; pp < 6; ++pp)
        for (int ks = 0; ks < kSub; ++ks) {
          const uint64_t da = tc::smemDescSw128(sA + (pa[pp] * kSub + ks) * kSubBytes);
          const uint64_t db = tc::smemDescSw128(sB + (pb[pp] * kSub + ks) * kSubBytes);
          for (int kk = 0; kk < 4; ++kk) {  // 4 x K16 per 64-wide sub-tile
            const int step = ks * 4 + kk;   // K16 step in the chunk, 0..7
            const uint32_t acc_col = static_cast<uint32_t>(step >> 1) * 128;
            tc::mmaBf16(tmem + acc_col, tc::descAdvance(da, kk * 32), tc::descAdvance(db, kk * 32), idesc,
                        (pp | (step & 1)) != 0);
          }
        }
      tc::commitTo(bar);
    }
    const bool done = mbarWait(bar, kc & 1, err);
    tc::fenceAfterThreadSync();
    if (!__syncthreads_and(done))
      break;
    float re[16], im[16], pr[16], pi[16];
    for (int c0 = 0; c0 < kTileNc; c0 += 16) {
      tc::ld32x32bx16(tmem + lane_base + c0, re);
      tc::ld32x32bx16(tmem + lane_base + kTileNc + c0, im);
      tc::waitLd();
#pragma unroll
      for (int g = 1; g < kAccs; ++g) {
        tc::ld32x32bx16(tmem + lane_base + g * 128 + c0, pr);
        tc::ld32x32bx16(tmem + lane_base + g * 128 + kTileNc + c0, pi);
        tc::waitLd();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          re[i] += pr[i];
          im[i] += pi[i];
        }
      }
      const int n0 = nb * kTileNc + c0;
      if (row < M) {
        float2* o = out + (prob * M + n0) * M + row;
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (n0 + i < M) {
            float2 v = make_float2(re[i], im[i]);
            if (kc > 0) {
              const float2 prev = o[static_cast<long>(i) * M];
              v.x += prev.x;
              v.y += prev.y;
            }
            o[static_cast<long>(i) * M] = v;
          }
      }
    }
    tc::fenceBeforeThreadSync();
  }
  tc::fenceBeforeThreadSync();
  __syncthreads();
  if (warp == 0)
    tc::tmemDealloc(tmem, kTmemCols);
}

}  // namespace

size_t discScratchBytes(const TpDims& d, int max_batch) {
  const DiscShape s = discShape(d, max_batch);
  return size_t(s.probs) * kPlanes * (s.plane_a + s.plane_b) * sizeof(__nv_bfloat16) +
         size_t(s.probs) * s.M * s.M * sizeof(float2);
}

const float2* launchDiscGemm(const G4Args& a, const float2* G, long g_sector_stride, cudaStream_t stream) {
  const TpDims& d = a.dims;
  const DiscShape s = discShape(d, a.n_slots);
  if (!a.disc_scratch || discScratchBytes(d, a.n_slots) > a.disc_scratch_bytes)
    return nullptr;
  __nv_bfloat16* Ap = static_cast<__nv_bfloat16*>(a.disc_scratch);
  __nv_bfloat16* Bpl = Ap + size_t(s.probs) * kPlanes * s.plane_a;
  float2* out = reinterpret_cast<float2*>(Bpl + size_t(s.probs) * kPlanes * s.plane_b);
  {
    const long work = long(s.Bp / 8) * s.P;
    const dim3 grid(static_cast<unsigned>(std::max(1L, std::min(1024L, (work + 255) / 256))), d.nq * d.nwq,
                    d.n_channels);
    discPlanesKernel<<<grid, 256, 0, stream>>>(d, G, g_sector_stride, a.signs, a.n_slots, s.Bp, s.P, a.k_add,
                                               a.q_list, a.wex_list, Ap, Bpl);
    DCAACC_LAUNCH_CHECK();
  }
  {
    DCAACC_CUDA_CHECK(
        cudaFuncSetAttribute(discGemmKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem));
    const dim3 grid(s.P / kTileM, (s.M + kTileNc - 1) / kTileNc, s.probs);
    discGemmKernel<<<grid, 128, kGemmSmem, stream>>>(Ap, Bpl, s.M, s.P, static_cast<int>(s.kp), out, a.err);
    DCAACC_LAUNCH_CHECK();
  }
  return out;
}

}  // namespace dcaacc
