// Direct term of the batched single-band G4 update on the tensor cores (Nc = 16, all momentum
// transfers, PH-magnetic / PH-charge), the mixed path's replacement of updateG4SinglebandOuter.
//
// Grouped by d = k1 - k2 (tp_g4_batched.cu), the direct term of a frequency tile (w1, w2) is, for
// each d, a 16 x 16 complex product whose contraction index K runs over the batch:
//   D_d(k1, l1) = sum_m (-s_m / 2) sum_s alpha_sd(k1) beta_sd(l1),
//   alpha_sd(k1) = G_s(k1 w1; k1 - d w2),   beta_sd(l1) = G_s(l1 - d w2 + x; l1 w1 + x),
// (G4 entry k2 = k1 - d, q = l1 - k1; the reference sums the same products entry by entry,
// tp_accumulator_gpu kernels updateG4 / g4_helper).  At 16 x 16 per d this is exactly the shape of
// the warp-level m16n8k16 MMA: a tcgen05 MMA is at least 64 rows high and takes one B operand, so
// it would spend three quarters or more of its work on the block-diagonal zeros that separate
// different d.  So warp w of a CTA owns d = w and computes D_d as two 16 x 8 tiles, K = 16 = eight
// measurements x two spins per MMA step, in split FP16: x = 2^e (hi + lo) with the three products
// lo*hi, hi*lo, hi*hi (smallest first) per real product and the complex product as
//   Re = ar br + (-ai) bi,   Im = ar bi + ai br
// (12 MMAs per 16 x 8 tile and step).  Each step's chain starts from zero and is promoted into FP32
// registers with the exact factor 2^-2e, like the front-end GEMM's per-chunk promotion.  The step
// exponent e comes from the largest |G| of the step's sixteen sectors, which the column step
// records per sector (gmax).
//
// Layout choices that make every fragment gather conflict-free: MMA row i of warp d is k2 = i, k1 =
// i + d (so the alpha of row i sits in column i of its G block: row i of the fragment reads bank
// column i), MMA column n is l1 = n (beta_d(l1) sits in column l1), and the eight measurement slots
// of a stage are 8 KB + 32 bytes apart, so the four lanes of a fragment row (four measurements)
// land on four different 32-byte bank groups.  The 16 consumer warps are fed by one producer warp
// (bulk copies of the four 2 KB G blocks of each measurement into a three-deep stage ring, full /
// empty mbarriers); the CTA is persistent over the tiles, so the producer runs ahead across tile
// boundaries while the consumers flush.  The step exponents depend on the batch only and are
// computed once, before the tile loop.  The flush goes through a shared table [q][k2][k1 ^ q]
// (conflict-free both ways) so that consecutive threads touch consecutive k1 of G4 and of the
// disconnected terms, as in the SIMT kernel.
//
// Half G (dims.half_g): a block whose row frequency lies in the lower half is not stored; the
// producer copies its mirror (w' = NwExt - 1 - w on both frequencies) and the consumers read
// element (k1, k2) as the conjugate of the mirror's (-k1, -k2).  So that the gathers stay
// conflict-free, a mirrored A block takes MMA row i as k2 = -i and a mirrored B block takes MMA
// column n as l1 = -n (the mirror's element then sits in column i / n again).
//
// Every mbarrier wait is bounded (async_copy.cuh); after a timeout a warp stops waiting and
// computing but still takes part in the two named barriers per tile, so no thread can be left
// waiting, and the host reports the error word.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "async_copy.cuh"
#include "common.cuh"
#include "tp_g4.hpp"

namespace dcaacc {
namespace {

constexpr int kNc = 16;
constexpr int kBlk = kNc * kNc;                        // one G block: 16 x 16 complex
constexpr int kMeasPerStep = 8;                        // K = 16 = 8 measurements x 2 spins
constexpr uint32_t kBlkBytes = kBlk * sizeof(float2);  // 2 KB
constexpr uint32_t kSlotBytes = 4 * kBlkBytes + 32;    // A0 B0 A1 B1 + 32-byte bank skew
constexpr uint32_t kStageBytes = kMeasPerStep * kSlotBytes;
constexpr int kStages = 3;
constexpr int kConsumerWarps = kNc;  // warp w owns d = w
constexpr int kConsumers = 32 * kConsumerWarps;
constexpr int kThreads = kConsumers + 32;  // + the producer warp
constexpr uint32_t kTableBytes = kBlk * kNc * sizeof(float2);
constexpr uint32_t kOffTable = kStages * kStageBytes;
constexpr uint32_t kOffBars = kOffTable + kTableBytes;
constexpr int kMaxSteps = 32;  // batches of up to 256 measurements
constexpr uint32_t kOffExp = kOffBars + 2 * kStages * 8;
constexpr uint32_t kOffKplus = kOffExp + 4 * kMaxSteps;
constexpr uint32_t kOffKsub = kOffKplus + kBlk;
constexpr uint32_t kOffQinv = kOffKsub + kBlk;
constexpr uint32_t kOffKneg = kOffQinv + 16;
constexpr uint32_t kOffSigns = kOffKneg + 16;
constexpr size_t kSmem = kOffSigns + kMaxSteps * kMeasPerStep;
constexpr int kExpMax = 60;  // |e| <= 60 keeps 2^{+-2e} a normal FP32 number
constexpr int kMaxCh = 2;    // PH-magnetic and PH-charge
static_assert(kSlotBytes % 16 == 0 && kOffTable % 16 == 0 && kOffBars % 8 == 0, "alignment");
static_assert(kSmem <= 227 * 1024, "shared memory per CTA");

__device__ inline uint32_t asU32(__half2 h) {
  return *reinterpret_cast<uint32_t*>(&h);
}

// (x0, x1) = hi + lo with both halves rounded to nearest (x0 in the low 16 bits, the first K
// element of an MMA fragment register).
__device__ inline void splitPair(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const __half2 h = __floats2half2_rn(x0, x1);
  const float2 hf = __half22float2(h);
  hi = asU32(h);
  lo = asU32(__floats2half2_rn(x0 - hf.x, x1 - hf.y));
}

// c += A B for one m16n8k16 tile (A row-major 16 x 16 FP16, B column-major 16 x 8, FP32 c).
__device__ inline void mma16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Fragments of one step from the staged G blocks S: A (alphas, rows k2 = g, g + 8; register 2j + r
// holds row g + 8r and K = (measurement t4 + 4j, spin 0 / 1)) pre-scaled by -s_m/2 2^e, and B
// (betas; N tile n, register j: column g + 8n, K = (measurement t4 + 4j, spin)) scaled by 2^e, each
// split into FP16 hi / lo.  FULL: all eight measurements of the step exist (no predicates).
template <bool FULL>
__device__ __forceinline__ void buildFragments(const float2* S, const int (&oa)[2], const int (&ob)[2], int t4,
                                               int m0, int n_slots, const signed char* sgn, float sc, float ca,
                                               float cb,
                                               uint32_t (&arh)[4], uint32_t (&arl)[4], uint32_t (&aih)[4],
                                               uint32_t (&ail)[4], uint32_t (&brh)[2][2], uint32_t (&brl)[2][2],
                                               uint32_t (&bih)[2][2], uint32_t (&bil)[2][2]) {
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int mi = t4 + 4 * j;
    const bool valid = FULL || m0 + mi < n_slots;
    const float fa = valid ? -0.5f * static_cast<float>(sgn[m0 + mi]) * sc : 0.f;
    const float fb = valid ? sc : 0.f;
    const float fai = fa * ca, fbi = fb * cb;  // imaginary parts (conjugated mirrors: negated)
    const float2* slot = S + mi * (kSlotBytes / sizeof(float2));
    const float2 z = make_float2(0.f, 0.f);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const float2 a0 = valid ? slot[oa[r]] : z;
      const float2 a1 = valid ? slot[2 * kBlk + oa[r]] : z;
      splitPair(a0.x * fa, a1.x * fa, arh[2 * j + r], arl[2 * j + r]);
      splitPair(a0.y * fai, a1.y * fai, aih[2 * j + r], ail[2 * j + r]);
      const float2 b0 = valid ? slot[kBlk + ob[r]] : z;
      const float2 b1 = valid ? slot[3 * kBlk + ob[r]] : z;
      splitPair(b0.x * fb, b1.x * fb, brh[r][j], brl[r][j]);
      splitPair(b0.y * fbi, b1.y * fbi, bih[r][j], bil[r][j]);
    }
  }
}

__device__ inline void namedSync() {
  asm volatile("bar.sync 1, %0;" ::"n"(kConsumers) : "memory");
}

// Exponent e (|e| <= kExpMax) with mx 2^e in [2^14, 2^15).
__device__ inline int stepExp(float mx) {
  return mx > 0.f ? max(-kExpMax, min(kExpMax, 14 - ilogbf(mx))) : 0;
}
__device__ inline float pow2(int e) {
  return __int_as_float((127 + e) << 23);  // |e| <= 126
}

// Tile index -> (w1, w2): the Nw diagonal tiles first, then the pairs (a, b), (b, a) next to each
// other, so that the second read of each G block of a pair comes from L2.
__device__ inline void tilePair(int idx, int nw, int& w1, int& w2) {
  if (idx < nw) {
    w1 = w2 = idx;
    return;
  }
  const int j = idx - nw;
  const int p = j >> 1;
  int b = static_cast<int>((1.0 + sqrt(1.0 + 8.0 * p)) * 0.5);
  while (b * (b - 1) / 2 > p)
    --b;
  while ((b + 1) * b / 2 <= p)
    ++b;
  const int a = p - b * (b - 1) / 2;
  w1 = (j & 1) ? b : a;
  w2 = (j & 1) ? a : b;
}

__global__ void __launch_bounds__(kThreads, 1)
updateG4DirectMma(const TpDims dims, const float2* __restrict__ G, long g_sector_stride,
                  const int* __restrict__ signs, int n_slots, const int* __restrict__ k_sub,
                  const int* __restrict__ q_list, const int* __restrict__ wex_list,
                  const int* __restrict__ gmax, const unsigned* __restrict__ tile_order,
                  const float2* __restrict__ disc, double2* const* __restrict__ G4, bool atomic,
                  int* __restrict__ err, uint32_t wait_limit, int fault_stop_step) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* table = reinterpret_cast<float2*>(smem + kOffTable);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kOffBars);
  uint64_t* empty = full + kStages;
  int* step_exp = reinterpret_cast<int*>(smem + kOffExp);  // [step] exponent of the step's operands
  unsigned char* kplus = smem + kOffKplus;  // [d][i] -> k1 with k1 - d = i
  unsigned char* ksub = smem + kOffKsub;    // [a + 16 b] = b - a
  unsigned char* qinv = smem + kOffQinv;    // q -> its position in q_list
  unsigned char* kneg = smem + kOffKneg;    // k -> -k (half G)
  signed char* sgn = reinterpret_cast<signed char*>(smem + kOffSigns);  // [m] measurement signs

  const int t = threadIdx.x, warp = t / 32, lane = t % 32;
  const int nw = dims.nw, nw_ext = dims.nw_ext, nq = dims.nq;
  const int per_wq = dims.half_g4 ? nw * nw / 2 : nw * nw;  // half G4: the tiles with w1 >= Nw / 2
  const int n_tiles = per_wq * dims.nwq;
  auto tileOf = [&](int tile, int& w1, int& w2) {
    if (dims.half_g4) {
      const unsigned v = tile_order[tile % per_wq];
      w1 = static_cast<int>(v & 0xffffu);
      w2 = static_cast<int>(v >> 16);
    }
    else {
      tilePair(tile % per_wq, nw, w1, w2);
    }
  };
  const int n_steps = (n_slots + kMeasPerStep - 1) / kMeasPerStep;

  for (int e = t; e < kBlk; e += kThreads) {
    const int a = e % kNc, b = e / kNc;  // k_sub[a + 16 b] = b - a
    const int s = k_sub[e];
    ksub[e] = static_cast<unsigned char>(s);
    kplus[a * kNc + s] = static_cast<unsigned char>(b);  // d = a, k1 = b, i = b - d
  }
  for (int e = t; e < kNc; e += kThreads) {
    qinv[q_list[e]] = static_cast<unsigned char>(e);
    kneg[e] = dims.half_g ? dims.kneg[e] : static_cast<unsigned char>(e);
  }
  for (int m = t; m < n_slots; m += kThreads)
    sgn[m] = static_cast<signed char>(signs[m]);
  for (int step = warp; step < n_steps; step += kThreads / 32) {
    const int m0 = step * kMeasPerStep;
    float mx = lane < 2 * min(kMeasPerStep, n_slots - m0) ? __int_as_float(gmax[2 * m0 + lane]) : 0.f;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if (lane == 0)
      step_exp[step] = stepExp(mx);
  }
  if (t == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbarInit(&full[s], 1);
      mbarInit(&empty[s], kConsumerWarps);
    }
    fenceBarrierInit();
  }
  __syncthreads();

  if (warp == kConsumerWarps) {
    // ---- producer warp: per step, the four G blocks of eight measurements and the step exponent
    int gs = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
      int w1, w2;
      tileOf(tile, w1, w2);
      const int wex = wex_list[tile / per_wq];
      const int w1e = w1 + dims.ext, w2e = w2 + dims.ext, w1x = w1e + wex, w2x = w2e + wex;
      // A = block (w1e, w2e), B = block (w2x, w1x), or their mirrors (half G).
      const bool mir_a = dims.half_g && 2 * w1e < nw_ext, mir_b = dims.half_g && 2 * w2x < nw_ext;
      const long b_A = mir_a ? (static_cast<long>(nw_ext - 1 - w1e) * nw_ext + nw_ext - 1 - w2e) * kBlk
                             : (static_cast<long>(w1e) * nw_ext + w2e) * kBlk;
      const long b_B = mir_b ? (static_cast<long>(nw_ext - 1 - w2x) * nw_ext + nw_ext - 1 - w1x) * kBlk
                             : (static_cast<long>(w2x) * nw_ext + w1x) * kBlk;
      for (int step = 0; step < n_steps; ++step, ++gs) {
        const int st = gs % kStages, use = gs / kStages;
        // Injected failure (tests of the error path): CTA 0's producer stops before step gs, as if
        // its copies never came, so the consumers' bounded wait for that stage runs out.
        if (blockIdx.x == 0 && gs == fault_stop_step) {
          ok = false;
          break;
        }
        if (use > 0 && !__all_sync(0xffffffffu, mbarWait(&empty[st], (use - 1) & 1, err, wait_limit))) {
          ok = false;
          break;
        }
        const int m0 = step * kMeasPerStep;
        const int nvalid = min(kMeasPerStep, n_slots - m0);
        if (lane == 0)
          mbarArriveExpectTx(&full[st], static_cast<uint32_t>(nvalid) * 4 * kBlkBytes);
        __syncwarp();
        if (lane < 4 * nvalid) {
          const int mi = lane / 4, part = lane % 4;  // part: A spin 0, B spin 0, A spin 1, B spin 1
          const float2* src = G + g_sector_stride * (2 * (m0 + mi) + (part >> 1)) + ((part & 1) ? b_B : b_A);
          unsigned char* dst = smem + st * kStageBytes + mi * kSlotBytes + part * kBlkBytes;
          bulkCopyG2S(dst, src, kBlkBytes, &full[st]);
        }
      }
    }
    // Copies still in flight land before the CTA exits (on the normal path all were consumed).
    if (lane == 0)
      for (int c = max(0, gs - kStages); c < gs; ++c)
        mbarWait(&full[c % kStages], (c / kStages) & 1, err);
    return;
  }

  // ---- consumer warps: warp d = warp
  const int d = warp;
  const int g = lane >> 2, t4 = lane & 3;
  const long M = static_cast<long>(kNc) * nw;
  const long s_w1 = kNc, s_k2 = s_w1 * nw, s_w2 = s_k2 * kNc, s_q = s_w2 * nw, s_wq = s_q * nq;
  const int n_ch = dims.n_channels;
  // Flush of a tile: entry x = t + kConsumers j (j < 8 n_ch) of [channel][q][k2][k1], so
  // consecutive threads take consecutive k1.  A thread keeps k1 = t % 16 and k2 = (t / 16) % 16; its
  // entry j has channel c = j / 8 and q position qi = t / 256 + 2 (j % 8).  The entries go two at a
  // time ("chunks"); the chunks of tile t are spread over the steps of the CTA's next tile: the loads
  // of chunk s are issued at step s and consumed (add, store) at step s + 1, so the G4
  // read-modify-write overlaps the MMAs.
  static_assert(kConsumers == 2 * kBlk, "entry layout of the flush");
  const int n_chunks = n_ch * kBlk * kNc / (2 * kConsumers);
  const int fk1 = t % kNc, fk2 = (t / kNc) % kNc, fq0 = t / kBlk;
  long g4_base = 0, di_base = 0;  // offsets of the tile being flushed, without the q / channel terms
  bool have_prev = false;
  int pend = -1;  // chunk whose loads are in flight
  double2 po[2];
  float2 pdv[2];
  const long MM = M * M;
  auto issue = [&](int chunk) {
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int j = 2 * chunk + u, c = j / 8, qi = fq0 + 2 * (j % 8);
      pdv[u] = __ldg(disc + di_base + (static_cast<long>(qi) * n_ch + c) * MM);
      po[u] = atomic ? make_double2(0., 0.) : G4[c][g4_base + qi * s_q];
    }
  };
  auto consume = [&](int chunk) {
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int j = 2 * chunk + u, c = j / 8, qi = fq0 + 2 * (j % 8);
      const float2 v = table[(qi * kNc + fk2) * kNc + (fk1 ^ qi)];
      double2* p = G4[c] + g4_base + qi * s_q;
      const double re = static_cast<double>(v.x + pdv[u].x), im = static_cast<double>(v.y + pdv[u].y);
      if (atomic) {
        atomicAdd(&p->x, re);
        atomicAdd(&p->y, im);
      }
      else {
        *p = make_double2(po[u].x + re, po[u].y + im);
      }
    }
  };

  int gs = 0;
  bool ok = true;
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    int w1, w2;
    tileOf(tile, w1, w2);
    const int iwq = tile / per_wq;
    const int w1e = w1 + dims.ext, w2x = w2 + dims.ext + wex_list[iwq];
    const bool mir_a = dims.half_g && 2 * w1e < nw_ext, mir_b = dims.half_g && 2 * w2x < nw_ext;
    // Fragment gathers (float2 offsets inside a staged block).  MMA row i: k2 = i (mirrored: -i),
    // k1 = k2 + d, element A[k1][k2] (mirrored: A'[-k1][i]); MMA column n (N tile r): l1 = n
    // (mirrored: -n), element B[l1 - d][l1] (mirrored: B'[-(l1 - d)][n]).
    int oa[2], ob[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int i = g + 8 * r;
      const int k2 = mir_a ? kneg[i] : i, k1 = kplus[d * kNc + k2];
      oa[r] = (mir_a ? kneg[k1] : k1) * kNc + i;
      const int l1 = mir_b ? kneg[i] : i, lr = ksub[d + kNc * l1];
      ob[r] = (mir_b ? kneg[lr] : lr) * kNc + i;
    }
    const float ca = mir_a ? -1.f : 1.f, cb = mir_b ? -1.f : 1.f;  // conjugation of the mirrors
    float acc_re[2][4], acc_im[2][4];
#pragma unroll
    for (int n = 0; n < 2; ++n)
#pragma unroll
      for (int k = 0; k < 4; ++k)
        acc_re[n][k] = acc_im[n][k] = 0.f;

    for (int step = 0; step < n_steps; ++step, ++gs) {
      const int st = gs % kStages;
      if (have_prev) {  // previous tile's flush: finish the chunk in flight, start the next one
        if (pend >= 0)
          consume(pend);
        pend = -1;
        if (step < n_chunks) {
          issue(step);
          pend = step;
        }
      }
      if (ok)
        ok = __all_sync(0xffffffffu, mbarWait(&full[st], (gs / kStages) & 1, err, wait_limit));
      if (ok) {
        const int e = step_exp[step];
        const float sc = pow2(e), inv = pow2(-2 * e);
        const int m0 = step * kMeasPerStep;
        const float2* S = reinterpret_cast<const float2*>(smem + st * kStageBytes);
        uint32_t arh[4], arl[4], aih[4], ail[4];
        uint32_t brh[2][2], brl[2][2], bih[2][2], bil[2][2];
        if (m0 + kMeasPerStep <= n_slots)
          buildFragments<true>(S, oa, ob, t4, m0, n_slots, sgn, sc, ca, cb, arh, arl, aih, ail, brh, brl, bih,
                               bil);
        else
          buildFragments<false>(S, oa, ob, t4, m0, n_slots, sgn, sc, ca, cb, arh, arl, aih, ail, brh, brl, bih,
                                bil);
        uint32_t naih[4], nail[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          naih[k] = aih[k] ^ 0x80008000u;
          nail[k] = ail[k] ^ 0x80008000u;
        }
        float tr[2][4], ti[2][4];
#pragma unroll
        for (int n = 0; n < 2; ++n)
#pragma unroll
          for (int k = 0; k < 4; ++k)
            tr[n][k] = ti[n][k] = 0.f;
        // Re = ar br - ai bi, Im = ar bi + ai br; small products first, the four chains interleaved.
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          mma16816(tr[n], arh, brl[n][0], brl[n][1]);
          mma16816(ti[n], arh, bil[n][0], bil[n][1]);
        }
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          mma16816(tr[n], arl, brh[n][0], brh[n][1]);
          mma16816(ti[n], arl, bih[n][0], bih[n][1]);
        }
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          mma16816(tr[n], naih, bil[n][0], bil[n][1]);
          mma16816(ti[n], aih, brl[n][0], brl[n][1]);
        }
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          mma16816(tr[n], nail, bih[n][0], bih[n][1]);
          mma16816(ti[n], ail, brh[n][0], brh[n][1]);
        }
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          mma16816(tr[n], arh, brh[n][0], brh[n][1]);
          mma16816(ti[n], arh, bih[n][0], bih[n][1]);
        }
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          mma16816(tr[n], naih, bih[n][0], bih[n][1]);
          mma16816(ti[n], aih, brh[n][0], brh[n][1]);
        }
#pragma unroll
        for (int n = 0; n < 2; ++n)
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            acc_re[n][k] = fmaf(tr[n][k], inv, acc_re[n][k]);
            acc_im[n][k] = fmaf(ti[n][k], inv, acc_im[n][k]);
          }
      }
      __syncwarp();
      if (lane == 0)
        mbarArrive(&empty[st]);  // release: this warp's reads of the stage are done
    }
    if (have_prev) {  // the rest of the previous tile's flush (batches with fewer steps than chunks)
      if (pend >= 0)
        consume(pend);
      pend = -1;
      for (int c = n_steps; c < n_chunks; ++c) {
        issue(c);
        consume(c);
      }
    }
    namedSync();  // the previous table has been read
    // This tile's table.  Accumulator element (n, k): row i = g + 8 (k >> 1) -> k2 = i, k1 = i + d;
    // column l1 = 8 n + 2 t4 + (k & 1) -> q = l1 - k1.
    if (ok) {
#pragma unroll
      for (int n = 0; n < 2; ++n)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int i = g + 8 * (k >> 1), nn = 8 * n + 2 * t4 + (k & 1);
          const int k2 = mir_a ? kneg[i] : i, k1 = kplus[d * kNc + k2];
          const int l1 = mir_b ? kneg[nn] : nn;
          const int qi = qinv[ksub[k1 + kNc * l1]];
          table[(qi * kNc + k2) * kNc + (k1 ^ qi)] = make_float2(acc_re[n][k], acc_im[n][k]);
        }
    }
    namedSync();  // the table is complete
    g4_base = fk1 + w1 * s_w1 + fk2 * s_k2 + w2 * s_w2 + iwq * s_wq;
    di_base = static_cast<long>(iwq) * nq * n_ch * MM + (fk2 + static_cast<long>(kNc) * w2) * M + fk1 +
              static_cast<long>(kNc) * w1;
    have_prev = ok;
  }
  if (have_prev)  // the CTA's last tile
    for (int c = 0; c < n_chunks; ++c) {
      issue(c);
      consume(c);
    }
}

}  // namespace

bool directTcApplies(const G4Args& a) {
  return a.dims.nb == 1 && a.dims.nc == kNc && a.q_all && a.dims.nq == kNc && a.gmax != nullptr &&
         a.dims.n_channels <= kMaxCh && a.n_slots <= kMaxSteps * kMeasPerStep;
}

void launchDirectTc(const G4Args& a, const float2* G, long g_sector_stride, const float2* disc, int n_sm,
                    cudaStream_t stream) {
  const TpDims& d = a.dims;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(updateG4DirectMma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kSmem)));
  const long tiles = long(d.nw) * d.nw * d.nwq / (d.half_g4 ? 2 : 1);
  const unsigned grid = static_cast<unsigned>(std::max(1L, std::min<long>(tiles, n_sm)));
  updateG4DirectMma<<<grid, kThreads, kSmem, stream>>>(d, G, g_sector_stride, a.signs, a.n_slots, a.k_sub,
                                                       a.q_list, a.wex_list, a.gmax, a.tile_order, disc, a.G4,
                                                       a.atomic, a.err, a.wait_limit ? a.wait_limit : kWaitLimit,
                                                       a.fault_stop_step);
  DCAACC_LAUNCH_CHECK();
}

}  // namespace dcaacc
