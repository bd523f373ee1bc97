// Batched single-band G4 update (the mixed path's PH-magnetic / PH-charge kernel).
//
// Same mathematics as updateG4SinglebandPH in tp_g4.cu (see the channel formulas there), tuned
// for long batches with FP32 G and FP32 partial sums:
//   * the cluster size is a compile-time constant, so the per-thread loop over k2 is fully
//     unrolled and all shared-memory offsets that do not depend on the measurement are computed
//     once, before the batch loop;
//   * per measurement, the A blocks are pre-scaled by sign/2 in shared memory, so the direct term
//     D = sum_s A_s B_s arrives scaled;
//   * consecutive threads take consecutive q: a warp's A reads are broadcasts, its B reads fall in
//     distinct banks, and the U/V rows are padded so their writes and reads are conflict free;
//   * tiles (w1, w2) and (w2, w1), which read the same two G blocks A and B (swapped), are launched
//     next to each other so the second read of each block comes from L2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "async_copy.cuh"
#include "common.cuh"
#include "tp_g4.hpp"

namespace dcaacc {

namespace {

// Tile order: the Nw diagonal tiles first, then the off-diagonal pairs (a, b), (b, a) next to each
// other.
__device__ inline void tileOfIndex(int idx, int nw, int& w1, int& w2) {
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
  if (j & 1) {
    w1 = b;
    w2 = a;
  }
  else {
    w1 = a;
    w2 = b;
  }
}

template <int NC, bool MAG, bool CHARGE>
__global__ void __launch_bounds__(256, 2)
updateG4SinglebandBatched(const TpDims dims, const float2* __restrict__ G, long g_sector_stride,
                          const int* __restrict__ signs, int n_slots, const int* __restrict__ k_add,
                          const int* __restrict__ q_list, const int* __restrict__ wex_list,
                          double2* const* __restrict__ G4, bool atomic, int q_chunk, int* __restrict__ err) {
  constexpr int R = NC;
  constexpr int BLK = R * R;
  const int nw = dims.nw, nw_ext = dims.nw_ext, nq = dims.nq;
  const int tiles = nw * nw;
  const int n_qchunks = (nq + q_chunk - 1) / q_chunk;
  int w1, w2;
  tileOfIndex(blockIdx.x % tiles, nw, w1, w2);
  const int rest = blockIdx.x / tiles;
  const int iwq = rest / n_qchunks, q0 = (rest % n_qchunks) * q_chunk;
  const int wex = wex_list[iwq];
  const int ext = dims.ext;
  const int t = threadIdx.x;
  const int qp = q_chunk + 1;  // padded row of the U / V tables
  // Main-phase mapping: q fastest.
  const int ql = t % q_chunk, k1 = t / q_chunk;
  const int iq = q0 + ql;
  const bool active = iq < nq && k1 < NC;
  const int q = active ? q_list[iq] : 0;
  // U/V-phase mapping: k fastest.
  const int kv = t % NC, qv = t / NC;
  const bool active_v = qv < q_chunk && q0 + qv < nq;
  const int q_v = active_v ? q_list[q0 + qv] : 0;

  const int w1e = w1 + ext, w2e = w2 + ext, w1x = w1e + wex, w2x = w2e + wex;
  const long b_A = (static_cast<long>(w1e) * nw_ext + w2e) * BLK;
  const long b_B = (static_cast<long>(w2x) * nw_ext + w1x) * BLK;
  const long b_C = (static_cast<long>(w1e) * nw_ext + w1x) * BLK;
  const long b_E = (static_cast<long>(w2x) * nw_ext + w2e) * BLK;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);       // [2]
  float2* stage = reinterpret_cast<float2*>(smem_raw + 16);    // [2][spin][A B C E][BLK]
  float2* Um = stage + 2 * 8 * BLK;                            // [NC][qp]
  float2* Uc = Um + NC * qp;
  float2* Vm = Uc + NC * qp;
  float2* Vc = Vm + NC * qp;

  int b_off[NC];
  const int k1q = k_add[k1 % NC + NC * q];
#pragma unroll
  for (int j = 0; j < NC; ++j)
    b_off[j] = k_add[j + NC * q] * R + k1q;
  const int a_off = (k1 % NC) * R;
  const int v_c = k_add[kv + NC * q_v];  // k + q for the U/V phase

  constexpr uint32_t blk_bytes = BLK * sizeof(float2);
  auto issue = [&](int slot, int st) {
    float2* dst = stage + st * 8 * BLK;
    mbarArriveExpectTx(&bar[st], 8 * blk_bytes);
    const float2* src0 = G + g_sector_stride * (2 * slot);
    const float2* src1 = src0 + g_sector_stride;
    bulkCopyG2S(dst + 0 * BLK, src0 + b_A, blk_bytes, &bar[st]);
    bulkCopyG2S(dst + 1 * BLK, src0 + b_B, blk_bytes, &bar[st]);
    bulkCopyG2S(dst + 2 * BLK, src0 + b_C, blk_bytes, &bar[st]);
    bulkCopyG2S(dst + 3 * BLK, src0 + b_E, blk_bytes, &bar[st]);
    bulkCopyG2S(dst + 4 * BLK, src1 + b_A, blk_bytes, &bar[st]);
    bulkCopyG2S(dst + 5 * BLK, src1 + b_B, blk_bytes, &bar[st]);
    bulkCopyG2S(dst + 6 * BLK, src1 + b_C, blk_bytes, &bar[st]);
    bulkCopyG2S(dst + 7 * BLK, src1 + b_E, blk_bytes, &bar[st]);
  };
  if (t == 0) {
    mbarInit(&bar[0], 1);
    mbarInit(&bar[1], 1);
    fenceBarrierInit();
  }
  __syncthreads();
  if (t == 0) {
    issue(0, 0);
    if (n_slots > 1)
      issue(1, 1);
  }

  float2 acc_m[NC], acc_c[NC];
#pragma unroll
  for (int j = 0; j < NC; ++j) {
    acc_m[j] = make_float2(0.f, 0.f);
    acc_c[j] = make_float2(0.f, 0.f);
  }

  for (int m = 0; m < n_slots; ++m) {
    const int st = m & 1;
    const bool ok = mbarWait(&bar[st], (m >> 1) & 1, err);
    if (!__syncthreads_and(ok))
      return;  // uniform bail-out; the host reports the error word
    float2* S = stage + st * 8 * BLK;
    const float hs = 0.5f * static_cast<float>(signs[m]);
    // Phase 1: scale A_0, A_1 by s/2; U = s/2 (C_0 -+ C_1)(k, k+q), V = (E_0 -+ E_1)(k+q, k).
    for (int e = t; e < BLK; e += blockDim.x) {
      float2 a = S[e];
      S[e] = make_float2(hs * a.x, hs * a.y);
      a = S[4 * BLK + e];
      S[4 * BLK + e] = make_float2(hs * a.x, hs * a.y);
    }
    if (active_v) {
      const float2 c0 = S[2 * BLK + kv * R + v_c], c1 = S[6 * BLK + kv * R + v_c];
      const float2 e0 = S[3 * BLK + v_c * R + kv], e1 = S[7 * BLK + v_c * R + kv];
      const int o = kv * qp + qv;
      if (MAG) {
        Um[o] = make_float2(hs * (c0.x - c1.x), hs * (c0.y - c1.y));
        Vm[o] = make_float2(e0.x - e1.x, e0.y - e1.y);
      }
      if (CHARGE) {
        Uc[o] = make_float2(hs * (c0.x + c1.x), hs * (c0.y + c1.y));
        Vc[o] = make_float2(e0.x + e1.x, e0.y + e1.y);
      }
    }
    __syncthreads();
    // Phase 2: the tile's entries (k1, k2 = 0..NC-1, q).
    if (active) {
      const float2* A0 = S + a_off;
      const float2* A1 = S + 4 * BLK + a_off;
      const float2* B0 = S + 1 * BLK;
      const float2* B1 = S + 5 * BLK;
      const int o = k1 * qp + ql;
      const float2 um = MAG ? Um[o] : make_float2(0.f, 0.f);
      const float2 uc = CHARGE ? Uc[o] : make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < NC; ++j) {
        const float2 a0 = A0[j], a1 = A1[j], b0 = B0[b_off[j]], b1 = B1[b_off[j]];
        float2 d = cmul(a0, b0);
        cfma(d, a1, b1);
        if (MAG) {
          const float2 v = Vm[j * qp + ql];
          float2& ac = acc_m[j];
          ac.x = fma(um.x, v.x, ac.x);
          ac.x = fma(-um.y, v.y, ac.x);
          ac.y = fma(um.x, v.y, ac.y);
          ac.y = fma(um.y, v.x, ac.y);
          ac.x -= d.x;
          ac.y -= d.y;
        }
        if (CHARGE) {
          const float2 v = Vc[j * qp + ql];
          float2& ac = acc_c[j];
          ac.x = fma(uc.x, v.x, ac.x);
          ac.x = fma(-uc.y, v.y, ac.x);
          ac.y = fma(uc.x, v.y, ac.y);
          ac.y = fma(uc.y, v.x, ac.y);
          ac.x -= d.x;
          ac.y -= d.y;
        }
      }
    }
    fenceProxyAsync();  // this thread's generic writes to the stage precede the next bulk copy
    __syncthreads();    // stage st and the U/V tables are free again
    if (t == 0 && m + 2 < n_slots)
      issue(m + 2, st);
  }

  if (!active)
    return;
  const long s_w1 = NC, s_k2 = s_w1 * nw, s_w2 = s_k2 * NC, s_q = s_w2 * nw, s_wq = s_q * nq;
  const long base = k1 + w1 * s_w1 + w2 * s_w2 + iq * s_q + iwq * s_wq;
#pragma unroll
  for (int c = 0; c < kMaxChannels; ++c) {
    if (c >= dims.n_channels)
      break;
    const bool mag = dims.channels[c] == 2;
    double2* g4 = G4[c] + base;
#pragma unroll
    for (int j = 0; j < NC; ++j) {
      const float2 v = mag ? acc_m[j] : acc_c[j];
      double2* p = g4 + j * s_k2;
      if (atomic) {
        atomicAdd(&p->x, static_cast<double>(v.x));
        atomicAdd(&p->y, static_cast<double>(v.y));
      }
      else {
        double2 o = *p;
        o.x += static_cast<double>(v.x);
        o.y += static_cast<double>(v.y);
        *p = o;
      }
    }
  }
}

// Direct term only: sum_m sum_s -s_m/2 G_s(k1 w1; k2 w2) G_s(k2+q w2+x; k1+q w1+x), which is the same
// for PH-magnetic and PH-charge with one band.  The disconnected terms come from the tensor-core
// GEMM (tp_g4_disc.cu) in `disc`: per problem (iwq, iq, channel) an M x M matrix (M = Nc Nw) with
// m = k1 + Nc w1 fastest.  Only the A and B blocks are staged.  The flush goes through shared
// memory so that consecutive lanes touch consecutive k1 of G4 and of `disc`.
template <int NC>
__global__ void __launch_bounds__(256, 2)
updateG4SinglebandDirect(const TpDims dims, const float2* __restrict__ G, long g_sector_stride,
                         const int* __restrict__ signs, int n_slots, const int* __restrict__ k_add,
                         const int* __restrict__ q_list, const int* __restrict__ wex_list,
                         const float2* __restrict__ disc, double2* const* __restrict__ G4, bool atomic,
                         int q_chunk, int* __restrict__ err) {
  constexpr int R = NC;
  constexpr int BLK = R * R;
  const int nw = dims.nw, nw_ext = dims.nw_ext, nq = dims.nq;
  const int tiles = nw * nw;
  const int n_qchunks = (nq + q_chunk - 1) / q_chunk;
  int w1, w2;
  tileOfIndex(blockIdx.x % tiles, nw, w1, w2);
  const int rest = blockIdx.x / tiles;
  const int iwq = rest / n_qchunks, q0 = (rest % n_qchunks) * q_chunk;
  const int wex = wex_list[iwq];
  const int ext = dims.ext;
  const int t = threadIdx.x;
  const int qp = q_chunk + 1;  // padded row of the flush table
  const int ql = t % q_chunk, k1 = t / q_chunk;
  const int iq = q0 + ql;
  const bool active = iq < nq && k1 < NC;
  const int q = active ? q_list[iq] : 0;

  const int w1e = w1 + ext, w2e = w2 + ext, w1x = w1e + wex, w2x = w2e + wex;
  const long b_A = (static_cast<long>(w1e) * nw_ext + w2e) * BLK;
  const long b_B = (static_cast<long>(w2x) * nw_ext + w1x) * BLK;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);     // [2]
  float2* stage = reinterpret_cast<float2*>(smem_raw + 16);  // [2][A0 B0 A1 B1][BLK]

  int b_off[NC];
  const int k1q = k_add[k1 % NC + NC * q];
#pragma unroll
  for (int j = 0; j < NC; ++j)
    b_off[j] = k_add[j + NC * q] * R + k1q;
  const int a_off = (k1 % NC) * R;

  constexpr uint32_t blk_bytes = BLK * sizeof(float2);
  auto issue = [&](int slot, int st) {
    float2* dst = stage + st * 4 * BLK;
    mbarArriveExpectTx(&bar[st], 4 * blk_bytes);
    const float2* src0 = G + g_sector_stride * (2 * slot);
    const float2* src1 = src0 + g_sector_stride;
    bulkCopyG2S(dst + 0 * BLK, src0 + b_A, blk_bytes, &bar[st]);
    bulkCopyG2S(dst + 1 * BLK, src0 + b_B, blk_bytes, &bar[st]);
    bulkCopyG2S(dst + 2 * BLK, src1 + b_A, blk_bytes, &bar[st]);
    bulkCopyG2S(dst + 3 * BLK, src1 + b_B, blk_bytes, &bar[st]);
  };
  if (t == 0) {
    mbarInit(&bar[0], 1);
    mbarInit(&bar[1], 1);
    fenceBarrierInit();
  }
  __syncthreads();
  if (t == 0) {
    issue(0, 0);
    if (n_slots > 1)
      issue(1, 1);
  }

  float2 acc[NC];
#pragma unroll
  for (int j = 0; j < NC; ++j)
    acc[j] = make_float2(0.f, 0.f);

  for (int m = 0; m < n_slots; ++m) {
    const int st = m & 1;
    const bool ok = mbarWait(&bar[st], (m >> 1) & 1, err);
    if (!__syncthreads_and(ok))
      return;  // uniform bail-out; the host reports the error word
    float2* S = stage + st * 4 * BLK;
    const float nhs = -0.5f * static_cast<float>(signs[m]);
    for (int e = t; e < BLK; e += blockDim.x) {  // A_0, A_1 *= -s/2
      float2 a = S[e];
      S[e] = make_float2(nhs * a.x, nhs * a.y);
      a = S[2 * BLK + e];
      S[2 * BLK + e] = make_float2(nhs * a.x, nhs * a.y);
    }
    __syncthreads();
    if (active) {
      const float2* A0 = S + a_off;
      const float2* B0 = S + 1 * BLK;
      const float2* A1 = S + 2 * BLK + a_off;
      const float2* B1 = S + 3 * BLK;
#pragma unroll
      for (int j = 0; j < NC; ++j) {
        cfma(acc[j], A0[j], B0[b_off[j]]);
        cfma(acc[j], A1[j], B1[b_off[j]]);
      }
    }
    fenceProxyAsync();  // this thread's generic writes to the stage precede the next bulk copy
    __syncthreads();    // stage st is free again
    if (t == 0 && m + 2 < n_slots)
      issue(m + 2, st);
  }

  // Flush: table T[j][k1][ql] (rows padded to qp), then lanes take consecutive k1.
  float2* T = stage;
  if (active) {
#pragma unroll
    for (int j = 0; j < NC; ++j)
      T[(j * NC + k1) * qp + ql] = acc[j];
  }
  __syncthreads();
  const long M = static_cast<long>(NC) * nw;
  const long s_w1 = NC, s_k2 = s_w1 * nw, s_w2 = s_k2 * NC, s_q = s_w2 * nw, s_wq = s_q * nq;
  const int n_ch = dims.n_channels;
  for (int idx = t; idx < NC * NC * q_chunk; idx += blockDim.x) {
    const int fk1 = idx % NC, j = (idx / NC) % NC, fql = idx / (NC * NC);
    const int fiq = q0 + fql;
    if (fiq >= nq)
      continue;
    const float2 v = T[(j * NC + fk1) * qp + fql];
    const long g4i = fk1 + w1 * s_w1 + j * s_k2 + w2 * s_w2 + fiq * s_q + iwq * s_wq;
    const long di = (j + static_cast<long>(NC) * w2) * M + fk1 + static_cast<long>(NC) * w1;
    for (int c = 0; c < n_ch; ++c) {
      const float2 dv = disc[(static_cast<long>(iwq * nq + fiq) * n_ch + c) * M * M + di];
      double2* p = G4[c] + g4i;
      const double re = static_cast<double>(v.x + dv.x), im = static_cast<double>(v.y + dv.y);
      if (atomic) {
        atomicAdd(&p->x, re);
        atomicAdd(&p->y, im);
      }
      else {
        double2 o = *p;
        o.x += re;
        o.y += im;
        *p = o;
      }
    }
  }
}

// Direct term, all momentum transfers (nq = Nc, q_list a permutation of the cluster momenta).
// Grouping the entries by d = k1 - k2 turns the term into outer products: with l1 = k1 + q,
//   D(k1, k2 = k1 - d, q = l1 - k1) = sum_m sum_s alpha_sd(k1) beta_sd(l1),
//   alpha_sd(k1) = -s_m/2 G_s(k1 w1; k1-d w2),   beta_sd(l1) = G_s(l1-d w2+x; l1 w1+x),
// (the cluster momenta form a group, so k2 + q = l1 - d).  Thread (d, k1 block, l1 block) keeps a
// TA x TB tile of complex sums in registers and, per measurement and spin, gathers its TA alphas
// and TB betas straight from the staged G blocks (fixed shared-memory offsets, computed once) for
// TA TB complex FMAs.  Measurements are staged eight deep (bulk copies); per-stage "empty"
// barriers let the warps drift apart instead of meeting at a block barrier per measurement.  The flush goes through a shared table so that lanes touch consecutive k1
// of G4 and of `disc`.
template <int NC, int TA, int TB>
__global__ void __launch_bounds__(NC * (NC / TA) * (NC / TB))
updateG4SinglebandOuter(const TpDims dims, const float2* __restrict__ G, long g_sector_stride,
                        const int* __restrict__ signs, int n_slots, const int* __restrict__ k_sub,
                        const int* __restrict__ q_list, const int* __restrict__ wex_list,
                        const float2* __restrict__ disc, double2* const* __restrict__ G4, bool atomic,
                        int* __restrict__ err) {
  constexpr int BLK = NC * NC;
  constexpr int NKB = NC / TA, NLB = NC / TB;
  constexpr int NT = NC * NKB * NLB;  // threads
  constexpr int QP = NC + 1;          // padded row of the flush table
  constexpr int DEPTH = 8;            // staged measurements
  const int nw = dims.nw, nw_ext = dims.nw_ext, nq = dims.nq;
  int w1, w2;
  tileOfIndex(blockIdx.x % (nw * nw), nw, w1, w2);
  const int iwq = blockIdx.x / (nw * nw);
  const int wex = wex_list[iwq];
  const int ext = dims.ext;
  const int t = threadIdx.x;
  const int d = t / (NKB * NLB), sub = t % (NKB * NLB);
  const int k1_0 = (sub / NLB) * TA, l1_0 = (sub % NLB) * TB;

  const int w1e = w1 + ext, w2e = w2 + ext, w1x = w1e + wex, w2x = w2e + wex;
  const long b_A = (static_cast<long>(w1e) * nw_ext + w2e) * BLK;
  const long b_B = (static_cast<long>(w2x) * nw_ext + w1x) * BLK;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);      // [DEPTH] copies landed
  uint64_t* empty = full + DEPTH;                               // [DEPTH] all warps done reading
  int* ksub = reinterpret_cast<int*>(smem_raw + 16 * DEPTH);   // [NC * NC]
  int* qinv = ksub + BLK;                                      // [NC]
  float2* region = reinterpret_cast<float2*>(smem_raw + 16 * DEPTH + 4 * (BLK + NC + 4));
  static_assert((16 * DEPTH + 4 * (BLK + NC + 4)) % 16 == 0, "bulk-copy destinations need 16-byte alignment");
  const int lane = t % 32;
  float2* stage = region;                                      // [DEPTH][A0 B0 A1 B1][BLK]
  float2* T = region;                                          // flush table, after the batch loop

  for (int e = t; e < BLK; e += NT)
    ksub[e] = k_sub[e];
  for (int e = t; e < NC; e += NT)
    qinv[q_list[e]] = e;

  constexpr uint32_t blk_bytes = BLK * sizeof(float2);
  auto issue = [&](int slot) {
    const int st = slot % DEPTH;
    float2* dst = stage + st * 4 * BLK;
    mbarArriveExpectTx(&full[st], 4 * blk_bytes);
    const float2* src0 = G + g_sector_stride * (2 * slot);
    const float2* src1 = src0 + g_sector_stride;
    bulkCopyG2S(dst + 0 * BLK, src0 + b_A, blk_bytes, &full[st]);
    bulkCopyG2S(dst + 1 * BLK, src0 + b_B, blk_bytes, &full[st]);
    bulkCopyG2S(dst + 2 * BLK, src1 + b_A, blk_bytes, &full[st]);
    bulkCopyG2S(dst + 3 * BLK, src1 + b_B, blk_bytes, &full[st]);
  };
  if (t == 0) {
    for (int s2 = 0; s2 < DEPTH; ++s2) {
      mbarInit(&full[s2], 1);
      mbarInit(&empty[s2], NT / 32);
    }
    fenceBarrierInit();
  }
  __syncthreads();
  if (t == 0)
    for (int m = 0; m < DEPTH && m < n_slots; ++m)
      issue(m);

  // Fixed gather offsets inside a staged block: alpha from A (row k1, column k1 - d), beta from B
  // (row l1 - d, column l1).
  int oa[TA], ob[TB];
#pragma unroll
  for (int a = 0; a < TA; ++a)
    oa[a] = (k1_0 + a) * NC + ksub[d + NC * (k1_0 + a)];
#pragma unroll
  for (int b = 0; b < TB; ++b)
    ob[b] = ksub[d + NC * (l1_0 + b)] * NC + l1_0 + b;

  // Sums of -s_m alpha beta (the factor 1/2 is applied at the flush); the sign selects the loop
  // body (uniform across the CTA), so no multiply is spent on it.
  float2 acc[TA][TB];
#pragma unroll
  for (int a = 0; a < TA; ++a)
#pragma unroll
    for (int b = 0; b < TB; ++b)
      acc[a][b] = make_float2(0.f, 0.f);

  // Each warp arrives on empty[stage] when it is done with a measurement; thread 0 waits for all
  // warps there before re-filling the stage, so the other warps can run up to DEPTH - 1
  // measurements ahead of the slowest one instead of meeting at a block barrier.
  bool ok = true;
  int sg = n_slots > 0 ? signs[0] : 1;
  for (int m = 0; m < n_slots; ++m) {
    const int st = m % DEPTH;
    const int sg_next = m + 1 < n_slots ? signs[m + 1] : 1;
    ok = __all_sync(0xffffffffu, mbarWait(&full[st], (m / DEPTH) & 1, err));
    if (!ok)
      break;
    const float2* S = stage + st * 4 * BLK;
    const bool add = sg < 0;
#pragma unroll
    for (int spin = 0; spin < 2; ++spin) {
      const float2* A = S + (2 * spin) * BLK;
      const float2* B = S + (2 * spin + 1) * BLK;
      float2 av[TA], bv[TB];
#pragma unroll
      for (int a = 0; a < TA; ++a)
        av[a] = A[oa[a]];
#pragma unroll
      for (int b = 0; b < TB; ++b)
        bv[b] = B[ob[b]];
      if (add) {
#pragma unroll
        for (int a = 0; a < TA; ++a)
#pragma unroll
          for (int b = 0; b < TB; ++b)
            cfma(acc[a][b], av[a], bv[b]);
      }
      else {
#pragma unroll
        for (int a = 0; a < TA; ++a)
#pragma unroll
          for (int b = 0; b < TB; ++b) {
            float2& c = acc[a][b];
            c.x = fmaf(-av[a].x, bv[b].x, c.x);
            c.x = fmaf(av[a].y, bv[b].y, c.x);
            c.y = fmaf(-av[a].x, bv[b].y, c.y);
            c.y = fmaf(-av[a].y, bv[b].x, c.y);
          }
      }
    }
    sg = sg_next;
    __syncwarp();
    if (lane == 0)
      mbarArrive(&empty[st]);  // release: this warp's reads of the stage are done
    if (t == 0 && m + DEPTH < n_slots) {
      if (!mbarWait(&empty[st], (m / DEPTH) & 1, err)) {
        ok = false;  // the other warps see the missing copy as a timeout of their own
        break;
      }
      issue(m + DEPTH);
    }
  }
  if (__syncthreads_or(!ok))
    return;  // uniform bail-out; the host reports the error word

  // Flush table T[k2][k1][qi] (rows padded to QP), then lanes take consecutive k1.
#pragma unroll
  for (int a = 0; a < TA; ++a)
#pragma unroll
    for (int b = 0; b < TB; ++b) {
      const int k1 = k1_0 + a, l1 = l1_0 + b;
      const int k2 = ksub[d + NC * k1];
      const int qi = qinv[ksub[k1 + NC * l1]];
      T[(k2 * NC + k1) * QP + qi] = make_float2(0.5f * acc[a][b].x, 0.5f * acc[a][b].y);
    }
  __syncthreads();
  const long M = static_cast<long>(NC) * nw;
  const long s_w1 = NC, s_k2 = s_w1 * nw, s_w2 = s_k2 * NC, s_q = s_w2 * nw, s_wq = s_q * nq;
  const int n_ch = dims.n_channels;
  // Four entries per thread and pass, all their loads issued before any add, so the DRAM round
  // trips of the flush overlap instead of running one entry at a time.
  constexpr int U = 4;
  const int total = NC * NC * nq;
  for (int base = t; base < total; base += U * NT) {
    float2 v[U];
    long g4i[U], di[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = min(base + u * NT, total - 1);
      const int fk1 = idx % NC, j = (idx / NC) % NC, fqi = idx / (NC * NC);
      v[u] = T[(j * NC + fk1) * QP + fqi];
      g4i[u] = fk1 + w1 * s_w1 + j * s_k2 + w2 * s_w2 + fqi * s_q + iwq * s_wq;
      di[u] = (static_cast<long>(iwq * nq + fqi) * n_ch * M + j + static_cast<long>(NC) * w2) * M + fk1 +
              static_cast<long>(NC) * w1;
    }
    for (int c = 0; c < n_ch; ++c) {
      float2 dv[U];
      double2 o[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        dv[u] = __ldg(disc + di[u] + static_cast<long>(c) * M * M);
        o[u] = atomic ? make_double2(0., 0.) : G4[c][g4i[u]];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (base + u * NT >= total)
          continue;
        double2* p = G4[c] + g4i[u];
        const double re = static_cast<double>(v[u].x + dv[u].x), im = static_cast<double>(v[u].y + dv[u].y);
        if (atomic) {
          atomicAdd(&p->x, re);
          atomicAdd(&p->y, im);
        }
        else {
          o[u].x += re;
          o[u].y += im;
          *p = o[u];
        }
      }
    }
  }
}

// Direct term for clusters whose NC^3 sums per (w1, w2, wq) tile do not fit one CTA's registers
// (Nc = 36: 46,656 complex sums): the same outer products as updateG4SinglebandOuter, with
// NC / KG CTAs per tile, CTA g owning the rows k1 in [g KG, (g + 1) KG).  Per measurement and spin
// a CTA stages the KG rows of the A block it reads and the whole B block (bulk copies, DEPTH
// measurements deep); thread (d, k1 block, l1 block) keeps a TA x TB tile of sums in registers.
// The flush table T[k2][k1 - g KG][q] covers the CTA's entries, and lanes write runs of KG
// consecutive k1 of G4 (and read the disconnected terms in the same order).
// Half G (dims.half_g): a block in the lower frequency half is read as the conjugate of its mirror
// block with k -> -k (G(k1 w; k2 w') = conj G(-k1 w*; -k2 w'*), w* = NwExt - 1 - w): the A rows are
// staged one by one (row -k1 of the mirror block into the slot of k1), the B block whole, and the
// gather offsets take -k on the mirrored indices.  Half G4 (tile_order non-null): only the tiles
// listed there (w1 >= Nw / 2) run.
constexpr int kSplitMaxSlots = 256;  // measurements per launch (the signs sit in shared memory)

template <int NC, int KG, int TA, int TB, int DEPTH>
__global__ void __launch_bounds__(NC * (KG / TA) * (NC / TB), 1)
updateG4SinglebandOuterSplit(const TpDims dims, const float2* __restrict__ G, long g_sector_stride,
                             const int* __restrict__ signs, int n_slots, const int* __restrict__ k_sub,
                             const int* __restrict__ q_list, const int* __restrict__ wex_list,
                             const unsigned* __restrict__ tile_order, const float2* __restrict__ disc,
                             double2* const* __restrict__ G4, bool atomic, int* __restrict__ err) {
  constexpr int BLK = NC * NC;
  constexpr int AR = KG * NC;         // staged rows of A
  constexpr int SP = AR + BLK;        // one spin's staged A rows + B block
  constexpr int NKB = KG / TA, NLB = NC / TB;
  constexpr int NT = NC * NKB * NLB;  // threads
  constexpr int KSPLIT = NC / KG;
  constexpr int QP = NC + 1;          // padded row of the flush table
  static_assert(NC % KG == 0 && KG % TA == 0 && NC % TB == 0 && NT % 32 == 0, "tile shape");
  const int nw = dims.nw, nw_ext = dims.nw_ext, nq = dims.nq;
  const int grp = blockIdx.x % KSPLIT;
  const int tile = blockIdx.x / KSPLIT;  // the KSPLIT CTAs of a tile run next to each other
  const int per_wq = tile_order ? nw * nw / 2 : nw * nw;
  int w1, w2;
  if (tile_order) {
    const unsigned v = tile_order[tile % per_wq];
    w1 = static_cast<int>(v & 0xffffu);
    w2 = static_cast<int>(v >> 16);
  }
  else {
    tileOfIndex(tile % per_wq, nw, w1, w2);
  }
  const int iwq = tile / per_wq;
  const int wex = wex_list[iwq];
  const int ext = dims.ext;
  const int t = threadIdx.x;
  const int d = t / (NKB * NLB), sub = t % (NKB * NLB);
  const int kg0 = grp * KG;
  const int k1_0 = kg0 + (sub / NLB) * TA, l1_0 = (sub % NLB) * TB;

  const int w1e = w1 + ext, w2e = w2 + ext, w1x = w1e + wex, w2x = w2e + wex;
  const bool mir_a = dims.half_g && 2 * w1e < nw_ext, mir_b = dims.half_g && 2 * w2x < nw_ext;
  // A: the KG rows of block (w1e, w2e) from row kg0 on, or (mirrored) rows -k1 of block
  // (w1e*, w2e*); B: block (w2x, w1x) or its mirror (w2x*, w1x*).
  const long b_A = mir_a ? (static_cast<long>(nw_ext - 1 - w1e) * nw_ext + nw_ext - 1 - w2e) * BLK
                         : (static_cast<long>(w1e) * nw_ext + w2e) * BLK + static_cast<long>(kg0) * NC;
  const long b_B = mir_b ? (static_cast<long>(nw_ext - 1 - w2x) * nw_ext + nw_ext - 1 - w1x) * BLK
                         : (static_cast<long>(w2x) * nw_ext + w1x) * BLK;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);     // [DEPTH] copies landed
  uint64_t* empty = full + DEPTH;                              // [DEPTH] all warps done reading
  int* ksub = reinterpret_cast<int*>(smem_raw + 16 * DEPTH);  // [NC * NC]
  int* qinv = ksub + BLK;                                     // [NC]
  int* kneg = qinv + NC;                                      // [NC] index of -k (half G)
  int* arow = kneg + NC;                                      // [KG] mirrored A: offset of row -k1
  int* sgn = arow + KG;                                       // [kSplitMaxSlots] measurement signs
  constexpr int kHead = (16 * DEPTH + 4 * (BLK + 2 * NC + KG + kSplitMaxSlots) + 15) / 16 * 16;
  float2* stage = reinterpret_cast<float2*>(smem_raw + kHead);  // [DEPTH][A0 rows, B0, A1 rows, B1]
  float2* T = stage;                                           // flush table, after the batch loop
  const int lane = t % 32;

  for (int e = t; e < BLK; e += NT)
    ksub[e] = k_sub[e];
  // -k = k_z - k with z = k_0 - k_0 the zero momentum: k_sub gives it without reading dims' table.
  const int z0 = k_sub[0];
  for (int e = t; e < NC; e += NT) {
    qinv[q_list[e]] = e;
    kneg[e] = k_sub[e + NC * z0];
  }
  for (int r = t; r < KG; r += NT)
    arow[r] = k_sub[kg0 + r + NC * z0] * NC;
  for (int m = t; m < n_slots; m += NT)
    sgn[m] = signs[m];
  __syncthreads();
  auto kn = [&](int k) { return kneg[k]; };

  constexpr uint32_t a_bytes = AR * sizeof(float2), b_bytes = BLK * sizeof(float2), row_bytes = NC * sizeof(float2);
  static_assert(row_bytes % 16 == 0, "bulk copies of single rows");
  auto issue = [&](int slot) {
    const int st = slot % DEPTH;
    float2* dst = stage + st * 2 * SP;
    mbarArriveExpectTx(&full[st], 2 * (a_bytes + b_bytes));
    const float2* src0 = G + g_sector_stride * (2 * slot);
    const float2* src1 = src0 + g_sector_stride;
    if (mir_a) {
      for (int r = 0; r < KG; ++r) {  // row -k1 of the mirror block into the slot of k1
        const float2* row = src0 + b_A + arow[r];
        bulkCopyG2S(dst + r * NC, row, row_bytes, &full[st]);
        bulkCopyG2S(dst + SP + r * NC, row + g_sector_stride, row_bytes, &full[st]);
      }
    }
    else {
      bulkCopyG2S(dst, src0 + b_A, a_bytes, &full[st]);
      bulkCopyG2S(dst + SP, src1 + b_A, a_bytes, &full[st]);
    }
    bulkCopyG2S(dst + AR, src0 + b_B, b_bytes, &full[st]);
    bulkCopyG2S(dst + SP + AR, src1 + b_B, b_bytes, &full[st]);
  };
  if (t == 0) {
    for (int s2 = 0; s2 < DEPTH; ++s2) {
      mbarInit(&full[s2], 1);
      mbarInit(&empty[s2], NT / 32);
    }
    fenceBarrierInit();
  }
  __syncthreads();
  if (t == 0)
    for (int m = 0; m < DEPTH && m < n_slots; ++m)
      issue(m);

  // Fixed gather offsets: alpha from the staged A rows (row k1 - kg0, column k1 - d), beta from B
  // (row l1 - d, column l1).
  // The beta offsets two to a register (SP < 2^16), so that the TA x TB sums stay in registers.
  static_assert(SP < 65536, "16-bit gather offsets");
  int oa[TA];
  uint32_t ob2[(TB + 1) / 2];
#pragma unroll
  for (int a = 0; a < TA; ++a) {
    const int k2 = ksub[d + NC * (k1_0 + a)];  // k1 - d
    oa[a] = (k1_0 + a - kg0) * NC + (mir_a ? kn(k2) : k2);
  }
#pragma unroll
  for (int i = 0; i < (TB + 1) / 2; ++i)
    ob2[i] = 0;
#pragma unroll
  for (int b = 0; b < TB; ++b) {
    const int l1 = l1_0 + b, lr = ksub[d + NC * l1];  // row l1 - d, column l1
    ob2[b / 2] |= static_cast<uint32_t>(AR + (mir_b ? kn(lr) * NC + kn(l1) : lr * NC + l1)) << (16 * (b & 1));
  }
  auto ob = [&](int b) {
    return static_cast<int>((b & 1) ? (ob2[b / 2] >> 16) : __byte_perm(ob2[b / 2], 0u, 0x4410u));
  };

  float2 acc[TA][TB];
#pragma unroll
  for (int a = 0; a < TA; ++a)
#pragma unroll
    for (int b = 0; b < TB; ++b)
      acc[a][b] = make_float2(0.f, 0.f);

  // acc += alpha' beta with alpha' = -s (conj if mirrored) alpha, folded into the TA alphas once per
  // spin; a mirrored B block's conjugation is a compile-time variant of the product (CB).
  bool ok = true;
  auto run = [&](auto cb_tag) {
    constexpr bool CB = decltype(cb_tag)::value;
    const float ia = mir_a ? -1.f : 1.f;
    for (int m = 0; m < n_slots; ++m) {
      const int st = m % DEPTH;
      ok = __all_sync(0xffffffffu, mbarWait(&full[st], (m / DEPTH) & 1, err));
      if (!ok)
        break;
      const float ns = -static_cast<float>(sgn[m]);
#pragma unroll
      for (int spin = 0; spin < 2; ++spin) {
        const float2* S = stage + (st * 2 + spin) * SP;
        float2 av[TA];
#pragma unroll
        for (int a = 0; a < TA; ++a) {
          const float2 x = S[oa[a]];
          av[a] = make_float2(ns * x.x, ns * ia * x.y);
        }
#pragma unroll
        for (int b = 0; b < TB; ++b) {
          const float2 bv = S[ob(b)];
#pragma unroll
          for (int a = 0; a < TA; ++a) {
            float2& c = acc[a][b];
            if constexpr (CB) {  // av conj(bv)
              c.x = fmaf(av[a].x, bv.x, c.x);
              c.x = fmaf(av[a].y, bv.y, c.x);
              c.y = fmaf(av[a].y, bv.x, c.y);
              c.y = fmaf(-av[a].x, bv.y, c.y);
            }
            else {
              cfma(c, av[a], bv);
            }
          }
        }
      }
      __syncwarp();
      if (lane == 0)
        mbarArrive(&empty[st]);  // release: this warp's reads of the stage are done
      if (t == 0 && m + DEPTH < n_slots) {
        if (!mbarWait(&empty[st], (m / DEPTH) & 1, err)) {
          ok = false;  // the other warps see the missing copy as a timeout of their own
          break;
        }
        issue(m + DEPTH);
      }
    }
  };
  if (mir_b)
    run(std::true_type{});
  else
    run(std::false_type{});
  if (__syncthreads_or(!ok))
    return;  // uniform bail-out; the host reports the error word

#pragma unroll
  for (int a = 0; a < TA; ++a)
#pragma unroll
    for (int b = 0; b < TB; ++b) {
      const int k1 = k1_0 + a, l1 = l1_0 + b;
      const int k2 = ksub[d + NC * k1];
      const int qi = qinv[ksub[k1 + NC * l1]];
      T[(k2 * KG + k1 - kg0) * QP + qi] = make_float2(0.5f * acc[a][b].x, 0.5f * acc[a][b].y);
    }
  __syncthreads();
  const long M = static_cast<long>(NC) * nw;
  const long s_w1 = NC, s_k2 = s_w1 * nw, s_w2 = s_k2 * NC, s_q = s_w2 * nw, s_wq = s_q * nq;
  const int n_ch = dims.n_channels;
  constexpr int U = 4;
  const int total = KG * NC * nq;
  for (int base = t; base < total; base += U * NT) {
    float2 v[U];
    long g4i[U], di[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = min(base + u * NT, total - 1);
      const int fk1l = idx % KG, j = (idx / KG) % NC, fqi = idx / (KG * NC);
      const int fk1 = kg0 + fk1l;
      v[u] = T[(j * KG + fk1l) * QP + fqi];
      g4i[u] = fk1 + w1 * s_w1 + j * s_k2 + w2 * s_w2 + fqi * s_q + iwq * s_wq;
      di[u] = (static_cast<long>(iwq * nq + fqi) * n_ch * M + j + static_cast<long>(NC) * w2) * M + fk1 +
              static_cast<long>(NC) * w1;
    }
    for (int c = 0; c < n_ch; ++c) {
      float2 dv[U];
      double2 o[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        dv[u] = __ldg(disc + di[u] + static_cast<long>(c) * M * M);
        o[u] = atomic ? make_double2(0., 0.) : G4[c][g4i[u]];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (base + u * NT >= total)
          continue;
        double2* p = G4[c] + g4i[u];
        const double re = static_cast<double>(v[u].x + dv[u].x), im = static_cast<double>(v[u].y + dv[u].y);
        if (atomic) {
          atomicAdd(&p->x, re);
          atomicAdd(&p->y, im);
        }
        else {
          o[u].x += re;
          o[u].y += im;
          *p = o[u];
        }
      }
    }
  }
}

// Nc = 36: 3 CTAs per tile (12 rows k1 each), 6 measurements staged (166 KB; the flush table,
// 128 KB, reuses the staging); per thread 3 x 9 sums (576 threads) or 6 x 9 (288 threads), which
// the launch-shape tuner chooses between (same sums in the same order either way).
constexpr int kSplitNc = 36, kSplitKG = 12, kSplitTB = 9, kSplitDepth = 6;

size_t outerSplitSmem() {
  constexpr int BLK = kSplitNc * kSplitNc;
  constexpr size_t head = (16 * kSplitDepth + 4 * (BLK + 2 * kSplitNc + kSplitKG + kSplitMaxSlots) + 15) / 16 * 16;
  const size_t loop = sizeof(float2) * kSplitDepth * 2 * (kSplitKG * kSplitNc + BLK);
  const size_t table = sizeof(float2) * size_t(kSplitNc) * kSplitKG * (kSplitNc + 1);
  return head + std::max(loop, table);
}

template <int TA>
void launchOuterSplitTA(const G4Args& a, const float2* G, long stride, const float2* disc, cudaStream_t stream) {
  const TpDims& d = a.dims;
  const size_t smem = outerSplitSmem();
  auto k = updateG4SinglebandOuterSplit<kSplitNc, kSplitKG, TA, kSplitTB, kSplitDepth>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long tiles = long(d.nw) * d.nw * d.nwq / (a.tile_order ? 2 : 1);  // half G4: w1 >= Nw / 2 only
  const long blocks = tiles * (kSplitNc / kSplitKG);
  constexpr int threads = kSplitNc * (kSplitKG / TA) * (kSplitNc / kSplitTB);
  k<<<static_cast<unsigned>(blocks), threads, smem, stream>>>(d, G, stride, a.signs, a.n_slots, a.k_sub,
                                                              a.q_list, a.wex_list, a.tile_order, disc, a.G4,
                                                              a.atomic, a.err);
  DCAACC_LAUNCH_CHECK();
}

void launchOuterSplit(const G4Args& a, const float2* G, long stride, const float2* disc, cudaStream_t stream) {
  const TpDims& d = a.dims;
  const auto pk = tunePick(a.tuner, tuneKey("g4split", d.nb, d.nc, d.nw_ext, d.nq, a.n_slots, 8), 2, stream);
  if (pk.choice == 1)
    launchOuterSplitTA<6>(a, G, stride, disc, stream);
  else
    launchOuterSplitTA<3>(a, G, stride, disc, stream);
  tuneEnd(a.tuner, pk, stream);
}

template <int NC>
struct OuterTile;  // per-thread tile (k1 x l1) of the outer-product kernel
// A beta gather B[l1 - d][l1] falls in the bank of column l1, so the threads of a warp that read
// betas at once should span few d values: with 4 x 4 tiles a warp holds two d values (2-way at
// most), and the alphas A[k1][k1 - d] spread over distinct banks.
template <>
struct OuterTile<16> {
  static constexpr int TA = 4, TB = 4;
};
template <>
struct OuterTile<8> {
  static constexpr int TA = 2, TB = 2;
};
template <>
struct OuterTile<4> {
  static constexpr int TA = 1, TB = 1;
};

template <int NC>
size_t outerSmem() {
  constexpr int BLK = NC * NC;
  const size_t loop = sizeof(float2) * 8 * 4 * BLK;
  const size_t table = sizeof(float2) * size_t(NC) * NC * (NC + 1);
  return 16 * 8 + 4 * (BLK + NC + 4) + std::max(loop, table);
}

template <int NC>
void launchOuter(const G4Args& a, const float2* G, long stride, const float2* disc, cudaStream_t stream) {
  const TpDims& d = a.dims;
  constexpr int TA = OuterTile<NC>::TA, TB = OuterTile<NC>::TB;
  const size_t smem = outerSmem<NC>();
  auto k = updateG4SinglebandOuter<NC, TA, TB>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long blocks = long(d.nw) * d.nw * d.nwq;
  constexpr int threads = NC * (NC / TA) * (NC / TB);
  k<<<static_cast<unsigned>(blocks), threads, smem, stream>>>(d, G, stride, a.signs, a.n_slots, a.k_sub, a.q_list,
                                                              a.wex_list, disc, a.G4, a.atomic, a.err);
  DCAACC_LAUNCH_CHECK();
}

template <int NC, bool MAG, bool CHARGE>
void launchBatched(const G4Args& a, const float2* G, long stride, cudaStream_t stream) {
  const TpDims& d = a.dims;
  const int q_chunk = std::max(1, std::min(d.nq, 256 / NC));
  const int threads = NC * q_chunk;
  const int qp = q_chunk + 1;
  const size_t smem = 16 + sizeof(float2) * (2 * 8 * NC * NC + 4 * NC * qp);
  auto k = updateG4SinglebandBatched<NC, MAG, CHARGE>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int n_qchunks = (d.nq + q_chunk - 1) / q_chunk;
  const long blocks = long(d.nw) * d.nw * d.nwq * n_qchunks;
  k<<<static_cast<unsigned>(blocks), threads, smem, stream>>>(d, G, stride, a.signs, a.n_slots, a.k_add,
                                                              a.q_list, a.wex_list, a.G4, a.atomic, q_chunk,
                                                              a.err);
  DCAACC_LAUNCH_CHECK();
}

template <int NC>
void launchDirect(const G4Args& a, const float2* G, long stride, const float2* disc, cudaStream_t stream) {
  const TpDims& d = a.dims;
  const int q_chunk = std::max(1, std::min(d.nq, 256 / NC));
  const int threads = NC * q_chunk;
  const int qp = q_chunk + 1;
  const size_t smem = 16 + sizeof(float2) * std::max<size_t>(2 * 4 * NC * NC, size_t(NC) * NC * qp);
  auto k = updateG4SinglebandDirect<NC>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int n_qchunks = (d.nq + q_chunk - 1) / q_chunk;
  const long blocks = long(d.nw) * d.nw * d.nwq * n_qchunks;
  k<<<static_cast<unsigned>(blocks), threads, smem, stream>>>(d, G, stride, a.signs, a.n_slots, a.k_add,
                                                              a.q_list, a.wex_list, disc, a.G4, a.atomic,
                                                              q_chunk, a.err);
  DCAACC_LAUNCH_CHECK();
}

template <int NC>
int launchForNc(const G4Args& a, const float2* G, long stride, bool mag, bool charge, cudaStream_t s) {
  if (const float2* disc = launchDiscGemm(a, G, stride, s)) {
    if (NC == 16 && directTcApplies(a))
      launchDirectTc(a, G, stride, disc, a.n_sm, s);
    else if (a.q_all)
      launchOuter<NC>(a, G, stride, disc, s);
    else
      launchDirect<NC>(a, G, stride, disc, s);
    return 3;
  }
  if (mag && charge)
    launchBatched<NC, true, true>(a, G, stride, s);
  else if (mag)
    launchBatched<NC, true, false>(a, G, stride, s);
  else
    launchBatched<NC, false, true>(a, G, stride, s);
  return 1;
}

}  // namespace

int launchUpdateG4SinglebandBatched(const G4Args& a, const float2* G, long g_sector_stride,
                                    cudaStream_t stream) {
  const TpDims& d = a.dims;
  if (!singlebandBatchedApplies(d))
    return 0;
  bool mag = false, charge = false;
  for (int c = 0; c < d.n_channels; ++c)
    (d.channels[c] == 2 ? mag : charge) = true;
  switch (d.nc) {
    case 4:
      return launchForNc<4>(a, G, g_sector_stride, mag, charge, stream);
    case 8:
      return launchForNc<8>(a, G, g_sector_stride, mag, charge, stream);
    case kSplitNc:
      // Disconnected terms on the tensor cores and the split direct term (both read mirrored
      // blocks for half G and run the w1 >= Nw / 2 tiles for half G4); without the workspace or
      // with a subset of the transfers, the general one-band kernel (return 0; half G is never
      // enabled then).
      if (!a.q_all || a.n_slots > kSplitMaxSlots)
        return 0;
      if (const float2* disc = launchDiscGemm(a, G, g_sector_stride, stream)) {
        launchOuterSplit(a, G, g_sector_stride, disc, stream);
        return 3;
      }
      return 0;
    default:
      return launchForNc<16>(a, G, g_sector_stride, mag, charge, stream);
  }
}

bool singlebandBatchedApplies(const TpDims& d) {
  if (d.nb != 1 || (d.nc != 4 && d.nc != 8 && d.nc != 16 && d.nc != kSplitNc))
    return false;
  for (int c = 0; c < d.n_channels; ++c)
    if (d.channels[c] != 2 && d.channels[c] != 3)
      return false;
  return d.n_channels > 0;
}

}  // namespace dcaacc
