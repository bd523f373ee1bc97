// Particle-particle up-down update of a multiband model, mixed path (FP32 G, FP32 batch sums).
//
// Channel PARTICLE_PARTICLE_UP_DOWN (tp_accumulator_cpu.hpp:628-661, updateG4Kernel's PP branch in
// tp_accumulator_kernels.cu):
//   G4(k1, w1, k2, w2, q, wq; b1, b2, b3, b4) += s/2 sum_sigma G_sigma(k1, w1; k2, w2)[b1, b3]
//                                               x G_-sigma(q - k1, m1; q - k2, m2)[b2, b4],
//   m = wq + Nw - 1 - w.
// For fixed (k1, k2, q, w1, w2, wq) the nb^4 entries are a sum of Kronecker products of two nb x nb
// band blocks.  A thread owns one (k1, k2, q, b4) and keeps the nb^3 entries (b1, b2, b3) in
// registers for the whole batch: per measurement and spin it reads nb^2 elements of the A block
// G(w1; w2) and nb of the P block G(m1; m2) and does nb^3 complex FMAs (27 per 12 reads for three
// bands), where the generic staged kernel (tp_g4.cu) reads two elements per entry.  CTA = one
// (w1, w2, wq) tile; per measurement the two spins' A and P blocks (R x R each, R = nb Nc) arrive in
// shared memory by the bulk-copy engine through a four-stage ring.  Items (k1, k2, q, b4) are
// numbered q fastest, then k2, so that the A reads of a warp are broadcasts; items beyond the
// CTA's threads take further passes over the batch.  The batch sum of each entry goes into the
// FP64 running sum with one read-modify-write, as in the staged kernel, spread over the next pass;
// the band indices follow its G layout (element (b3, k1; b1, k2) of the A block, (b4, q - k1;
// b2, q - k2) of the P block).
#include <cuda_runtime.h>

#include "async_copy.cuh"
#include "common.cuh"
#include "tp_g4.hpp"
#include "tp_layout.hpp"

namespace dcaacc {

namespace {

constexpr int kPPThreads = 512;
constexpr int kPPStages = 4;  // ring of per-measurement block sets: copies run three steps ahead

template <int NB, int NC>
__global__ void __launch_bounds__(kPPThreads, 1)
updateG4PPMultibandKernel(const TpDims dims, const float2* __restrict__ G, long g_sector_stride,
                          const int* __restrict__ signs, int n_slots, const int* __restrict__ k_sub,
                          const int* __restrict__ q_list, const int* __restrict__ wex_list,
                          double2* const* __restrict__ G4, bool atomic, int* __restrict__ err, uint32_t wait_limit) {
  constexpr int NB2 = NB * NB, NB3 = NB2 * NB, NB4 = NB3 * NB;
  constexpr int nc = NC, R = NB * NC;  // compile-time block shape: the band offsets are immediates
  const int nw = dims.nw, nw_ext = dims.nw_ext, nq = dims.nq, ext = dims.ext;
  // wq fastest: the CTAs that read the same A block G(w1; w2) run side by side (one L2 fetch).
  const int iwq = blockIdx.x, w2 = blockIdx.y, w1 = blockIdx.z;
  const int wex = wex_list[iwq];
  constexpr long blk = static_cast<long>(R) * R;
  const int n_items = nc * nc * nq * NB;
  const int n_passes = (n_items + kPPThreads - 1) / kPPThreads;
  const long n_steps = static_cast<long>(n_passes) * n_slots;
  const int m1 = wex + nw - 1 - w1 + ext, m2 = wex + nw - 1 - w2 + ext;
  const long offA = (static_cast<long>(w1 + ext) * nw_ext + w2 + ext) * blk;
  const long offP = (static_cast<long>(m1) * nw_ext + m2) * blk;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);     // [kPPStages] a stage's copies landed
  uint64_t* empty = bar + kPPStages;                         // [kPPStages] every warp is done with it
  float2* stage = reinterpret_cast<float2*>(smem_raw + 64);  // [kPPStages][spin][A, P][R * R]
  const uint32_t blk_bytes = static_cast<uint32_t>(blk * sizeof(float2));
  auto issue = [&](long step) {
    const int st = static_cast<int>(step % kPPStages);
    const int slot = static_cast<int>(step % n_slots);
    float2* dst = stage + st * 4 * blk;
    mbarArriveExpectTx(&bar[st], 4 * blk_bytes);
    for (int s = 0; s < 2; ++s) {
      const float2* src = G + g_sector_stride * (2 * slot + s);
      bulkCopyG2S(dst + (2 * s) * blk, src + offA, blk_bytes, &bar[st]);
      bulkCopyG2S(dst + (2 * s + 1) * blk, src + offP, blk_bytes, &bar[st]);
    }
  };
  const int t = threadIdx.x;
  const int lane = t % 32;
  if (t == 0) {
    for (int i = 0; i < kPPStages; ++i) {
      mbarInit(&bar[i], 1);
      mbarInit(&empty[i], kPPThreads / 32);
    }
    fenceBarrierInit();
  }
  __syncthreads();
  if (t == 0)
    for (long i = 0; i < kPPStages && i < n_steps; ++i)
      issue(i);

  // G4 strides: entry (b1, b2, b3, b4) + nb^4 (k1 + Nc (w1 + Nw (k2 + Nc (w2 + Nw (q + Nq wq))))).
  const long s_w1 = static_cast<long>(NB4) * nc, s_k2 = s_w1 * nw, s_w2 = s_k2 * nc, s_q = s_w2 * nw,
             s_wq = s_q * nq;
  double2* g4t = G4[0] + w1 * s_w1 + w2 * s_w2 + iwq * s_wq;
  const uint32_t limit = wait_limit ? wait_limit : kWaitLimit;
  // A pass's batch sums wait in shared memory ([entry][thread]) and go into the FP64 running sum
  // one entry per measurement step of the next pass, so that the read-modify-write latency hides
  // behind that step's FMAs (the last pass's sums go at the end).
  float2* fb = stage + kPPStages * 4 * blk;
  int* sgn = reinterpret_cast<int*>(fb + NB3 * kPPThreads);  // [n_slots] the measurements' signs
  for (int i = t; i < n_slots; i += kPPThreads)
    sgn[i] = signs[i];
  __syncthreads();  // the signs are in place before any warp's first step
  long pend = -1;  // G4 offset of this thread's pending item
  int fe = NB3;    // its next entry to write
  auto flushEntry = [&](double2* dst, float2 v, double2 old) {
    if (atomic) {
      atomicAdd(&dst->x, static_cast<double>(v.x));
      atomicAdd(&dst->y, static_cast<double>(v.y));
    }
    else {
      old.x += static_cast<double>(v.x);
      old.y += static_cast<double>(v.y);
      *dst = old;
    }
  };
  auto entryPtr = [&](int e) {  // e = b1 + nb b2 + nb^2 b3: consecutive entries are contiguous
    return g4t + pend + e;
  };
  auto flushRest = [&]() {
    if (pend >= 0 && fe == 0 && !atomic) {  // a whole item: all reads before the writes
      double2 old[NB3];
#pragma unroll
      for (int e = 0; e < NB3; ++e)
        old[e] = *entryPtr(e);
#pragma unroll
      for (int e = 0; e < NB3; ++e)
        flushEntry(entryPtr(e), fb[e * kPPThreads + t], old[e]);
      fe = NB3;
    }
    for (; pend >= 0 && fe < NB3; ++fe) {
      double2* dst = entryPtr(fe);
      flushEntry(dst, fb[fe * kPPThreads + t], atomic ? make_double2(0., 0.) : *dst);
    }
  };
  long step = 0;
  bool ok = true;
  for (int pass = 0; pass < n_passes; ++pass) {
    const int item = t + kPPThreads * pass;
    const bool live = item < n_items;
    const int it = live ? item : 0;
    const int iq = it % nq, k2 = (it / nq) % nc, b4 = (it / (nq * nc)) % NB, k1 = it / (nq * nc * NB);
    const int q = q_list[iq];
    const int qk1 = k_sub[k1 + nc * q], qk2 = k_sub[k2 + nc * q];
    const int aoff = NB * k1 * R + NB * k2;          // element (b1, b3) at + b3 R + b1
    const int poff = (b4 + NB * qk1) * R + NB * qk2;  // element b2 at + b2
    const long g4o = NB3 * b4 + static_cast<long>(NB4) * k1 + k2 * s_k2 + iq * s_q;
    float2 acc[NB][NB][NB];  // [b1][b2][b3]
#pragma unroll
    for (int b1 = 0; b1 < NB; ++b1)
#pragma unroll
      for (int b2 = 0; b2 < NB; ++b2)
#pragma unroll
        for (int b3 = 0; b3 < NB; ++b3)
          acc[b1][b2][b3] = make_float2(0.f, 0.f);

    for (int slot = 0; slot < n_slots; ++slot, ++step) {
      const int st = static_cast<int>(step % kPPStages);
      // One pending entry of the previous pass: its FP64 value is read here, written after the FMAs.
      double2* fdst = nullptr;
      float2 fv = make_float2(0.f, 0.f);
      double2 fold = make_double2(0., 0.);
      if (pend >= 0 && fe < NB3) {
        fdst = entryPtr(fe);
        fv = fb[fe * kPPThreads + t];
        if (!atomic)
          fold = *fdst;
      }
      const uint32_t phase = static_cast<uint32_t>((step / kPPStages) & 1);
      ok = __all_sync(0xffffffffu, mbarWait(&bar[st], phase, err, limit));
      if (!ok)
        break;
      const float2* A0 = stage + st * 4 * blk;
      const float2* P0 = A0 + blk;
      const float2* A1 = A0 + 2 * blk;
      const float2* P1 = A0 + 3 * blk;
      if (live) {
        const float hs = 0.5f * static_cast<float>(sgn[slot]);
        float2 p0[NB], p1[NB];  // s/2 P_sigma(b4, q - k1; b2, q - k2)
#pragma unroll
        for (int b2 = 0; b2 < NB; ++b2) {
          const float2 x0 = P0[poff + b2], x1 = P1[poff + b2];
          p0[b2] = make_float2(hs * x0.x, hs * x0.y);
          p1[b2] = make_float2(hs * x1.x, hs * x1.y);
        }
#pragma unroll
        for (int b3 = 0; b3 < NB; ++b3)
#pragma unroll
          for (int b1 = 0; b1 < NB; ++b1) {
            const float2 a0 = A0[aoff + b3 * R + b1], a1 = A1[aoff + b3 * R + b1];
#pragma unroll
            for (int b2 = 0; b2 < NB; ++b2) {
              cfma(acc[b1][b2][b3], a0, p1[b2]);
              cfma(acc[b1][b2][b3], a1, p0[b2]);
            }
          }
      }
      if (fdst) {
        flushEntry(fdst, fv, fold);
        ++fe;
      }
      __syncwarp();
      if (lane == 0)
        mbarArrive(&empty[st]);  // release: this warp's reads of the stage are done
      if (t == 0 && step + kPPStages < n_steps) {
        if (!mbarWait(&empty[st], phase, err, limit)) {
          ok = false;  // the other warps see the missing copies as a timeout of their own
          break;
        }
        fenceProxyAsync();
        issue(step + kPPStages);
      }
    }
    if (__syncthreads_or(!ok))
      return;  // uniform bail-out; the host reports the error word
    flushRest();  // batches shorter than nb^3 measurements leave entries of the previous pass
    if (live) {
#pragma unroll
      for (int b3 = 0; b3 < NB; ++b3)
#pragma unroll
        for (int b2 = 0; b2 < NB; ++b2)
#pragma unroll
          for (int b1 = 0; b1 < NB; ++b1)
            fb[(b1 + NB * b2 + NB2 * b3) * kPPThreads + t] = acc[b1][b2][b3];
      pend = g4o;
      fe = 0;
    }
    else {
      pend = -1;
    }
  }
  flushRest();
}

}  // namespace

bool launchUpdateG4PPMultiband(const G4Args& a, const float2* G, long g_sector_stride, cudaStream_t stream) {
  const TpDims& d = a.dims;
  if (d.n_channels != 1 || d.channels[0] != 4 /* PARTICLE_PARTICLE_UP_DOWN */ || d.nb != 3 || d.half_g4 || d.half_g ||
      a.n_slots < 1 || (d.nc != 4 && d.nc != 8))
    return false;
  const size_t smem = 64 + kPPStages * 4 * size_t(d.R) * d.R * sizeof(float2) +
                      27 * size_t(kPPThreads) * sizeof(float2) + sizeof(int) * size_t(a.n_slots);
  if (smem > 220 * 1024)
    return false;
  auto k = d.nc == 4 ? updateG4PPMultibandKernel<3, 4> : updateG4PPMultibandKernel<3, 8>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const dim3 grid(d.nwq, d.nw, d.nw);
  k<<<grid, kPPThreads, smem, stream>>>(d, G, g_sector_stride, a.signs, a.n_slots, a.k_sub, a.q_list, a.wex_list,
                                         a.G4, a.atomic, a.err, a.wait_limit);
  DCAACC_LAUNCH_CHECK();
  return true;
}

}  // namespace dcaacc
