// G4 update: G4(b1,b2,b3,b4,k1,w1,k2,w2,q,wq) += sum over a batch of measurements.
//
// Replaces the reference's updateG4Kernel (tp_accumulator_kernels.cu:255-681, one thread per G4
// entry with a 10-level div/mod unroll of its linear index and one launch per channel per
// measurement) by one kernel that:
//   * assigns a CTA to a (w1, w2, wq) tile and lets its threads walk the tile's entries in G4's
//     memory order (b1..b4, k1 contiguous; k2, q strided), so every G4 load and store is coalesced
//     and each G4 entry is read and written exactly once per launch;
//   * updates every configured channel in the same pass (the channels share the G blocks);
//   * loops over all measurements of a batch with the partial sums in registers, then adds them
//     to the FP64 running G4 once (the FP32-partials mode of the mixed path); with a batch of one
//     and FP64 G and partials it is the plain FP64 update.
//
// Channel formulas (spin-symmetric branch of TpAccumulator<CPU>::updateG4,
// tp_accumulator_cpu.hpp:452-666), written with Gd_s(r, wr; c, wc) = G_(b_r, b_c, s, k_r, k_c, wr, wc),
// r = b + nb k, the band transpose of getGMultiband (tp_accumulator_cpu.hpp:389-405) applied:
//   PH_MAGNETIC  s/2 [ dG(b1 k1, w1; b2 k1+q, w1+x) dG(b4 k2+q, w2+x; b3 k2, w2)
//                      - sum_s Gd_s(b1 k1, w1; b3 k2, w2) Gd_s(b4 k2+q, w2+x; b2 k1+q, w1+x) ],
//                dG = Gd_0 - Gd_1
//   PH_CHARGE    s/2 [ sG(b1 k1, w1; b2 k1+q, w1+x) sG(b4 k2+q, w2+x; b3 k2, w2)
//                      - sum_s Gd_s(b4 k1, w1; b1 k2, w2) Gd_s(b3 k2+q, w2+x; b2 k1+q, w1+x) ],
//                sG = Gd_0 + Gd_1
//   PH_TRANSVERSE  -s/2 sum_s Gd_s(b4 k1, w1; b2 k2, w2) Gd_{!s}(b1 k2+q, w2+x; b3 k1+q, w1+x)
//   PP_UP_DOWN      s/2 sum_s Gd_s(b3 k1, w1; b1 k2, w2) Gd_{!s}(b4 q-k1, m1; b2 q-k2, m2),
//                m = x + Nw - 1 - w
// with s the measurement sign, x the frequency transfer, compact w shifted by ext onto the
// extended mesh of G.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "async_copy.cuh"
#include "common.cuh"
#include "tp_g4.hpp"

namespace dcaacc {

namespace {

template <typename GT, typename AT>
__device__ inline cplx_t<AT> ldG(const GT* p) {
  const GT v = __ldg(p);
  return mk(static_cast<AT>(v.x), static_cast<AT>(v.y));
}

template <typename GT, typename AT, int EPT>
__global__ void __launch_bounds__(256)
updateG4Kernel(const TpDims dims, const GT* __restrict__ G, long g_sector_stride,
               const int* __restrict__ signs, int n_slots, const int* __restrict__ k_add,
               const int* __restrict__ k_sub, const int* __restrict__ q_list,
               const int* __restrict__ wex_list, double2* const* __restrict__ G4, bool atomic) {
  using C = cplx_t<AT>;
  const int nb = dims.nb, nc = dims.nc, nw = dims.nw, nw_ext = dims.nw_ext, R = dims.R;
  const int w1 = blockIdx.x, w2 = blockIdx.y, iwq = blockIdx.z;
  const int wex = wex_list[iwq];
  const int ext = dims.ext;
  const int nb2 = nb * nb, nb4 = nb2 * nb2;
  const int inner = nb4 * nc;                 // (b1, b2, b3, b4, k1)
  const long per_tile = static_cast<long>(inner) * nc * dims.nq;
  const long blk_stride = static_cast<long>(R) * R;

  // Extended frequency indices of the blocks this tile reads.
  const int w1e = w1 + ext, w2e = w2 + ext;
  const int w1x = w1e + wex, w2x = w2e + wex;
  const int m1 = wex + nw - 1 - w1 + ext, m2 = wex + nw - 1 - w2 + ext;
  auto blk = [&](int wr, int wc) { return (static_cast<long>(wr) * nw_ext + wc) * blk_stride; };
  const long bA = blk(w1e, w2e), bB = blk(w2x, w1x), bC = blk(w1e, w1x), bE = blk(w2x, w2e),
             bP = blk(m1, m2);

  // G4 offset of (b=0, k1=0, w1, k2=0, w2, q=0, wq): strides of the (k2, q) part follow.
  const long s_w1 = inner;
  const long s_k2 = s_w1 * nw;
  const long s_w2 = s_k2 * nc;
  const long s_q = s_w2 * nw;
  const long s_wq = s_q * dims.nq;
  const long tile_base = w1 * s_w1 + w2 * s_w2 + iwq * s_wq;

  for (long chunk = 0; chunk < per_tile; chunk += static_cast<long>(EPT) * blockDim.x) {
    C acc[EPT][kMaxChannels];
#pragma unroll
    for (int e = 0; e < EPT; ++e)
#pragma unroll
      for (int c = 0; c < kMaxChannels; ++c)
        acc[e][c] = mk(AT(0), AT(0));

    for (int slot = 0; slot < n_slots; ++slot) {
      const AT half_sign = AT(0.5) * static_cast<AT>(signs[slot]);
      const GT* G0s = G + g_sector_stride * (2 * slot);
      const GT* G1s = G0s + g_sector_stride;
#pragma unroll
      for (int e = 0; e < EPT; ++e) {
        const long idx = chunk + threadIdx.x + static_cast<long>(e) * blockDim.x;
        if (idx >= per_tile)
          break;
        const int in = static_cast<int>(idx % inner);
        const int outer = static_cast<int>(idx / inner);  // k2 + nc * q
        const int b1 = in % nb, b2 = (in / nb) % nb, b3 = (in / nb2) % nb, b4 = (in / (nb2 * nb)) % nb;
        const int k1 = in / nb4;
        const int k2 = outer % nc, iq = outer / nc;
        const int q = q_list[iq];
        const int k1q = k_add[k1 + nc * q], k2q = k_add[k2 + nc * q];
        auto rc = [&](int b, int k) { return b + nb * k; };
#pragma unroll
        for (int c = 0; c < kMaxChannels; ++c) {
          if (c >= dims.n_channels)
            break;
          const int ch = dims.channels[c];
          C v = mk(AT(0), AT(0));
          if (ch == 2 || ch == 3) {  // PH_MAGNETIC / PH_CHARGE
            const long ia = bC + rc(b1, k1) * R + rc(b2, k1q);
            const long ib = bE + rc(b4, k2q) * R + rc(b3, k2);
            const C a0 = ldG<GT, AT>(G0s + ia), a1 = ldG<GT, AT>(G1s + ia);
            const C e0 = ldG<GT, AT>(G0s + ib), e1 = ldG<GT, AT>(G1s + ib);
            const AT sg = ch == 2 ? AT(-1) : AT(1);
            const C u = mk(a0.x + sg * a1.x, a0.y + sg * a1.y);
            const C w = mk(e0.x + sg * e1.x, e0.y + sg * e1.y);
            v = cmul(u, w);
            long id, ie;
            if (ch == 2) {
              id = bA + rc(b1, k1) * R + rc(b3, k2);
              ie = bB + rc(b4, k2q) * R + rc(b2, k1q);
            }
            else {
              id = bA + rc(b4, k1) * R + rc(b1, k2);
              ie = bB + rc(b3, k2q) * R + rc(b2, k1q);
            }
            C d = cmul(ldG<GT, AT>(G0s + id), ldG<GT, AT>(G0s + ie));
            cfma(d, ldG<GT, AT>(G1s + id), ldG<GT, AT>(G1s + ie));
            v = csub(v, d);
          }
          else if (ch == 1) {  // PH_TRANSVERSE
            const long id = bA + rc(b4, k1) * R + rc(b2, k2);
            const long ie = bB + rc(b1, k2q) * R + rc(b3, k1q);
            C d = cmul(ldG<GT, AT>(G0s + id), ldG<GT, AT>(G1s + ie));
            cfma(d, ldG<GT, AT>(G1s + id), ldG<GT, AT>(G0s + ie));
            v = mk(-d.x, -d.y);
          }
          else if (ch == 4) {  // PP_UP_DOWN
            const int qk1 = k_sub[k1 + nc * q], qk2 = k_sub[k2 + nc * q];
            const long id = bA + rc(b3, k1) * R + rc(b1, k2);
            const long ie = bP + rc(b4, qk1) * R + rc(b2, qk2);
            v = cmul(ldG<GT, AT>(G0s + id), ldG<GT, AT>(G1s + ie));
            cfma(v, ldG<GT, AT>(G1s + id), ldG<GT, AT>(G0s + ie));
          }
          acc[e][c].x = fma(half_sign, v.x, acc[e][c].x);
          acc[e][c].y = fma(half_sign, v.y, acc[e][c].y);
        }
      }
    }

    // One read-modify-write of the FP64 running sum per entry and channel.
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const long idx = chunk + threadIdx.x + static_cast<long>(e) * blockDim.x;
      if (idx >= per_tile)
        break;
      const int in = static_cast<int>(idx % inner);
      const int outer = static_cast<int>(idx / inner);
      const int k2 = outer % nc, iq = outer / nc;
      const long g4i = tile_base + in + k2 * s_k2 + iq * s_q;
#pragma unroll
      for (int c = 0; c < kMaxChannels; ++c) {
        if (c >= dims.n_channels)
          break;
        double2* p = G4[c] + g4i;
        if (atomic) {
          atomicAdd(&p->x, static_cast<double>(acc[e][c].x));
          atomicAdd(&p->y, static_cast<double>(acc[e][c].y));
        }
        else {
          double2 old = *p;
          old.x += static_cast<double>(acc[e][c].x);
          old.y += static_cast<double>(acc[e][c].y);
          *p = old;
        }
      }
    }
  }
}


// Any number of bands, at most two channels: the same entries and formulas as updateG4Kernel,
// with the G blocks a tile reads (A, B, C, E, P below, per channel set) staged in shared memory
// for each measurement by the bulk-copy engine (two-stage ring) instead of gathered from L2 per
// entry and measurement.  A thread keeps EPT entries; their block offsets are computed once per
// chunk of entries, the measurement loop then reads shared memory only.  The (chunk, measurement)
// steps form one sequence, so the ring keeps running across chunks.
//   A = G(w1; w2)  B = G(w2+x; w1+x)  C = G(w1; w1+x)  E = G(w2+x; w2)  P = G(m1; m2)
constexpr int kStagedMaxCh = 2;

// EPT entries per thread: every chunk of EPT x 256 entries re-stages the tile's blocks for each
// measurement, so a larger EPT cuts that traffic; NCH = number of channels (registers for NCH only).
// The sum of an entry is the same whatever EPT, so the launch-shape tuner chooses it.
template <typename GT, typename AT, int EPT, int NCH>
__global__ void __launch_bounds__(256)
updateG4StagedKernel(const TpDims dims, const GT* __restrict__ G, long g_sector_stride,
                     const int* __restrict__ signs, int n_slots, const int* __restrict__ k_add,
                     const int* __restrict__ k_sub, const int* __restrict__ q_list,
                     const int* __restrict__ wex_list, double2* const* __restrict__ G4, bool atomic,
                     int* __restrict__ err) {
  using C = cplx_t<AT>;
  static_assert(NCH >= 1 && NCH <= kStagedMaxCh, "channels");
  const int nb = dims.nb, nc = dims.nc, nw = dims.nw, nw_ext = dims.nw_ext, R = dims.R;
  const int w1 = blockIdx.x, w2 = blockIdx.y, iwq = blockIdx.z;
  const int wex = wex_list[iwq];
  const int ext = dims.ext;
  const int nb2 = nb * nb, nb4 = nb2 * nb2;
  const int inner = nb4 * nc;
  const long per_tile = static_cast<long>(inner) * nc * dims.nq;
  const long blk = static_cast<long>(R) * R;
  const int n_ch = dims.n_channels;

  // Blocks of this tile: slot index in the stage (-1: not needed).
  bool need[5] = {false, false, false, false, false};  // A B C E P
  for (int c = 0; c < n_ch; ++c) {
    const int ch = dims.channels[c];
    need[0] = true;
    if (ch == 1 || ch == 2 || ch == 3)
      need[1] = true;
    if (ch == 2 || ch == 3)
      need[2] = need[3] = true;
    if (ch == 4)
      need[4] = true;
  }
  const int w1e = w1 + ext, w2e = w2 + ext, w1x = w1e + wex, w2x = w2e + wex;
  const int m1 = wex + nw - 1 - w1 + ext, m2 = wex + nw - 1 - w2 + ext;
  auto blkOff = [&](int wr, int wc) { return (static_cast<long>(wr) * nw_ext + wc) * blk; };
  const long boffAll[5] = {blkOff(w1e, w2e), blkOff(w2x, w1x), blkOff(w1e, w1x), blkOff(w2x, w2e), blkOff(m1, m2)};
  int sidx[5];
  long boff[5];
  int nblk = 0;
  for (int b = 0; b < 5; ++b) {
    sidx[b] = need[b] ? nblk : -1;
    if (need[b])
      boff[nblk++] = boffAll[b];
  }

  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);  // [2]
  GT* stage = reinterpret_cast<GT*>(smem_raw + 16);       // [2][2 spins][nblk][R*R]
  const long stage_elems = 2L * nblk * blk;
  const uint32_t blk_bytes = static_cast<uint32_t>(blk * sizeof(GT));
  const long n_chunks = (per_tile + static_cast<long>(EPT) * blockDim.x - 1) / (static_cast<long>(EPT) * blockDim.x);
  const long n_steps = n_chunks * n_slots;
  auto issue = [&](long step) {
    const int st = static_cast<int>(step & 1);
    const int slot = static_cast<int>(step % n_slots);
    GT* dst = stage + st * stage_elems;
    mbarArriveExpectTx(&bar[st], 2 * nblk * blk_bytes);
    for (int s = 0; s < 2; ++s) {
      const GT* src = G + g_sector_stride * (2 * slot + s);
      for (int b = 0; b < nblk; ++b)
        bulkCopyG2S(dst + (s * nblk + b) * blk, src + boff[b], blk_bytes, &bar[st]);
    }
  };
  const int t = threadIdx.x;
  if (t == 0) {
    mbarInit(&bar[0], 1);
    mbarInit(&bar[1], 1);
    fenceBarrierInit();
  }
  __syncthreads();
  if (t == 0) {
    issue(0);
    if (n_steps > 1)
      issue(1);
  }

  const long s_w1 = inner, s_k2 = s_w1 * nw, s_w2 = s_k2 * nc, s_q = s_w2 * nw, s_wq = s_q * dims.nq;
  const long tile_base = w1 * s_w1 + w2 * s_w2 + iwq * s_wq;
  long step = 0;
  for (long chunk = 0; chunk < n_chunks; ++chunk) {
    // This chunk's entries: G4 index and, per channel, the shared-memory offsets of the two G
    // elements of the second-order term (id in A, ie in B or P) and, for PH magnetic / charge,
    // of the disconnected-term elements (iu in C, iv in E).
    int g4o[EPT];  // offset from the tile base (a tile holds fewer than 2^31 entries)
    int id[EPT][NCH], ie[EPT][NCH], iu[EPT], iv[EPT];
    bool live[EPT];
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const long idx = chunk * EPT * blockDim.x + t + static_cast<long>(e) * blockDim.x;
      live[e] = idx < per_tile;
      const long ii = live[e] ? idx : 0;
      const int in = static_cast<int>(ii % inner);
      const int outer = static_cast<int>(ii / inner);
      const int b1 = in % nb, b2 = (in / nb) % nb, b3 = (in / nb2) % nb, b4 = (in / (nb2 * nb)) % nb;
      const int k1 = in / nb4;
      const int k2 = outer % nc, iq = outer / nc;
      const int q = q_list[iq];
      const int k1q = k_add[k1 + nc * q], k2q = k_add[k2 + nc * q];
      auto rc = [&](int b, int k) { return b + nb * k; };
      g4o[e] = static_cast<int>(in + k2 * s_k2 + iq * s_q);
      iu[e] = rc(b1, k1) * R + rc(b2, k1q);
      iv[e] = rc(b4, k2q) * R + rc(b3, k2);
#pragma unroll
      for (int c = 0; c < NCH; ++c) {
        const int ch = dims.channels[c];
        if (ch == 2) {
          id[e][c] = rc(b1, k1) * R + rc(b3, k2);
          ie[e][c] = rc(b4, k2q) * R + rc(b2, k1q);
        }
        else if (ch == 3) {
          id[e][c] = rc(b4, k1) * R + rc(b1, k2);
          ie[e][c] = rc(b3, k2q) * R + rc(b2, k1q);
        }
        else if (ch == 1) {
          id[e][c] = rc(b4, k1) * R + rc(b2, k2);
          ie[e][c] = rc(b1, k2q) * R + rc(b3, k1q);
        }
        else {
          const int qk1 = k_sub[k1 + nc * q], qk2 = k_sub[k2 + nc * q];
          id[e][c] = rc(b3, k1) * R + rc(b1, k2);
          ie[e][c] = rc(b4, qk1) * R + rc(b2, qk2);
        }
      }
    }
    C acc[EPT][NCH];
#pragma unroll
    for (int e = 0; e < EPT; ++e)
#pragma unroll
      for (int c = 0; c < NCH; ++c)
        acc[e][c] = mk(AT(0), AT(0));

    for (int slot = 0; slot < n_slots; ++slot, ++step) {
      const int st = static_cast<int>(step & 1);
      const bool ok = mbarWait(&bar[st], static_cast<uint32_t>((step >> 1) & 1), err);
      if (!__syncthreads_and(ok))
        return;  // uniform bail-out; the host reports the error word
      const GT* S0 = stage + st * stage_elems;
      const GT* S1 = S0 + nblk * blk;
      auto ld = [](const GT* p) { return mk(static_cast<AT>(p->x), static_cast<AT>(p->y)); };
      const AT half_sign = AT(0.5) * static_cast<AT>(signs[slot]);
#pragma unroll
      for (int e = 0; e < EPT; ++e) {
        if (!live[e])
          continue;
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
          const int ch = dims.channels[c];
          C v;
          if (ch == 2 || ch == 3) {
            const GT* Cb0 = S0 + sidx[2] * blk;
            const GT* Cb1 = S1 + sidx[2] * blk;
            const GT* Eb0 = S0 + sidx[3] * blk;
            const GT* Eb1 = S1 + sidx[3] * blk;
            const C a0 = ld(Cb0 + iu[e]), a1 = ld(Cb1 + iu[e]), e0 = ld(Eb0 + iv[e]), e1 = ld(Eb1 + iv[e]);
            const AT sg = ch == 2 ? AT(-1) : AT(1);
            v = cmul(mk(a0.x + sg * a1.x, a0.y + sg * a1.y), mk(e0.x + sg * e1.x, e0.y + sg * e1.y));
            const GT* Ab0 = S0 + sidx[0] * blk;
            const GT* Ab1 = S1 + sidx[0] * blk;
            const GT* Bb0 = S0 + sidx[1] * blk;
            const GT* Bb1 = S1 + sidx[1] * blk;
            C d = cmul(ld(Ab0 + id[e][c]), ld(Bb0 + ie[e][c]));
            cfma(d, ld(Ab1 + id[e][c]), ld(Bb1 + ie[e][c]));
            v = csub(v, d);
          }
          else if (ch == 1) {
            const GT* Ab0 = S0 + sidx[0] * blk;
            const GT* Ab1 = S1 + sidx[0] * blk;
            const GT* Bb0 = S0 + sidx[1] * blk;
            const GT* Bb1 = S1 + sidx[1] * blk;
            C d = cmul(ld(Ab0 + id[e][c]), ld(Bb1 + ie[e][c]));
            cfma(d, ld(Ab1 + id[e][c]), ld(Bb0 + ie[e][c]));
            v = mk(-d.x, -d.y);
          }
          else {
            const GT* Ab0 = S0 + sidx[0] * blk;
            const GT* Ab1 = S1 + sidx[0] * blk;
            const GT* Pb0 = S0 + sidx[4] * blk;
            const GT* Pb1 = S1 + sidx[4] * blk;
            v = cmul(ld(Ab0 + id[e][c]), ld(Pb1 + ie[e][c]));
            cfma(v, ld(Ab1 + id[e][c]), ld(Pb0 + ie[e][c]));
          }
          acc[e][c].x = fma(half_sign, v.x, acc[e][c].x);
          acc[e][c].y = fma(half_sign, v.y, acc[e][c].y);
        }
      }
      __syncthreads();  // stage st is free again
      if (t == 0 && step + 2 < n_steps) {
        fenceProxyAsync();
        issue(step + 2);
      }
    }

    // One read-modify-write of the FP64 running sum per entry and channel.
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      if (!live[e])
        continue;
#pragma unroll
      for (int c = 0; c < NCH; ++c) {
        double2* p = G4[c] + tile_base + g4o[e];
        if (atomic) {
          atomicAdd(&p->x, static_cast<double>(acc[e][c].x));
          atomicAdd(&p->y, static_cast<double>(acc[e][c].y));
        }
        else {
          double2 old = *p;
          old.x += static_cast<double>(acc[e][c].x);
          old.y += static_cast<double>(acc[e][c].y);
          *p = old;
        }
      }
    }
  }
}

// Single-band PH-magnetic / PH-charge update with the G blocks staged in shared memory.
//
// CTA = one (w1, w2, wq) tile and a chunk of momentum transfers q; thread = (k1, q, k2-chunk),
// holding the partial sums of its KT entries (k1, k2, q) for both channels in registers across
// the whole batch.  Per measurement the CTA needs four R x R blocks per spin,
//   A = G(., w1; ., w2)   B = G(., w2+x; ., w1+x)   C = G(., w1; ., w1+x)   E = G(., w2+x; ., w2),
// fetched by the bulk-copy engine (cp.async.bulk, one copy per block) into a two-stage ring while
// the previous measurement is being consumed.  With u_s(k1) = C_s(k1, k1+q), v_s(k2) = E_s(k2+q, k2):
//   magnetic += s/2 [(u_0 - u_1)(v_0 - v_1) - D],  charge += s/2 [(u_0 + u_1)(v_0 + v_1) - D],
//   D = sum_s A_s(k1, k2) B_s(k2+q, k1+q)
// (for one band the two channels share D).
// QFAST: consecutive threads take consecutive q (the A-block reads of a warp are broadcasts and
// the B-block reads fall in distinct banks) -- used for long batches.  Otherwise consecutive
// threads take consecutive k1 (coalesced G4 read-modify-write) and the running sums are read
// before the G blocks arrive (PREFETCH) -- used for the bandwidth-bound single-measurement case.
template <typename GT, typename AT, int KT, bool QFAST, bool PREFETCH, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
updateG4SinglebandPH(const TpDims dims, const GT* __restrict__ G, long g_sector_stride,
                     const int* __restrict__ signs, int n_slots, const int* __restrict__ k_add,
                     const int* __restrict__ q_list, const int* __restrict__ wex_list,
                     double2* const* __restrict__ G4, bool atomic, int q_chunk, int n_kc,
                     int* __restrict__ err) {
  using C = cplx_t<AT>;
  const int nc = dims.nc, nw = dims.nw, nw_ext = dims.nw_ext, R = dims.R, nq = dims.nq;
  const int w1 = blockIdx.x, w2 = blockIdx.y;
  const int n_qchunks = (nq + q_chunk - 1) / q_chunk;
  const int iwq = blockIdx.z / n_qchunks, q0 = (blockIdx.z % n_qchunks) * q_chunk;
  const int wex = wex_list[iwq];
  const int ext = dims.ext;
  const int t = threadIdx.x;
  const int k1 = QFAST ? (t / q_chunk) % nc : t % nc;
  const int ql = QFAST ? t % q_chunk : (t / nc) % q_chunk;
  const int kc = t / (nc * q_chunk);
  const int iq = q0 + ql;
  const bool active = iq < nq && kc < n_kc;
  const int q = active ? q_list[iq] : 0;

  bool has_mag = false, has_charge = false;
  for (int c = 0; c < dims.n_channels; ++c) {
    has_mag |= dims.channels[c] == 2;
    has_charge |= dims.channels[c] == 3;
  }

  const long blk_elems = static_cast<long>(R) * R;
  const int w1e = w1 + ext, w2e = w2 + ext, w1x = w1e + wex, w2x = w2e + wex;
  const long boff[4] = {(static_cast<long>(w1e) * nw_ext + w2e) * blk_elems,
                        (static_cast<long>(w2x) * nw_ext + w1x) * blk_elems,
                        (static_cast<long>(w1e) * nw_ext + w1x) * blk_elems,
                        (static_cast<long>(w2x) * nw_ext + w2e) * blk_elems};

  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);                   // [2]
  GT* stage = reinterpret_cast<GT*>(smem_raw + 16);                        // [2][2 spins][4][R*R]
  const int n_stages = n_slots > 1 ? 2 : 1;
  C* Um = reinterpret_cast<C*>(stage + n_stages * 8 * blk_elems);          // [nc][q_chunk]
  C* Uc = Um + q_chunk * nc;
  C* Vm = Uc + q_chunk * nc;
  C* Vc = Vm + q_chunk * nc;
  int* kadd = reinterpret_cast<int*>(Vc + q_chunk * nc);                  // [nc][nc]

  for (int i = t; i < nc * nc; i += blockDim.x)
    kadd[i] = k_add[i];
  // Slot-independent shared-memory offsets of this thread's A and B elements.
  const int k1q_t = k_add[k1 + nc * q];
  const int a_off = k1 * R + kc * KT;
  int b_off[KT];
#pragma unroll
  for (int j = 0; j < KT; ++j) {
    const int k2 = min(kc * KT + j, nc - 1);
    b_off[j] = k_add[k2 + nc * q] * R + k1q_t;
  }
  const uint32_t blk_bytes = static_cast<uint32_t>(blk_elems * sizeof(GT));
  auto issue = [&](int slot, int st) {
    GT* dst = stage + static_cast<long>(st) * 8 * blk_elems;
    mbarArriveExpectTx(&bar[st], 8 * blk_bytes);
    for (int s = 0; s < 2; ++s) {
      const GT* src = G + g_sector_stride * (2 * slot + s);
      for (int b = 0; b < 4; ++b)
        bulkCopyG2S(dst + (s * 4 + b) * blk_elems, src + boff[b], blk_bytes, &bar[st]);
    }
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

  C acc_m[KT], acc_c[KT];
#pragma unroll
  for (int j = 0; j < KT; ++j) {
    acc_m[j] = mk(AT(0), AT(0));
    acc_c[j] = mk(AT(0), AT(0));
  }
  const long s_w1 = nc, s_k2 = s_w1 * nw, s_w2 = s_k2 * nc, s_q = s_w2 * nw, s_wq = s_q * nq;
  const long g4_base = k1 + w1 * s_w1 + w2 * s_w2 + iq * s_q + iwq * s_wq;
  double2 old[PREFETCH ? 2 * KT : 1];
  if constexpr (PREFETCH) {
    // Running sums of (at most) two channels, loaded while the G blocks are in flight.
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
      for (int j = 0; j < KT; ++j) {
        const int k2 = kc * KT + j;
        old[c * KT + j] = (active && c < dims.n_channels && k2 < nc) ? G4[c][g4_base + k2 * s_k2]
                                                                     : make_double2(0, 0);
      }
  }

  for (int m = 0; m < n_slots; ++m) {
    const int st = m & 1;
    const bool ok = mbarWait(&bar[st], (m >> 1) & 1, err);
    if (!__syncthreads_and(ok))
      return;  // uniform bail-out; the host reports the error word
    const GT* S = stage + static_cast<long>(st) * 8 * blk_elems;
    const GT *A0 = S, *B0 = S + blk_elems, *C0 = S + 2 * blk_elems, *E0 = S + 3 * blk_elems;
    const GT *A1 = S + 4 * blk_elems, *B1 = S + 5 * blk_elems, *C1 = S + 6 * blk_elems,
             *E1 = S + 7 * blk_elems;
    const AT hs = AT(0.5) * static_cast<AT>(signs[m]);
    auto ld = [](const GT* p) { return mk(static_cast<AT>(p->x), static_cast<AT>(p->y)); };
    if (active && kc == 0) {
      const int k1q = kadd[k1 + nc * q];
      const C c0 = ld(C0 + k1 * R + k1q), c1 = ld(C1 + k1 * R + k1q);
      const C e0 = ld(E0 + k1q * R + k1), e1 = ld(E1 + k1q * R + k1);  // v(k2 = k1)
      Um[k1 * q_chunk + ql] = mk(hs * (c0.x - c1.x), hs * (c0.y - c1.y));
      Uc[k1 * q_chunk + ql] = mk(hs * (c0.x + c1.x), hs * (c0.y + c1.y));
      Vm[k1 * q_chunk + ql] = mk(e0.x - e1.x, e0.y - e1.y);
      Vc[k1 * q_chunk + ql] = mk(e0.x + e1.x, e0.y + e1.y);
    }
    __syncthreads();
    if (active) {
      const C um = Um[k1 * q_chunk + ql], uc = Uc[k1 * q_chunk + ql];
#pragma unroll
      for (int j = 0; j < KT; ++j) {
        const int k2 = kc * KT + j;
        if (k2 < nc) {
          const int ob = b_off[j];
          C d = cmul(ld(A0 + a_off + j), ld(B0 + ob));
          cfma(d, ld(A1 + a_off + j), ld(B1 + ob));
          d = cscale(d, hs);
          if (has_mag) {
            C v = cmul(um, Vm[k2 * q_chunk + ql]);
            acc_m[j] = cadd(acc_m[j], csub(v, d));
          }
          if (has_charge) {
            C v = cmul(uc, Vc[k2 * q_chunk + ql]);
            acc_c[j] = cadd(acc_c[j], csub(v, d));
          }
        }
      }
    }
    __syncthreads();  // stage st and U/V free again
    if (t == 0 && m + 2 < n_slots) {
      fenceProxyAsync();
      issue(m + 2, st);
    }
  }

  if (!active)
    return;
  // One read-modify-write of the FP64 running sums.
#pragma unroll
  for (int c = 0; c < kMaxChannels; ++c) {
    if (c >= dims.n_channels)
      break;
    const bool mag = dims.channels[c] == 2;
    double2* g4 = G4[c] + g4_base;
#pragma unroll
    for (int j = 0; j < KT; ++j) {
      const int k2 = kc * KT + j;
      if (k2 >= nc)
        break;
      const C v = mag ? acc_m[j] : acc_c[j];
      double2* p = g4 + k2 * s_k2;
      if (atomic) {
        atomicAdd(&p->x, static_cast<double>(v.x));
        atomicAdd(&p->y, static_cast<double>(v.y));
      }
      else {
        double2 o;
        if constexpr (PREFETCH)
          o = (c < 2) ? old[c * KT + j] : *p;
        else
          o = *p;
        o.x += static_cast<double>(v.x);
        o.y += static_cast<double>(v.y);
        *p = o;
      }
    }
  }
}

// Single-band PH-magnetic / PH-charge update of ONE measurement, streaming: the bandwidth-bound
// case (the plain FP64 path feeds measurements one at a time).  Persistent CTAs walk the (w1, w2,
// wq) tiles; per tile the eight R x R blocks (A, B, C, E of both spins, see updateG4SinglebandPH)
// are bulk-copied into one of two shared-memory stages while the previous tile is processed, and
// the tile's G4 entries are streamed in memory order (k1 contiguous, then k2, then q).  With NC
// (= Nc) a power of two and NC^2 <= 256, thread t keeps k1 = t % NC and k2 = (t / NC) % NC for every
// tile (so A_s(k1, k2) is one shared-memory read per tile) and walks the transfers q = t / NC^2,
// + 256 / NC^2, ...: kRound entries at a time it issues their G4 loads, then adds and stores them.
// A's rows are staged with a one-element pad (row stride R + 1) so that lanes of consecutive k1
// read distinct banks.  Each G4 entry is read and written once; G is read from L2 once per tile.
template <typename GT, typename AT, int NC>
__global__ void __launch_bounds__(256, sizeof(GT) == 16 ? 2 : 3)
updateG4SinglebandStream(const TpDims dims, const GT* __restrict__ G, long g_sector_stride,
                         const int* __restrict__ signs, const int* __restrict__ k_add,
                         const int* __restrict__ q_list, const int* __restrict__ wex_list,
                         double2* const* __restrict__ G4, bool atomic, int* __restrict__ err) {
  using C = cplx_t<AT>;
  constexpr int kRound = 4;            // transfers in flight per thread (two channels each)
  constexpr int R = NC, RP = NC + 1;   // one band
  constexpr int blk = R * R, blkA = R * RP;
  constexpr int stage_elems = 2 * (blkA + 3 * blk);  // per spin: A (padded), B, C, E
  constexpr int QSTEP = 256 / (NC * NC);             // transfers between a thread's entries
  const int nw = dims.nw, nw_ext = dims.nw_ext, nq = dims.nq, ext = dims.ext;
  const int n_tiles = nw * nw * dims.nwq;
  const int t = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);  // [2]
  int* kadd = reinterpret_cast<int*>(smem_raw + 16);      // [NC][NC]
  int* qtab = kadd + NC * NC;                             // [nq]
  GT* stage = reinterpret_cast<GT*>(smem_raw + 16 + ((sizeof(int) * (NC * NC + nq) + 15) / 16) * 16);

  for (int i = t; i < NC * NC; i += blockDim.x)
    kadd[i] = k_add[i];
  for (int i = t; i < nq; i += blockDim.x)
    qtab[i] = q_list[i];
  if (t == 0) {
    mbarInit(&bar[0], 1);
    mbarInit(&bar[1], 1);
    fenceBarrierInit();
  }
  __syncthreads();

  // Warp 0 issues a tile's copies: per spin, A row by row (padded), then B, C, E whole.
  constexpr uint32_t row_bytes = R * sizeof(GT), blk_bytes = row_bytes * R;
  auto issue = [&](int tile, int st) {
    const int w1 = tile % nw, w2 = (tile / nw) % nw, iwq = tile / (nw * nw);
    const int wex = wex_list[iwq];
    const int w1e = w1 + ext, w2e = w2 + ext, w1x = w1e + wex, w2x = w2e + wex;
    const long bA = (static_cast<long>(w1e) * nw_ext + w2e) * blk, bB = (static_cast<long>(w2x) * nw_ext + w1x) * blk,
               bC = (static_cast<long>(w1e) * nw_ext + w1x) * blk, bE = (static_cast<long>(w2x) * nw_ext + w2e) * blk;
    GT* dst = stage + static_cast<long>(st) * stage_elems;
    const int lane = t & 31;
    if (lane == 0)
      mbarArriveExpectTx(&bar[st], 2 * (blk_bytes * 4));
    __syncwarp();
    for (int c = lane; c < 2 * (R + 3); c += 32) {  // per spin: R row copies of A, 3 block copies
      const int s = c / (R + 3), j = c % (R + 3);
      const GT* src = G + g_sector_stride * s;
      GT* d = dst + s * (blkA + 3 * blk);
      if (j < R)
        bulkCopyG2S(d + j * RP, src + bA + j * R, row_bytes, &bar[st]);
      else {
        const int b = j - R;  // 0: B, 1: C, 2: E
        bulkCopyG2S(d + blkA + b * blk, src + (b == 0 ? bB : b == 1 ? bC : bE), blk_bytes, &bar[st]);
      }
    }
  };

  // Positions of the PH-magnetic and PH-charge channels in G4 (-1: not accumulated); static
  // indices keep dims in registers.
  int c_mag = -1, c_chg = -1;
#pragma unroll
  for (int c = 0; c < kMaxChannels; ++c) {
    if (c < dims.n_channels && dims.channels[c] == 2)
      c_mag = c;
    if (c < dims.n_channels && dims.channels[c] == 3)
      c_chg = c;
  }
  const AT hs = AT(0.5) * static_cast<AT>(signs[0]);
  const int k1 = t % NC, k2 = (t / NC) % NC, q0 = t / (NC * NC);
  // k1 + q and k2 + q of this thread's transfers (at most 16, each < NC <= 16): 4 bits apiece.
  uint64_t kq1p = 0, kq2p = 0;
  for (int iq = q0, m = 0; iq < nq; iq += QSTEP, ++m) {
    const int q = qtab[iq];
    kq1p |= static_cast<uint64_t>(kadd[k1 + NC * q]) << (4 * m);
    kq2p |= static_cast<uint64_t>(kadd[k2 + NC * q]) << (4 * m);
  }
  // G4 offsets: s_k2 = Nc Nw, s_q = (Nc Nw)^2 (< 2^31 for Nc <= 16, Nw <= 2048), tile base long.
  const int s_k2 = NC * nw, s_q = NC * nw * NC * nw;
  const long s_w2 = static_cast<long>(s_k2) * NC, s_wq = static_cast<long>(s_q) * nq;
  const int own = k1 + k2 * s_k2;  // this thread's entry inside a (tile, q)
  double2* const g4m = c_mag >= 0 ? G4[c_mag] : nullptr;
  double2* const g4c = c_chg >= 0 ? G4[c_chg] : nullptr;

  int it = 0;
  if (t < 32 && blockIdx.x < n_tiles)
    issue(blockIdx.x, 0);
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++it) {
    const int st = it & 1;
    // The next tile's copies into the other stage (released by the __syncthreads that ended the
    // previous iteration).
    if (t < 32 && tile + gridDim.x < n_tiles) {
      if (t == 0)
        fenceProxyAsync();
      __syncwarp();
      issue(tile + gridDim.x, st ^ 1);
    }
    const int w1 = tile % nw, w2 = (tile / nw) % nw, iwq = tile / (nw * nw);
    const long base = static_cast<long>(w1) * NC + w2 * s_w2 + iwq * s_wq + own;
    const bool ok = mbarWait(&bar[st], (it >> 1) & 1, err);
    if (!__syncthreads_and(ok)) {
      // Give up; the copies of the other stage (if issued) land before the CTA exits.
      if (t == 0 && tile + gridDim.x < n_tiles)
        mbarWait(&bar[st ^ 1], ((it + 1) >> 1) & 1, err);
      __syncthreads();
      return;
    }
    const GT* S = stage + static_cast<long>(st) * stage_elems;
    const GT *A0 = S, *B0 = S + blkA, *C0 = B0 + blk, *E0 = C0 + blk;
    const GT *A1 = S + blkA + 3 * blk, *B1 = A1 + blkA, *C1 = B1 + blk, *E1 = C1 + blk;
    auto ld = [](const GT* p) { return mk(static_cast<AT>(p->x), static_cast<AT>(p->y)); };
    const C a0 = ld(A0 + k1 * RP + k2), a1 = ld(A1 + k1 * RP + k2);
    // Both channels per entry: they share D = sum_s A_s B_s and u_s, v_s up to the spin signs.
    for (int iq0 = q0, m0 = 0; iq0 < nq; iq0 += kRound * QSTEP, m0 += kRound) {
      double2 om[kRound], oc[kRound];
#pragma unroll
      for (int r = 0; r < kRound; ++r) {
        const long o = static_cast<long>(iq0 + r * QSTEP) * s_q;
        if (!atomic && iq0 + r * QSTEP < nq) {
          if (g4m)
            om[r] = g4m[base + o];
          if (g4c)
            oc[r] = g4c[base + o];
        }
      }
#pragma unroll
      for (int r = 0; r < kRound; ++r) {
        const int iq = iq0 + r * QSTEP;
        if (iq >= nq)
          break;
        const int kq1 = static_cast<int>((kq1p >> (4 * (m0 + r))) & 15u);
        const int kq2 = static_cast<int>((kq2p >> (4 * (m0 + r))) & 15u);
        C d = cmul(a0, ld(B0 + kq2 * R + kq1));
        cfma(d, a1, ld(B1 + kq2 * R + kq1));
        const C u0 = ld(C0 + k1 * R + kq1), u1 = ld(C1 + k1 * R + kq1);
        const C v0 = ld(E0 + kq2 * R + k2), v1 = ld(E1 + kq2 * R + k2);
        const long o = base + static_cast<long>(iq) * s_q;
        if (g4m) {
          const C val = cscale(csub(cmul(csub(u0, u1), csub(v0, v1)), d), hs);
          if (atomic) {
            atomicAdd(&g4m[o].x, static_cast<double>(val.x));
            atomicAdd(&g4m[o].y, static_cast<double>(val.y));
          }
          else {
            g4m[o] = make_double2(om[r].x + static_cast<double>(val.x), om[r].y + static_cast<double>(val.y));
          }
        }
        if (g4c) {
          const C val = cscale(csub(cmul(cadd(u0, u1), cadd(v0, v1)), d), hs);
          if (atomic) {
            atomicAdd(&g4c[o].x, static_cast<double>(val.x));
            atomicAdd(&g4c[o].y, static_cast<double>(val.y));
          }
          else {
            g4c[o] = make_double2(oc[r].x + static_cast<double>(val.x), oc[r].y + static_cast<double>(val.y));
          }
        }
      }
    }
    __syncthreads();  // stage st is free for the tile after next
  }
}

}  // namespace

template <typename GT>
static bool singlebandPHApplies(const TpDims& d) {
  if (d.nb != 1)
    return false;
  for (int c = 0; c < d.n_channels; ++c)
    if (d.channels[c] != 2 && d.channels[c] != 3)
      return false;
  return (size_t(d.R) * d.R * sizeof(GT)) % 16 == 0;
}

// Momentum transfers per CTA of updateG4SinglebandPH for a thread target, and its shared memory;
// 0 when one transfer does not fit the launch bound or the CTA's shared memory.
template <typename GT, typename AT, int KT, int MAXT>
static int singlebandPHChunk(const G4Args& a, int target_threads, size_t* smem_out) {
  const TpDims& d = a.dims;
  const int per_q = d.nc * ((d.nc + KT - 1) / KT);
  if (per_q > MAXT)  // one q per CTA must fit the kernel's launch bound
    return 0;
  const int q_chunk = std::max(1, std::min(d.nq, std::min(target_threads, MAXT) / per_q));
  const int n_stages = a.n_slots > 1 ? 2 : 1;
  const size_t smem = 16 + sizeof(GT) * n_stages * 8 * size_t(d.R) * d.R +
                      sizeof(cplx_t<AT>) * 4 * q_chunk * d.nc + sizeof(int) * d.nc * d.nc;
  if (smem > 220 * 1024)
    return 0;
  if (smem_out)
    *smem_out = smem;
  return q_chunk;
}

// Every G4 entry is summed over the batch by one thread in slot order whatever the number of
// transfers per CTA, so the tuner may choose it: the q chunk for 256 threads or for 128.
template <typename GT, typename AT, int KT, bool QFAST, bool PREFETCH, int MAXT, int MINB>
static bool launchSinglebandPH(const G4Args& a, const GT* G, long g_sector_stride, cudaStream_t stream) {
  const TpDims& d = a.dims;
  size_t smem = 0;
  const int chunk_a = singlebandPHChunk<GT, AT, KT, MAXT>(a, 256, nullptr);
  if (chunk_a == 0)
    return false;
  const int chunk_b = singlebandPHChunk<GT, AT, KT, MAXT>(a, 128, nullptr);
  const auto pk = tunePick(a.tuner, tuneKey("g4ph", d.nb, d.nc, d.nw_ext, d.nq, a.n_slots, sizeof(GT)),
                           chunk_b != chunk_a ? 2 : 1, stream);
  const int q_chunk = singlebandPHChunk<GT, AT, KT, MAXT>(a, pk.choice == 0 ? 256 : 128, &smem);
  const int n_kc = (d.nc + KT - 1) / KT;
  const int threads = d.nc * n_kc * q_chunk;
  auto k = updateG4SinglebandPH<GT, AT, KT, QFAST, PREFETCH, MAXT, MINB>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int n_qchunks = (d.nq + q_chunk - 1) / q_chunk;
  const dim3 grid(d.nw, d.nw, d.nwq * n_qchunks);
  k<<<grid, threads, smem, stream>>>(d, G, g_sector_stride, a.signs, a.n_slots, a.k_add, a.q_list,
                                     a.wex_list, a.G4, a.atomic, q_chunk, n_kc, a.err);
  DCAACC_LAUNCH_CHECK();
  tuneEnd(a.tuner, pk, stream);
  return true;
}

// The streaming single-measurement kernel: one band, PH channels, Nc in {4, 8, 16} (two stages of
// eight blocks in shared memory; Nc a compile-time power of two).
template <typename GT>
static bool launchSinglebandStream(const G4Args& a, const GT* G, long g_sector_stride, cudaStream_t stream) {
  const TpDims& d = a.dims;
  if (a.n_slots != 1 || !singlebandPHApplies<GT>(d) || a.n_sm <= 0 || (d.nc != 4 && d.nc != 8 && d.nc != 16))
    return false;
  using AT = std::conditional_t<std::is_same_v<GT, double2>, double, float>;
  const size_t tables = ((sizeof(int) * (d.nc * d.nc + d.nq) + 15) / 16) * 16;
  const size_t smem = 16 + tables + 2 * sizeof(GT) * 2 * (size_t(d.R) * (d.R + 1) + 3 * size_t(d.R) * d.R);
  auto k = d.nc == 16 ? updateG4SinglebandStream<GT, AT, 16>
           : d.nc == 8 ? updateG4SinglebandStream<GT, AT, 8> : updateG4SinglebandStream<GT, AT, 4>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const long tiles = long(d.nw) * d.nw * d.nwq;
  const int grid = int(std::max(1L, std::min<long>(tiles, (sizeof(GT) == 16 ? 2L : 3L) * a.n_sm)));
  k<<<grid, 256, smem, stream>>>(d, G, g_sector_stride, a.signs, a.k_add, a.q_list, a.wex_list, a.G4, a.atomic,
                                 a.err);
  DCAACC_LAUNCH_CHECK();
  return true;
}

template <typename GT>
int launchUpdateG4(const G4Args& a, const GT* G, long g_sector_stride, cudaStream_t stream) {
  if constexpr (std::is_same_v<GT, float2>) {
    if (const int n = launchUpdateG4SinglebandBatched(a, G, g_sector_stride, stream))
      return n;
    const char* pp_env = std::getenv("DCAACC_TP_PP_GENERIC");  // =1: the generic staged kernel instead
    if (!(pp_env && std::strcmp(pp_env, "1") == 0) && launchUpdateG4PPMultiband(a, G, g_sector_stride, stream))
      return 1;
  }
  if (launchSinglebandStream<GT>(a, G, g_sector_stride, stream))
    return 1;
  if (singlebandPHApplies<GT>(a.dims)) {
    bool done;
    if constexpr (std::is_same_v<GT, double2>)
      done = launchSinglebandPH<double2, double, 2, false, true, 256, 4>(a, G, g_sector_stride, stream);
    else
      done = launchSinglebandPH<float2, float, 16, true, false, 256, 2>(a, G, g_sector_stride, stream);
    if (done)
      return 1;
  }
  const dim3 grid(a.dims.nw, a.dims.nw, a.dims.nwq);
  // Batches: the staged kernel (a single measurement reads each block element a few times only, and
  // the direct gathers of updateG4Kernel cost less than staging).
  if (a.n_slots >= 2 && a.dims.n_channels <= kStagedMaxCh && (size_t(a.dims.R) * a.dims.R * sizeof(GT)) % 16 == 0) {
    int nblk = 1;  // A, and B / C, E / P as the channels need them
    bool needB = false, needCE = false, needP = false;
    for (int c = 0; c < a.dims.n_channels; ++c) {
      const int ch = a.dims.channels[c];
      needB |= ch == 1 || ch == 2 || ch == 3;
      needCE |= ch == 2 || ch == 3;
      needP |= ch == 4;
    }
    nblk += needB + 2 * needCE + needP;
    const size_t smem = 16 + 2 * 2 * size_t(nblk) * a.dims.R * a.dims.R * sizeof(GT);
    if (smem <= 200 * 1024) {
      using AT = std::conditional_t<std::is_same_v<GT, double2>, double, float>;
      // Entries per thread: 4 (candidate 0), 8 or 16.
      const auto pk = tunePick(a.tuner, tuneKey("g4staged", a.dims.nb, a.dims.nc, a.dims.nw_ext, a.dims.nq,
                                                a.n_slots, sizeof(GT)), 3, stream);
      const bool two = a.dims.n_channels == 2;
      auto k = pk.choice == 2 ? (two ? updateG4StagedKernel<GT, AT, 16, 2> : updateG4StagedKernel<GT, AT, 16, 1>)
               : pk.choice == 1 ? (two ? updateG4StagedKernel<GT, AT, 8, 2> : updateG4StagedKernel<GT, AT, 8, 1>)
                                : (two ? updateG4StagedKernel<GT, AT, 4, 2> : updateG4StagedKernel<GT, AT, 4, 1>);
      DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      k<<<grid, 256, smem, stream>>>(a.dims, G, g_sector_stride, a.signs, a.n_slots, a.k_add, a.k_sub, a.q_list,
                                     a.wex_list, a.G4, a.atomic, a.err);
      DCAACC_LAUNCH_CHECK();
      tuneEnd(a.tuner, pk, stream);
      return 1;
    }
  }
  if constexpr (std::is_same_v<GT, double2>) {
    updateG4Kernel<double2, double, 4><<<grid, 256, 0, stream>>>(
        a.dims, G, g_sector_stride, a.signs, a.n_slots, a.k_add, a.k_sub, a.q_list, a.wex_list,
        a.G4, a.atomic);
  }
  else {
    updateG4Kernel<float2, float, 8><<<grid, 256, 0, stream>>>(
        a.dims, G, g_sector_stride, a.signs, a.n_slots, a.k_add, a.k_sub, a.q_list, a.wex_list,
        a.G4, a.atomic);
  }
  DCAACC_LAUNCH_CHECK();
  return 1;
}

template int launchUpdateG4<double2>(const G4Args&, const double2*, long, cudaStream_t);
template int launchUpdateG4<float2>(const G4Args&, const float2*, long, cudaStream_t);

}  // namespace dcaacc

namespace dcaacc {

namespace {
__global__ void addAndClearKernel(double2* __restrict__ dst, double2* __restrict__ src, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const double2 a = src[i];
    double2 b = dst[i];
    b.x += a.x;
    b.y += a.y;
    dst[i] = b;
    src[i] = make_double2(0.0, 0.0);
  }
}
}  // namespace

namespace {

// G4 entry index (one band: k1 + Nc (w1 + Nw (k2 + Nc (w2 + Nw (iq + Nq iwq))))) of the mirror of
// entry e, and whether e lies in the lower half (w1 < Nw / 2) that the mirror provides.
__device__ inline bool g4Mirror(const TpDims& d, const int* q_mirror, const int* wq_mirror, size_t e, size_t& m) {
  const int nc = d.nc, nw = d.nw;
  size_t r = e;
  const int k1 = static_cast<int>(r % nc);
  r /= nc;
  const int w1 = static_cast<int>(r % nw);
  r /= nw;
  const int k2 = static_cast<int>(r % nc);
  r /= nc;
  const int w2 = static_cast<int>(r % nw);
  r /= nw;
  const int iq = static_cast<int>(r % d.nq);
  const int iwq = static_cast<int>(r / d.nq);
  if (2 * w1 >= nw)
    return false;
  m = d.kneg[k1] + nc * (nw - 1 - w1 + size_t(nw) * (d.kneg[k2] + nc * (nw - 1 - w2 +
      size_t(nw) * (q_mirror[iq] + size_t(d.nq) * wq_mirror[iwq]))));
  return true;
}

__global__ void g4MirrorKernel(double2* __restrict__ G4, const TpDims d, const int* __restrict__ q_mirror,
                               const int* __restrict__ wq_mirror, size_t n) {
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    size_t m;
    if (g4Mirror(d, q_mirror, wq_mirror, e, m)) {
      const double2 v = G4[m];
      G4[e] = make_double2(v.x, -v.y);
    }
  }
}

__global__ void g4WindowKernel(const double2* __restrict__ G4, const TpDims d, const int* __restrict__ q_mirror,
                               const int* __restrict__ wq_mirror, size_t offset, size_t count,
                               double2* __restrict__ out) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x) {
    size_t m;
    if (d.half_g4 && g4Mirror(d, q_mirror, wq_mirror, offset + i, m)) {
      const double2 v = G4[m];
      out[i] = make_double2(v.x, -v.y);
    }
    else {
      out[i] = G4[offset + i];
    }
  }
}

size_t g4Entries(const TpDims& d) {
  return size_t(d.nb) * d.nb * d.nb * d.nb * d.nc * d.nc * d.nw * d.nw * d.nq * d.nwq;
}

}  // namespace

void launchG4Mirror(double2* G4, const TpDims& d, const int* q_mirror, const int* wq_mirror, cudaStream_t stream) {
  const size_t n = g4Entries(d);
  const int blocks = static_cast<int>(std::min<size_t>((n + 255) / 256, 148 * 16));
  g4MirrorKernel<<<blocks, 256, 0, stream>>>(G4, d, q_mirror, wq_mirror, n);
  DCAACC_LAUNCH_CHECK();
}

void launchG4Window(const double2* G4, const TpDims& d, const int* q_mirror, const int* wq_mirror, size_t offset,
                    size_t count, double2* out, cudaStream_t stream) {
  if (!count)
    return;
  const int blocks = static_cast<int>(std::min<size_t>((count + 255) / 256, 148 * 16));
  g4WindowKernel<<<blocks, 256, 0, stream>>>(G4, d, q_mirror, wq_mirror, offset, count, out);
  DCAACC_LAUNCH_CHECK();
}

void launchAddAndClear(double2* dst, double2* src, size_t n, cudaStream_t stream) {
  if (!n)
    return;
  const int blocks = static_cast<int>(std::min<size_t>((n + 255) / 256, 148 * 16));
  addAndClearKernel<<<blocks, 256, 0, stream>>>(dst, src, n);
  DCAACC_LAUNCH_CHECK();
}

}  // namespace dcaacc
