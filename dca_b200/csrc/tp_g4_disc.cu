// Disconnected (spin-difference / spin-sum) terms of the batched PH-magnetic / PH-charge G4 update
// as a tensor-core GEMM.
//
// For one band, PH-magnetic and PH-charge contain (tp_accumulator_cpu.hpp:491-575)
//   sum_m s_m/2 u_m(k1, w1; q) v_m(k2, w2; q),   u = G_0(k1 w1; k1+q w1+x) -+ G_1(...),
//                                                v = G_0(k2+q w2+x; k2 w2) -+ G_1(...),
// (- for magnetic, + for charge), i.e. for each (q, x, channel) problem the product U V^T of two
// (Nc Nw x B) complex matrices over the batch index m.  This file builds U (with s_m/2 folded in)
// and V from the diagonal G blocks of the batch as two FP16 planes each (each row scaled by a power
// of two that puts its maximum over the batch in [2^14, 2^15)), and runs them through the shared
// persistent tcgen05 GEMM (tc_gemm.cuh, MODE 2), which writes the FP32 result per problem as an
// M x M matrix, m = k1 + Nc w1 fastest, for the direct-term kernel (tp_g4_batched.cu) to add at
// its flush.  Rows are padded to a multiple of 128 and the batch to a power of two >= 32.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "async_copy.cuh"
#include "common.cuh"
#include "tc_gemm.cuh"
#include "tp_g4.hpp"

namespace dcaacc {

namespace {

using namespace tcg;

struct DiscShape {
  int M;      // Nc * Nw
  int Mp;     // M rounded up to 128
  int Kb;     // batch rounded up to a power of two >= 32 (<= 256)
  int probs;  // nq * nwq * n_channels
  size_t plane_elems;  // FP16 elements of one operand's planes over all problems
};

DiscShape discShape(const TpDims& d, int batch) {
  DiscShape s;
  s.M = d.nc * d.nw;
  s.Mp = (s.M + kBM - 1) / kBM * kBM;
  s.Kb = 32;
  while (s.Kb < batch)
    s.Kb *= 2;
  s.probs = d.nq * d.nwq * d.n_channels;
  s.plane_elems = size_t(s.probs) * kPl * s.Mp * 2 * s.Kb;
  return s;
}

size_t align256(size_t b) {
  return (b + 255) / 256 * 256;
}

// One thread per (row, group of 8 measurements) of one problem (blockIdx.y = iwq * nq + iq,
// blockIdx.z = channel); the Kb / 8 groups of a row are adjacent lanes of one warp, which reduce
// the row's maxima with shuffles.  U and V planes: [problem][plane][Mp rows][2 Kb], real part at
// column m, imaginary part at Kb + m; eU / eV: [problem][Mp].
__global__ void __launch_bounds__(256)
discPlanesKernel(const TpDims dims, const float2* __restrict__ G, long g_sector_stride,
                 const int* __restrict__ signs, int n_slots, int Kb, int Mp, const int* __restrict__ k_add,
                 const int* __restrict__ q_list, const int* __restrict__ wex_list, __half* __restrict__ Up,
                 __half* __restrict__ Vp, int* __restrict__ eU, int* __restrict__ eV) {
  const int nc = dims.nc, ext = dims.ext;
  const int M = nc * dims.nw;
  const int p = blockIdx.y;
  const int ch = blockIdx.z;
  const float sg = dims.channels[ch] == 2 ? -1.f : 1.f;  // magnetic: difference, charge: sum
  const int iq = p % dims.nq, iwq = p / dims.nq;
  const int q = q_list[iq], wex = wex_list[iwq];
  const long kp = 2L * Kb;
  const long plane = static_cast<long>(Mp) * kp;
  const long prob = static_cast<long>(p) * gridDim.z + ch;
  __half* U = Up + prob * kPl * plane;
  __half* V = Vp + prob * kPl * plane;
  const int groups = Kb / 8;  // a power of two <= 32: a row's groups share a warp
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < long(groups) * Mp;
       idx += long(gridDim.x) * blockDim.x) {
    const int grp = static_cast<int>(idx % groups);
    const int row = static_cast<int>(idx / groups);
    const int slot0 = grp * 8;
    long bc = 0, be = 0;
    bool cc = false, ce = false;  // read from the conjugated mirror (half G)
    const bool in_row = row < M;
    // Half G4: the GEMM reads U only for the rows (k1, w1) with w1 >= Nw / 2.
    const bool need_u = in_row && !(dims.half_g4 && 2 * (row / nc) < dims.nw);
    if (in_row) {
      const int k = row % nc, w = row / nc;
      const int kq = k_add[k + nc * q];
      const int we = w + ext, wx = we + wex;
      bc = gIndexMirrored(dims, we, wx, k, kq, cc);
      be = gIndexMirrored(dims, wx, we, kq, k, ce);
    }
    float2 u[8], v[8];
    float mu = 0.f, mv = 0.f;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int slot = slot0 + e;
      u[e] = v[e] = make_float2(0.f, 0.f);
      if (in_row && slot < n_slots) {
        const float hs = 0.5f * static_cast<float>(signs[slot]);
        const float2* G0s = G + g_sector_stride * (2 * slot);
        const float2* G1s = G0s + g_sector_stride;
        float2 c0 = make_float2(0.f, 0.f), c1 = c0;
        if (need_u) {
          c0 = G0s[bc];
          c1 = G1s[bc];
        }
        float2 e0 = G0s[be], e1 = G1s[be];
        if (cc) {
          c0.y = -c0.y;
          c1.y = -c1.y;
        }
        if (ce) {
          e0.y = -e0.y;
          e1.y = -e1.y;
        }
        u[e] = make_float2(hs * (c0.x + sg * c1.x), hs * (c0.y + sg * c1.y));
        v[e] = make_float2(e0.x + sg * e1.x, e0.y + sg * e1.y);
      }
      mu = fmaxf(mu, fmaxf(fabsf(u[e].x), fabsf(u[e].y)));
      mv = fmaxf(mv, fmaxf(fabsf(v[e].x), fabsf(v[e].y)));
    }
    for (int off = groups / 2; off > 0; off >>= 1) {
      mu = fmaxf(mu, __shfl_xor_sync(0xffffffffu, mu, off));
      mv = fmaxf(mv, __shfl_xor_sync(0xffffffffu, mv, off));
    }
    const int xu = scaleExp(mu), xv = scaleExp(mv);
    const float su = pow2f(xu), sv = pow2f(xv);
    Pack8 ur[kPl], ui[kPl], vr[kPl], vi[kPl];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const Split2 a = split2f(u[e].x, su), b = split2f(u[e].y, su), c = split2f(v[e].x, sv),
                   d = split2f(v[e].y, sv);
      ur[0].v[e] = a.h, ur[1].v[e] = a.l;
      ui[0].v[e] = b.h, ui[1].v[e] = b.l;
      vr[0].v[e] = c.h, vr[1].v[e] = c.l;
      vi[0].v[e] = d.h, vi[1].v[e] = d.l;
    }
    const long o = static_cast<long>(row) * kp + slot0;
#pragma unroll
    for (int pl = 0; pl < kPl; ++pl) {
      if (need_u || !dims.half_g4) {
        store8(U + pl * plane + o, ur[pl]);
        store8(U + pl * plane + o + Kb, ui[pl]);
      }
      store8(V + pl * plane + o, vr[pl]);
      store8(V + pl * plane + o + Kb, vi[pl]);
    }
    if (grp == 0) {
      eU[prob * Mp + row] = xu;
      eV[prob * Mp + row] = xv;
    }
  }
}

}  // namespace

bool discGemmApplies(const TpDims& d, int max_batch) {
  return singlebandBatchedApplies(d) && max_batch <= 256;
}

size_t discScratchBytes(const TpDims& d, int max_batch) {
  const DiscShape s = discShape(d, max_batch);
  return 2 * align256(s.plane_elems * sizeof(__half)) + 2 * align256(sizeof(int) * s.probs * s.Mp) +
         align256(sizeof(float2) * s.probs * size_t(s.M) * s.M);
}

void discInit(DiscWorkspace& w, const TpDims& d, int max_batch, void* mem, size_t bytes) {
  const DiscShape s = discShape(d, max_batch);
  if (bytes < discScratchBytes(d, max_batch))
    throw Error(DCAACC_INVALID_ARG, "disconnected-term workspace too small");
  unsigned char* b = static_cast<unsigned char*>(mem);
  size_t off = 0;
  w.U = b + off;
  off += align256(s.plane_elems * sizeof(__half));
  w.V = b + off;
  off += align256(s.plane_elems * sizeof(__half));
  w.eU = reinterpret_cast<int*>(b + off);
  off += align256(sizeof(int) * s.probs * s.Mp);
  w.eV = reinterpret_cast<int*>(b + off);
  off += align256(sizeof(int) * s.probs * s.Mp);
  w.out = reinterpret_cast<float2*>(b + off);
  w.max_batch = max_batch;
  makePlaneMap(&w.tm_u, w.U, 2L * s.Kb, s.Mp, long(s.probs) * kPl);
  makePlaneMap(&w.tm_v, w.V, 2L * s.Kb, s.Mp, long(s.probs) * kPl);
  int dev = 0;
  DCAACC_CUDA_CHECK(cudaGetDevice(&dev));
  DCAACC_CUDA_CHECK(cudaDeviceGetAttribute(&w.n_sm, cudaDevAttrMultiProcessorCount, dev));
}

const float2* launchDiscGemm(const G4Args& a, const float2* G, long g_sector_stride, cudaStream_t stream) {
  const DiscWorkspace* w = a.disc;
  if (!w || a.n_slots > w->max_batch)
    return nullptr;
  const TpDims& d = a.dims;
  const DiscShape s = discShape(d, w->max_batch);
  {
    const long work = long(s.Kb / 8) * s.Mp;
    const dim3 grid(static_cast<unsigned>(std::max(1L, std::min(1024L, (work + 255) / 256))), d.nq * d.nwq,
                    d.n_channels);
    discPlanesKernel<<<grid, 256, 0, stream>>>(d, G, g_sector_stride, a.signs, a.n_slots, s.Kb, s.Mp, a.k_add,
                                               a.q_list, a.wex_list, static_cast<__half*>(w->U),
                                               static_cast<__half*>(w->V), w->eU, w->eV);
    DCAACC_LAUNCH_CHECK();
  }
  GemmParams p{};
  p.dims = d;
  p.n_sectors = s.probs;
  p.D = s.M;
  p.Dp = s.Mp;
  p.Kr = s.Kb;
  p.mt0 = d.half_g4 ? s.M / 2 / kBM : 0;  // half G4: the rows (k1, w1) with w1 >= Nw / 2 only
  p.mt = s.Mp / kBM - p.mt0;
  p.nt = s.Mp / kBN;
  p.err = a.err;
  p.n_slots = a.n_slots;
  p.Md = s.M;
  p.eU = w->eU;
  p.eV = w->eV;
  p.disc = w->out;
  const auto pk = tunePick(a.tuner, tuneKey("tc_disc_order", d.nb, d.nc, d.nw_ext, a.n_slots, s.probs, 2), 2,
                           stream);
  p.order = pk.choice;
  launchGemm<2>(p, w->tm_u, w->tm_v, w->n_sm, stream);
  tuneEnd(a.tuner, pk, stream);
  return w->out;
}

}  // namespace dcaacc
