// Column step factored by orbital with the per-site sums in tensor memory (one band, 4 x 4
// cluster, mixed path): tcgen05 form of tp_colfactor.cu's two stages,
//   Z(rho1, w2, r)  = sum_{j in site r} X'(rho1, j) conj T(w2, j)
//   G(rho1; k2, w2) = -(1/Nc) G0_s(k2, w2) sum_r e^{-i k2 x_r} Z(rho1, w2, r) + beta G0_s delta,
// (CachedNdft<GPU>::performFT, cached_ndft_gpu.hpp:193-252; SpaceTransform2DGpu::execute,
// space_transform_2D_gpu.hpp:116-159).
//
// CTA = (sector, 128 rows rho1, 8 frequencies w2); Z of all 16 sites for that tile lives in 256
// tensor-memory columns (site r: columns 16 r .. 16 r + 15, (re, im) of w2 = 2 w, 2 w + 1), so the
// on-chip capacity that capped the shared-memory forms is the tensor memory's, and two CTAs fit an
// SM.  Warp roles:
//   warp 0     TMA loads of the X' chunks (the row step's split-FP16 planes, 128 rows x 32 vertices
//              per plane, 64-byte swizzle; the column GEMM's descriptors), two stages;
//   warp 1     tensor-memory allocation and the MMA issue: the sites a chunk touches are consecutive
//              in site order, so their sums are contiguous columns and up to four of them take one
//              MMA: per (chunk, site group) item and 16-vertex step, D += Xr B_re + Xi B_im with split
//              FP16 (lo hi, hi lo, hi hi), six M128 x N(16 per site) x K16 MMAs (a tcgen05 MMA costs
//              about as long to issue whatever its N, so the sites share instructions);
//   warps 2-5  zero the tensor memory (so that every MMA accumulates), then build each item's B
//              operands in shared memory: per site 8 frequencies x 32 vertices, B_re = [Tr; -Ti],
//              B_im = [Ti; Tr] (rows 16 i + 2 w, + 1), the vertices of other sites zeroed, split into
//              FP16 hi / lo planes, in a ring of 2 items; the chunk twiddles are loaded one chunk
//              ahead; then the epilogue.
// The X' chunk scales 2^-e_c fold into B exactly (T 2^12 s_c / s_max), so each site sums all of its
// chunks in tensor memory without promotion: a site spans one or two 16-vertex steps per chunk, so
// every tensor-memory sum is a short chain (the precision the dense GEMM gets from promoting every
// chunk).  Epilogue: thread = row rho1 (tensor-memory lane); per pair of frequencies it loads the
// 16 sites' Z in the FFT's slot order, runs the 4 x 4 FFT, applies the G0 factor and the delta
// term, and writes its row of 16 momenta through a warp-private shared-memory transpose, so each
// store instruction writes 512 contiguous bytes of G.
// Measured on B200 (c3: 4x4 cluster, Nw = 64, n ~ U[50, 400], batch 64): 0.44 ms per batch, the
// same as the dense tcgen05 GEMM, and the batch saves the dense step's Q operand planes.  A CTA
// (about 30 us) spends about 15 us issuing its MMAs and taking the builders' operands and 11 us in
// the FFT epilogue; two CTAs per SM overlap those phases.
#include <cuda.h>
#include <algorithm>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "async_copy.cuh"
#include "common.cuh"
#include "tc_gemm.cuh"
#include "tcgen05.cuh"
#include "tp_frontend.hpp"
#include "tp_layout.hpp"

namespace dcaacc {
namespace {

constexpr int kW = 8;                         // frequencies w2 per CTA
constexpr int kN = 2 * kW;                    // MMA N: (re, im) of each frequency
constexpr int kSites = 16;
constexpr uint32_t kTmemCols = kSites * kN;   // 256
constexpr int kXStages = 2;
constexpr uint32_t kXBox = 128 * 32 * 2;      // one X' plane box: 8 KB
constexpr uint32_t kXStage = 4 * kXBox;       // re hi, re lo, im hi, im lo
constexpr int kMaxGroup = 4;                  // consecutive sites stacked into one MMA (N <= 64)
constexpr uint32_t kBTile = kMaxGroup * kN * 64;  // one B plane: up to 64 rows x 64 bytes
constexpr uint32_t kBItem = 4 * kBTile;       // B_re hi, B_re lo, B_im hi, B_im lo
constexpr int kBSlots = 2;
constexpr int kBuilders = 128;                // warps 2..5
constexpr int kThreads = 64 + kBuilders;
constexpr float kTScale = 4096.f;
// Shared memory (from a 1024-byte aligned base): X' stages, B ring, then the rest.
constexpr uint32_t kOffB = kXStages * kXStage;                  // 64 KB
constexpr uint32_t kOffT = kOffB + kBSlots * kBItem;            // chunk twiddles, float2 [2][kW][32]
constexpr uint32_t kOffC = kOffT + 2 * kW * 32 * 8;             // Cg, Ds: float2 [kW][16] each
constexpr uint32_t kOffTab = kOffC + 2 * kW * 16 * 8;           // cs[17], rm[16], km[16], smax
constexpr uint32_t kOffBar = kOffTab + 4 * 64;                  // barriers, tensor-memory slot
constexpr uint32_t kSmemUsed = kOffBar + 8 * (2 * kXStages + 2 * kBSlots + 1) + 16;
__host__ __device__ constexpr size_t colFactorTcSmem(int) {
  return 1024 + kSmemUsed;
}
constexpr int kEpiRowB = 144;  // epilogue transpose: one row of 16 momenta (+16 bytes)
static_assert(kXStages * kXStage >= 4 * 32 * kEpiRowB, "epilogue staging fits in the X' stages");
static_assert(kOffT % 16 == 0 && kOffC % 16 == 0, "table alignment");

__device__ inline void ld32x32bx4(uint32_t taddr, float (&v)[4]) {
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 4; ++i)
    v[i] = __uint_as_float(r[i]);
}

// Zeros into 32 consecutive columns of the warp's 32 lanes.
__device__ inline void stZero32x32bx32(uint32_t taddr) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,"
      "%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr), "r"(0u)
      : "memory");
}

__device__ inline void namedSync128() {
  asm volatile("bar.sync 1, 128;" ::: "memory");
}

// 4-point DFT X[m] = sum_x e^{-i pi m x / 2} z[x] in place.
__device__ inline void dft4tc(float2& z0, float2& z1, float2& z2, float2& z3) {
  const float2 t0 = cadd(z0, z2), t1 = csub(z0, z2), t2 = cadd(z1, z3), t3 = csub(z1, z3);
  const float2 mt3 = make_float2(t3.y, -t3.x);
  z0 = cadd(t0, t2);
  z2 = csub(t0, t2);
  z1 = cadd(t1, mt3);
  z3 = csub(t1, mt3);
}

// Byte offset of 16-byte unit q (0..3) of row r in a K-major 64-byte-swizzled tile.
__device__ inline uint32_t sw64(int r, int q) {
  return static_cast<uint32_t>(r * 64 + ((q ^ ((r >> 1) & 3)) << 4));
}

// The sites whose vertex ranges meet chunk [c0, c0 + 32): ra .. rb (consecutive in site order;
// sites without vertices in between are included and add nothing).
__device__ inline void chunkSites(const int* cs, int c0, int n, int& ra, int& rb) {
  const int c1 = min(c0 + 32, n);
  ra = kSites;
  rb = -1;
  for (int r = 0; r < kSites; ++r) {
    if (cs[r + 1] > c0 && ra == kSites)
      ra = r;
    if (cs[r] < c1 && cs[r + 1] > cs[r])
      rb = r;
  }
}

__global__ void __launch_bounds__(kThreads, 2)
colFactorTcKernel(const __grid_constant__ CUtensorMap tmX, const TpDims dims, const SectorDesc* __restrict__ sectors,
                  const int* __restrict__ col_start, const double2* __restrict__ T, const float* __restrict__ xInv,
                  int Dp, int Kr, const double2* __restrict__ Fb, const double2* __restrict__ G0,
                  float2* __restrict__ G, long g_sector_stride, int* __restrict__ gmax, int row0, const ColFft fft,
                  int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  float2* Ts = reinterpret_cast<float2*>(base + kOffT);  // [2][kW][32] a chunk's T 2^12 s_c / s_max
  float2* Cg = reinterpret_cast<float2*>(base + kOffC);  // [kW][FFT slot g] -(1/Nc) G0 conj Fb(r0, km[g])
  float2* Ds = Cg + kW * 16;                             // [kW][k2] beta G0, the delta term
  int* cs = reinterpret_cast<int*>(base + kOffTab);      // [17] site starts (column order)
  int* rm = cs + 17;                                     // [16] FFT slot -> site
  int* km = rm + 16;                                     // [16] FFT slot -> momentum
  float* smax = reinterpret_cast<float*>(km + 16);       // the tile's largest X' chunk scale
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kOffBar);
  uint64_t* full_x = bars;                        // [kXStages] TMA -> MMA
  uint64_t* empty_x = full_x + kXStages;          // [kXStages] MMA -> TMA
  uint64_t* full_b = empty_x + kXStages;          // [kBSlots] builders -> MMA
  uint64_t* empty_b = full_b + kBSlots;           // [kBSlots] MMA -> builders
  uint64_t* acc_full = empty_b + kBSlots;         // MMA -> epilogue
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_full + 1);

  const int t = threadIdx.x, warp = t / 32, lane = t % 32;
  const SectorDesc sd = sectors[blockIdx.z];
  const int n = sd.n, nw_ext = dims.nw_ext, R = dims.R;
  const int mt = row0 / 128 + blockIdx.x;  // X' / G row tile
  const int w2_0 = blockIdx.y * kW;
  const int n_chunks = (n + 31) / 32;
  const int kxc = Kr / 32;
  const float* xs = xInv + (static_cast<long>(blockIdx.z) * (Dp / 128) + mt) * kxc;

  if (warp == 1) {
    tc::tmemAlloc(tmem_slot, kTmemCols);
    tc::tmemRelinquish();
  }
  if (t == 0) {
    for (int s = 0; s < kXStages; ++s) {
      mbarInit(&full_x[s], 1);
      mbarInit(&empty_x[s], 1);
    }
    for (int s = 0; s < kBSlots; ++s) {
      mbarInit(&full_b[s], kBuilders / 32);  // one arrival per builder warp
      mbarInit(&empty_b[s], 1);
    }
    mbarInit(acc_full, 1);
    fenceBarrierInit();
    tc::prefetchTensorMap(&tmX);
  }
  if (t <= 16)
    cs[t] = col_start[sd.orb_off + t];
  if (t < 16) {
#pragma unroll
    for (int g = 0; g < 16; ++g)
      if (g == t) {
        rm[g] = fft.rmap[g];
        km[g] = fft.kmap[g];
      }
  }
  if (warp == 2) {  // the tile's largest chunk scale: the B operands carry s_c / s_max <= 1
    float m = 0.f;
    for (int c = lane; c < n_chunks; c += 32)
      m = fmaxf(m, xs[c]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    if (lane == 0)
      *smax = m > 0.f ? m : 1.f;
  }
  for (int i = t; i < kW * 16; i += kThreads) {
    const int k = i % 16, w2 = w2_0 + i / 16;
    const double2 g0d = G0[static_cast<long>(sd.spin) * nw_ext * 16 + k + 16 * w2];  // G0_s(k, w2), one band
    Ds[i] = make_float2(static_cast<float>(dims.beta * g0d.x), static_cast<float>(dims.beta * g0d.y));
    // Slot order: entry (w, g) holds the factor of momentum km[g].
    int kg = 0;
#pragma unroll
    for (int g = 0; g < 16; ++g)
      if (g == k)
        kg = fft.kmap[g];
    double2 g0 = G0[static_cast<long>(sd.spin) * nw_ext * 16 + kg + 16 * w2];
    const double2 f = Fb[kg * 16 + fft.r0];  // the band phase e^{-i k a}: conj Fb(r0, k) (x_r0 = 0)
    g0 = make_double2(g0.x * f.x + g0.y * f.y, g0.y * f.x - g0.x * f.y);
    Cg[i] = make_float2(static_cast<float>(-g0.x / 16), static_cast<float>(-g0.y / 16));
  }
  tc::fenceBeforeThreadSync();
  __syncthreads();
  tc::fenceAfterThreadSync();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;
  {  // the tile's scale s_max 2^-12 of the tensor-memory sums into the G0 factors (exact: powers of two)
    const float zs = *smax * (1.f / kTScale);
    for (int i = t; i < kW * 16; i += kThreads)
      Cg[i] = make_float2(Cg[i].x * zs, Cg[i].y * zs);
  }
  if (warp >= 2) {  // every site's sums start at zero, so that each MMA accumulates
    const uint32_t qa = tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16);
#pragma unroll
    for (uint32_t c = 0; c < kTmemCols; c += 32)
      stZero32x32bx32(qa + c);
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
  }
  tc::fenceBeforeThreadSync();
  __syncthreads();
  tc::fenceAfterThreadSync();

  if (warp == 0) {
    if (lane == 0) {
      for (int c = 0; c < n_chunks && ok; ++c) {
        const int s = c % kXStages, use = c / kXStages;
        if (use > 0 && !mbarWait(&empty_x[s], (use - 1) & 1, err)) {
          ok = false;
          break;
        }
        unsigned char* st = base + s * kXStage;
        mbarArriveExpectTx(&full_x[s], kXStage);
#pragma unroll
        for (int pl = 0; pl < 2; ++pl) {
          const int z = static_cast<int>(blockIdx.z) * 2 + pl;
          tc::tmaLoad3d(st + (0 + pl) * kXBox, &tmX, c * 32, mt * 128, z, &full_x[s]);       // re
          tc::tmaLoad3d(st + (2 + pl) * kXBox, &tmX, Kr + c * 32, mt * 128, z, &full_x[s]);  // im
        }
      }

      // Loads still in flight are waited for (bounded) before the CTA can exit.
      for (int c = max(0, n_chunks - kXStages); c < n_chunks; ++c)
        mbarWait(&full_x[c % kXStages], (c / kXStages) & 1, err);
    }
  }
  else if (warp == 1) {
    if (lane == 0) {
      const int pa[3] = {1, 0, 0};  // (A plane, B plane) products, smallest first: lo hi, hi lo, hi hi
      const int pb[3] = {0, 1, 0};
      // Descriptors of stage 0 / slot 0; the others differ by the stage / slot stride (>> 4).
      uint64_t dA[4], dB[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        dA[i] = tc::smemDescSw64(base + i * kXBox);
        dB[i] = tc::smemDescSw64(base + kOffB + i * kBTile);
      }
      int item = 0;
      for (int c = 0; c < n_chunks && ok; ++c) {
        const int s = c % kXStages;
        if (!mbarWait(&full_x[s], (c / kXStages) & 1, err)) {
          ok = false;
          break;
        }
        tc::fenceAfterThreadSync();
        const int c0 = c * 32;
        int ra, rb;
        chunkSites(cs, c0, n, ra, rb);
        for (int g0 = ra; g0 <= rb; g0 += kMaxGroup) {
          const int ng = min(kMaxGroup, rb - g0 + 1);
          const int lo = cs[g0], hi = cs[g0 + ng];
          const int slot = item % kBSlots;
          if (!mbarWait(&full_b[slot], (item / kBSlots) & 1, err)) {
            ok = false;
            break;
          }
          tc::fenceAfterThreadSync();
          const uint32_t d = tmem + g0 * kN;
          const uint32_t idesc = tc::instrDescF16F32(128, kN * ng);
          // The small products of both 16-vertex steps first, then the hi x hi ones.
#pragma unroll
          for (int pp = 0; pp < 3; ++pp) {
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
              if (hi <= c0 + 16 * kk || lo >= c0 + 16 * kk + 16)
                continue;  // this 16-vertex step holds none of the group's vertices
              const uint64_t xo = (s * kXStage + kk * 32) >> 4, bo = (slot * kBItem + kk * 32) >> 4;
              const uint64_t ar = dA[0 + pa[pp]] + xo, ai = dA[2 + pa[pp]] + xo;
              const uint64_t br = dB[0 + pb[pp]] + bo, bi = dB[2 + pb[pp]] + bo;
              tc::mmaBf16(d, ar, br, idesc, 1);
              tc::mmaBf16(d, ai, bi, idesc, 1);
            }
          }
          tc::commitTo(&empty_b[slot]);  // the builders may refill this slot once these MMAs finish
          ++item;
        }
        if (!ok)
          break;
        tc::commitTo(&empty_x[s]);
      }
      tc::commitTo(acc_full);  // every MMA of the tile issued (none for an empty sector)
    }
  }
  else {
    // Builders: the same (chunk, site group) item sequence as the MMA issuer.
    const int bt = t - 64;
    const float s_max = *smax;
    // A chunk's twiddles T(w2, j) (8 frequencies x 32 vertices, two per thread) are loaded one chunk
    // ahead into registers, scaled by the chunk's 2^12 s_c / s_max (exact: powers of two) and
    // stored into one of two buffers; one named barrier per chunk publishes them (and orders the
    // reuse of the buffer the chunk before last read).
    const double2* Tsec = T + static_cast<long>(sd.vtx_off) * nw_ext + static_cast<long>(w2_0) * n;
    auto loadT = [&](int c, double2 (&v)[2]) {
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int i = bt + u * kBuilders, wl = i / 32, j = c * 32 + i % 32;
        v[u] = (c < n_chunks && j < n) ? Tsec[static_cast<long>(wl) * n + j] : make_double2(0., 0.);
      }
    };
    double2 tcur[2], tnext[2];
    loadT(0, tcur);

    int item = 0;
    for (int c = 0; c < n_chunks; ++c) {
      const int c0 = c * 32;
      loadT(c + 1, tnext);
      {
        const float f = xs[c] / s_max * kTScale;
        float2* tb = Ts + (c & 1) * kW * 32;
#pragma unroll
        for (int u = 0; u < 2; ++u)
          tb[bt + u * kBuilders] = make_float2(static_cast<float>(tcur[u].x) * f, static_cast<float>(tcur[u].y) * f);
      }
      namedSync128();
      const float2* tb = Ts + (c & 1) * kW * 32;
      int ra, rb;
      chunkSites(cs, c0, n, ra, rb);
      for (int g0 = ra; g0 <= rb && ok; g0 += kMaxGroup) {
        const int ng = min(kMaxGroup, rb - g0 + 1);
        const int slot = item % kBSlots, use = item / kBSlots;
        if (use > 0 && !__all_sync(0xffffffffu, mbarWait(&empty_b[slot], (use - 1) & 1, err))) {
          ok = false;  // the issuer sees the missing item as a timeout of its own
          continue;
        }
        // Units (part, row, 8 vertices): row 16 i + 2 w + p of B_re = (Tr, -Ti), of B_im = (Ti, Tr)
        // for site g0 + i; vertices outside that site are zero.  ng units per thread.
        for (int u = 0; u < ng; ++u) {
          const int ui = bt + kBuilders * u;
          const int q = ui % 4, row = (ui / 4) % (kN * ng), part = ui / (4 * kN * ng);
          const int site = g0 + row / kN, w = (row % kN) / 2, p = row % 2;
          const int lo = cs[site], hi = cs[site + 1];
          float y[8];
#pragma unroll
          for (int x = 0; x < 8; ++x) {
            const int jl = 8 * q + x, j = c0 + jl;
            const float2 tv = tb[w * 32 + jl];
            const float val = part == 0 ? (p == 0 ? tv.x : -tv.y) : (p == 0 ? tv.y : tv.x);
            y[x] = (j >= lo && j < hi) ? val : 0.f;
          }
          tcg::Pack8 h, l;
          tcg::split8(y, h, l);
          unsigned char* bst = base + kOffB + slot * kBItem + (2 * part) * kBTile + sw64(row, q);
          tcg::store8(reinterpret_cast<__half*>(bst), h);
          tcg::store8(reinterpret_cast<__half*>(bst + kBTile), l);
        }
        fenceProxyAsync();  // generic-proxy writes -> the tensor core's reads
        __syncwarp();
        if (lane == 0)
          mbarArrive(&full_b[slot]);
        ++item;
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
        tcur[u] = tnext[u];
    }
  }

  // Epilogue (warps 2..5): thread = tensor-memory lane = row of the tile.
  if (warp >= 2) {
    const bool got = __all_sync(0xffffffffu, mbarWait(acc_full, 0, err));  // uniform: the loads are warp-wide
    tc::fenceAfterThreadSync();
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    const int rho = mt * 128 + row;
    const int k1 = rho % R, w1 = rho / R;
    const uint32_t lane_addr = tmem + (static_cast<uint32_t>(quarter * 32) << 16);
    unsigned char* stg = base + (warp - 2) * 32 * kEpiRowB;  // warp-private transpose buffer (X' stages)
    float2* gsec = G + g_sector_stride * (2 * sd.slot + sd.spin);
    float gabs = 0.f;
    int kmr[16];  // FFT slot -> momentum, in registers
#pragma unroll
    for (int g = 0; g < 16; ++g)
      kmr[g] = km[g];
    // The X' stages become the transpose buffers: every TMA load has landed and every MMA that
    // read them has completed (acc_full).
    for (int wp = 0; wp < kW / 2; ++wp) {
      float z4[16][4];  // slot g: (re, im) of w2 = 2 wp and 2 wp + 1
#pragma unroll
      for (int g = 0; g < 16; ++g) {
        if (got)  // every site's columns hold its sums (zero for sites without vertices)
          ld32x32bx4(lane_addr + rm[g] * kN + 4 * wp, z4[g]);
        else
          z4[g][0] = z4[g][1] = z4[g][2] = z4[g][3] = 0.f;
      }
      tc::waitLd();
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int wl = 2 * wp + h, w2 = w2_0 + wl;
        float2 z[16];
#pragma unroll
        for (int g = 0; g < 16; ++g)
          z[g] = make_float2(z4[g][2 * h], z4[g][2 * h + 1]);
#pragma unroll
        for (int b = 0; b < 4; ++b)
          dft4tc(z[4 * b], z[4 * b + 1], z[4 * b + 2], z[4 * b + 3]);
#pragma unroll
        for (int m = 0; m < 4; ++m)
          dft4tc(z[m], z[m + 4], z[m + 8], z[m + 12]);
        const float2* cw = Cg + wl * 16;
        __syncwarp();  // the previous frequency's copy-out reads are done
#pragma unroll
        for (int g = 0; g < 16; ++g) {
          const float2 x = cmul(cw[g], z[g]);
          gabs = fmaxf(gabs, fmaxf(fabsf(x.x), fabsf(x.y)));
          *reinterpret_cast<float2*>(stg + lane * kEpiRowB + kmr[g] * 8) = x;
        }
        if (w2 == w1) {  // the delta term at k2 = k1 of the diagonal block
          float2* e = reinterpret_cast<float2*>(stg + lane * kEpiRowB + k1 * 8);
          const float2 x = cadd(*e, Ds[wl * 16 + k1]);
          gabs = fmaxf(gabs, fmaxf(fabsf(x.x), fabsf(x.y)));
          *e = x;
        }
        __syncwarp();
        // The warp's 32 rows (two (w1, w2) blocks of 16 k1 x 16 k2, 2 KB each, contiguous in G):
        // per instruction four rows, lane: row it * 4 + lane / 8, momenta 2 (lane % 8), + 1.
#pragma unroll
        for (int it = 0; it < 8; ++it) {
          const int rl = it * 4 + lane / 8, qq = lane % 8;
          const int rr = mt * 128 + quarter * 32 + rl;
          const float4 v = *reinterpret_cast<const float4*>(stg + rl * kEpiRowB + qq * 16);
          float2* out = gsec + ((static_cast<long>(rr / R) * nw_ext + w2) * R + rr % R) * R + 2 * qq;
          *reinterpret_cast<float4*>(out) = v;
        }
      }
    }
    if (gmax) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1)
        gabs = fmaxf(gabs, __shfl_xor_sync(0xffffffffu, gabs, off));
      if (lane == 0)
        atomicMax(gmax + 2 * sd.slot + sd.spin, __float_as_int(gabs));
    }
  }
  tc::fenceBeforeThreadSync();
  __syncthreads();
  if (warp == 1) {
    tc::fenceAfterThreadSync();
    tc::tmemDealloc(tmem, kTmemCols);
  }
}

}  // namespace

bool colFactorTcApplies(const TpDims& d, int D, int row0, int max_order) {
  return d.nb == 1 && d.nc == 16 && d.nw_ext % kW == 0 && D % 128 == 0 && row0 % 128 == 0 &&
         colFactorTcSmem(max_order) <= 227 * 1024;
}

int launchColFactorTc(const FrontendArgs& a, const FrontTcWorkspace& w, float2* G, long g_sector_stride, int* gmax,
                      int* err, cudaStream_t stream) {
  const TpDims& d = a.dims;
  const FrontTcShape& s = w.shape;
  if (gmax)
    DCAACC_CUDA_CHECK(cudaMemsetAsync(gmax, 0, sizeof(int) * size_t(a.n_sectors), stream));
  const int row0 = d.half_g ? s.D / 2 : 0;
  const size_t smem = colFactorTcSmem(0);
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(colFactorTcKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  // Two CTAs per SM (their tensor memory halves fill it) need the largest shared-memory carveout.
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(colFactorTcKernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         int(cudaSharedmemCarveoutMaxShared)));
  const dim3 grid((s.D - row0) / 128, d.nw_ext / kW, a.n_sectors);
  colFactorTcKernel<<<grid, kThreads, smem, stream>>>(w.tm_ac, d, a.sectors, a.col_start, a.Tc, w.xInv, s.Dp, s.Kr,
                                                       a.Fb, a.G0, G, g_sector_stride, gmax, row0, w.fft, err);
  DCAACC_LAUNCH_CHECK();
  return 1;
}

}  // namespace dcaacc

