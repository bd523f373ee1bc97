// Column step of the mixed path, factored by orbital (one band).
//
// The dense column step computes G = X' Q^H with K = every vertex j of the sector, although Q only
// varies with j through the vertex's site and time:
//   Q(rho2, j) = -(1/Nc) e^{i k2 x_j} e^{i w2 tau_j} conj G0_s(k2, w2),   rho2 = k2 + Nc w2.
// Grouping the column vertices by orbital r (= site, one band) -- the reference's own order of
// work, the column NDFT per orbital (CachedNdft<GPU>::performFT, cached_ndft_gpu.hpp:193-252)
// followed by the cluster transform (SpaceTransform2DGpu::execute, space_transform_2D_gpu.hpp:
// 116-159) -- gives
//   Z(rho1, w2, r)  = sum_{j in orbital r} X'(rho1, j) conj T(w2, j),     T(w, j) = e^{i w tau_j}
//   G(rho1; k2, w2) = -(1/Nc) G0_s(k2, w2) sum_r e^{-i k2 x_r} Z(rho1, w2, r)
//                     + beta G0_s(k2, w2) delta_{rho1, rho2}
// whose work is 8 D NwExt n + 8 D^2 Nc flops per sector instead of 8 D^2 n (12x less on the 4x4
// benchmark cluster).  Two kernels, both selected by DCAACC_TP_FACTORED_COL=1 (the dense tcgen05
// GEMM stays the default, being faster on B200: see the tensor-core form below):
//  - colFactorMmaKernel (4 x 4 clusters): stage A on the tensor cores, stage B as a 4 x 4 FFT;
//  - colFactorKernel (any 16-site cluster, or DCAACC_TP_COL_FFT=0): both stages in FP32 on the
//    CUDA cores of one CTA per (sector, 32 rows rho1, 16 frequencies w2):
//   stage A  the column-sorted vertices are staged in chunks of kVC: X' (decoded from the row
//            step's two FP16 planes and their per-chunk power-of-two scale, exact in FP32) and
//            conj T; warp w accumulates Z for the orbitals r = w, w + 8, ... in registers, each
//            lane a 4 x 4 tile of (rho1, w2) over the orbital's vertices;
//   stage B  Z goes to shared memory (over the staging buffers), and each thread transforms the r
//            axis of two (rho1, w2) pairs into k2 with the G0 factor and the delta term, stores the
//            16 complex values of a G block row (128 bytes), and records the sector's largest |G|
//            for the G4 kernel's operand scaling.
// With half G (mirror symmetry) only the rows rho1 of the upper frequency half are computed, as in
// the dense step.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "tp_frontend.hpp"
#include "tp_layout.hpp"

namespace dcaacc {

namespace {

constexpr int kRT = 32;    // rows rho1 per CTA
constexpr int kWT = 16;    // frequencies w2 per CTA
constexpr int kVC = 128;   // vertices per staged chunk
constexpr int kVP = kVC + 1;  // padded row of the staging buffers
constexpr int kRTP = kRT + 8;  // padded row of Z (lanes with w2 four apart fall in other banks)
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

template <int NC>
constexpr size_t colFactorSmem() {
  constexpr size_t stage = sizeof(float2) * (size_t(kRT) * kVP + size_t(kWT) * kVP);
  constexpr size_t zs = sizeof(float2) * size_t(NC) * kWT * kRTP;
  return (stage > zs ? stage : zs) + sizeof(float2) * (NC * NC + 2 * kWT * NC) + sizeof(int) * (NC + 1);
}

// 4-point DFT X[m] = sum_x e^{-i pi m x / 2} z[x] in place (additions only).
__device__ inline void dft4(float2& z0, float2& z1, float2& z2, float2& z3) {
  const float2 t0 = cadd(z0, z2), t1 = csub(z0, z2), t2 = cadd(z1, z3), t3 = csub(z1, z3);
  const float2 mt3 = make_float2(t3.y, -t3.x);  // -i t3
  z0 = cadd(t0, t2);
  z2 = csub(t0, t2);
  z1 = cadd(t1, mt3);
  z3 = csub(t1, mt3);
}

template <int NC, bool FFT>
__global__ void __launch_bounds__(kThreads, 2)
colFactorKernel(const TpDims dims, const SectorDesc* __restrict__ sectors, const int* __restrict__ col_start,
                const double2* __restrict__ T, const __half* __restrict__ ac, const float* __restrict__ xInv,
                int Dp, int Kr, const double2* __restrict__ Fb, const double2* __restrict__ G0,
                float2* __restrict__ G, long g_sector_stride, int* __restrict__ gmax, int row0, const ColFft fft) {
  constexpr int NO = (NC + kWarps - 1) / kWarps;  // orbitals per warp
  extern __shared__ __align__(16) unsigned char smem[];
  float2* Xs = reinterpret_cast<float2*>(smem);   // [kRT][kVP]   stage A
  float2* Ts = Xs + kRT * kVP;                     // [kWT][kVP]   stage A
  float2* Zs = reinterpret_cast<float2*>(smem);   // [NC][kWT][kRTP] stage B (over the staging)
  constexpr size_t stage_bytes = sizeof(float2) * (size_t(kRT) * kVP + size_t(kWT) * kVP);
  constexpr size_t zs_bytes = sizeof(float2) * size_t(NC) * kWT * kRTP;
  float2* Fs = reinterpret_cast<float2*>(smem + (stage_bytes > zs_bytes ? stage_bytes : zs_bytes));  // [k2][r]
  float2* Cs = Fs + NC * NC;   // [kWT][NC] -(1/Nc) G0_s(k2, w2) (FFT: times conj Fb(r0, k2))
  float2* Ds = Cs + kWT * NC;  // [kWT][NC] beta G0_s(k2, w2), the delta term
  int* cs = reinterpret_cast<int*>(Ds + kWT * NC);  // [NC + 1] orbital starts (column order)

  const int t = threadIdx.x, warp = t / 32, lane = t % 32;
  const SectorDesc sd = sectors[blockIdx.z];
  const int n = sd.n, nw_ext = dims.nw_ext;
  const int rho_0 = row0 + blockIdx.x * kRT;  // first row of this CTA
  const int w2_0 = blockIdx.y * kWT;
  const int xtiles = Dp / 128, kxc = Kr / 32;
  const long plane = static_cast<long>(Dp) * 2 * Kr;
  const __half* xp = ac + static_cast<long>(blockIdx.z) * 2 * plane;  // hi plane; lo at + plane
  const float* xs_scale = xInv + static_cast<long>(blockIdx.z) * xtiles * kxc;
  const double2* Tsec = T + static_cast<long>(sd.vtx_off) * nw_ext;

  // F(k2, r) = e^{-i k2 (x_r + a_0)} = conj Fb(r, k2, band 0).
  for (int i = t; i < NC * NC; i += kThreads) {
    const double2 f = Fb[i];  // (k * NC + r)
    Fs[i] = make_float2(static_cast<float>(f.x), -static_cast<float>(f.y));
  }
  for (int i = t; i <= NC; i += kThreads)
    cs[i] = col_start[sd.orb_off + i];
  {
    const double2* g0s = G0 + static_cast<long>(sd.spin) * nw_ext * NC;  // G0_s(k, w) at k + NC w (one band)
    for (int i = t; i < kWT * NC; i += kThreads) {
      const int k = i % NC, w2 = w2_0 + i / NC;
      double2 g0 = w2 < nw_ext ? g0s[k + NC * w2] : make_double2(0., 0.);
      Ds[i] = make_float2(static_cast<float>(dims.beta * g0.x), static_cast<float>(dims.beta * g0.y));
      if (FFT) {  // the band phase e^{-i k a}: conj Fb(r0, k) (x_r0 = 0)
        const double2 f = Fb[k * NC + fft.r0];
        g0 = make_double2(g0.x * f.x + g0.y * f.y, g0.y * f.x - g0.x * f.y);
      }
      Cs[i] = make_float2(static_cast<float>(-g0.x / NC), static_cast<float>(-g0.y / NC));
    }
  }

  // Lane tile of stage A: rows rg + 8 a, frequencies wg + 4 b (a, b < 4): interleaved, so that the
  // eight row groups of a warp read distinct shared-memory banks.
  const int rg = lane / 4, wg = lane % 4;
  float2 acc[NO][4][4];
#pragma unroll
  for (int o = 0; o < NO; ++o)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
        acc[o][a][b] = make_float2(0.f, 0.f);

  for (int c0 = 0; c0 < n; c0 += kVC) {
    const int vc = min(kVC, n - c0);
    __syncthreads();  // the previous chunk's reads are done (and Fs / cs are in place)
    // X'(rho_0 + row, c0 + jl) = (hi + lo) 2^{-e(row tile, chunk)}, real part at column j of the
    // plane row, imaginary part at column Kr + j: per work item 8 consecutive vertices of one row,
    // read as four 16-byte vectors (hi re, hi im, lo re, lo im), all loads of a thread issued first.
    // A half-warp takes 16 rows at one vertex group (a warp: two adjacent groups, i.e. one 32-byte
    // sector per row and plane part), so that its shared-memory stores fall in distinct banks.
    {
      constexpr int kItems = kRT * kVC / 8;                  // 512
      constexpr int kPer = (kItems + kThreads - 1) / kThreads;  // 2
      uint4 hr[kPer], hi[kPer], lr[kPer], li[kPer];
      float sc[kPer];
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int it = t + u * kThreads;
        const int row = (it % 16) + 16 * ((it / 32) % 2), g8 = 2 * (it / 64) + (it / 16) % 2;
        const int rho = rho_0 + row, j = c0 + 8 * g8;
        if (it < kItems && rho < Dp && 8 * g8 < vc) {
          const long o = static_cast<long>(rho) * 2 * Kr + j;
          hr[u] = *reinterpret_cast<const uint4*>(xp + o);
          hi[u] = *reinterpret_cast<const uint4*>(xp + o + Kr);
          lr[u] = *reinterpret_cast<const uint4*>(xp + o + plane);
          li[u] = *reinterpret_cast<const uint4*>(xp + o + plane + Kr);
          sc[u] = xs_scale[(rho / 128) * kxc + j / 32];
        }
        else {
          hr[u] = hi[u] = lr[u] = li[u] = make_uint4(0, 0, 0, 0);
          sc[u] = 0.f;
        }
      }
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int it = t + u * kThreads;
        if (it >= kItems)
          break;
        const int row = (it % 16) + 16 * ((it / 32) % 2), g8 = 2 * (it / 64) + (it / 16) % 2;
        const __half* a = reinterpret_cast<const __half*>(&hr[u]);
        const __half* b = reinterpret_cast<const __half*>(&hi[u]);
        const __half* c = reinterpret_cast<const __half*>(&lr[u]);
        const __half* d = reinterpret_cast<const __half*>(&li[u]);
#pragma unroll
        for (int x = 0; x < 8; ++x) {
          // Vertices beyond the sector's order are zero in the planes (and sc is 0 past the rows).
          const bool in = 8 * g8 + x < vc;
          Xs[row * kVP + 8 * g8 + x] =
              in ? make_float2((__half2float(a[x]) + __half2float(c[x])) * sc[u],
                               (__half2float(b[x]) + __half2float(d[x])) * sc[u])
                 : make_float2(0.f, 0.f);
        }
      }
    }
    {
      constexpr int kPer = kWT * kVC / kThreads;  // 8
      double2 tv[kPer];
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int idx = t + u * kThreads, wl = idx / kVC, jl = idx % kVC;
        tv[u] = (jl < vc && w2_0 + wl < nw_ext) ? Tsec[static_cast<long>(w2_0 + wl) * n + c0 + jl]
                                                : make_double2(0., 0.);
      }
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int idx = t + u * kThreads, wl = idx / kVC, jl = idx % kVC;
        Ts[wl * kVP + jl] = make_float2(static_cast<float>(tv[u].x), -static_cast<float>(tv[u].y));  // conj T
      }
    }
    __syncthreads();
#pragma unroll
    for (int o = 0; o < NO; ++o) {
      const int r = warp + kWarps * o;
      if (r >= NC)
        break;
      const int j0 = max(cs[r], c0) - c0, j1 = min(cs[r + 1], c0 + vc) - c0;
      for (int jl = j0; jl < j1; ++jl) {
        float2 x[4], y[4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
          x[a] = Xs[(rg + 8 * a) * kVP + jl];
#pragma unroll
        for (int b = 0; b < 4; ++b)
          y[b] = Ts[(wg + 4 * b) * kVP + jl];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b)
            cfma(acc[o][a][b], x[a], y[b]);
      }
    }
  }
  __syncthreads();  // the staging buffers become Zs
#pragma unroll
  for (int o = 0; o < NO; ++o) {
    const int r = warp + kWarps * o;
    if (r >= NC)
      break;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
        Zs[(r * kWT + wg + 4 * b) * kRTP + rg + 8 * a] = acc[o][a][b];
  }
  __syncthreads();

  // Stage B: pair (row, w2l) -> G(rho; k2, w2) for all k2 (one G block row, 16 complex for Nc 16).
  const int R = dims.R;
  float2* gsec = G + g_sector_stride * (2 * sd.slot + sd.spin);
  float gabs = 0.f;
  for (int p = t; p < kRT * kWT; p += kThreads) {
    const int row = p % kRT, wl = p / kRT;
    const int rho = rho_0 + row, w2 = w2_0 + wl;
    if (rho >= dims.R * nw_ext || w2 >= nw_ext)
      continue;
    const int k1 = rho % R, w1 = rho / R;
    float2* out = gsec + ((static_cast<long>(w1) * nw_ext + w2) * R + k1) * R;
    const float2* cw = Cs + wl * NC;
    const float2* dw = Ds + wl * NC;
    const bool diag = w2 == w1;  // the delta term sits at k2 = k1 of the diagonal block
    if constexpr (FFT) {
      // sum_r e^{-i k2 x_r} Z(r) on the 4 x 4 grid: z[a + 4 b] = Z(site at (a, b)), output
      // [m + 4 n] = momentum 2 pi (m, n) / 4, by 4-point DFTs along a, then along b.
      float2 z[16];
#pragma unroll
      for (int g = 0; g < 16; ++g)
        z[g] = Zs[(fft.rmap[g] * kWT + wl) * kRTP + row];
#pragma unroll
      for (int b = 0; b < 4; ++b)
        dft4(z[4 * b], z[4 * b + 1], z[4 * b + 2], z[4 * b + 3]);
#pragma unroll
      for (int m = 0; m < 4; ++m)
        dft4(z[m], z[m + 4], z[m + 8], z[m + 12]);
      // Output g is momentum kmap[g]: put it back in k2 order through this pair's own 16 Z slots
      // (already read into registers; no other thread touches them), then store 16 bytes at a time.
      float2* zp = Zs + wl * kRTP + row;  // slot of r: zp[r * kWT * kRTP]
#pragma unroll
      for (int g = 0; g < 16; ++g) {
        const int k2 = fft.kmap[g];
        float2 x = cmul(cw[k2], z[g]);
        if (diag && k2 == k1)
          x = cadd(x, dw[k2]);
        zp[k2 * kWT * kRTP] = x;
        gabs = fmaxf(gabs, fmaxf(fabsf(x.x), fabsf(x.y)));
      }
#pragma unroll
      for (int k2 = 0; k2 < 16; k2 += 2) {
        const float2 a = zp[k2 * kWT * kRTP], b = zp[(k2 + 1) * kWT * kRTP];
        *reinterpret_cast<float4*>(out + k2) = make_float4(a.x, a.y, b.x, b.y);
      }
    }
    else {
      float2 z[NC];
#pragma unroll
      for (int r = 0; r < NC; ++r)
        z[r] = Zs[(r * kWT + wl) * kRTP + row];
#pragma unroll 2
      for (int k2 = 0; k2 < NC; k2 += 2) {
        float2 v[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float2 g = make_float2(0.f, 0.f);
#pragma unroll
          for (int r = 0; r < NC; ++r)
            cfma(g, Fs[(k2 + h) * NC + r], z[r]);
          v[h] = cmul(cw[k2 + h], g);
          if (diag && k2 + h == k1)
            v[h] = cadd(v[h], dw[k2 + h]);
          gabs = fmaxf(gabs, fmaxf(fabsf(v[h].x), fabsf(v[h].y)));
        }
        *reinterpret_cast<float4*>(out + k2) = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
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

// ---- Tensor-core form (4 x 4 cluster, the FFT cluster transform) ----
//
// Stage A as warp-level tensor-core products (mma.sync m16n8k16, FP16 in, FP32 accumulate), split
// FP16 on both sides (hi hi + hi lo + lo hi): A = the row step's X' planes as they lie in global
// memory (hi / lo, real / imaginary, each 32-vertex chunk of a 128-row tile at its own power-of-two
// scale), B = the column twiddles T(w2, j) 2^12 split into FP16 planes by colTwiddlePlanesKernel.
// The vertices are sorted by site, but the sites' blocks do not start on 16-vertex boundaries: a
// 16-vertex step is multiplied once per site it overlaps, with the other sites' vertices masked to
// zero in the A fragments (about twice the products of the site sums, at 16-vertex granularity).
// CTA: 16 rows rho1 (k1 = 0..15 of one w1) x 32 frequencies w2; its
// four warps each take a quarter of the sites (r = warp mod 4) over the whole 16 x 32 tile (four n8
// tiles, 48 products per site and step).  A warp walks its sites in vertex order with one open
// accumulator (the site that runs on into the next chunk keeps it) and stores each finished site's
// Z tile to shared memory.  Stage B (thread = one (row, w2) pair at a time): the 4 x 4 FFT over the
// sites, the G0 factor and the delta term, written back over the pair's own Z slots in momentum
// order; G then leaves as whole (w1, w2) blocks of 16 k1 x 16 k2 (2 KB, contiguous in G), 512
// bytes per warp store.
// Measured on B200 (4x4 cluster, Nw = 64, n ~ U[50, 400]): about 4.7 us per sector against 3.5 us
// for the dense tcgen05 GEMM.  Z (16 x 32 x 16 sites, 74 KB) must stay on chip until the FFT, which
// caps the CTA tile: every CTA re-reads the twiddle planes of its sector (32x per sector) and X'
// (2x), with two 12 KB stages in flight per CTA, and the kernel waits on those loads (tensor pipe
// 16 %, L2 throughput 13 %, issue 27 %).
namespace tcf {

constexpr int kRows = 16;      // rows rho1 per CTA: one m16 tile, k1 = 0..15 of one w1
constexpr int kCols = 32;      // frequencies w2 per CTA: four n8 tiles
constexpr int kChunk = 32;     // vertices per staged chunk (the X' scale chunk)
constexpr int kStages = 2;
constexpr int kThreads = 128;  // 4 warps: site groups r = warp (mod 4)
constexpr int kWarps = kThreads / 32;
constexpr float kTScale = 4096.f;  // T is split at 2^12 |T| (the low part stays a normal FP16)
constexpr int kXPlane = kRows * 64;            // 16 rows x 32 vertices of one FP16 plane
constexpr int kTPlane = kCols * 64;            // 32 frequencies x 32 vertices
constexpr int kStageBytes = 4 * kXPlane + 4 * kTPlane;  // X' re hi, re lo, im hi, im lo; T the same
// Z(site, w2, row) as float2: rows of 16 (+2) entries, sites 32 w2 rows (+8 bytes) apart, so that
// the fragment stores, the FFT's row reads and the output's momentum-pair reads are conflict-free.
constexpr int kZRow = (kRows + 2) * 8;         // 144 bytes
constexpr int kZSite = kCols * kZRow + 8;      // 4616 bytes
constexpr int kZBytes = 16 * kZSite;
constexpr int kSmem = kZBytes + kStages * kStageBytes + 2 * kCols * 16 * 8 + (17 + 2 * 16) * 4;

__device__ inline void ldsm4(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(p))));
}

__device__ inline void mma(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ inline void cpAsync16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ inline void cpAsyncCommit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ inline void cpAsyncWait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Byte offset of 16-byte unit q (0..3) of row r in a 32 x 64-byte plane: q ^ ((r >> 1) & 3), so
// that the eight rows an ldmatrix phase reads fall in distinct banks.
__device__ inline int swz(int r, int q) {
  return r * 64 + ((q ^ ((r >> 1) & 3)) << 4);
}

// T(w, j) 2^12 of each sector's column-sorted vertices as four FP16 planes [re hi, re lo, im hi,
// im lo][w][Kr] (zero for j >= n).
__global__ void colTwiddlePlanesKernel(const TpDims dims, const SectorDesc* __restrict__ sectors,
                                       const double2* __restrict__ T, __half* __restrict__ tp, int Kr) {
  const SectorDesc sd = sectors[blockIdx.y];
  const int nw = dims.nw_ext;
  const long per = static_cast<long>(nw) * Kr;
  __half* o = tp + static_cast<long>(blockIdx.y) * 4 * per;
  const double2* Ts = T + static_cast<long>(sd.vtx_off) * nw;
  for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < per;
       i += static_cast<long>(gridDim.x) * blockDim.x) {
    const int w = static_cast<int>(i / Kr), j = static_cast<int>(i % Kr);
    const double2 v = j < sd.n ? Ts[static_cast<long>(w) * sd.n + j] : make_double2(0., 0.);
    const float re = static_cast<float>(v.x) * kTScale, im = static_cast<float>(v.y) * kTScale;
    const __half rh = __float2half_rn(re), ih = __float2half_rn(im);
    o[i] = rh;
    o[per + i] = __float2half_rn(re - __half2float(rh));
    o[2 * per + i] = ih;
    o[3 * per + i] = __float2half_rn(im - __half2float(ih));
  }
}

__global__ void __launch_bounds__(kThreads, 2)
colFactorMmaKernel(const TpDims dims, const SectorDesc* __restrict__ sectors, const int* __restrict__ col_start,
                   const __half* __restrict__ tplanes, const __half* __restrict__ ac, const float* __restrict__ xInv,
                   int Dp, int Kr, const double2* __restrict__ Fb, const double2* __restrict__ G0,
                   float2* __restrict__ G, long g_sector_stride, int* __restrict__ gmax, int row0, const ColFft fft) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* Zs = smem;                                              // [site][w2][row] (padded)
  unsigned char* stg = smem + kZBytes;                                   // [stage] X' and T planes
  float2* Cs = reinterpret_cast<float2*>(stg + kStages * kStageBytes);  // [w2][k2] -(1/Nc) G0 conj Fb(r0, k2)
  float2* Ds = Cs + kCols * 16;                                          // [w2][k2] beta G0, the delta term
  int* cs = reinterpret_cast<int*>(Ds + kCols * 16);                     // [17] site starts (column order)
  int* rm = cs + 17;                                                     // [16] FFT slot -> site
  int* km = rm + 16;                                                     // [16] FFT slot -> momentum

  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g8 = lane / 4, t4 = lane % 4;
  const SectorDesc sd = sectors[blockIdx.z];
  const int n = sd.n, nw_ext = dims.nw_ext, R = dims.R;
  const int rho_0 = row0 + blockIdx.x * kRows, w2_0 = blockIdx.y * kCols;
  const long kp = 2L * Kr, plane = static_cast<long>(Dp) * kp;
  const __half* xsec = ac + static_cast<long>(blockIdx.z) * 2 * plane + static_cast<long>(rho_0) * kp;
  const long tper = static_cast<long>(nw_ext) * Kr;
  const __half* tsec = tplanes + static_cast<long>(blockIdx.z) * 4 * tper + static_cast<long>(w2_0) * Kr;
  const int kxc = Kr / 32;
  const float* xs_scale = xInv + (static_cast<long>(blockIdx.z) * (Dp / 128) + rho_0 / 128) * kxc;

  // Stage a chunk: 256 16-byte units of X' (4 planes x 16 rows x 4) and 512 of T (4 planes x 32
  // frequencies x 4), six per thread.
  auto stage = [&](int c) {
    unsigned char* base = stg + (c % kStages) * kStageBytes;
#pragma unroll
    for (int u = 0; u < 6; ++u) {
      const int idx = tid + u * kThreads;
      if (idx < 256) {
        const int p = idx / 64, r = (idx % 64) / 4, q = idx % 4;
        cpAsync16(base + p * kXPlane + swz(r, q), xsec + (p & 1) * plane + r * kp + (p >> 1) * Kr + c * kChunk + 8 * q);
      }
      else {
        const int rem = idx - 256, p = rem / 128, r = (rem % 128) / 4, q = rem % 4;
        cpAsync16(base + 4 * kXPlane + p * kTPlane + swz(r, q), tsec + p * tper + static_cast<long>(r) * Kr + c * kChunk + 8 * q);
      }
    }
  };
  const int n_chunks = (n + kChunk - 1) / kChunk;
  if (n_chunks > 0)
    stage(0);
  cpAsyncCommit();

  for (int i = tid; i < kZBytes / 16; i += kThreads)  // sites without vertices keep Z = 0
    reinterpret_cast<float4*>(Zs)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  {
    const double2* g0s = G0 + static_cast<long>(sd.spin) * nw_ext * 16;  // G0_s(k, w) at k + 16 w (one band)
    for (int i = tid; i < kCols * 16; i += kThreads) {
      const int k = i % 16, w2 = w2_0 + i / 16;
      double2 g0 = g0s[k + 16 * w2];
      Ds[i] = make_float2(static_cast<float>(dims.beta * g0.x), static_cast<float>(dims.beta * g0.y));
      const double2 f = Fb[k * 16 + fft.r0];  // the band phase e^{-i k a}: conj Fb(r0, k) (x_r0 = 0)
      g0 = make_double2(g0.x * f.x + g0.y * f.y, g0.y * f.x - g0.x * f.y);
      Cs[i] = make_float2(static_cast<float>(-g0.x / 16), static_cast<float>(-g0.y / 16));
    }
    if (tid <= 16)
      cs[tid] = col_start[sd.orb_off + tid];
    if (tid < 16) {
#pragma unroll
      for (int g = 0; g < 16; ++g)
        if (g == tid) {
          rm[g] = fft.rmap[g];
          km[g] = fft.kmap[g];
        }
    }
  }

  // Stage A.  Warp w takes the sites r = w, w + 4, ... in vertex order with one open accumulator
  // (the site that runs on into the next chunk keeps it).  The products of one site within one
  // chunk sum in a fresh tensor-core accumulator, which then joins the open one at the chunk's
  // power-of-two scale (a long chain of tensor-core additions into a large running sum loses
  // precision).
  float zr[4][4], zi[4][4];  // Z re / im of the open site, n8 tile j (w2 8 j + 2 t4 + e % 2)
  int carry = -1;
  for (int c = 0; c < n_chunks; ++c) {
    cpAsyncWait<0>();
    __syncthreads();  // chunk c is in place for every warp; the other stage is free
    if (c + 1 < n_chunks)
      stage(c + 1);
    cpAsyncCommit();
    const unsigned char* base = stg + (c % kStages) * kStageBytes;
    const int c0 = c * kChunk, c1 = c0 + kChunk;
    const float s = xs_scale[c] * (1.f / kTScale);
    for (int r = warp; r < 16; r += kWarps) {
      const int lo = cs[r], hi = cs[r + 1];
      if (lo >= c1 || lo >= n)
        break;  // this and the later sites start beyond the chunk
      if (hi <= c0 || lo == hi)
        continue;
      if (r != carry) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e)
            zr[j][e] = zi[j][e] = 0.f;
      }
      // This chunk's products: Xr Tr, Xi Ti, Xi Tr, -Xr Ti in separate tensor-core accumulators.
      float prr[4][4], pii[4][4], pir[4][4], pri[4][4];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
          prr[j][e] = pii[j][e] = pir[j][e] = pri[j][e] = 0.f;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int k0 = c0 + 16 * h;
        if (k0 >= hi || k0 + 16 <= lo)
          continue;
        // A: X' rows, vertices k0 + 2 t4, + 1 (registers 0, 1) and + 8, + 9 (2, 3), masked to the site.
        const int kt = k0 + 2 * t4;
        const uint32_t m0 = (kt >= lo && kt < hi ? 0xffffu : 0u) | (kt + 1 >= lo && kt + 1 < hi ? 0xffff0000u : 0u);
        const uint32_t m1 =
            (kt + 8 >= lo && kt + 8 < hi ? 0xffffu : 0u) | (kt + 9 >= lo && kt + 9 < hi ? 0xffff0000u : 0u);
        uint32_t a[4][4], na[2][4];  // X' re hi, re lo, im hi, im lo; -X' re hi, re lo
        {
          const int ra = (lane % 8) + 8 * ((lane / 8) % 2), qa = 2 * h + lane / 16;
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            ldsm4(a[p], base + p * kXPlane + swz(ra, qa));
            a[p][0] &= m0;
            a[p][1] &= m0;
            a[p][2] &= m1;
            a[p][3] &= m1;
          }
#pragma unroll
          for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int i = 0; i < 4; ++i)
              na[p][i] = a[p][i] ^ 0x80008000u;
        }
        const int rb = lane % 8, qb = 2 * h + (lane / 8) % 2, pb = lane / 16;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          uint32_t br[4], bi[4];  // T re: hi k0..7, hi k8..15, lo k0..7, lo k8..15; T im the same
          ldsm4(br, base + 4 * kXPlane + pb * kTPlane + swz(8 * j + rb, qb));
          ldsm4(bi, base + 4 * kXPlane + (2 + pb) * kTPlane + swz(8 * j + rb, qb));
          // Z = X' conj T: re = Xr Tr + Xi Ti, im = Xi Tr - Xr Ti; the hi x lo terms first.
          mma(prr[j], a[0], br[2], br[3]);
          mma(pii[j], a[2], bi[2], bi[3]);
          mma(pir[j], a[2], br[2], br[3]);
          mma(pri[j], na[0], bi[2], bi[3]);
          mma(prr[j], a[1], br[0], br[1]);
          mma(pii[j], a[3], bi[0], bi[1]);
          mma(pir[j], a[3], br[0], br[1]);
          mma(pri[j], na[1], bi[0], bi[1]);
          mma(prr[j], a[0], br[0], br[1]);
          mma(pii[j], a[2], bi[0], bi[1]);
          mma(pir[j], a[2], br[0], br[1]);
          mma(pri[j], na[0], bi[0], bi[1]);
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          zr[j][e] = fmaf(s, prr[j][e] + pii[j][e], zr[j][e]);
          zi[j][e] = fmaf(s, pir[j][e] + pri[j][e], zi[j][e]);
        }
      if (hi <= c1) {  // the site ends in this chunk: Z(r) to shared memory
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int row = g8 + 8 * (e / 2), w2l = 8 * j + 2 * t4 + (e % 2);
            *reinterpret_cast<float2*>(Zs + r * kZSite + w2l * kZRow + row * 8) = make_float2(zr[j][e], zi[j][e]);
          }
        carry = -1;
      }
      else {
        carry = r;
      }
    }
  }
  cpAsyncWait<0>();
  __syncthreads();  // Z of every site is in place

  // Stage B: thread = (row, w2) pairs: the 4 x 4 FFT over the sites, the G0 factor and the delta
  // term, written back over the pair's own Z slots in momentum order.
  const int w1 = rho_0 / R;  // the CTA's rows: k1 = 0..15 of one w1
  float gabs = 0.f;
#pragma unroll 1
  for (int pp = 0; pp < kRows * kCols / kThreads; ++pp) {
    const int pidx = tid + pp * kThreads, k1 = pidx % kRows, w2l = pidx / kRows, w2 = w2_0 + w2l;
    unsigned char* zp = Zs + w2l * kZRow + k1 * 8;
    float2 z[16];
#pragma unroll
    for (int g = 0; g < 16; ++g)
      z[g] = *reinterpret_cast<const float2*>(zp + rm[g] * kZSite);
#pragma unroll
    for (int b = 0; b < 4; ++b)
      dft4(z[4 * b], z[4 * b + 1], z[4 * b + 2], z[4 * b + 3]);
#pragma unroll
    for (int m = 0; m < 4; ++m)
      dft4(z[m], z[m + 4], z[m + 8], z[m + 12]);
    const bool diag = w2 == w1;  // the delta term sits at k2 = k1 of the diagonal block
    const float2* cw = Cs + w2l * 16;
    const float2* dw = Ds + w2l * 16;
#pragma unroll
    for (int g = 0; g < 16; ++g) {
      const int k2 = km[g];
      float2 x = cmul(cw[k2], z[g]);
      if (diag && k2 == k1)
        x = cadd(x, dw[k2]);
      gabs = fmaxf(gabs, fmaxf(fabsf(x.x), fabsf(x.y)));
      *reinterpret_cast<float2*>(zp + k2 * kZSite) = x;
    }
  }
  __syncthreads();
  // Out: the CTA's kCols (w1, w2) blocks of 16 k1 x 16 k2 (2 KB each, contiguous in G), one per
  // iteration, 512 bytes per warp store; thread: row k1, momenta 2 cc, 2 cc + 1.
  float2* gsec = G + g_sector_stride * (2 * sd.slot + sd.spin);
  const int cc = tid % 8, k1 = tid / 8;
  const unsigned char* zq = Zs + k1 * 8 + (2 * cc) * kZSite;
  float2* out = gsec + ((static_cast<long>(w1) * nw_ext + w2_0) * R + k1) * R + 2 * cc;
#pragma unroll 4
  for (int w2l = 0; w2l < kCols; ++w2l) {
    const float2 va = *reinterpret_cast<const float2*>(zq + w2l * kZRow);
    const float2 vb = *reinterpret_cast<const float2*>(zq + w2l * kZRow + kZSite);
    *reinterpret_cast<float4*>(out + static_cast<long>(w2l) * R * R) = make_float4(va.x, va.y, vb.x, vb.y);
  }
  if (gmax) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      gabs = fmaxf(gabs, __shfl_xor_sync(0xffffffffu, gabs, off));
    if (lane == 0)
      atomicMax(gmax + 2 * sd.slot + sd.spin, __float_as_int(gabs));
  }
}

}  // namespace tcf

// ---- 6 x 6 clusters (one band, Nc = 36) on the CUDA cores ----
//
// The same two stages for a cluster whose per-site sums do not fit the 16-site tiles above.
// CTA = (sector, 32 rows rho1, 8 frequencies w2), 8 warps, one CTA per SM.
//  stage A  the warps take the sites one at a time from a shared counter (every site, empty ones
//           included, so that each site's Z slot is written).  A warp stages its site's vertices
//           in blocks of up to 32 in its own shared-memory area -- X' decoded from the row step's
//           FP16 planes (hi + lo at the 32-vertex chunk's power-of-two scale, exact in FP32), lane
//           = row, and conj T, lane = vertex -- and each lane sums a 4 x 2 tile of (rho1, w2) over
//           them; the site's Z then goes to shared memory.  No CTA-wide barrier until every site
//           is done, so a warp is never held up by the vertex counts of the other warps' sites.
//  stage B  thread = one (rho1, w2) pair: the 6 x 6 FFT over the sites (6-point DFTs along both
//           grid axes), the G0 factor and the delta term, written back over the pair's own Z
//           slots in momentum order; then G leaves as whole 36-entry rows (k2 fastest), a warp
//           writing 256 contiguous bytes per store instruction.
// Work: 8 D NwExt n flops of site sums per sector (24x less than the dense GEMM's 8 D^2 n at
// Nc = 36) plus the FFTs.
namespace wide {

constexpr int kRows = 32;                       // rows rho1 per CTA
constexpr int kCols = 8;                        // frequencies w2 per CTA
constexpr int kBlk = 32;                        // vertices per staged block of a site
constexpr int kBP = kBlk + 1;                   // padded staging row (float2)
constexpr int kWarps = 8;
constexpr int kThreads = 32 * kWarps;           // = kRows * kCols: one (rho1, w2) pair per thread in stage B
constexpr int kZP = kRows + 4;                  // Z row of one (site, w2), float2: conflict-free lane tiles
constexpr int kZS = kCols * kZP + 1;            // one site's Z; odd, so that the output's reads spread
constexpr int kStageW = (kRows + kCols) * kBP;  // one warp's staging: X' [kRows][kBP], conj T [kCols][kBP]
static_assert(kThreads == kRows * kCols, "stage B: one pair per thread");

template <int NC>
constexpr size_t smemBytes() {
  return sizeof(float2) * (size_t(NC) * kZS + size_t(kWarps) * kStageW + 2 * size_t(kCols) * NC) +
         sizeof(int) * (3 * size_t(NC) + 2);
}

// X_m = sum_x e^{-2 pi i m x / 3} x_x in place.
__device__ inline void dft3(float2& x0, float2& x1, float2& x2) {
  constexpr float s = 0.86602540378443865f;  // sin(pi / 3)
  const float2 t = cadd(x1, x2), u = csub(x1, x2);
  const float2 m = make_float2(x0.x - 0.5f * t.x, x0.y - 0.5f * t.y);
  const float2 v = make_float2(s * u.y, -s * u.x);  // -i s u
  x0 = cadd(x0, t);
  x1 = cadd(m, v);
  x2 = csub(m, v);
}

// X_m = sum_x e^{-2 pi i m x / 6} z_x in place: 3-point DFTs of the even and odd samples, then
// X_m = E_{m mod 3} + e^{-i pi m / 3} O_{m mod 3}.
__device__ inline void dft6(float2& z0, float2& z1, float2& z2, float2& z3, float2& z4, float2& z5) {
  constexpr float s = 0.86602540378443865f;
  float2 e0 = z0, e1 = z2, e2 = z4, o0 = z1, o1 = z3, o2 = z5;
  dft3(e0, e1, e2);
  dft3(o0, o1, o2);
  const float2 p1 = cmul(make_float2(0.5f, -s), o1);   // e^{-i pi / 3} O_1
  const float2 p2 = cmul(make_float2(-0.5f, -s), o2);  // e^{-2 i pi / 3} O_2
  z0 = cadd(e0, o0);
  z3 = csub(e0, o0);
  z1 = cadd(e1, p1);
  z4 = csub(e1, p1);
  z2 = cadd(e2, p2);
  z5 = csub(e2, p2);
}

template <int NC, int L>
__global__ void __launch_bounds__(kThreads, 1)
colFactorWideKernel(const TpDims dims, const SectorDesc* __restrict__ sectors, const int* __restrict__ col_start,
                    const double2* __restrict__ T, const __half* __restrict__ ac, const float* __restrict__ xInv,
                    int Dp, int Kr, const double2* __restrict__ Fb, const double2* __restrict__ G0,
                    float2* __restrict__ G, long g_sector_stride, int* __restrict__ gmax, int row0, const ColFft fft) {
  static_assert(L == 6 && L * L == NC, "6 x 6 cluster");
  extern __shared__ __align__(16) unsigned char smem[];
  float2* Zs = reinterpret_cast<float2*>(smem);      // [site][w2][row], site stride kZS
  float2* Sw = Zs + NC * kZS;                         // [warp] staging
  float2* Cs = Sw + kWarps * kStageW;                 // [w2][k2] -(1/Nc) G0_s(k2, w2) conj Fb(r0, k2)
  float2* Ds = Cs + kCols * NC;                       // [w2][k2] beta G0_s(k2, w2), the delta term
  int* cs = reinterpret_cast<int*>(Ds + kCols * NC);  // [NC + 1] site starts (column order)
  int* rm = cs + NC + 1;                              // [NC] FFT slot -> site
  int* km = rm + NC;                                  // [NC] FFT slot -> momentum
  int* next = km + NC;                                // the next unclaimed site

  const int t = threadIdx.x, warp = t / 32, lane = t % 32;
  const SectorDesc sd = sectors[blockIdx.z];
  const int n = sd.n, nw_ext = dims.nw_ext, R = dims.R, D = R * nw_ext;
  const int rho_0 = row0 + blockIdx.x * kRows, w2_0 = blockIdx.y * kCols;
  const int kxc = Kr / 32;
  const long plane = static_cast<long>(Dp) * 2 * Kr;
  const __half* xp = ac + static_cast<long>(blockIdx.z) * 2 * plane;  // hi plane; lo at + plane
  const float* xs_scale = xInv + static_cast<long>(blockIdx.z) * (Dp / 128) * kxc;
  const double2* Tsec = T + static_cast<long>(sd.vtx_off) * nw_ext;  // T(w, j) at w n + j (column order)

  for (int i = t; i <= NC; i += kThreads)
    cs[i] = col_start[sd.orb_off + i];
  if (t < NC) {
    int rv = 0, kv = 0;
#pragma unroll
    for (int g = 0; g < NC; ++g)
      if (g == t) {
        rv = fft.rmap[g];
        kv = fft.kmap[g];
      }
    rm[t] = rv;
    km[t] = kv;
  }
  if (t == 0)
    *next = 0;
  {
    const double2* g0s = G0 + static_cast<long>(sd.spin) * nw_ext * NC;  // G0_s(k, w) at k + NC w (one band)
    for (int i = t; i < kCols * NC; i += kThreads) {
      const int k = i % NC, w2 = w2_0 + i / NC;
      double2 g0 = w2 < nw_ext ? g0s[k + NC * w2] : make_double2(0., 0.);
      Ds[i] = make_float2(static_cast<float>(dims.beta * g0.x), static_cast<float>(dims.beta * g0.y));
      const double2 f = Fb[k * NC + fft.r0];  // the band phase e^{-i k a}: conj Fb(r0, k) (x_r0 = 0)
      g0 = make_double2(g0.x * f.x + g0.y * f.y, g0.y * f.x - g0.x * f.y);
      Cs[i] = make_float2(static_cast<float>(-g0.x / NC), static_cast<float>(-g0.y / NC));
    }
  }
  __syncthreads();

  // Stage A.
  const int rg = lane / 4, wg = lane % 4;  // lane tile: rows rg + 8 a, frequencies wg + 4 b
  float2* Xw = Sw + warp * kStageW;        // [kRows][kBP]
  float2* Tw = Xw + kRows * kBP;           // [kCols][kBP]
  const int rho_l = rho_0 + lane;          // the row this lane stages
  const bool row_in = rho_l < D;           // rows past D (last tile) stay zero
  const __half* xrow = xp + static_cast<long>(row_in ? rho_l : 0) * 2 * Kr;
  const float* srow = xs_scale + (row_in ? rho_l / 128 : 0) * kxc;
  for (;;) {
    int r = 0;
    if (lane == 0)
      r = atomicAdd(next, 1);
    r = __shfl_sync(0xffffffffu, r, 0);
    if (r >= NC)
      break;
    const int lo = cs[r], hi = cs[r + 1];
    float2 acc[4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
        acc[a][b] = make_float2(0.f, 0.f);
    for (int b0 = lo; b0 < hi; b0 += kBlk) {
      const int cnt = min(kBlk, hi - b0);
      __syncwarp();  // the previous block's reads are done
      // X'(rho_l, j) for j in [b0, b0 + cnt): 8-vertex groups (16-byte vectors of each plane part).
      for (int g = b0 / 8; 8 * g < b0 + cnt; ++g) {
        uint4 hr = make_uint4(0, 0, 0, 0), hm = hr, lr = hr, lm = hr;
        float sc = 0.f;
        if (row_in) {
          const __half* p = xrow + 8 * g;
          hr = *reinterpret_cast<const uint4*>(p);
          hm = *reinterpret_cast<const uint4*>(p + Kr);
          lr = *reinterpret_cast<const uint4*>(p + plane);
          lm = *reinterpret_cast<const uint4*>(p + plane + Kr);
          sc = srow[g / 4];  // the 32-vertex chunk of this group
        }
        const __half* a = reinterpret_cast<const __half*>(&hr);
        const __half* b = reinterpret_cast<const __half*>(&hm);
        const __half* c = reinterpret_cast<const __half*>(&lr);
        const __half* d = reinterpret_cast<const __half*>(&lm);
#pragma unroll
        for (int x = 0; x < 8; ++x) {
          const int v = 8 * g + x - b0;
          if (v >= 0 && v < cnt)
            Xw[lane * kBP + v] = make_float2((__half2float(a[x]) + __half2float(c[x])) * sc,
                                             (__half2float(b[x]) + __half2float(d[x])) * sc);
        }
      }
#pragma unroll
      for (int u = 0; u < kCols; ++u) {
        const int w2 = w2_0 + u;
        const double2 tv =
            (lane < cnt && w2 < nw_ext) ? Tsec[static_cast<long>(w2) * n + b0 + lane] : make_double2(0., 0.);
        Tw[u * kBP + lane] = make_float2(static_cast<float>(tv.x), -static_cast<float>(tv.y));  // conj T
      }
      __syncwarp();
#pragma unroll 2
      for (int v = 0; v < cnt; ++v) {
        float2 x[4], y[2];
#pragma unroll
        for (int a = 0; a < 4; ++a)
          x[a] = Xw[(rg + 8 * a) * kBP + v];
#pragma unroll
        for (int b = 0; b < 2; ++b)
          y[b] = Tw[(wg + 4 * b) * kBP + v];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 2; ++b)
            cfma(acc[a][b], x[a], y[b]);
      }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
        Zs[r * kZS + (wg + 4 * b) * kZP + rg + 8 * a] = acc[a][b];
  }
  __syncthreads();  // Z of every site is in place

  // Stage B: the pair (row, wl) -> G(rho; k2, w2) for all k2.
  const int row = t % kRows, wl = t / kRows;
  const int rho = rho_0 + row, w2 = w2_0 + wl;
  float gabs = 0.f;
  {
    float2* zp = Zs + wl * kZP + row;  // slot of site r: zp[r * kZS]
    float2 z[NC];
#pragma unroll
    for (int g = 0; g < NC; ++g)
      z[g] = zp[rm[g] * kZS];
#pragma unroll
    for (int b = 0; b < L; ++b)  // along the first grid axis
      dft6(z[L * b], z[L * b + 1], z[L * b + 2], z[L * b + 3], z[L * b + 4], z[L * b + 5]);
#pragma unroll
    for (int m = 0; m < L; ++m)  // along the second
      dft6(z[m], z[m + L], z[m + 2 * L], z[m + 3 * L], z[m + 4 * L], z[m + 5 * L]);
    const int k1 = rho % R, w1 = rho / R;
    const bool diag = w2 == w1;  // the delta term sits at k2 = k1 of the diagonal block
    const bool in = rho < D && w2 < nw_ext;
    const float2* cw = Cs + wl * NC;
    const float2* dw = Ds + wl * NC;
#pragma unroll
    for (int g = 0; g < NC; ++g) {
      const int k2 = km[g];
      float2 x = cmul(cw[k2], z[g]);
      if (diag && k2 == k1)
        x = cadd(x, dw[k2]);
      if (in)
        gabs = fmaxf(gabs, fmaxf(fabsf(x.x), fabsf(x.y)));
      zp[k2 * kZS] = x;
    }
  }
  __syncthreads();
  // Out: segment s = row + kRows wl is G's row (k1, w1; w2) of NC entries k2, contiguous in G;
  // consecutive segments are consecutive rows k1 of one (w1, w2) block.
  float2* gsec = G + g_sector_stride * (2 * sd.slot + sd.spin);
  for (int idx = t; idx < kRows * kCols * NC; idx += kThreads) {
    const int s = idx / NC, k2 = idx % NC;
    const int rs = s % kRows, ws = s / kRows;
    const int rho_s = rho_0 + rs, w2_s = w2_0 + ws;
    if (rho_s < D && w2_s < nw_ext) {
      const int k1 = rho_s % R, w1 = rho_s / R;
      gsec[((static_cast<long>(w1) * nw_ext + w2_s) * R + k1) * R + k2] = Zs[k2 * kZS + ws * kZP + rs];
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

}  // namespace wide

}  // namespace

bool colFactorApplies(const TpDims& d) {
  return d.nb == 1 && d.nc == 16 && d.nw_ext % tcf::kCols == 0;
}

bool colFactorWideApplies(const TpDims& d) {
  return d.nb == 1 && d.nc == 36;
}

size_t colTwiddlePlaneBytes(const TpDims& d, int n_sectors, int Kr) {
  return sizeof(__half) * 4 * size_t(n_sectors) * d.nw_ext * Kr;
}

int launchColFactor(const FrontendArgs& a, const FrontTcWorkspace& w, float2* G, long g_sector_stride, int* gmax,
                    cudaStream_t stream) {
  const TpDims& d = a.dims;
  const FrontTcShape& s = w.shape;
  if (gmax)
    DCAACC_CUDA_CHECK(cudaMemsetAsync(gmax, 0, sizeof(int) * size_t(a.n_sectors), stream));
  const int row0 = d.half_g ? s.D / 2 : 0;  // half G: the rows of the upper frequency half
  if (colFactorWideApplies(d)) {  // 6 x 6 cluster, the 6 x 6 FFT (the caller checked fft)
    constexpr size_t smem = wide::smemBytes<36>();
    auto k = wide::colFactorWideKernel<36, 6>;
    DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const dim3 grid((s.D - row0 + wide::kRows - 1) / wide::kRows, (d.nw_ext + wide::kCols - 1) / wide::kCols,
                    a.n_sectors);
    k<<<grid, wide::kThreads, smem, stream>>>(d, a.sectors, a.col_start, a.Tc, static_cast<const __half*>(w.ac),
                                              w.xInv, s.Dp, s.Kr, a.Fb, a.G0, G, g_sector_stride, gmax, row0, w.fft);
    DCAACC_LAUNCH_CHECK();
    return 1;
  }
  if (w.fft.on && w.tp) {
    auto* tp = static_cast<__half*>(w.tp);
    const long per = long(d.nw_ext) * s.Kr;
    const dim3 pgrid(unsigned((per + 255) / 256), a.n_sectors);
    tcf::colTwiddlePlanesKernel<<<pgrid, 256, 0, stream>>>(d, a.sectors, a.Tc, tp, s.Kr);
    DCAACC_LAUNCH_CHECK();
    DCAACC_CUDA_CHECK(
        cudaFuncSetAttribute(tcf::colFactorMmaKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tcf::kSmem));
    const dim3 grid((s.D - row0) / tcf::kRows, d.nw_ext / tcf::kCols, a.n_sectors);
    tcf::colFactorMmaKernel<<<grid, tcf::kThreads, tcf::kSmem, stream>>>(
        d, a.sectors, a.col_start, tp, static_cast<const __half*>(w.ac), w.xInv, s.Dp, s.Kr, a.Fb, a.G0, G,
        g_sector_stride, gmax, row0, w.fft);
    DCAACC_LAUNCH_CHECK();
    return 2;
  }
  constexpr size_t smem = colFactorSmem<16>();
  auto k = w.fft.on ? colFactorKernel<16, true> : colFactorKernel<16, false>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const dim3 grid((s.D - row0 + kRT - 1) / kRT, d.nw_ext / kWT, a.n_sectors);
  k<<<grid, kThreads, smem, stream>>>(d, a.sectors, a.col_start, a.Tc, static_cast<const __half*>(w.ac), w.xInv,
                                      s.Dp, s.Kr, a.Fb, a.G0, G, g_sector_stride, gmax, row0, w.fft);
  DCAACC_LAUNCH_CHECK();
  return 1;
}

}  // namespace dcaacc
