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
// benchmark cluster).  Both stages run in FP32 on the CUDA cores of one CTA per (sector, 32 rows
// rho1, 16 frequencies w2):
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

}  // namespace

bool colFactorApplies(const TpDims& d) {
  return d.nb == 1 && d.nc == 16 && d.nw_ext % kWT == 0;
}

void launchColFactor(const FrontendArgs& a, const FrontTcWorkspace& w, float2* G, long g_sector_stride, int* gmax,
                     cudaStream_t stream) {
  const TpDims& d = a.dims;
  const FrontTcShape& s = w.shape;
  if (gmax)
    DCAACC_CUDA_CHECK(cudaMemsetAsync(gmax, 0, sizeof(int) * size_t(a.n_sectors), stream));
  const int row0 = d.half_g ? s.D / 2 : 0;  // half G: the rows of the upper frequency half
  constexpr size_t smem = colFactorSmem<16>();
  auto k = w.fft.on ? colFactorKernel<16, true> : colFactorKernel<16, false>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const dim3 grid((s.D - row0 + kRT - 1) / kRT, d.nw_ext / kWT, a.n_sectors);
  k<<<grid, kThreads, smem, stream>>>(d, a.sectors, a.col_start, a.Tc, static_cast<const __half*>(w.ac), w.xInv,
                                      s.Dp, s.Kr, a.Fb, a.G0, G, g_sector_stride, gmax, row0, w.fft);
  DCAACC_LAUNCH_CHECK();
}

}  // namespace dcaacc
