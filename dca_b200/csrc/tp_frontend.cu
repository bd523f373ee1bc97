// Two-particle front-end: M(tau, tau') -> G(k1, w1; k2, w2) for every sector of a batch.
//
// Replaces the reference's CachedNdft<GPU>::execute (cached_ndft_gpu.hpp:131-252: sortM,
// computeT, two MAGMA vbatched GEMMs, rearrange), SpaceTransform2DGpu::execute
// (space_transform_2D_gpu.hpp:116-171: two MAGMA batched GEMMs + phaseFactorsAndRearrange) and
// computeGSingleband / computeGMultiband (tp_accumulator_kernels.cu:73-217) with three kernels:
//
//   twiddle_kernel      T(w, v) = exp(i w tau_v) over the extended frequency mesh, in both the
//                       row-sorted and column-sorted vertex orders.
//   row_transform       X'(b1 k1 w1, j) = sum_{r1} e^{i k1 (r1 + a_b1)} sum_{i in orbital (b1,r1)}
//                       T(w1, i) M(i, j)      (row NDFT fused with the row cluster transform)
//   col_transform       G~(r, w1; b2 k2 w2) = 1/Nc sum_{r2} e^{-i k2 (r2 + a_b2)}
//                       sum_{j in orbital (b2,r2)} X'(r w1, j) conj(T(w2, j)), then the epilogue
//                       G = -G0(k1,w1) G~ G0(k2,w2) + beta G0(k1,w1) delta_{k1k2} delta_{w1w2}
//                       (band-matrix products when nb > 1), written in frequency-block layout.
//
// Both transforms exploit the orbital structure (each vertex belongs to one orbital, so the
// inner sums run over that orbital's vertices only, as the reference's per-orbital-pair
// products do) and keep the cluster transform (K = Nc) in shared memory, so M, X' and G each
// cross global memory once.  Templated on the working precision: double for the FP64 path,
// float for the FP32 SIMT variant of the mixed path.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "tp_frontend.hpp"

namespace dcaacc {

namespace {

// Matsubara frequency of extended index w: +-pi (2l+1) / beta, ordered as the reference's
// vertex_frequency_domain<EXTENDED> (vertex_frequency_domain.hpp EXTENDED initialize).
__device__ inline double extFrequency(int w, int nw_ext, double beta) {
  const int half = nw_ext / 2;
  if (w >= half)
    return M_PI / beta * (1 + 2 * (w - half));
  return -M_PI / beta * (1 + 2 * (half - 1 - w));
}

__global__ void twiddleKernel(const SectorDesc* __restrict__ sectors,
                              const double* __restrict__ tau,     // packed, original vertex order
                              const int* __restrict__ perm,       // packed, sorted -> original
                              double2* __restrict__ T,            // packed sorted x NwExt
                              int nw_ext, double beta) {
  const SectorDesc sd = sectors[blockIdx.y];
  const int ii = blockIdx.x;
  if (ii >= sd.n)
    return;
  const int v = perm[sd.vtx_off + ii];
  const double t = tau[sd.vtx_off + v];
  for (int w = threadIdx.x; w < nw_ext; w += blockDim.x) {
    // x = tau * w as in CachedNdft<CPU>::computeT (cached_ndft_cpu.hpp:151-156).
    const double x = t * extFrequency(w, nw_ext, beta);
    double s, c;
    sincos(x, &s, &c);
    T[static_cast<long>(sd.vtx_off + ii) * nw_ext + w] = make_double2(c, s);
  }
}

template <typename Real>
__device__ inline cplx_t<Real> loadC(const double2* p) {
  const double2 v = *p;
  return mk(static_cast<Real>(v.x), static_cast<Real>(v.y));
}

// Row transform.  grid (ceil(n_max / JC), ceil(NwExt / WC), n_sectors), 256 threads.
template <typename Real, int JC, int WC>
__global__ void __launch_bounds__(256)
rowTransformKernel(const TpDims dims, const SectorDesc* __restrict__ sectors,
                   const int* __restrict__ perm_r, const int* __restrict__ perm_c,
                   const int* __restrict__ row_start, const double2* __restrict__ Tr,
                   const double2* __restrict__ Fb,  // (r, k, b): e^{i k (r + a_b)}
                   cplx_t<Real>* __restrict__ Xp, int n_max) {
  using C = cplx_t<Real>;
  const SectorDesc sd = sectors[blockIdx.z];
  const int n = sd.n;
  const int jj0 = blockIdx.x * JC;
  const int w0 = blockIdx.y * WC;
  if (jj0 >= n)
    return;
  const int nw_ext = dims.nw_ext, n_orb = dims.n_orb, R = dims.R, nb = dims.nb, nc = dims.nc;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Xs = reinterpret_cast<C*>(smem_raw);                      // [JC][WC][n_orb]
  C* Fs = Xs + JC * WC * n_orb;                                // [nb][nc][nc]
  Real* Ms = reinterpret_cast<Real*>(Fs + nb * nc * nc);       // [JC][n]

  const int* pr = perm_r + sd.vtx_off;
  const int* pc = perm_c + sd.vtx_off;
  const int* rs = row_start + sd.orb_off;

  for (int idx = threadIdx.x; idx < nb * nc * nc; idx += blockDim.x)
    Fs[idx] = loadC<Real>(Fb + idx);
  const int jc_count = min(JC, n - jj0);
  for (int jc = 0; jc < jc_count; ++jc) {
    const double* col = sd.M + static_cast<long>(sd.ldm) * pc[jj0 + jc];
    for (int ii = threadIdx.x; ii < n; ii += blockDim.x)
      Ms[jc * n_max + ii] = static_cast<Real>(col[pr[ii]]);
  }
  __syncthreads();

  // Row NDFT per orbital: X(o1, w; jc) = sum_{ii in seg(o1)} T(w, ii) M(ii, jc).
  for (int p = threadIdx.x; p < WC * n_orb; p += blockDim.x) {
    const int w = p % WC, o1 = p / WC, we = w0 + w;
    C acc[JC];
#pragma unroll
    for (int jc = 0; jc < JC; ++jc)
      acc[jc] = mk(Real(0), Real(0));
    if (we < nw_ext) {
      for (int ii = rs[o1]; ii < rs[o1 + 1]; ++ii) {
        const C t = loadC<Real>(Tr + static_cast<long>(sd.vtx_off + ii) * nw_ext + we);
#pragma unroll
        for (int jc = 0; jc < JC; ++jc) {
          const Real m = Ms[jc * n_max + ii];
          acc[jc].x = fma(t.x, m, acc[jc].x);
          acc[jc].y = fma(t.y, m, acc[jc].y);
        }
      }
    }
#pragma unroll
    for (int jc = 0; jc < JC; ++jc)
      Xs[(jc * WC + w) * n_orb + o1] = acc[jc];
  }
  __syncthreads();

  // Row cluster transform with band phases: X'(b1 + nb k1) = sum_r1 Fb(b1, k1, r1) X(b1 + nb r1).
  for (int q = threadIdx.x; q < jc_count * WC * R; q += blockDim.x) {
    const int row = q % R, w = (q / R) % WC, jc = q / (R * WC), we = w0 + w;
    if (we >= nw_ext)
      continue;
    const int b1 = row % nb, k1 = row / nb;
    const C* x = Xs + (jc * WC + w) * n_orb + b1;
    const C* f = Fs + (b1 * nc + k1) * nc;
    C acc = mk(Real(0), Real(0));
    for (int r1 = 0; r1 < nc; ++r1)
      cfma(acc, f[r1], x[nb * r1]);
    Xp[sd.x_off + (static_cast<long>(we) * n + jj0 + jc) * R + row] = acc;
  }
}

// Column transform + G epilogue.  grid (NwExt, ceil(NwExt / WC2), n_sectors), R * WC2 threads.
template <typename Real>
__global__ void colTransformKernel(const TpDims dims, const SectorDesc* __restrict__ sectors,
                                   const int* __restrict__ col_start,
                                   const double2* __restrict__ Tc, const double2* __restrict__ Fb,
                                   const double2* __restrict__ G0,  // (b1, b2, k, w, s)
                                   const cplx_t<Real>* __restrict__ Xp, cplx_t<Real>* __restrict__ G,
                                   long g_sector_stride, int WC2) {
  using C = cplx_t<Real>;
  const SectorDesc sd = sectors[blockIdx.z];
  const int n = sd.n;
  const int w1 = blockIdx.x;
  const int nw_ext = dims.nw_ext, n_orb = dims.n_orb, R = dims.R, nb = dims.nb, nc = dims.nc;
  const int row = threadIdx.x % R, w2l = threadIdx.x / R;
  const int w2 = blockIdx.y * WC2 + w2l;
  const bool active = w2 < nw_ext;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Zs = reinterpret_cast<C*>(smem_raw);  // [R][WC2][n_orb]
  C* Gs = Zs + R * WC2 * n_orb;            // [R][WC2][R]
  C* Fs = Gs + R * WC2 * R;                // [nb][nc][nc]
  for (int idx = threadIdx.x; idx < nb * nc * nc; idx += blockDim.x)
    Fs[idx] = loadC<Real>(Fb + idx);

  const int* cs = col_start + sd.orb_off;
  C* z = Zs + (row * WC2 + w2l) * n_orb;
  if (active) {
    // Column NDFT per orbital: Z(o2) = sum_{jj in seg(o2)} X'(row, w1; jj) conj(T(w2, jj)).
    const C* xrow = Xp + sd.x_off + static_cast<long>(w1) * n * R + row;
    const double2* tcol = Tc + static_cast<long>(sd.vtx_off) * nw_ext + w2;
    for (int o2 = 0; o2 < n_orb; ++o2) {
      C acc = mk(Real(0), Real(0));
      for (int jj = cs[o2]; jj < cs[o2 + 1]; ++jj)
        cfmac(acc, xrow[static_cast<long>(jj) * R], loadC<Real>(tcol + static_cast<long>(jj) * nw_ext));
      z[o2] = acc;
    }
  }
  __syncthreads();
  C* g = Gs + (row * WC2 + w2l) * R;
  if (active) {
    // Column cluster transform with band phases and the 1/Nc normalisation
    // (space_transform_2D.hpp:79-89).
    const Real norm = Real(1) / Real(nc);
    for (int col = 0; col < R; ++col) {
      const int b2 = col % nb, k2 = col / nb;
      const C* f = Fs + (b2 * nc + k2) * nc;
      C acc = mk(Real(0), Real(0));
      for (int r2 = 0; r2 < nc; ++r2)
        cfmac(acc, z[b2 + nb * r2], f[r2]);
      g[col] = cscale(acc, norm);
    }
  }
  __syncthreads();
  if (!active)
    return;

  // Epilogue: G = -G0(k1, w1) G~ G0(k2, w2) + beta G0(k1, w1) delta (tp_accumulator_cpu.hpp:309-375).
  const int s = sd.spin;
  const int b1 = row % nb, k1 = row / nb;
  const double2* g0s = G0 + static_cast<long>(s) * nw_ext * nc * nb * nb;
  auto g0 = [&](int ba, int bb, int k, int w) {
    return loadC<Real>(g0s + ba + nb * (bb + nb * (k + nc * w)));
  };
  C* out = G + g_sector_stride * (2 * sd.slot + s) +
             (static_cast<long>(w1) * nw_ext + w2) * R * R + static_cast<long>(row) * R;
  const Real beta = static_cast<Real>(dims.beta);
  for (int col = 0; col < R; ++col) {
    const int b2 = col % nb, k2 = col / nb;
    C v;
    if (nb == 1) {
      v = cmul(cmul(g0(0, 0, k1, w1), g[col]), g0(0, 0, k2, w2));
      v = mk(-v.x, -v.y);
    }
    else {
      v = mk(Real(0), Real(0));
      const C* gs_k1 = Gs + (static_cast<long>(k1 * nb) * WC2 + w2l) * R;  // row (c1 = 0, k1)
      for (int c2 = 0; c2 < nb; ++c2) {
        C t = mk(Real(0), Real(0));  // (G0_w1 G~)(b1, c2) at (k1, k2)
        for (int c1 = 0; c1 < nb; ++c1)
          cfma(t, g0(b1, c1, k1, w1), gs_k1[c1 * WC2 * R + c2 + nb * k2]);
        cfma(v, t, g0(c2, b2, k2, w2));
      }
      v = mk(-v.x, -v.y);
    }
    if (k1 == k2 && w1 == w2) {
      const C d = g0(b1, b2, k1, w1);
      v.x += d.x * beta;
      v.y += d.y * beta;
    }
    out[col] = v;
  }
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// Host launchers
// ------------------------------------------------------------------------------------------------
void launchTwiddles(const FrontendArgs& a, cudaStream_t stream) {
  const dim3 grid(a.n_max, a.n_sectors);
  twiddleKernel<<<grid, 128, 0, stream>>>(a.sectors, a.tau, a.perm_r, a.Tr, a.dims.nw_ext, a.dims.beta);
  DCAACC_LAUNCH_CHECK();
  if (a.Tc != a.Tr) {
    twiddleKernel<<<grid, 128, 0, stream>>>(a.sectors, a.tau, a.perm_c, a.Tc, a.dims.nw_ext, a.dims.beta);
    DCAACC_LAUNCH_CHECK();
  }
}

template <typename Real>
static size_t rowSmem(const TpDims& d, int n_max, int JC, int WC) {
  return sizeof(cplx_t<Real>) * (JC * WC * d.n_orb + d.nb * d.nc * d.nc) + sizeof(Real) * JC * n_max;
}

template <typename Real>
static int pickWC2(const TpDims& d) {
  // Largest power of two <= 16 with R * WC2 <= 1024 threads and Zs + Gs <= 96 KB.
  int wc2 = 16;
  while (wc2 > 1 && (d.R * wc2 > 1024 || 2 * sizeof(cplx_t<Real>) * d.R * d.R * wc2 > 96 * 1024))
    wc2 /= 2;
  return wc2;
}

template <typename Real>
static size_t colSmem(const TpDims& d, int wc2) {
  return sizeof(cplx_t<Real>) * (2 * d.R * wc2 * d.R + d.nb * d.nc * d.nc);
}

template <typename Real>
void launchRowTransform(const FrontendArgs& a, cplx_t<Real>* Xp, cudaStream_t stream) {
  constexpr int JC = 8, WC = 8;
  const TpDims& d = a.dims;
  if (a.n_max == 0)
    return;
  const size_t smem = rowSmem<Real>(d, a.n_max, JC, WC);
  auto k = rowTransformKernel<Real, JC, WC>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const dim3 grid(ceil_div(a.n_max, JC), ceil_div(d.nw_ext, WC), a.n_sectors);
  k<<<grid, 256, smem, stream>>>(d, a.sectors, a.perm_r, a.perm_c, a.row_start, a.Tr, a.Fb, Xp,
                                 a.n_max);
  DCAACC_LAUNCH_CHECK();
}

template <typename Real>
void launchColTransform(const FrontendArgs& a, const cplx_t<Real>* Xp, cplx_t<Real>* G,
                        long g_sector_stride, cudaStream_t stream) {
  const TpDims& d = a.dims;
  const int wc2 = pickWC2<Real>(d);
  const size_t smem = colSmem<Real>(d, wc2);
  auto k = colTransformKernel<Real>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const dim3 grid(d.nw_ext, ceil_div(d.nw_ext, wc2), a.n_sectors);
  k<<<grid, d.R * wc2, smem, stream>>>(d, a.sectors, a.col_start, a.Tc, a.Fb, a.G0, Xp, G,
                                       g_sector_stride, wc2);
  DCAACC_LAUNCH_CHECK();
}

size_t frontendSmemRequirement(const TpDims& d, int n_max, bool fp64) {
  if (fp64)
    return std::max(rowSmem<double>(d, n_max, 8, 8), colSmem<double>(d, pickWC2<double>(d)));
  return std::max(rowSmem<float>(d, n_max, 8, 8), colSmem<float>(d, pickWC2<float>(d)));
}

template void launchRowTransform<double>(const FrontendArgs&, double2*, cudaStream_t);
template void launchRowTransform<float>(const FrontendArgs&, float2*, cudaStream_t);
template void launchColTransform<double>(const FrontendArgs&, const double2*, double2*, long, cudaStream_t);
template void launchColTransform<float>(const FrontendArgs&, const float2*, float2*, long, cudaStream_t);

}  // namespace dcaacc
