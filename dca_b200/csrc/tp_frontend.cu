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

// Row transform.  grid (ceil(n_max / JC), ceil(NwExt / WC), n_sectors), WC * JC threads.
// Thread (w, jc) walks the row-sorted vertices once; the vertices of one orbital are contiguous,
// so its running sum is flushed to shared memory at each orbital boundary (the same boundaries
// for every thread, so no divergence).  M columns and twiddles are staged through shared memory
// in chunks of IB vertices.
template <typename Real, int JC, int WC, int IB>
__global__ void __launch_bounds__(JC * WC)
rowTransformKernel(const TpDims dims, const SectorDesc* __restrict__ sectors,
                   const int* __restrict__ perm_r, const int* __restrict__ perm_c,
                   const int* __restrict__ row_start, const double2* __restrict__ Tr,
                   const double2* __restrict__ Fb,  // (r, k, b): e^{i k (r + a_b)}
                   cplx_t<Real>* __restrict__ Xp) {
  using C = cplx_t<Real>;
  const SectorDesc sd = sectors[blockIdx.z];
  const int n = sd.n;
  const int jj0 = blockIdx.x * JC;
  const int w0 = blockIdx.y * WC;
  if (jj0 >= n)
    return;
  const int nw_ext = dims.nw_ext, n_orb = dims.n_orb, R = dims.R, nb = dims.nb, nc = dims.nc;
  const int t = threadIdx.x;
  const int w = t % WC, jc = t / WC;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int MS = IB + 1;               // padded row of Ms (no bank conflicts across jc)
  C* Xs = reinterpret_cast<C*>(smem_raw);   // [n_orb][JC][WC]
  C* Fs = Xs + JC * WC * n_orb;             // [nb][r][k]: lanes that differ in k read distinct banks
  C* Ts = Fs + nb * nc * nc;                // [IB][WC]
  Real* Ms = reinterpret_cast<Real*>(Ts + IB * WC);  // [JC][MS]
  int* rs = reinterpret_cast<int*>(Ms + JC * MS);    // [n_orb + 1]

  const int* pr = perm_r + sd.vtx_off;
  const int* pc = perm_c + sd.vtx_off;
  for (int idx = t; idx < nb * nc * nc; idx += blockDim.x) {  // Fb is (b, k, r); Fs is (b, r, k)
    const int b = idx / (nc * nc), k = (idx / nc) % nc, r = idx % nc;
    Fs[(b * nc + r) * nc + k] = loadC<Real>(Fb + idx);
  }
  for (int idx = t; idx <= n_orb; idx += blockDim.x)
    rs[idx] = row_start[sd.orb_off + idx];
  const int jc_count = min(JC, n - jj0);

  // Row NDFT per orbital: X(o1, w; jc) = sum_{ii in seg(o1)} T(w, ii) M(ii, jc).
  C acc = mk(Real(0), Real(0));
  int o1 = 0;
  __syncthreads();
  int seg_end = rs[1];
  while (o1 < n_orb && seg_end == 0) {  // leading empty orbitals
    Xs[o1 * JC * WC + t] = acc;
    ++o1;
    seg_end = o1 < n_orb ? rs[o1 + 1] : n;
  }
  for (int i0 = 0; i0 < n; i0 += IB) {
    const int ib_count = min(IB, n - i0);
    for (int idx = t; idx < ib_count * WC; idx += blockDim.x) {
      const int ib = idx / WC, ww = idx % WC;
      Ts[ib * WC + ww] = (w0 + ww < nw_ext) ? loadC<Real>(Tr + static_cast<long>(sd.vtx_off + i0 + ib) * nw_ext + w0 + ww)
                                           : mk(Real(0), Real(0));
    }
    for (int idx = t; idx < JC * ib_count; idx += blockDim.x) {
      const int c = idx / ib_count, ib = idx % ib_count;
      Ms[c * MS + ib] = c < jc_count
                            ? static_cast<Real>(loadM(sd, static_cast<long>(sd.ldm) * pc[jj0 + c] + pr[i0 + ib]))
                            : Real(0);
    }
    __syncthreads();
    for (int ib = 0; ib < ib_count; ++ib) {
      const int ii = i0 + ib;
      while (ii >= seg_end) {  // orbital boundary: uniform across the CTA
        Xs[o1 * JC * WC + t] = acc;
        acc = mk(Real(0), Real(0));
        ++o1;
        seg_end = o1 < n_orb ? rs[o1 + 1] : n;
      }
      const C tv = Ts[ib * WC + w];
      const Real m = Ms[jc * MS + ib];
      acc.x = fma(tv.x, m, acc.x);
      acc.y = fma(tv.y, m, acc.y);
    }
    __syncthreads();
  }
  for (; o1 < n_orb; ++o1) {
    Xs[o1 * JC * WC + t] = acc;
    acc = mk(Real(0), Real(0));
  }
  __syncthreads();

  // Row cluster transform with band phases: X'(b1 + nb k1) = sum_r1 Fb(b1, k1, r1) X(b1 + nb r1).
  for (int q = t; q < jc_count * WC * R; q += blockDim.x) {
    const int row = q % R, ww = (q / R) % WC, c = q / (R * WC), we = w0 + ww;
    if (we >= nw_ext)
      continue;
    const int b1 = row % nb, k1 = row / nb;
    const C* x = Xs + b1 * JC * WC + c * WC + ww;
    const C* f = Fs + b1 * nc * nc + k1;
    C a = mk(Real(0), Real(0));
    for (int r1 = 0; r1 < nc; ++r1)
      cfma(a, f[r1 * nc], x[nb * r1 * JC * WC]);
    Xp[sd.x_off + (static_cast<long>(we) * n + jj0 + c) * R + row] = a;
  }
}

// Column transform + G epilogue.  grid (NwExt, ceil(NwExt / WC2), n_sectors), R * WC2 threads.
// X' rows of frequency w1 and the twiddles of the CTA's w2 chunk are staged through shared
// memory in chunks of JB vertices; thread (row, w2) walks the column-sorted vertices once and
// flushes its running sum at each column-orbital boundary.
template <typename Real, int JB>
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
  const int t = threadIdx.x;
  const int row = t % R, w2l = t / R;
  const int w2c0 = blockIdx.y * WC2;
  const int w2 = w2c0 + w2l;
  const bool active = w2 < nw_ext;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Zs = reinterpret_cast<C*>(smem_raw);  // [n_orb][WC2][R]; reused as the output tile
  C* Gs = Zs + WC2 * R * (R + 1);          // [R cols][WC2][R rows]; Zs space holds the padded tile
  C* Fs = Gs + R * WC2 * R;                // [nb][nc][nc]
  C* Xst = Fs + nb * nc * nc;              // [JB][R]
  C* Tst = Xst + JB * R;                   // [JB][WC2]
  int* cs = reinterpret_cast<int*>(Tst + JB * WC2);  // [n_orb + 1]
  for (int idx = t; idx < nb * nc * nc; idx += blockDim.x)
    Fs[idx] = loadC<Real>(Fb + idx);
  for (int idx = t; idx <= n_orb; idx += blockDim.x)
    cs[idx] = col_start[sd.orb_off + idx];
  __syncthreads();

  // Column NDFT per orbital: Z(o2) = sum_{jj in seg(o2)} X'(row, w1; jj) conj(T(w2, jj)).
  const int zs = WC2 * R;  // stride between orbitals of one thread's Z
  C* z = Zs + t;
  C acc = mk(Real(0), Real(0));
  int o2 = 0;
  int seg_end = cs[1];
  while (o2 < n_orb && seg_end == 0) {
    z[o2 * zs] = acc;
    ++o2;
    seg_end = o2 < n_orb ? cs[o2 + 1] : n;
  }
  const C* xrow = Xp + sd.x_off + static_cast<long>(w1) * n * R;
  for (int j0 = 0; j0 < n; j0 += JB) {
    const int jb_count = min(JB, n - j0);
    for (int idx = t; idx < jb_count * R; idx += blockDim.x)
      Xst[idx] = xrow[static_cast<long>(j0) * R + idx];
    for (int idx = t; idx < jb_count * WC2; idx += blockDim.x) {
      const int jb = idx / WC2, ww = idx % WC2;
      Tst[idx] = (w2c0 + ww < nw_ext)
                     ? loadC<Real>(Tc + static_cast<long>(sd.vtx_off + j0 + jb) * nw_ext + w2c0 + ww)
                     : mk(Real(0), Real(0));
    }
    __syncthreads();
    for (int jb = 0; jb < jb_count; ++jb) {
      const int jj = j0 + jb;
      while (jj >= seg_end) {
        z[o2 * zs] = acc;
        acc = mk(Real(0), Real(0));
        ++o2;
        seg_end = o2 < n_orb ? cs[o2 + 1] : n;
      }
      cfmac(acc, Xst[jb * R + row], Tst[jb * WC2 + w2l]);
    }
    __syncthreads();
  }
  for (; o2 < n_orb; ++o2) {
    z[o2 * zs] = acc;
    acc = mk(Real(0), Real(0));
  }
  __syncthreads();
  C* g = Gs + t;  // column col of this thread's row at g[col * zs]
  if (active) {
    // Column cluster transform with band phases and the 1/Nc normalisation
    // (space_transform_2D.hpp:79-89).
    const Real norm = Real(1) / Real(nc);
    for (int col = 0; col < R; ++col) {
      const int b2 = col % nb, k2 = col / nb;
      const C* f = Fs + (b2 * nc + k2) * nc;
      C a = mk(Real(0), Real(0));
      for (int r2 = 0; r2 < nc; ++r2)
        cfmac(a, z[(b2 + nb * r2) * zs], f[r2]);
      g[col * zs] = cscale(a, norm);
    }
  }
  __syncthreads();
  // Epilogue: G = -G0(k1, w1) G~ G0(k2, w2) + beta G0(k1, w1) delta (tp_accumulator_cpu.hpp:309-375),
  // staged as row-major blocks (row stride R + 1 against bank conflicts) in the Zs space.
  C* Os = Zs;  // [WC2][R][R + 1]
  if (active) {
    const int s = sd.spin;
    const int b1 = row % nb, k1 = row / nb;
    const double2* g0s = G0 + static_cast<long>(s) * nw_ext * nc * nb * nb;
    auto g0 = [&](int ba, int bb, int k, int w) {
      return loadC<Real>(g0s + ba + nb * (bb + nb * (k + nc * w)));
    };
    const Real beta = static_cast<Real>(dims.beta);
    C* o = Os + (w2l * R + row) * (R + 1);
    for (int col = 0; col < R; ++col) {
      const int b2 = col % nb, k2 = col / nb;
      C v;
      if (nb == 1) {
        v = cmul(cmul(g0(0, 0, k1, w1), g[col * zs]), g0(0, 0, k2, w2));
        v = mk(-v.x, -v.y);
      }
      else {
        v = mk(Real(0), Real(0));
        for (int c2 = 0; c2 < nb; ++c2) {
          C tt = mk(Real(0), Real(0));  // (G0_w1 G~)(b1, c2) at (k1, k2)
          for (int c1 = 0; c1 < nb; ++c1)
            cfma(tt, g0(b1, c1, k1, w1), Gs[((c2 + nb * k2) * WC2 + w2l) * R + c1 + nb * k1]);
          cfma(v, tt, g0(c2, b2, k2, w2));
        }
        v = mk(-v.x, -v.y);
      }
      if (k1 == k2 && w1 == w2) {
        const C d = g0(b1, b2, k1, w1);
        v.x += d.x * beta;
        v.y += d.y * beta;
      }
      o[col] = v;
    }
  }
  __syncthreads();
  // Coalesced store of the CTA's blocks (w1, w2c0 .. w2c0 + WC2 - 1), each R x R contiguous.
  const int n_w2 = min(WC2, nw_ext - w2c0);
  C* out = G + g_sector_stride * (2 * sd.slot + sd.spin) +
           (static_cast<long>(w1) * nw_ext + w2c0) * R * R;
  for (int idx = t; idx < n_w2 * R * R; idx += blockDim.x) {
    const int wl = idx / (R * R), rem = idx % (R * R);
    out[idx] = Os[(wl * R + rem / R) * (R + 1) + rem % R];
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

constexpr int kRowJC = 32, kRowWC = 8, kRowIB = 64, kColJB = 64;

template <typename Real, int JC = kRowJC, int WC = kRowWC, int IB = kRowIB>
static size_t rowSmem(const TpDims& d) {
  return sizeof(cplx_t<Real>) * (JC * WC * d.n_orb + d.nb * d.nc * d.nc + IB * WC) +
         sizeof(Real) * JC * (IB + 1) + sizeof(int) * (d.n_orb + 1);
}

template <typename Real>
static int pickWC2(const TpDims& d) {
  // Largest power of two <= 16 with R * WC2 <= 1024 threads and Zs + Gs <= 96 KB.
  int wc2 = 16;
  while (wc2 > 1 && (d.R * wc2 > 1024 || sizeof(cplx_t<Real>) * (d.R * d.R * wc2 + d.R * (d.R + 1) * wc2) > 96 * 1024))
    wc2 /= 2;
  return wc2;
}

template <typename Real>
static size_t colSmem(const TpDims& d, int wc2) {
  // Zs (also the padded output tile) + Gs + Fs + staging + column starts.
  const size_t zs = std::max(size_t(d.R) * wc2 * d.n_orb, size_t(wc2) * d.R * (d.R + 1));
  return sizeof(cplx_t<Real>) * (zs + size_t(d.R) * wc2 * d.R + d.nb * d.nc * d.nc + kColJB * (d.R + wc2)) +
         sizeof(int) * (d.n_orb + 1);
}

template <typename Real, int JC, int WC>
static void launchRowTile(const FrontendArgs& a, cplx_t<Real>* Xp, cudaStream_t stream) {
  const TpDims& d = a.dims;
  const size_t smem = rowSmem<Real, JC, WC>(d);
  auto k = rowTransformKernel<Real, JC, WC, kRowIB>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const dim3 grid(ceil_div(a.n_max, JC), ceil_div(d.nw_ext, WC), a.n_sectors);
  k<<<grid, JC * WC, smem, stream>>>(d, a.sectors, a.perm_r, a.perm_c, a.row_start, a.Tr, a.Fb, Xp);
  DCAACC_LAUNCH_CHECK();
}

// Tile shapes (vertices JC x frequencies WC per CTA, 256 threads) the tuner chooses among: each
// X' element is the same sum in the same order whatever the tile.
template <typename Real>
void launchRowTransform(const FrontendArgs& a, cplx_t<Real>* Xp, cudaStream_t stream) {
  const TpDims& d = a.dims;
  if (a.n_max == 0)
    return;
  const size_t lim = 227 * 1024;
  const bool fit16 = rowSmem<Real, 16, 16>(d) <= lim, fit64 = rowSmem<Real, 64, 4>(d) <= lim;
  const int n_cand = fit16 ? (fit64 ? 3 : 2) : 1;
  const auto pk = tunePick(a.tuner, tuneKey("row", d.nb, d.nc, d.nw_ext, a.n_max, a.n_sectors, sizeof(Real)),
                           n_cand, stream);
  if (pk.choice == 1)
    launchRowTile<Real, 16, 16>(a, Xp, stream);
  else if (pk.choice == 2)
    launchRowTile<Real, 64, 4>(a, Xp, stream);
  else
    launchRowTile<Real, kRowJC, kRowWC>(a, Xp, stream);
  tuneEnd(a.tuner, pk, stream);
}

template <typename Real>
void launchColTransform(const FrontendArgs& a, const cplx_t<Real>* Xp, cplx_t<Real>* G,
                        long g_sector_stride, cudaStream_t stream) {
  const TpDims& d = a.dims;
  // Candidates: the heuristic's column-frequency width and the next two halvings (each G element
  // is the same sum in the same order whatever the width).
  const int wc2_max = pickWC2<Real>(d);
  const int n_cand = wc2_max >= 4 ? 3 : wc2_max == 2 ? 2 : 1;
  const auto pk = tunePick(a.tuner, tuneKey("col", d.nb, d.nc, d.nw_ext, a.n_max, a.n_sectors, sizeof(Real)),
                           n_cand, stream);
  const int wc2 = wc2_max >> pk.choice;
  const size_t smem = colSmem<Real>(d, wc2);
  auto k = colTransformKernel<Real, kColJB>;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const dim3 grid(d.nw_ext, ceil_div(d.nw_ext, wc2), a.n_sectors);
  k<<<grid, d.R * wc2, smem, stream>>>(d, a.sectors, a.col_start, a.Tc, a.Fb, a.G0, Xp, G,
                                       g_sector_stride, wc2);
  DCAACC_LAUNCH_CHECK();
  tuneEnd(a.tuner, pk, stream);
}

size_t frontendSmemRequirement(const TpDims& d, int /*n_max*/, bool fp64) {
  if (fp64)
    return std::max(rowSmem<double>(d), colSmem<double>(d, pickWC2<double>(d)));
  return std::max(rowSmem<float>(d), colSmem<float>(d, pickWC2<float>(d)));
}

template void launchRowTransform<double>(const FrontendArgs&, double2*, cudaStream_t);
template void launchRowTransform<float>(const FrontendArgs&, float2*, cudaStream_t);
template void launchColTransform<double>(const FrontendArgs&, const double2*, double2*, long, cudaStream_t);
template void launchColTransform<float>(const FrontendArgs&, const float2*, float2*, long, cudaStream_t);

}  // namespace dcaacc
