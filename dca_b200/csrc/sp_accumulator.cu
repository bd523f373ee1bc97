// Single-particle accumulator: the delayed NFFT of sign * M(tau_i - tau_j) onto a padded time
// grid per (b_i, b_j, r_i - r_j) label, and its transform to Matsubara frequencies.
//
// Replaces Dnfft1DGpu (dnfft_1d_gpu.hpp:38-276) whose accumulateOnDeviceKernel
// (dnfft_1d_kernels.cu:56-138) issues one FP64 global atomicAdd per (i, j, tap), and whose
// finalize copies f(tau) to the host for FFTW.  Here:
//   * vertices are sorted by orbital on the host (as for the two-particle NDFT), so one CTA owns
//     one output label and visits exactly the (i, j) pairs that land in it; the 16-tap cubic
//     convolution (dnfft_1d.hpp:353-399, nfft_atomic_convolution.hpp:20-35) accumulates into a
//     shared-memory copy of the label's row, which is then added to f(tau) with plain stores;
//   * finalize folds the halos (dnfft_1d.hpp:401-418) and evaluates the transform only at the
//     Matsubara indices (the values transformFTauToFW, dnfft_1d.hpp:427-489, picks from its FFT),
//     divides by the window's phi(w_n) and by n, and scales by 1/Nc
//     (sp_accumulator.hpp:205-220) -- all on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/dcaacc.h"
#include "common.cuh"
#include "sp_accumulator.hpp"

namespace dcaacc {

namespace {

constexpr int kOversampling = 8;
constexpr int kWindowSampling = 32;

struct NfftGrid {
  int n_padded, n, nb, nc, n_labels;
  double T0, Delta, one_div_Delta, t0_window, delta, one_div_delta, one_div_two_beta;
};

// One CTA per (label, spin).  Vertices of the sector are sorted by row orbital (right band/site)
// and by column orbital (left band/site).
__global__ void spAccumulateKernel(const NfftGrid g, const SpSector* __restrict__ sectors,
                                   const int* __restrict__ perm_r, const int* __restrict__ perm_c,
                                   const int* __restrict__ row_start, const int* __restrict__ col_start,
                                   const double* __restrict__ tau, const int* __restrict__ r_of,
                                   const double* __restrict__ coeff, double factor,
                                   double* __restrict__ f_tau, double* __restrict__ f_tau_sqr,
                                   double* __restrict__ f_tau_single) {
  extern __shared__ __align__(16) double sp_smem[];
  double* row = sp_smem;
  double* row_sqr = sp_smem + g.n_padded;
  const int label = blockIdx.x;
  const int spin = blockIdx.y;
  const SpSector sd = sectors[spin];
  const bool sqr = f_tau_sqr != nullptr;
  for (int t = threadIdx.x; t < g.n_padded * (sqr ? 2 : 1); t += blockDim.x)
    sp_smem[t] = 0.0;
  __syncthreads();

  // label = b_i + nb (b_j + nb dr), dr = index of r_i - r_j (sp_accumulator.hpp:185-191).
  const int b_i = label % g.nb, b_j = (label / g.nb) % g.nb, dr = label / (g.nb * g.nb);
  const int* pr = perm_r + sd.vtx_off;
  const int* pc = perm_c + sd.vtx_off;
  const int* rs = row_start + spin * (g.nb * g.nc + 1);
  const int* cs = col_start + spin * (g.nb * g.nc + 1);
  const double* tv = tau + sd.vtx_off;
  for (int r_j = 0; r_j < g.nc; ++r_j) {
    const int r_i = r_of[r_j + g.nc * dr];  // x_{r_i} = x_{r_j} + x_dr
    const int oi = b_i + g.nb * r_i, oj = b_j + g.nb * r_j;
    const int i0 = rs[oi], ni = rs[oi + 1] - i0;
    const int j0 = cs[oj], nj = cs[oj + 1] - j0;
    const long pairs = long(ni) * nj * (2 * kOversampling);
    for (long p = threadIdx.x; p < pairs; p += blockDim.x) {
      const int tap = static_cast<int>(p % (2 * kOversampling)) + 1;
      const long ij = p / (2 * kOversampling);
      const int i = pr[i0 + static_cast<int>(ij % ni)];
      const int j = pc[j0 + static_cast<int>(ij / ni)];
      // convoluteToFTauFineCubicInterpolation (dnfft_1d.hpp:353-399), FP64.
      const double t_val = (tv[i] - tv[j]) * g.one_div_two_beta;
      const int tau_0 = static_cast<int>((t_val - g.T0) * g.one_div_Delta);
      const double t0_val_lb = g.T0 + tau_0 * g.Delta;
      const int tau_1 = static_cast<int>((t0_val_lb - t_val - g.t0_window) * g.one_div_delta);
      const double t1_val_lb = g.t0_window + tau_1 * g.delta;
      const double d = t0_val_lb - t_val - t1_val_lb;
      const int dti = tau_1 - kOversampling * kWindowSampling;
      const int jw = dti % kWindowSampling;
      const int iw = (dti - jw) / kWindowSampling;
      const int t_out = tau_0 - kOversampling + tap;
      const int ci = iw + tap;
      if (t_out < 0 || t_out >= g.n_padded || ci < 0 || ci >= 4 * kOversampling || jw < 0)
        continue;  // only reachable for |t_val| > 1/2, which the host rejects
      const double* cf = coeff + 4 * (ci + 4 * kOversampling * jw);
      const double m = sd.M[i + static_cast<long>(sd.ldm) * j];
      const double f = factor * m;
      const double d2 = d * d;
      const double w = cf[0] + cf[1] * d + cf[2] * d2 + cf[3] * d2 * d;
      atomicAdd(row + t_out, f * w);
      if (sqr)
        atomicAdd(row_sqr + t_out, f * m * w);
    }
  }
  __syncthreads();
  double* out = f_tau + (static_cast<long>(spin) * g.n_labels + label) * g.n_padded;
  for (int t = threadIdx.x; t < g.n_padded; t += blockDim.x)
    out[t] += row[t];
  if (f_tau_single) {  // this measurement alone (replaces the previous one)
    double* one = f_tau_single + (static_cast<long>(spin) * g.n_labels + label) * g.n_padded;
    for (int t = threadIdx.x; t < g.n_padded; t += blockDim.x)
      one[t] = row[t];
  }
  if (sqr) {
    double* out2 = f_tau_sqr + (static_cast<long>(spin) * g.n_labels + label) * g.n_padded;
    for (int t = threadIdx.x; t < g.n_padded; t += blockDim.x)
      out2[t] += row_sqr[t];
  }
}

// One CTA per (label, spin): fold, then f(w) = -(1/n) sum_x f(x) e^{2 pi i x nu_w / n} / phi(w) / Nc.
__global__ void spFinalizeKernel(const NfftGrid g, const double* __restrict__ f_tau,
                                 const double* __restrict__ inv_phi, int n_sp,
                                 double2* __restrict__ out) {
  extern __shared__ __align__(16) double fin_smem[];
  double* row = fin_smem;                                       // n folded samples
  double2* tw = reinterpret_cast<double2*>(fin_smem + g.n);     // e^{2 pi i m / n}
  const int label = blockIdx.x, spin = blockIdx.y;
  const int pad = (g.n_padded - g.n) / 2;
  const double* f = f_tau + (static_cast<long>(spin) * g.n_labels + label) * g.n_padded;
  for (int x = threadIdx.x; x < g.n; x += blockDim.x) {
    double v = f[pad + x];
    // foldTimeDomainBack: halo t < pad lands on t + n, halo t >= n_padded - pad on t - n.
    const int t = pad + x;
    if (t >= g.n && t - g.n < pad)
      v += f[t - g.n];
    if (t + g.n >= g.n_padded - pad && t + g.n < g.n_padded)
      v += f[t + g.n];
    row[x] = v;
    double s, c;
    sincospi(2.0 * x / g.n, &s, &c);
    tw[x] = make_double2(c, s);
  }
  __syncthreads();
  const int b1 = label % g.nb, b2 = (label / g.nb) % g.nb, r = label / (g.nb * g.nb);
  const int nb = g.nb;
  for (int w = threadIdx.x; w < 2 * n_sp; w += blockDim.x) {
    const int nu = w >= n_sp ? 2 * (w - n_sp) + 1 : -(2 * (n_sp - 1 - w) + 1);
    const int step = ((nu % g.n) + g.n) % g.n;
    double re = 0, im = 0;
    int m = 0;
    for (int x = 0; x < g.n; ++x) {
      const double2 e = tw[m];
      re = fma(row[x], e.x, re);
      im = fma(row[x], e.y, im);
      m += step;
      if (m >= g.n)
        m -= g.n;
    }
    const double scale = -inv_phi[w] / (double(g.n) * g.nc);
    // (b1, s, b2, s, r, w)
    const long o = b1 + nb * (spin + 2 * (b2 + nb * (spin + 2 * (r + static_cast<long>(g.nc) * w))));
    out[o] = make_double2(re * scale, im * scale);
  }
}

__global__ void addKernel(double* __restrict__ dst, const double* __restrict__ src, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    dst[i] += src[i];
}

// Kaiser-Bessel window, restated from kaiser_bessel_function.cpp:28-116 (n = padded size,
// m = oversampling, sigma = 2); host only, used to build the cubic table and phi(w_n).
struct KaiserBessel {
  int n, m;
  double sigma;
  double b() const {
    return M_PI * (2. - 1. / sigma);
  }
  double renorm() const {
    return 1. / (M_PI * m) * std::sinh(M_PI * m * (2. * sigma - 1.) / sigma);
  }
  double phi_t(double x) const {
    double r = 0;
    const double val = double(m) * m - double(n) * n * x * x;
    if (val > 1.e-12)
      r = 1. / M_PI * std::sinh(b() * std::sqrt(val)) / std::sqrt(val);
    if (val < -1.e-12)
      r = 1. / M_PI * std::sin(b() * std::sqrt(-val)) / std::sqrt(-val);
    if (val >= -1.e-12 && val < 1.e-12)
      r = b() / M_PI;
    return r / renorm();
  }
  double d_phi_t(double x) const {
    double r = 0;
    const double val = double(m) * m - double(n) * n * x * x;
    if (val > 1.e-12)
      r = 1. / M_PI * (double(n) * n * x) *
          ((-b() * std::cosh(b() * std::sqrt(val))) / val + std::sinh(b() * std::sqrt(val)) / std::pow(val, 1.5));
    if (val < -1.e-12)
      r = 1. / M_PI * (double(n) * n * x) *
          ((b() * std::cos(b() * std::sqrt(-val))) / (-val) - std::sin(b() * std::sqrt(-val)) / std::pow(-val, 1.5));
    if (val >= -1.e-12 && val < 1.e-12)
      return 0;
    return r / renorm();
  }
  static double besselI0(double x) {
    double result = 0., gamma = 1, y = 1.;
    const double sq = x * x / 4.;
    for (int l = 0; l < 100000; l++) {
      const double term = y / gamma;
      if (std::abs(term) < 1.e-16)
        break;
      result += term;
      gamma *= ((l + 1) * (l + 1));
      y *= sq;
    }
    return result;
  }
  double phi_wn(int wn) const {
    if (std::pow(wn, 2) < std::pow(n * (1. - 1. / (2. * sigma)), 2))
      return 1. / double(n) *
             besselI0(m * std::sqrt(std::pow(b(), 2) - std::pow((2. * M_PI * double(wn) / double(n)), 2))) /
             renorm();
    throw Error(DCAACC_INVALID_ARG, "Matsubara index outside the window's support");
  }
};

}  // namespace

struct SpAccumulator::Impl {
  NfftGrid g{};
  int n_sp = 0, max_order = 0;
  double beta = 0;
  bool sqr = false;
  bool stamping = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaEvent_t upload_done = nullptr;
  std::vector<int> r_of;
  DevBuf<double> coeff, inv_phi, f_tau, f_tau_sqr, f_tau_single, tau_d, M_d;
  DevBuf<int> r_of_d, perm_r_d, perm_c_d, rs_d, cs_d;
  DevBuf<SpSector> sectors_d;
  DevBuf<double2> out_d;
  PinBuf<double> tau_h;
  PinBuf<int> perm_r_h, perm_c_h, rs_h, cs_h;
  PinBuf<SpSector> sectors_h;
  std::vector<double2> mrw, mrw_sqr;
  bool ready = false, finalized = false;
  uint64_t launches = 0;
};

SpAccumulator::SpAccumulator(const dcaacc_sp_config& c) : d_(new Impl) {
  auto& d = *d_;
  if (c.n_bands < 1 || c.n_sites < 1 || c.n_sp_freq < 1 || c.max_order < 1)
    throw Error(DCAACC_INVALID_ARG, "band, site, frequency counts and max_order must be positive");
  if (!(c.beta > 0) || !c.r_sub)
    throw Error(DCAACC_INVALID_ARG, "beta must be positive and r_sub non-null");
  const int nb = c.n_bands, nc = c.n_sites;
  d.n_sp = c.n_sp_freq;
  d.beta = c.beta;
  d.sqr = c.accumulate_m_sqr != 0;
  d.stamping = c.stamping != 0;
  d.max_order = c.max_order;
  // r_of[r_j + nc dr] = r_i with r_sub(r_j, r_i) = dr, i.e. x_{r_i} - x_{r_j} = x_dr.
  d.r_of.assign(nc * nc, -1);
  for (int rj = 0; rj < nc; ++rj)
    for (int ri = 0; ri < nc; ++ri) {
      const int dr = c.r_sub[rj + nc * ri];
      if (dr < 0 || dr >= nc)
        throw Error(DCAACC_INVALID_ARG, "r_sub entry out of range");
      d.r_of[rj + nc * dr] = ri;
    }
  for (int v : d.r_of)
    if (v < 0)
      throw Error(DCAACC_INVALID_ARG, "r_sub is not a group subtraction table");

  // nfft_time_domain (nfft_time_domain.hpp:112-176) with MAX_FREQUENCY = n_sp.
  auto& g = d.g;
  g.nb = nb;
  g.nc = nc;
  g.n_labels = nb * nb * nc;
  g.Delta = 1. / double(kOversampling * d.n_sp);
  g.delta = 1. / double(kOversampling * d.n_sp * kWindowSampling);
  g.one_div_Delta = 1. / g.Delta;
  g.one_div_delta = 1. / g.delta;
  g.n = kOversampling * d.n_sp;
  g.n_padded = g.n + 2 * kOversampling;
  g.T0 = -0.5 - kOversampling * g.Delta;
  g.t0_window = -2. / double(d.n_sp);
  g.one_div_two_beta = 1. / (2. * c.beta);

  // Cubic interpolation table of the window (dnfft_1d.hpp:198-250), layout (4, 4*os, ws).
  const KaiserBessel kb{g.n_padded, kOversampling, 2.0};
  const int n_os = 4 * kOversampling;
  std::vector<double> cf(4 * n_os * kWindowSampling);
  auto fine_tau = [&](int idx) { return g.t0_window + idx * g.delta; };
  const double dl = fine_tau(1) - fine_tau(0);
  for (int i = 0; i < n_os; ++i)
    for (int j = 0; j < kWindowSampling; ++j) {
      const double tau = fine_tau(j + i * kWindowSampling);
      const double f0 = kb.phi_t(tau), f1 = kb.phi_t(tau + dl);
      const double df0 = kb.d_phi_t(tau), df1 = kb.d_phi_t(tau + dl);
      double* p = &cf[4 * (i + n_os * j)];
      p[0] = f0;
      p[1] = df0;
      p[2] = -(3. * f0 - 3. * f1 + 2. * df0 * dl + df1 * dl) / std::pow(dl, 2);
      p[3] = -(-2. * f0 + 2. * f1 - 1. * df0 * dl - df1 * dl) / std::pow(dl, 3);
    }
  std::vector<double> ip(2 * d.n_sp);
  for (int w = 0; w < 2 * d.n_sp; ++w) {
    const int nu = w >= d.n_sp ? 2 * (w - d.n_sp) + 1 : -(2 * (d.n_sp - 1 - w) + 1);
    ip[w] = 1.0 / kb.phi_wn(nu);
  }

  DCAACC_CUDA_CHECK(cudaGetDevice(&d.device));
  DCAACC_CUDA_CHECK(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking));
  d.own_stream = true;
  DCAACC_CUDA_CHECK(cudaEventCreateWithFlags(&d.upload_done, cudaEventDisableTiming));
  d.coeff.alloc(cf.size());
  DCAACC_CUDA_CHECK(cudaMemcpy(d.coeff.get(), cf.data(), d.coeff.bytes(), cudaMemcpyHostToDevice));
  d.inv_phi.alloc(ip.size());
  DCAACC_CUDA_CHECK(cudaMemcpy(d.inv_phi.get(), ip.data(), d.inv_phi.bytes(), cudaMemcpyHostToDevice));
  d.r_of_d.alloc(d.r_of.size());
  DCAACC_CUDA_CHECK(cudaMemcpy(d.r_of_d.get(), d.r_of.data(), d.r_of_d.bytes(), cudaMemcpyHostToDevice));
  const size_t ft = 2 * size_t(g.n_labels) * g.n_padded;
  d.f_tau.alloc(ft);
  if (d.sqr)
    d.f_tau_sqr.alloc(ft);
  if (d.stamping)
    d.f_tau_single.alloc(ft);
  const size_t nv = 2 * size_t(d.max_order);
  d.tau_d.alloc(nv);
  d.M_d.alloc(2 * size_t(d.max_order) * d.max_order);
  d.perm_r_d.alloc(nv);
  d.perm_c_d.alloc(nv);
  d.rs_d.alloc(2 * size_t(nb * nc + 1));
  d.cs_d.alloc(2 * size_t(nb * nc + 1));
  d.sectors_d.alloc(2);
  d.out_d.alloc(size_t(2 * nb) * (2 * nb) * nc * 2 * d.n_sp);
  d.tau_h.alloc(nv);
  d.perm_r_h.alloc(nv);
  d.perm_c_h.alloc(nv);
  d.rs_h.alloc(2 * size_t(nb * nc + 1));
  d.cs_h.alloc(2 * size_t(nb * nc + 1));
  d.sectors_h.alloc(2);
  DCAACC_CUDA_CHECK(cudaEventRecord(d.upload_done, d.stream));
  if (sizeof(double) * 2 * g.n_padded > 200 * 1024 || sizeof(double) * 3 * g.n > 200 * 1024)
    throw Error(DCAACC_INVALID_ARG, "n_sp_freq too large for the shared-memory NFFT rows");
}

SpAccumulator::~SpAccumulator() {
  if (d_->stream)
    cudaStreamSynchronize(d_->stream);
  if (d_->upload_done)
    cudaEventDestroy(d_->upload_done);
  if (d_->own_stream && d_->stream)
    cudaStreamDestroy(d_->stream);
}

void SpAccumulator::reset() {
  auto& d = *d_;
  DCAACC_CUDA_CHECK(cudaMemsetAsync(d.f_tau.get(), 0, d.f_tau.bytes(), d.stream));
  if (d.sqr)
    DCAACC_CUDA_CHECK(cudaMemsetAsync(d.f_tau_sqr.get(), 0, d.f_tau_sqr.bytes(), d.stream));
  if (d.stamping)
    DCAACC_CUDA_CHECK(cudaMemsetAsync(d.f_tau_single.get(), 0, d.f_tau_single.bytes(), d.stream));
  d.ready = true;
  d.finalized = false;
}

void SpAccumulator::accumulate(const dcaacc_sector* sec, double factor) {
  auto& d = *d_;
  auto& g = d.g;
  if (!d.ready)
    throw Error(DCAACC_NOT_READY, "The accumulator was not initialized.");
  if (d.finalized)
    throw Error(DCAACC_NOT_READY, "The accumulator is already finalized.");
  if (!sec)
    throw Error(DCAACC_INVALID_ARG, "null sectors");
  const int n_orb = g.nb * g.nc;
  DCAACC_CUDA_CHECK(cudaEventSynchronize(d.upload_done));
  int vtx = 0;
  for (int s = 0; s < 2; ++s) {
    const auto& x = sec[s];
    if (x.n < 0 || x.n > d.max_order)
      throw Error(DCAACC_INVALID_ARG, "expansion order outside [0, max_order]");
    if (x.n && (!x.tau || !x.left_band || !x.right_band || !x.left_site || !x.right_site || !x.M ||
                x.ldm < x.n))
      throw Error(DCAACC_INVALID_ARG, "invalid sector");
    for (int i = 0; i < x.n; ++i) {
      if (x.left_band[i] < 0 || x.left_band[i] >= g.nb || x.right_band[i] < 0 || x.right_band[i] >= g.nb ||
          x.left_site[i] < 0 || x.left_site[i] >= g.nc || x.right_site[i] < 0 || x.right_site[i] >= g.nc)
        throw Error(DCAACC_INVALID_ARG, "vertex band or site out of range");
      if (!(x.tau[i] >= 0.0 && x.tau[i] <= d.beta))
        throw Error(DCAACC_INVALID_ARG, "vertex time outside [0, beta]");
    }
    // Rows: right band / site; columns: left band / site (sp_accumulator.hpp:181-187).
    auto sort_side = [&](bool left, int* perm, int* start) {
      std::fill(start, start + n_orb + 1, 0);
      for (int v = 0; v < x.n; ++v)
        start[(left ? x.left_band[v] + g.nb * x.left_site[v] : x.right_band[v] + g.nb * x.right_site[v]) + 1]++;
      for (int o = 0; o < n_orb; ++o)
        start[o + 1] += start[o];
      std::vector<int> fill(start, start + n_orb);
      for (int v = 0; v < x.n; ++v)
        perm[fill[left ? x.left_band[v] + g.nb * x.left_site[v] : x.right_band[v] + g.nb * x.right_site[v]]++] = v;
    };
    sort_side(false, d.perm_r_h.get() + vtx, d.rs_h.get() + s * (n_orb + 1));
    sort_side(true, d.perm_c_h.get() + vtx, d.cs_h.get() + s * (n_orb + 1));
    std::copy_n(x.tau, x.n, d.tau_h.get() + vtx);
    SpSector sd{};
    sd.n = x.n;
    sd.vtx_off = vtx;
    sd.M = x.M;
    sd.ldm = std::max(x.ldm, 1);
    if (x.n && !x.m_on_device) {
      double* dst = d.M_d.get() + size_t(s) * d.max_order * d.max_order;
      DCAACC_CUDA_CHECK(cudaMemcpy2DAsync(dst, sizeof(double) * x.n, x.M, sizeof(double) * x.ldm,
                                          sizeof(double) * x.n, x.n, cudaMemcpyHostToDevice, d.stream));
      sd.M = dst;
      sd.ldm = x.n;
    }
    d.sectors_h[s] = sd;
    vtx += x.n;
  }
  if (vtx == 0) {
    if (d.stamping)  // an empty measurement: its own f(tau) is zero
      DCAACC_CUDA_CHECK(cudaMemsetAsync(d.f_tau_single.get(), 0, d.f_tau_single.bytes(), d.stream));
    return;
  }
  auto h2d = [&](void* dst, const void* src, size_t bytes) {
    if (bytes)
      DCAACC_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, d.stream));
  };
  h2d(d.sectors_d.get(), d.sectors_h.get(), 2 * sizeof(SpSector));
  h2d(d.tau_d.get(), d.tau_h.get(), sizeof(double) * vtx);
  h2d(d.perm_r_d.get(), d.perm_r_h.get(), sizeof(int) * vtx);
  h2d(d.perm_c_d.get(), d.perm_c_h.get(), sizeof(int) * vtx);
  h2d(d.rs_d.get(), d.rs_h.get(), sizeof(int) * 2 * (n_orb + 1));
  h2d(d.cs_d.get(), d.cs_h.get(), sizeof(int) * 2 * (n_orb + 1));
  DCAACC_CUDA_CHECK(cudaEventRecord(d.upload_done, d.stream));
  const size_t smem = sizeof(double) * g.n_padded * (d.sqr ? 2 : 1);
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(spAccumulateKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  spAccumulateKernel<<<dim3(g.n_labels, 2), 256, smem, d.stream>>>(
      g, d.sectors_d.get(), d.perm_r_d.get(), d.perm_c_d.get(), d.rs_d.get(), d.cs_d.get(),
      d.tau_d.get(), d.r_of_d.get(), d.coeff.get(), factor, d.f_tau.get(),
      d.sqr ? d.f_tau_sqr.get() : nullptr, d.stamping ? d.f_tau_single.get() : nullptr);
  DCAACC_LAUNCH_CHECK();
  ++d.launches;
}

void SpAccumulator::finalize() {
  auto& d = *d_;
  if (d.finalized)
    return;
  finalizeInto(d.f_tau.get(), d.mrw);
  if (d.sqr)
    finalizeInto(d.f_tau_sqr.get(), d.mrw_sqr);
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(d.stream));
  d.finalized = true;
}

// Fold, DFT and window division of one f(tau) set into host memory (enqueued on the stream).
void SpAccumulator::finalizeInto(const double* f_tau, std::vector<double2>& host) {
  auto& d = *d_;
  auto& g = d.g;
  const size_t smem = sizeof(double) * 3 * g.n;
  DCAACC_CUDA_CHECK(cudaFuncSetAttribute(spFinalizeKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  DCAACC_CUDA_CHECK(cudaMemsetAsync(d.out_d.get(), 0, d.out_d.bytes(), d.stream));
  spFinalizeKernel<<<dim3(g.n_labels, 2), 256, smem, d.stream>>>(g, f_tau, d.inv_phi.get(), d.n_sp, d.out_d.get());
  DCAACC_LAUNCH_CHECK();
  ++d.launches;
  host.resize(d.out_d.size());
  DCAACC_CUDA_CHECK(cudaMemcpyAsync(host.data(), d.out_d.get(), d.out_d.bytes(), cudaMemcpyDeviceToHost, d.stream));
}

void SpAccumulator::singleMeasurementMrw(double* out, size_t count) {
  auto& d = *d_;
  if (!d.stamping)
    throw Error(DCAACC_NOT_READY, "single-measurement functions need stamping");
  if (count != d.out_d.size())
    throw Error(DCAACC_INVALID_ARG, "output size does not match");
  std::vector<double2> host;
  finalizeInto(d.f_tau_single.get(), host);
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(d.stream));
  std::memcpy(out, host.data(), 16 * count);
}

void SpAccumulator::singleMeasurementFtau(double* out, size_t count) {
  auto& d = *d_;
  if (!d.stamping)
    throw Error(DCAACC_NOT_READY, "single-measurement functions need stamping");
  if (count != d.f_tau_single.size())
    throw Error(DCAACC_INVALID_ARG, "output size does not match");
  DCAACC_CUDA_CHECK(cudaMemcpyAsync(out, d.f_tau_single.get(), d.f_tau_single.bytes(), cudaMemcpyDeviceToHost,
                                    d.stream));
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(d.stream));
}

void SpAccumulator::clearSingleMeasurement() {
  auto& d = *d_;
  if (!d.stamping)
    throw Error(DCAACC_NOT_READY, "single-measurement functions need stamping");
  DCAACC_CUDA_CHECK(cudaMemsetAsync(d.f_tau_single.get(), 0, d.f_tau_single.bytes(), d.stream));
}

size_t SpAccumulator::fTauSize() const {
  return d_->f_tau.size();
}

void SpAccumulator::get(bool sqr, double* out, size_t count) const {
  auto& d = *d_;
  if (!d.finalized)
    throw Error(DCAACC_NOT_READY, "The accumulator was not finalized.");
  if (sqr && !d.sqr)
    throw Error(DCAACC_NOT_READY, "M squared was not accumulated.");
  const auto& v = sqr ? d.mrw_sqr : d.mrw;
  if (count != v.size())
    throw Error(DCAACC_INVALID_ARG, "output size does not match");
  std::memcpy(out, v.data(), 16 * count);
}

void SpAccumulator::sumTo(SpAccumulator& other) const {
  auto& d = *d_;
  auto& o = *other.d_;
  if (o.g.n_padded != d.g.n_padded || o.g.n_labels != d.g.n_labels || o.sqr != d.sqr)
    throw Error(DCAACC_INVALID_ARG, "accumulators have different shapes");
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(d.stream));
  const int blocks = 148 * 4;
  addKernel<<<blocks, 256, 0, o.stream>>>(o.f_tau.get(), d.f_tau.get(), d.f_tau.size());
  DCAACC_LAUNCH_CHECK();
  ++o.launches;
  if (d.sqr) {
    addKernel<<<blocks, 256, 0, o.stream>>>(o.f_tau_sqr.get(), d.f_tau_sqr.get(), d.f_tau_sqr.size());
    DCAACC_LAUNCH_CHECK();
    ++o.launches;
  }
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(o.stream));
}

void SpAccumulator::setStream(cudaStream_t s) {
  auto& d = *d_;
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(d.stream));
  if (d.own_stream)
    DCAACC_CUDA_CHECK(cudaStreamDestroy(d.stream));
  d.own_stream = false;
  d.stream = s;
}

void SpAccumulator::synchronize() {
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(d_->stream));
}

size_t SpAccumulator::deviceFingerprint() const {
  auto& d = *d_;
  return d.coeff.bytes() + d.inv_phi.bytes() + d.f_tau.bytes() + d.f_tau_sqr.bytes() + d.f_tau_single.bytes() +
         d.tau_d.bytes() +
         d.M_d.bytes() + d.r_of_d.bytes() + d.perm_r_d.bytes() + d.perm_c_d.bytes() + d.rs_d.bytes() +
         d.cs_d.bytes() + d.sectors_d.bytes() + d.out_d.bytes();
}

uint64_t SpAccumulator::kernelLaunches() const {
  return d_->launches;
}

size_t SpAccumulator::outputSize() const {
  return d_->out_d.size();
}

}  // namespace dcaacc
