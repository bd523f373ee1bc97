// Allocation-free G computation for one measurement (dcaacc_tp_compute_g_noalloc).
//
// Who needs this: callers that cannot allocate device memory when they run.  Typical cases are
// host applications whose device memory is fully reserved by their own pool allocator (nothing
// is left for cudaMalloc), and tight per-measurement loops that must not pay the implicit
// device-wide synchronisation cudaMalloc / cudaFree perform.  The regular handle
// (dcaacc_tp_create) allocates all its buffers up front; this entry point instead keeps its
// scratch in one file-scope device array, so calling it allocates nothing.
//
// The scratch array is a static __device__ object: every GPU that loads this library holds its
// kStaticScratchBytes until the process exits.  In host code the array's name is only a
// host-side stand-in, not a device address, so its device address is looked up once per device
// with cudaGetSymbolAddress (on the first call made with that device current) and that address
// is what the kernels receive.  All calls share the array and it keeps the last call's
// contents: everything the kernels read is rewritten by each call before use, and calls whose
// work overlaps on the GPU (e.g. on two streams) race on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "../../include/dcaacc.h"
#include "common.cuh"
#include "tp_frontend.hpp"

namespace dcaacc {

namespace {

constexpr size_t kStaticScratchBytes = size_t(48) << 20;  // 48 MiB
constexpr int kMaxOrder = 512;                            // per spin sector
constexpr int kMaxOrbitals = 64;                          // nb * Nc
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once per device).
unsigned char* scratchOnCurrentDevice() {
  int dev = 0;
  DCAACC_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    throw Error(DCAACC_INVALID_ARG, "device ordinal out of range for the static scratch table");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess)
      throw Error(DCAACC_CUDA_ERR, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  return static_cast<unsigned char*>(g_scratch_ptr[dev]);
}

// G0_(b1, b2, k, w_ext, s) <- G0(b1, s, b2, s, k, w_ext + sp_offset) (tp_accumulator_base.hpp:210-221).
__global__ void sliceG0Kernel(const double2* __restrict__ G0, double2* __restrict__ out, int nb, int nc,
                              int nw_ext, int sp_offset) {
  const long total = 2L * nw_ext * nc * nb * nb;
  for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
    long r = i;
    const int b1 = r % nb;
    r /= nb;
    const int b2 = r % nb;
    r /= nb;
    const int k = r % nc;
    r /= nc;
    const int w = r % nw_ext;
    const int s = static_cast<int>(r / nw_ext);
    const long in = b1 + nb * (s + 2L * (b2 + nb * (s + 2L * (k + long(nc) * (w + sp_offset)))));
    out[i] = G0[in];
  }
}

// Fb(r, k, b) = e^{i k.r} e^{i k.a_b} (space_transform_2D.hpp:93-140).
__global__ void buildFbKernel(const double* __restrict__ vecs, double2* __restrict__ Fb, int nb, int nc) {
  const double* kv = vecs;
  const double* rv = vecs + 2 * nc;
  const double* av = vecs + 4 * nc;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb * nc * nc; i += gridDim.x * blockDim.x) {
    const int r = i % nc, k = (i / nc) % nc, b = i / (nc * nc);
    double s1, c1, s2, c2;
    sincos(kv[2 * k] * rv[2 * r] + kv[2 * k + 1] * rv[2 * r + 1], &s1, &c1);
    sincos(kv[2 * k] * av[2 * b] + kv[2 * k + 1] * av[2 * b + 1], &s2, &c2);
    Fb[i] = make_double2(c1 * c2 - s1 * s2, c1 * s2 + s1 * c2);
  }
}

size_t alignUp(size_t x) {
  return (x + 255) & ~size_t(255);
}

}  // namespace

void computeGNoAlloc(const dcaacc_tp_config& c, const double* G0_dev, const dcaacc_sector* sec,
                     double* G_out, cudaStream_t stream) {
  // ---- validation: everything is checked before the GPU is touched ----
  if (c.n_bands < 1 || c.n_sites < 1 || c.n_w_half < 1 || c.n_sp_freq < 1 || !(c.beta > 0))
    throw Error(DCAACC_INVALID_ARG, "band, site and frequency counts and beta must be positive");
  if (!G0_dev || !sec || !G_out || !c.k_vecs || !c.r_vecs || !c.a_vecs || !c.w_ex || c.n_w_ex < 1)
    throw Error(DCAACC_INVALID_ARG, "null argument");
  const int nb = c.n_bands, nc = c.n_sites, n_orb = nb * nc;
  if (n_orb > kMaxOrbitals)
    throw Error(DCAACC_INVALID_ARG, "nb * Nc exceeds 64, the limit of the allocation-free entry point");
  int ext = 0;
  for (int i = 0; i < c.n_w_ex; ++i)
    ext = std::max(ext, std::abs(c.w_ex[i]));
  const int nw_ext = 2 * c.n_w_half + 2 * ext;
  if (2 * c.n_sp_freq < nw_ext)
    throw Error(DCAACC_INVALID_ARG, "The number of single particle frequencies is too small.");
  int n[2];
  for (int s = 0; s < 2; ++s) {
    const auto& x = sec[s];
    n[s] = x.n;
    if (x.n < 0 || x.n > kMaxOrder)
      throw Error(DCAACC_INVALID_ARG, "expansion order outside [0, 512], the limit of the allocation-free entry point");
    if (x.n && (!x.m_on_device || !x.M || x.ldm < x.n || !x.tau || !x.left_band || !x.right_band ||
                !x.left_site || !x.right_site))
      throw Error(DCAACC_INVALID_ARG, "each non-empty sector needs host vertex arrays and a device M");
    for (int i = 0; i < x.n; ++i)
      if (x.left_band[i] < 0 || x.left_band[i] >= nb || x.right_band[i] < 0 || x.right_band[i] >= nb ||
          x.left_site[i] < 0 || x.left_site[i] >= nc || x.right_site[i] < 0 || x.right_site[i] >= nc ||
          !std::isfinite(x.tau[i]))
        throw Error(DCAACC_INVALID_ARG, "vertex band, site or time out of range");
  }
  const int n_vtx = n[0] + n[1];
  const bool non_density = c.non_density != 0;
  const int R = n_orb;
  TpDims d{};
  d.nb = nb;
  d.nc = nc;
  d.nw = 2 * c.n_w_half;
  d.ext = ext;
  d.nw_ext = nw_ext;
  d.n_orb = n_orb;
  d.R = R;
  d.beta = c.beta;
  // The FP64 front-end keeps per-CTA tiles of the cluster transform in shared memory; their size
  // grows with nb * Nc (for one band it passes 227 KB above Nc = 43).
  if (frontendSmemRequirement(d, std::max(n[0], n[1]), true) > 227 * 1024)
    throw Error(DCAACC_INVALID_ARG, "nb * Nc too large for the FP64 front-end's shared-memory tiles "
                                    "(more than 227 KB per block)");
  // Each call uploads its sorted vertex tables from stack memory: such copies cannot be recorded
  // into a graph (a replay would read a dead stack frame), so a capturing stream is refused.
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const cudaError_t ce = cudaStreamIsCapturing(stream, &cs);
    if (ce == cudaErrorStreamCaptureImplicit || (ce == cudaSuccess && cs != cudaStreamCaptureStatusNone)) {
      cudaGetLastError();
      throw Error(DCAACC_INVALID_ARG, "the allocation-free entry point cannot be called during stream capture");
    }
    DCAACC_CUDA_CHECK(ce);
  }

  // ---- carve the static scratch ----
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = alignUp(off + bytes);
    return o;
  };
  const size_t o_sec = take(2 * sizeof(SectorDesc));
  const size_t o_tau = take(sizeof(double) * std::max(n_vtx, 1));
  const size_t o_pr = take(sizeof(int) * std::max(n_vtx, 1));
  const size_t o_pc = take(sizeof(int) * std::max(n_vtx, 1));
  const size_t o_rs = take(sizeof(int) * 2 * (n_orb + 1));
  const size_t o_cs = take(sizeof(int) * 2 * (n_orb + 1));
  const size_t o_vec = take(sizeof(double) * (4 * nc + 2 * nb));
  const size_t o_g0 = take(sizeof(double2) * size_t(nb) * nb * nc * nw_ext * 2);
  const size_t o_fb = take(sizeof(double2) * size_t(nb) * nc * nc);
  const size_t o_tr = take(sizeof(double2) * size_t(std::max(n_vtx, 1)) * nw_ext);
  const size_t o_tc = non_density ? take(sizeof(double2) * size_t(std::max(n_vtx, 1)) * nw_ext) : o_tr;
  const size_t o_x = take(sizeof(double2) * size_t(R) * std::max(n_vtx, 1) * nw_ext);
  if (off > kStaticScratchBytes)
    throw Error(DCAACC_INVALID_ARG, "problem needs " + std::to_string(off >> 20) +
                                        " MiB of scratch; the allocation-free entry point has 48 MiB");
  unsigned char* base = scratchOnCurrentDevice();

  // ---- host-side sort into stack arrays (no heap use) ----
  int perm_r[2 * kMaxOrder], perm_c[2 * kMaxOrder], rstart[2 * (kMaxOrbitals + 1)],
      cstart[2 * (kMaxOrbitals + 1)];
  double tau[2 * kMaxOrder];
  SectorDesc sd[2];
  int vtx = 0;
  for (int s = 0; s < 2; ++s) {
    const auto& x = sec[s];
    auto sort_side = [&](bool left, int* perm, int* start) {
      int fill[kMaxOrbitals];
      std::fill(start, start + n_orb + 1, 0);
      for (int v = 0; v < x.n; ++v)
        start[(left ? x.left_band[v] + nb * x.left_site[v] : x.right_band[v] + nb * x.right_site[v]) + 1]++;
      for (int o = 0; o < n_orb; ++o)
        start[o + 1] += start[o];
      std::copy(start, start + n_orb, fill);
      for (int v = 0; v < x.n; ++v)
        perm[fill[left ? x.left_band[v] + nb * x.left_site[v] : x.right_band[v] + nb * x.right_site[v]]++] = v;
    };
    sort_side(false, perm_r + vtx, rstart + s * (n_orb + 1));
    if (non_density)
      sort_side(true, perm_c + vtx, cstart + s * (n_orb + 1));
    else {
      std::copy_n(perm_r + vtx, x.n, perm_c + vtx);
      std::copy_n(rstart + s * (n_orb + 1), n_orb + 1, cstart + s * (n_orb + 1));
    }
    std::copy_n(x.tau, x.n, tau + vtx);
    sd[s] = SectorDesc{};
    sd[s].M = x.M;
    sd[s].ldm = std::max(x.ldm, 1);
    sd[s].n = x.n;
    sd[s].vtx_off = vtx;
    sd[s].orb_off = s * (n_orb + 1);
    sd[s].spin = s;
    sd[s].slot = 0;
    sd[s].x_off = long(R) * vtx * nw_ext;
    vtx += x.n;
  }

  // ---- uploads into the scratch (copies from pageable host memory return once staged) ----
  auto h2d = [&](size_t o, const void* src, size_t bytes) {
    if (bytes)
      DCAACC_CUDA_CHECK(cudaMemcpyAsync(base + o, src, bytes, cudaMemcpyHostToDevice, stream));
  };
  h2d(o_sec, sd, 2 * sizeof(SectorDesc));
  h2d(o_tau, tau, sizeof(double) * n_vtx);
  h2d(o_pr, perm_r, sizeof(int) * n_vtx);
  h2d(o_pc, perm_c, sizeof(int) * n_vtx);
  h2d(o_rs, rstart, sizeof(int) * 2 * (n_orb + 1));
  h2d(o_cs, cstart, sizeof(int) * 2 * (n_orb + 1));
  h2d(o_vec, c.k_vecs, sizeof(double) * 2 * nc);
  h2d(o_vec + sizeof(double) * 2 * nc, c.r_vecs, sizeof(double) * 2 * nc);
  h2d(o_vec + sizeof(double) * 4 * nc, c.a_vecs, sizeof(double) * 2 * nb);

  sliceG0Kernel<<<64, 256, 0, stream>>>(reinterpret_cast<const double2*>(G0_dev),
                                        reinterpret_cast<double2*>(base + o_g0), nb, nc, nw_ext,
                                        (2 * c.n_sp_freq - nw_ext) / 2);
  DCAACC_LAUNCH_CHECK();
  buildFbKernel<<<8, 256, 0, stream>>>(reinterpret_cast<const double*>(base + o_vec),
                                       reinterpret_cast<double2*>(base + o_fb), nb, nc);
  DCAACC_LAUNCH_CHECK();

  FrontendArgs fa{};
  fa.dims = d;
  fa.sectors = reinterpret_cast<const SectorDesc*>(base + o_sec);
  fa.n_sectors = 2;
  fa.n_max = std::max(n[0], n[1]);
  fa.tau = reinterpret_cast<const double*>(base + o_tau);
  fa.perm_r = reinterpret_cast<const int*>(base + o_pr);
  fa.perm_c = reinterpret_cast<const int*>(base + o_pc);
  fa.row_start = reinterpret_cast<const int*>(base + o_rs);
  fa.col_start = reinterpret_cast<const int*>(base + o_cs);
  fa.Tr = reinterpret_cast<double2*>(base + o_tr);
  fa.Tc = reinterpret_cast<double2*>(base + o_tc);
  fa.Fb = reinterpret_cast<const double2*>(base + o_fb);
  fa.G0 = reinterpret_cast<const double2*>(base + o_g0);
  double2* Xp = reinterpret_cast<double2*>(base + o_x);
  if (fa.n_max > 0) {
    launchTwiddles(fa, stream);
    launchRowTransform<double>(fa, Xp, stream);
  }
  launchColTransform<double>(fa, Xp, reinterpret_cast<double2*>(G_out), long(nw_ext) * nw_ext * R * R,
                             stream);
}

size_t staticScratchBytes() {
  return kStaticScratchBytes;
}

}  // namespace dcaacc
