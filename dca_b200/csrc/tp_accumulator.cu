// Host side of the two-particle accumulator (see tp_accumulator.hpp).
#include "tp_accumulator.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "tp_frontend.hpp"
#include "tp_g4.hpp"
#include "tp_sort.hpp"

namespace dcaacc {

namespace {
[[noreturn]] void invalid(const std::string& msg) {
  throw Error(DCAACC_INVALID_ARG, msg);
}
}  // namespace

TpAccumulator::TpAccumulator(const dcaacc_tp_config& c, const double* G0) {
  // A failure part way (an invalid argument, or an allocation that fails) releases the streams
  // and events created so far; the device and pinned buffers release themselves.
  try {
    init(c, G0);
  }
  catch (...) {
    releaseStreamsAndEvents();
    throw;
  }
}

void TpAccumulator::init(const dcaacc_tp_config& c, const double* G0) {
  // ---- validation (the reference's logic_error cases, tp_accumulator_base.hpp:197-198,
  // tp_accumulator_gpu.hpp:456-468, plus the index tables G4Helper::set trusts) ----
  if (c.n_bands < 1 || c.n_sites < 1 || c.n_w_half < 1 || c.n_sp_freq < 1)
    invalid("band, site and frequency counts must be positive");
  if (c.n_k_ex < 1 || !c.k_ex || c.n_w_ex < 1 || !c.w_ex)
    invalid("at least one momentum and one frequency transfer are required");
  if (c.n_channels < 1 || c.n_channels > kMaxChannels || !c.channels)
    invalid("between 1 and 4 channels are supported");
  if (!(c.beta > 0) || !std::isfinite(c.beta))
    invalid("beta must be positive");
  if (!c.r_vecs || !c.k_vecs || !c.a_vecs || !c.k_add || !c.k_sub || !G0)
    invalid("null table pointer");
  if (c.precision != DCAACC_PRECISION_FP64 && c.precision != DCAACC_PRECISION_MIXED)
    invalid("unknown precision mode");
  if (c.max_batch < 1 || c.max_order < 1)
    invalid("max_batch and max_order must be positive");
  const int nc = c.n_sites, nb = c.n_bands;
  if (nb * nc > 1024)
    invalid("nb * Nc must not exceed 1024");
  for (int i = 0; i < nc * nc; ++i)
    if (c.k_add[i] < 0 || c.k_add[i] >= nc || c.k_sub[i] < 0 || c.k_sub[i] >= nc)
      invalid("momentum add/subtract table entry out of range");
  for (int i = 0; i < c.n_k_ex; ++i)
    if (c.k_ex[i] < 0 || c.k_ex[i] >= nc)
      invalid("momentum transfer index out of range");
  int ext = 0;
  for (int i = 0; i < c.n_w_ex; ++i)
    ext = std::max(ext, std::abs(c.w_ex[i]));
  for (int i = 0; i < c.n_channels; ++i)
    if (c.channels[i] < DCAACC_PH_TRANSVERSE || c.channels[i] > DCAACC_PP_UP_DOWN)
      throw Error(DCAACC_UNSUPPORTED, "Specified four point type not implemented.");
  const int nw = 2 * c.n_w_half, nw_ext = nw + 2 * ext;
  if (2 * c.n_sp_freq < nw_ext)
    invalid("The number of single particle frequencies is too small.");

  dims_.nb = nb;
  dims_.nc = nc;
  dims_.nw = nw;
  dims_.ext = ext;
  dims_.nw_ext = nw_ext;
  dims_.n_orb = nb * nc;
  dims_.R = nb * nc;
  dims_.nq = c.n_k_ex;
  dims_.nwq = c.n_w_ex;
  dims_.n_channels = c.n_channels;
  for (int i = 0; i < kMaxChannels; ++i)
    dims_.channels[i] = i < c.n_channels ? c.channels[i] : 0;
  dims_.beta = c.beta;
  mixed_ = c.precision == DCAACC_PRECISION_MIXED;
  non_density_ = c.non_density != 0;
  atomic_ = c.accumulators > 1;
  max_batch_ = c.max_batch;
  max_order_ = c.max_order;
  n_sp_ = c.n_sp_freq;
  k_add_.assign(c.k_add, c.k_add + nc * nc);
  k_sub_.assign(c.k_sub, c.k_sub + nc * nc);
  q_list_.assign(c.k_ex, c.k_ex + c.n_k_ex);
  wex_list_.assign(c.w_ex, c.w_ex + c.n_w_ex);
  g4_size_ = size_t(nb) * nb * nb * nb * nc * nc * nw * nw * c.n_k_ex * c.n_w_ex;
  // -k for the mirror-symmetric G of the mixed path: the identity z of the momentum group
  // (k_add[z + Nc k] = k for all k), then -k = z - k = k_sub[k + Nc z].
  std::vector<int> kneg;
  if (nc <= kMaxKneg)
    for (int z = 0; z < nc && kneg.empty(); ++z) {
      bool id = true;
      for (int k = 0; k < nc; ++k)
        id = id && k_add_[z + nc * k] == k;
      if (id)
        for (int k = 0; k < nc; ++k)
          kneg.push_back(k_sub_[k + nc * z]);
    }
  bool mirror_ok = !kneg.empty();
  for (size_t k = 0; k < kneg.size(); ++k)
    mirror_ok = mirror_ok && kneg[kneg[k]] == int(k);
  const long R = dims_.R;
  g_sector_stride_ = long(nw_ext) * nw_ext * R * R;

  DCAACC_CUDA_CHECK(cudaGetDevice(&device_));
  DCAACC_CUDA_CHECK(cudaDeviceGetAttribute(&n_sm_, cudaDevAttrMultiProcessorCount, device_));
  DCAACC_CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  own_stream_ = true;
  DCAACC_CUDA_CHECK(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
  for (auto& h : hstage_)
    DCAACC_CUDA_CHECK(cudaEventCreateWithFlags(&h.uploaded, cudaEventDisableTiming));
  for (auto& d : dstage_)
    DCAACC_CUDA_CHECK(cudaEventCreateWithFlags(&d.consumed, cudaEventDisableTiming));

  // ---- G0 slice over the extended mesh (tp_accumulator_base.hpp:210-221) ----
  {
    const int sp_offset = (2 * c.n_sp_freq - nw_ext) / 2;
    std::vector<double2> g0(size_t(nb) * nb * nc * nw_ext * 2);
    for (int s = 0; s < 2; ++s)
      for (int w = 0; w < nw_ext; ++w)
        for (int k = 0; k < nc; ++k)
          for (int b2 = 0; b2 < nb; ++b2)
            for (int b1 = 0; b1 < nb; ++b1) {
              const size_t in =
                  b1 + nb * (s + 2 * (b2 + nb * (s + 2 * (k + size_t(nc) * (w + sp_offset)))));
              g0[b1 + nb * (b2 + nb * (k + size_t(nc) * (w + size_t(nw_ext) * s)))] =
                  make_double2(G0[2 * in], G0[2 * in + 1]);
            }
    G0_.alloc(g0.size());
    DCAACC_CUDA_CHECK(cudaMemcpy(G0_.get(), g0.data(), G0_.bytes(), cudaMemcpyHostToDevice));
    // Mirror symmetry G0(-k, -w) = conj G0(k, w) (one band; time-reversal symmetric models).
    if (mirror_ok && nb == 1) {
      double mx = 0, dev = 0;
      for (int s = 0; s < 2; ++s)
        for (int w = 0; w < nw_ext; ++w)
          for (int k = 0; k < nc; ++k) {
            const double2 a = g0[k + size_t(nc) * (w + size_t(nw_ext) * s)];
            const double2 b = g0[kneg[k] + size_t(nc) * (nw_ext - 1 - w + size_t(nw_ext) * s)];
            mx = std::max(mx, std::hypot(a.x, a.y));
            dev = std::max(dev, std::hypot(a.x - b.x, a.y + b.y));
          }
      mirror_ok = dev <= 1e-12 * mx;
    }
    else {
      mirror_ok = false;
    }
  }
  // ---- cluster transform with band phases: Fb(r, k, b) = e^{i k.r} e^{i k.a_b}
  // (space_transform_2D.hpp:93-140) ----
  ColFft fft{};
  {
    std::vector<double2> fb(size_t(nb) * nc * nc);
    for (int b = 0; b < nb; ++b)
      for (int k = 0; k < nc; ++k) {
        const double kx = c.k_vecs[2 * k], ky = c.k_vecs[2 * k + 1];
        const std::complex<double> ph =
            std::exp(std::complex<double>(0, kx * c.a_vecs[2 * b] + ky * c.a_vecs[2 * b + 1]));
        for (int r = 0; r < nc; ++r) {
          const std::complex<double> t =
              std::exp(std::complex<double>(0, kx * c.r_vecs[2 * r] + ky * c.r_vecs[2 * r + 1]));
          const std::complex<double> v = t * ph;
          fb[(size_t(b) * nc + k) * nc + r] = make_double2(v.real(), v.imag());
        }
      }
    Fb_.alloc(fb.size());
    DCAACC_CUDA_CHECK(cudaMemcpy(Fb_.get(), fb.data(), Fb_.bytes(), cudaMemcpyHostToDevice));
    // An L x L square cluster (L = 4 or 6; integer sites (a, b), momenta 2 pi (m, n) / L) makes
    // the one-band cluster transform a 2D FFT: Fb(r, k) = e^{i 2 pi (m a + n b) / L} Fb(r0, k), r0
    // the origin.  Checked entry by entry; the column step uses it when it holds.
    if (nb == 1 && (nc == 16 || nc == 36)) {
      const int L = nc == 16 ? 4 : 6;
      int rmap[36], kmap[36], r0 = -1, ra[36], rb[36], km[36], kn[36];
      std::fill(rmap, rmap + 36, -1);
      std::fill(kmap, kmap + 36, -1);
      bool ok = true;
      for (int r = 0; r < nc && ok; ++r) {
        const double x = c.r_vecs[2 * r], y = c.r_vecs[2 * r + 1];
        const long a = std::lround(x), b = std::lround(y);
        ok = std::abs(x - a) < 1e-9 && std::abs(y - b) < 1e-9;
        ra[r] = int(((a % L) + L) % L);
        rb[r] = int(((b % L) + L) % L);
        const int g = ra[r] + L * rb[r];
        ok = ok && rmap[g] < 0;
        rmap[g] = r;
        if (a == 0 && b == 0)
          r0 = r;
      }
      for (int k = 0; k < nc && ok; ++k) {
        const double m = c.k_vecs[2 * k] * L / (2 * M_PI), n = c.k_vecs[2 * k + 1] * L / (2 * M_PI);
        const long mi = std::lround(m), ni = std::lround(n);
        ok = std::abs(m - mi) < 1e-9 && std::abs(n - ni) < 1e-9;
        km[k] = int(((mi % L) + L) % L);
        kn[k] = int(((ni % L) + L) % L);
        const int g = km[k] + L * kn[k];
        ok = ok && kmap[g] < 0;
        kmap[g] = k;
      }
      ok = ok && r0 >= 0;
      for (int k = 0; k < nc && ok; ++k)
        for (int r = 0; r < nc && ok; ++r) {
          const std::complex<double> f0(fb[size_t(k) * nc + r0].x, fb[size_t(k) * nc + r0].y);
          const std::complex<double> want =
              std::exp(std::complex<double>(0, 2 * M_PI * (km[k] * ra[r] + kn[k] * rb[r]) / double(L))) * f0;
          ok = std::abs(want - std::complex<double>(fb[size_t(k) * nc + r].x, fb[size_t(k) * nc + r].y)) < 1e-9;
        }
      if (ok) {
        fft.on = 1;
        fft.r0 = r0;
        fft.L = L;
        for (int g = 0; g < 36; ++g) {
          fft.rmap[g] = static_cast<unsigned char>(g < nc ? rmap[g] : 0);
          fft.kmap[g] = static_cast<unsigned char>(g < nc ? kmap[g] : 0);
        }
      }
    }
    // The cluster transform must map -k to the conjugate phases as well.
    if (mirror_ok)
      for (int k = 0; k < nc; ++k)
        for (int r = 0; r < nc; ++r) {
          const double2 a = fb[size_t(k) * nc + r], b = fb[size_t(kneg[k]) * nc + r];
          mirror_ok = mirror_ok && std::hypot(a.x - b.x, a.y + b.y) <= 1e-12;
        }
  }
  auto upload_ints = [](DevBuf<int>& d, const std::vector<int>& h) {
    d.alloc(h.size());
    DCAACC_CUDA_CHECK(cudaMemcpy(d.get(), h.data(), d.bytes(), cudaMemcpyHostToDevice));
  };
  upload_ints(k_add_d_, k_add_);
  upload_ints(k_sub_d_, k_sub_);
  upload_ints(q_d_, q_list_);
  upload_ints(wex_d_, wex_list_);

  // ---- G4 per channel ----
  g4s_ = std::make_shared<SharedG4>();
  g4s_->users.push_back(this);
  g4() = std::vector<DevBuf<double2>>(c.n_channels);
  for (auto& g : g4()) {
    g.alloc(g4_size_);
    DCAACC_CUDA_CHECK(cudaMemset(g.get(), 0, g.bytes()));
  }
  err_d_.alloc(1);
  DCAACC_CUDA_CHECK(cudaMemset(err_d_.get(), 0, sizeof(int)));
  G4_ptrs_.alloc(c.n_channels);
  uploadG4Ptrs();

  // ---- batch workspace ----
  const size_t n_sec = 2 * size_t(max_batch_);
  const size_t n_vtx = n_sec * max_order_;
  const size_t n_orb1 = dims_.n_orb + 1;
  for (auto& d : dstage_) {
    d.sectors.alloc(n_sec);
    d.tau.alloc(n_vtx);
    d.vb_r.alloc(n_vtx);
    d.vs_r.alloc(n_vtx);
    if (non_density_) {
      d.vb_c.alloc(n_vtx);
      d.vs_c.alloc(n_vtx);
    }
    d.perm_r.alloc(n_vtx);
    d.rstart.alloc(n_sec * n_orb1);
    if (non_density_) {
      d.perm_c.alloc(n_vtx);
      d.cstart.alloc(n_sec * n_orb1);
    }
    d.signs.alloc(max_batch_);
    d.M.alloc(n_sec * size_t(max_order_) * max_order_);
  }
  Tr_d_.alloc(n_vtx * nw_ext);
  if (non_density_)
    Tc_d_.alloc(n_vtx * nw_ext);
  // Launch-shape tuning (launch_tuner.hpp), unless DCAACC_TUNE=0 keeps the built-in shapes.
  const char* tune_env = std::getenv("DCAACC_TUNE");
  tuner_.setEnabled(!(tune_env && std::strcmp(tune_env, "0") == 0));
  const size_t x_elems = n_sec * size_t(R) * max_order_ * nw_ext;
  const size_t g_elems = n_sec * size_t(g_sector_stride_);
  if (mixed_) {
    // The mixed path runs its front-end and the disconnected terms of the one-band PH channels on
    // the tensor cores, unless DCAACC_TP_SIMT_ONLY=1 selects the all-SIMT kernels (kept to compare
    // both paths).
    const char* graphs_env = std::getenv("DCAACC_TP_GRAPHS");
    graphs_on_ = !(graphs_env && std::strcmp(graphs_env, "0") == 0);
    const char* simt_env = std::getenv("DCAACC_TP_SIMT_ONLY");
    const bool simt_only = simt_env && std::strcmp(simt_env, "1") == 0;
    G32_.alloc(g_elems);
    if (simt_only) {
      X32_.alloc(x_elems);
    }
    else {
      tc_front_ = true;
      const FrontTcShape fs = frontTcShape(dims_, int(n_sec), max_order_);
      ftc_mem_.alloc(frontTcBytes(fs));
      // Padding rows stay zero; ordered before the scale kernel frontTcInit launches on stream_.
      DCAACC_CUDA_CHECK(cudaMemsetAsync(ftc_mem_.get(), 0, ftc_mem_.bytes(), stream_));
      frontTcInit(ftc_, fs, ftc_mem_.get(), dims_, G0_.get(), stream_);
      // One band on a 4 x 4 cluster: the column step runs factored by orbital (12x fewer flops than
      // the dense GEMM) on tcgen05 with the per-site sums in tensor memory (tp_colfactor_tc.cu),
      // which also spares the dense step's Q operand.  DCAACC_TP_FACTORED_COL=0 keeps the dense
      // GEMM; =1 selects the other factored forms (mma.sync with the 4 x 4 FFT, or the CUDA cores
      // with the 16 x 16 matrix transform, which DCAACC_TP_COL_FFT=0 forces), both slower.  One
      // band on a 6 x 6 cluster: DCAACC_TP_FACTORED_COL=1 selects the factored form on the CUDA
      // cores with the 6 x 6 FFT (24x fewer flops than the dense GEMM, yet slower on B200: 57 ms
      // against 39 ms per batch of 128 at Nw = 128).
      const char* fact_env = std::getenv("DCAACC_TP_FACTORED_COL");
      const char* fft_env = std::getenv("DCAACC_TP_COL_FFT");
      ftc_.fft = fft;
      if (fft_env && std::strcmp(fft_env, "0") == 0)
        ftc_.fft.on = 0;
      const bool fact_off = fact_env && std::strcmp(fact_env, "0") == 0;
      const bool fact_on = fact_env && std::strcmp(fact_env, "1") == 0;
      const int row0 = dims_.half_g ? fs.D / 2 : 0;
      ftc_.col_tc = !fact_off && !fact_on && colFactorApplies(dims_) && ftc_.fft.on &&
                    colFactorTcApplies(dims_, fs.D, row0, max_order_);
      const bool wide = colFactorWideApplies(dims_) && ftc_.fft.on && ftc_.fft.L == 6 && fact_on;
      ftc_.factored_col = (colFactorApplies(dims_) && (fact_on || ftc_.col_tc)) || wide;
      if (ftc_.factored_col && ftc_.fft.on && !ftc_.col_tc && !wide) {
        col_tp_.alloc(colTwiddlePlaneBytes(dims_, int(n_sec), fs.Kr));
        ftc_.tp = col_tp_.get();
      }
      for (auto& d : dstage_) {
        d.orb_r.alloc(n_vtx);
        if (non_density_)
          d.orb_c.alloc(n_vtx);
      }
      gmax_d_.alloc(2 * size_t(max_batch_));
      if (discGemmApplies(dims_, max_batch_)) {
        disc_.alloc(discScratchBytes(dims_, max_batch_));
        discInit(disc_ws_, dims_, max_batch_, disc_.get(), disc_.bytes());
        have_disc_ = true;
      }
      // Half G (mirror symmetry) when the direct-term kernel reads mirrored G blocks: one band,
      // all momentum transfers, Nc = 16 (tensor-core direct term) or Nc = 36 (split FP32 direct
      // term), and half of D a whole number of 128-row tiles.  DCAACC_TP_FULL_G=1 computes the
      // whole of G instead (for comparisons).
      std::vector<int> seen(nc, 0);
      int distinct = 0;
      for (int q : q_list_)
        distinct += seen[q]++ == 0;
      const bool q_all = distinct == nc && int(q_list_.size()) == nc;
      const char* full_env = std::getenv("DCAACC_TP_FULL_G");
      const bool full_g = full_env && std::strcmp(full_env, "1") == 0;
      if (have_disc_ && mirror_ok && !full_g && nb == 1 && (nc == kMaxMirrorNc || nc == 36) && q_all &&
          c.n_channels <= 2 &&
          nw_ext % 2 == 0 && (long(R) * nw_ext / 2) % 128 == 0) {
        dims_.half_g = 1;
        for (int k = 0; k < nc; ++k)
          dims_.kneg[k] = static_cast<unsigned char>(kneg[k]);
        // Half G4 when the transfer lists are closed under negation.
        std::vector<int> qm(q_list_.size(), -1), wm(wex_list_.size(), -1);
        for (size_t i = 0; i < q_list_.size(); ++i)
          for (size_t j = 0; j < q_list_.size(); ++j)
            if (q_list_[j] == kneg[q_list_[i]])
              qm[i] = int(j);
        for (size_t i = 0; i < wex_list_.size(); ++i)
          for (size_t j = 0; j < wex_list_.size(); ++j)
            if (wex_list_[j] == -wex_list_[i])
              wm[i] = int(j);
        const bool closed = std::count(qm.begin(), qm.end(), -1) == 0 && std::count(wm.begin(), wm.end(), -1) == 0;
        if (closed && nw % 2 == 0 && (nc * nw / 2) % 128 == 0) {
          dims_.half_g4 = 1;
          upload_ints(q_mirror_d_, qm);
          upload_ints(wq_mirror_d_, wm);
          // Device window for reads of the running G4 (peek), whose lower half comes from the
          // mirror: allocated now, so that reads of up to kPeekWindow entries between batches
          // neither allocate nor synchronise.
          peek_d_.alloc(kPeekWindow);
          // Tiles (w1, w2) with w1 >= Nw / 2, each next to the tile that reads its B block as A:
          // (w2, w1) if w2 >= Nw / 2, else the mirror (Nw - 1 - w2, Nw - 1 - w1).
          std::vector<char> seen(size_t(nw) * nw, 0);
          std::vector<unsigned> order;
          auto push = [&](int a, int b) {
            if (!seen[size_t(a) * nw + b]) {
              seen[size_t(a) * nw + b] = 1;
              order.push_back(unsigned(a) | (unsigned(b) << 16));
            }
          };
          for (int a = nw / 2; a < nw; ++a)
            for (int b = 0; b < nw; ++b) {
              if (seen[size_t(a) * nw + b])
                continue;
              push(a, b);
              if (2 * b >= nw)
                push(b, a);
              else
                push(nw - 1 - b, nw - 1 - a);
            }
          tile_order_d_.alloc(order.size());
          DCAACC_CUDA_CHECK(cudaMemcpy(tile_order_d_.get(), order.data(), tile_order_d_.bytes(),
                                       cudaMemcpyHostToDevice));
        }
      }
    }
  }
  else {
    X64_.alloc(x_elems);
    G64_.alloc(g_elems);
  }
  for (auto& h : hstage_) {
    h.sectors.alloc(n_sec);
    h.tau.alloc(n_vtx);
    h.vb_r.alloc(n_vtx);
    h.vs_r.alloc(n_vtx);
    if (non_density_) {
      h.vb_c.alloc(n_vtx);
      h.vs_c.alloc(n_vtx);
    }
    h.signs.alloc(max_batch_);
    DCAACC_CUDA_CHECK(cudaEventRecord(h.uploaded, copy_stream_));
  }
  for (auto& d : dstage_)
    DCAACC_CUDA_CHECK(cudaEventRecord(d.consumed, stream_));

  if (!tc_front_ && frontendSmemRequirement(dims_, max_order_, !mixed_) > 227 * 1024)
    invalid("max_order too large for the front-end's shared-memory tiles");
  G4_host_.assign(c.n_channels, {});
}

TpAccumulator::~TpAccumulator() {
  if (g4s_) {
    std::lock_guard<std::mutex> lock(g4s_->m);
    auto& u = g4s_->users;
    u.erase(std::remove(u.begin(), u.end(), this), u.end());
  }
  releaseStreamsAndEvents();
}

void TpAccumulator::releaseStreamsAndEvents() {
  if (stream_)
    cudaStreamSynchronize(stream_);
  if (copy_stream_)
    cudaStreamSynchronize(copy_stream_);
  for (auto& t : timed_) {
    cudaEventDestroy(t.begin);
    cudaEventDestroy(t.end);
  }
  timed_.clear();
  releaseGraphs();
  for (auto& h : hstage_)
    if (h.uploaded) {
      cudaEventDestroy(h.uploaded);
      h.uploaded = nullptr;
    }
  for (auto& d : dstage_)
    if (d.consumed) {
      cudaEventDestroy(d.consumed);
      d.consumed = nullptr;
    }
  if (copy_stream_)
    cudaStreamDestroy(copy_stream_);
  copy_stream_ = nullptr;
  if (own_stream_ && stream_)
    cudaStreamDestroy(stream_);
  stream_ = nullptr;
}

// Error-path tests: see G4Args::wait_limit / fault_stop_step.  Launch arguments recorded in the
// CUDA graphs change, so the graphs are dropped.
void TpAccumulator::setFaultInjection(int stop_step, uint32_t wait_polls) {
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  releaseGraphs();
  fault_stop_step_ = stop_step;
  wait_limit_ = wait_polls;
}

void TpAccumulator::uploadG4Ptrs() {
  std::vector<double2*> ptrs;
  for (auto& g : g4())
    ptrs.push_back(g.get());
  DCAACC_CUDA_CHECK(cudaMemcpy(G4_ptrs_.get(), ptrs.data(), G4_ptrs_.bytes(), cudaMemcpyHostToDevice));
}

// This handle accumulates into owner's G4 from now on (its own is released when no handle uses it
// any more); both switch to atomic read-modify-writes, since their streams run concurrently.
// True when other accumulates the same G4 entries as this handle: same sizes, transfer lists,
// channels (in the same order) and beta.
bool TpAccumulator::sameG4(const TpAccumulator& o) const {
  if (o.g4_size_ != g4_size_ || o.g4().size() != g4().size() || o.dims_.nb != dims_.nb || o.dims_.nc != dims_.nc ||
      o.dims_.nw != dims_.nw || o.q_list_ != q_list_ || o.wex_list_ != wex_list_ || o.dims_.beta != dims_.beta)
    return false;
  for (int c = 0; c < dims_.n_channels; ++c)
    if (o.dims_.channels[c] != dims_.channels[c])
      return false;
  return true;
}

void TpAccumulator::shareG4(TpAccumulator& owner) {
  if (&owner == this || owner.g4s_ == g4s_)
    return;
  if (!sameG4(owner) || owner.dims_.half_g4 != dims_.half_g4)
    invalid("accumulators with different G4 shapes, transfers, channels, beta or mirror modes cannot share G4");
  if (owner.device_ != device_)
    invalid("sharing G4 requires both accumulators on the same device");
  process();
  owner.process();
  // What this handle has accumulated so far moves into the shared G4 (with its sign sum, which
  // stays with this handle), so no measurement is dropped with the released buffers.
  if (n_meas_ > 0) {
    // After every update already enqueued on the streams of the handles that use owner's G4.
    std::lock_guard<std::mutex> lock(owner.g4s_->m);
    for (TpAccumulator* u : owner.g4s_->users) {
      cudaEvent_t ev;
      DCAACC_CUDA_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      DCAACC_CUDA_CHECK(cudaEventRecord(ev, u->stream_));
      DCAACC_CUDA_CHECK(cudaStreamWaitEvent(stream_, ev, 0));
      DCAACC_CUDA_CHECK(cudaEventDestroy(ev));
    }
    for (size_t c = 0; c < g4().size(); ++c) {
      launchAddAndClear(owner.g4()[c].get(), g4()[c].get(), g4_size_, stream_);
      ++launches_;
    }
  }
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));  // this handle's kernels are done with its own G4
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(owner.stream_));
  {
    std::lock_guard<std::mutex> lock(g4s_->m);
    auto& u = g4s_->users;
    u.erase(std::remove(u.begin(), u.end(), this), u.end());
  }
  g4s_ = owner.g4s_;
  {
    std::lock_guard<std::mutex> lock(g4s_->m);
    g4s_->users.push_back(this);
  }
  uploadG4Ptrs();
  // The update mode is a kernel argument: graphs captured before are dropped on both sides.
  releaseGraphs();
  owner.releaseGraphs();
  atomic_ = true;
  owner.atomic_ = true;
}

void TpAccumulator::reset(long dca_loop) {
  // resetAccumulation: zero G4 and arm accumulate (tp_accumulator_gpu.hpp:285-296).
  for (auto& h : hstage_)
    DCAACC_CUDA_CHECK(cudaEventSynchronize(h.uploaded));
  slots_ = 0;
  vtx_used_ = 0;
  x_used_ = 0;
  m_used_ = 0;
  mcopy_bytes_ = 0;  // a copy of a discarded batch is not issued
  n_max_batch_ = 0;
  if (g4Shared()) {
    // Shared G4: zeroed once per DCA loop, by the first handle that resets for it
    // (callOncePerLoop in tp_accumulator_gpu.hpp:285-296); synchronously, so that no handle's
    // accumulation of this loop can run before the zeroing.
    std::lock_guard<std::mutex> lock(g4s_->m);
    if (dca_loop < 0 || dca_loop != g4s_->last_loop) {
      // Updates still in flight on the other sharing handles' streams (from the loop that ends
      // here) land before the zeroing; measurements they have queued but not yet launched count
      // toward the new loop.
      for (TpAccumulator* u : g4s_->users)
        if (u != this && u->stream_ != stream_) {
          cudaEvent_t ev;
          DCAACC_CUDA_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
          DCAACC_CUDA_CHECK(cudaEventRecord(ev, u->stream_));
          DCAACC_CUDA_CHECK(cudaStreamWaitEvent(stream_, ev, 0));
          DCAACC_CUDA_CHECK(cudaEventDestroy(ev));
        }
      for (auto& g : g4())
        DCAACC_CUDA_CHECK(cudaMemsetAsync(g.get(), 0, g.bytes(), stream_));
      DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));
      g4s_->last_loop = dca_loop;
    }
  }
  else {
    for (auto& g : g4())
      DCAACC_CUDA_CHECK(cudaMemsetAsync(g.get(), 0, g.bytes(), stream_));
  }
  sign_sum_ = 0;
  n_meas_ = 0;
  ready_ = true;
  finalized_ = false;
  have_g_ = false;
}

void TpAccumulator::validateSector(const dcaacc_sector& s) const {
  if (s.n < 0)
    invalid("negative expansion order");
  if (s.n > max_order_)
    invalid("expansion order " + std::to_string(s.n) + " exceeds max_order " +
            std::to_string(max_order_));
  if (s.n == 0)
    return;
  if (!s.tau || !s.left_band || !s.right_band || !s.left_site || !s.right_site || !s.M)
    invalid("null sector pointer");
  if (s.ldm < s.n)
    invalid("leading dimension of M smaller than n");
  for (int i = 0; i < s.n; ++i) {
    if (s.left_band[i] < 0 || s.left_band[i] >= dims_.nb || s.right_band[i] < 0 ||
        s.right_band[i] >= dims_.nb)
      invalid("vertex band out of range");
    if (s.left_site[i] < 0 || s.left_site[i] >= dims_.nc || s.right_site[i] < 0 ||
        s.right_site[i] >= dims_.nc)
      invalid("vertex site out of range");
    if (!std::isfinite(s.tau[i]))
      invalid("vertex time is not finite");
  }
}

double TpAccumulator::flopEstimate(const dcaacc_sector* sec) const {
  // Algorithmic flops of this implementation for one measurement: NDFT rows + columns,
  // both cluster transforms, the G0 epilogue, and the G4 update (18 / 26 flops per entry and
  // channel, the reference's convention in tp_accumulator_kernels.cu:704-723).
  const double nwe = dims_.nw_ext, R = dims_.R, D = R * nwe, nc = dims_.nc, nb = dims_.nb;
  double f = 0;
  for (int s = 0; s < 2; ++s) {
    const double n = sec[s].n;
    f += 8 * nwe * n * n / (nb * nc) * nb + 8 * D * n * nc;  // row NDFT per orbital + row transform
    f += 8 * D * nwe * n + 8 * D * D * nc;                    // column NDFT + column transform
    f += (nb == 1 ? 12 : 16 * nb) * D * D;                   // G0 epilogue
  }
  for (int c = 0; c < dims_.n_channels; ++c)
    f += (dims_.channels[c] == DCAACC_PH_MAGNETIC || dims_.channels[c] == DCAACC_PH_CHARGE ? 26.0 : 18.0) *
         double(g4_size_);
  return f;
}

void TpAccumulator::stage(const dcaacc_sector* sec, int sign, bool m_f32) {
  if (slots_ == 0) {
    DCAACC_CUDA_CHECK(cudaEventSynchronize(hs().uploaded));  // this staging set is free again
    // Copies into this device set wait for the kernels of the batch that last used it.
    DCAACC_CUDA_CHECK(cudaStreamWaitEvent(copy_stream_, dstage_[hset_].consumed, 0));
  }
  const int slot = slots_;
  const int n_orb = dims_.n_orb;
  for (int s = 0; s < 2; ++s) {
    const dcaacc_sector& x = sec[s];
    const int n = x.n;
    const int vtx_off = vtx_used_;
    const int sidx = 2 * slot + s;
    const int orb_off = sidx * (n_orb + 1);
    // The vertices as given; the device sorts them by orbital (tp_sort.cu): the row side by the
    // right band / site, the column side of non-density-density models by the left ones
    // (cached_ndft_base.hpp:97-103).
    std::copy_n(x.right_band, n, hs().vb_r.get() + vtx_off);
    std::copy_n(x.right_site, n, hs().vs_r.get() + vtx_off);
    if (non_density_) {
      std::copy_n(x.left_band, n, hs().vb_c.get() + vtx_off);
      std::copy_n(x.left_site, n, hs().vs_c.get() + vtx_off);
    }
    std::copy_n(x.tau, n, hs().tau.get() + vtx_off);

    const double* Mptr = x.M;
    int ldm = std::max(x.ldm, 1);
    const size_t esize = m_f32 ? sizeof(float) : sizeof(double);
    if (n && !x.m_on_device) {
      double* dst = dstage_[hset_].M.get() + m_used_;
      m_used_ += (esize * n * n + sizeof(double) - 1) / sizeof(double);
      const size_t bytes = esize * n * n;
      if (x.ldm == n) {
        if (mcopy_bytes_ && reinterpret_cast<const char*>(mcopy_src_) + mcopy_bytes_ == reinterpret_cast<const char*>(x.M) &&
            reinterpret_cast<char*>(mcopy_dst_) + mcopy_bytes_ == reinterpret_cast<char*>(dst)) {
          mcopy_bytes_ += bytes;  // contiguous on both sides: one larger copy
          if (mcopy_bytes_ >= (size_t(8) << 20))
            flushMCopy();  // in pieces of about 8 MB, overlapping the staging of the rest
        }
        else {
          flushMCopy();
          mcopy_src_ = x.M;
          mcopy_dst_ = dst;
          mcopy_bytes_ = bytes;
        }
      }
      else {
        flushMCopy();
        DCAACC_CUDA_CHECK(cudaMemcpy2DAsync(dst, esize * n, x.M, esize * x.ldm, esize * n, n, cudaMemcpyHostToDevice,
                                            copy_stream_));
      }
      Mptr = dst;
      ldm = n;
    }
    SectorDesc d{};
    d.M = Mptr;
    d.ldm = ldm;
    d.n = n;
    d.vtx_off = vtx_off;
    d.orb_off = orb_off;
    d.spin = s;
    d.slot = slot;
    d.m_f32 = m_f32 ? 1 : 0;
    d.x_off = x_used_;
    hs().sectors[sidx] = d;
    x_used_ += long(dims_.R) * n * dims_.nw_ext;
    vtx_used_ += n;
    n_max_batch_ = std::max(n_max_batch_, n);
  }
  hs().signs[slot] = sign;
  ++slots_;
}

void TpAccumulator::flushMCopy() {
  if (mcopy_bytes_)
    DCAACC_CUDA_CHECK(cudaMemcpyAsync(mcopy_dst_, mcopy_src_, mcopy_bytes_, cudaMemcpyHostToDevice, copy_stream_));
  mcopy_bytes_ = 0;
}

void TpAccumulator::process() {
  if (slots_ == 0)
    return;
  flushMCopy();
  const int n_sec = 2 * slots_;
  // Uploads on the copy stream (after the kernels that last read this device set, see stage());
  // the kernels below wait for them.
  DevStage& ds = dstage_[hset_];
  auto h2d = [&](void* dst, const void* src, size_t bytes) {
    if (bytes)
      DCAACC_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, copy_stream_));
  };
  h2d(ds.sectors.get(), hs().sectors.get(), sizeof(SectorDesc) * n_sec);
  h2d(ds.tau.get(), hs().tau.get(), sizeof(double) * vtx_used_);
  h2d(ds.vb_r.get(), hs().vb_r.get(), sizeof(int) * vtx_used_);
  h2d(ds.vs_r.get(), hs().vs_r.get(), sizeof(int) * vtx_used_);
  if (non_density_) {
    h2d(ds.vb_c.get(), hs().vb_c.get(), sizeof(int) * vtx_used_);
    h2d(ds.vs_c.get(), hs().vs_c.get(), sizeof(int) * vtx_used_);
  }
  h2d(ds.signs.get(), hs().signs.get(), sizeof(int) * slots_);
  DCAACC_CUDA_CHECK(cudaEventRecord(hs().uploaded, copy_stream_));
  DCAACC_CUDA_CHECK(cudaStreamWaitEvent(stream_, hs().uploaded, 0));
  const int set = hset_;
  hset_ ^= 1;

  FrontendArgs fa{};
  fa.dims = dims_;
  fa.sectors = ds.sectors.get();
  fa.n_sectors = n_sec;
  fa.n_max = n_max_batch_;
  fa.tau = ds.tau.get();
  fa.perm_r = ds.perm_r.get();
  fa.perm_c = non_density_ ? ds.perm_c.get() : ds.perm_r.get();
  fa.row_start = ds.rstart.get();
  fa.col_start = non_density_ ? ds.cstart.get() : ds.rstart.get();
  fa.Tr = Tr_d_.get();
  fa.Tc = non_density_ ? Tc_d_.get() : Tr_d_.get();
  fa.Fb = Fb_.get();
  fa.G0 = G0_.get();
  fa.tuner = &tuner_;
  // Tensor-core path: the launch shapes take the order bound in steps of 128 (the GEMM tile);
  // every kernel reads each sector's own order, so the results do not depend on it, and batches
  // of similar orders share one captured graph.
  if (tc_front_ && n_max_batch_ > 0)
    fa.n_max = (n_max_batch_ + 127) / 128 * 128;
  G4Args ga{};
  ga.dims = dims_;
  ga.signs = ds.signs.get();
  ga.n_slots = slots_;
  ga.k_add = k_add_d_.get();
  ga.k_sub = k_sub_d_.get();
  ga.q_list = q_d_.get();
  ga.wex_list = wex_d_.get();
  ga.G4 = G4_ptrs_.get();
  ga.atomic = atomic_;
  ga.err = err_d_.get();
  {
    std::vector<int> seen(dims_.nc, 0);
    int distinct = 0;
    for (int q : q_list_)
      distinct += seen[q]++ == 0;
    ga.q_all = distinct == dims_.nc && int(q_list_.size()) == dims_.nc;
  }
  ga.disc = have_disc_ ? &disc_ws_ : nullptr;
  ga.gmax = tc_front_ ? gmax_d_.get() : nullptr;
  ga.tile_order = dims_.half_g4 ? tile_order_d_.get() : nullptr;
  ga.n_sm = n_sm_;
  ga.tuner = &tuner_;
  ga.wait_limit = wait_limit_;
  ga.fault_stop_step = fault_stop_step_;

  const bool graphable = graphs_on_ && tc_front_ && !timing_ && n_max_batch_ > 0 && stream_ != nullptr &&
                         stream_ != cudaStreamLegacy && stream_ != cudaStreamPerThread;
  if (graphable)
    launches_ += launchBatchGraph(set, fa, ga, ds);
  else
    launches_ += launchBatch(fa, ga, ds);
  DCAACC_CUDA_CHECK(cudaEventRecord(ds.consumed, stream_));
  have_g_ = !mixed_;
  slots_ = 0;
  vtx_used_ = 0;
  x_used_ = 0;
  m_used_ = 0;
  n_max_batch_ = 0;
}

// The kernels of one batch, all on stream_ and nothing else (the sequence a graph captures).
int TpAccumulator::launchBatch(const FrontendArgs& fa, const G4Args& ga, DevStage& ds) {
  int launched = 0;
  cudaEvent_t b = nullptr;
  if (fa.n_max > 0) {
    timeBegin(DCAACC_STAGE_TWIDDLE, &b);
    // Vertex order and orbital runs of every sector (sortConfiguration), row side and, for
    // non-density-density models, column side.
    launchSortVertices(fa.sectors, fa.n_sectors, ds.vb_r.get(), ds.vs_r.get(), dims_.nb, dims_.n_orb,
                       ds.perm_r.get(), ds.rstart.get(), ds.orb_r.get(), stream_);
    launched += 1;
    if (non_density_) {
      launchSortVertices(fa.sectors, fa.n_sectors, ds.vb_c.get(), ds.vs_c.get(), dims_.nb, dims_.n_orb,
                         ds.perm_c.get(), ds.cstart.get(), ds.orb_c.get(), stream_);
      launched += 1;
    }
    int n_prep;
    if (tc_front_) {
      n_prep = launchFrontendTcPrep(fa, ftc_, ds.orb_r.get(), non_density_ ? ds.orb_c.get() : ds.orb_r.get(),
                                    stream_);
    }
    else {
      launchTwiddles(fa, stream_);
      n_prep = non_density_ ? 2 : 1;
    }
    launched += n_prep;
    timeEnd(DCAACC_STAGE_TWIDDLE, b, n_prep + (non_density_ ? 2 : 1));
  }
  timeBegin(DCAACC_STAGE_ROW, &b);
  if (tc_front_)
    launchFrontendTcRow(fa, ftc_, err_d_.get(), stream_);
  else if (mixed_)
    launchRowTransform<float>(fa, X32_.get(), stream_);
  else
    launchRowTransform<double>(fa, X64_.get(), stream_);
  timeEnd(DCAACC_STAGE_ROW, b, 1);
  timeBegin(DCAACC_STAGE_COL, &b);
  int col_launches = 1;
  if (tc_front_)
    col_launches = launchFrontendTcCol(fa, ftc_, G32_.get(), g_sector_stride_, gmax_d_.get(), err_d_.get(), stream_);
  else if (mixed_)
    launchColTransform<float>(fa, X32_.get(), G32_.get(), g_sector_stride_, stream_);
  else
    launchColTransform<double>(fa, X64_.get(), G64_.get(), g_sector_stride_, stream_);
  timeEnd(DCAACC_STAGE_COL, b, col_launches);
  timeBegin(DCAACC_STAGE_G4, &b);
  const int g4_launches = mixed_ ? launchUpdateG4<float2>(ga, G32_.get(), g_sector_stride_, stream_)
                                 : launchUpdateG4<double2>(ga, G64_.get(), g_sector_stride_, stream_);
  timeEnd(DCAACC_STAGE_G4, b, g4_launches);
  return launched + 1 + col_launches + g4_launches;
}

// Replays the batch's kernel sequence from a CUDA graph keyed by (device input set, batch size,
// order bound): the launch shapes and every pointer the kernels receive depend on nothing else
// (per-batch data reaches them through the device input set).  A key's batches run eagerly until
// one has run without launch-shape probes (so lazy setup such as shared-memory attributes happens
// outside any capture, and the tuned shapes are final); the next is captured and instantiated,
// later ones replay.  At most kMaxGraphs executables are kept.
int TpAccumulator::launchBatchGraph(int set, const FrontendArgs& fa, const G4Args& ga, DevStage& ds) {
  constexpr size_t kMaxGraphs = 32;
  BatchGraph* g = nullptr;
  for (auto& x : graphs_)
    if (x.set == set && x.slots == ga.n_slots && x.n_max == fa.n_max)
      g = &x;
  if (!g) {
    if (graphs_.size() >= kMaxGraphs) {
      auto lru = std::min_element(graphs_.begin(), graphs_.end(),
                                  [](const BatchGraph& a, const BatchGraph& b) { return a.last < b.last; });
      if (lru->exec) {
        DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));  // no launch of it may be pending
        cudaGraphExecDestroy(lru->exec);
      }
      graphs_.erase(lru);
    }
    graphs_.push_back(BatchGraph{set, ga.n_slots, fa.n_max, false, nullptr, 0, 0});
    g = &graphs_.back();
  }
  g->last = ++graph_stamp_;
  if (!g->clean) {
    const uint64_t p0 = tuner_.probes();
    const int n = launchBatch(fa, ga, ds);
    g->clean = tuner_.probes() == p0;
    return n;
  }
  if (!g->exec) {
    DCAACC_CUDA_CHECK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed));
    int n = 0;
    cudaGraph_t graph = nullptr;
    try {
      n = launchBatch(fa, ga, ds);
    }
    catch (...) {
      if (cudaStreamEndCapture(stream_, &graph) == cudaSuccess && graph)
        cudaGraphDestroy(graph);
      cudaGetLastError();
      throw;
    }
    DCAACC_CUDA_CHECK(cudaStreamEndCapture(stream_, &graph));
    const cudaError_t e = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      g->exec = nullptr;
      DCAACC_CUDA_CHECK(e);
    }
    g->launches = n;
    ++graph_captures_;
  }
  DCAACC_CUDA_CHECK(cudaGraphLaunch(g->exec, stream_));
  ++graph_replays_;
  return g->launches;
}

void TpAccumulator::releaseGraphs() {
  for (auto& g : graphs_)
    if (g.exec)
      cudaGraphExecDestroy(g.exec);
  graphs_.clear();
}

void TpAccumulator::setGraphs(bool on) {
  if (!on) {
    DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));  // no launch of them may be pending
    releaseGraphs();
  }
  graphs_on_ = on;
}

void TpAccumulator::graphStats(uint64_t* captures, uint64_t* replays) const {
  if (captures)
    *captures = graph_captures_;
  if (replays)
    *replays = graph_replays_;
}

double TpAccumulator::accumulate(const dcaacc_sector* sectors, int sign, bool m_f32) {
  if (!ready_)
    throw Error(DCAACC_NOT_READY, "The accumulator is not ready to measure.");
  if (!sectors)
    invalid("null sectors");
  if (sign != 1 && sign != -1)
    invalid("sign must be +1 or -1");
  validateSector(sectors[0]);
  validateSector(sectors[1]);
  sign_sum_ += sign;  // the solver's accumulated sign counts every measurement
  ++n_meas_;
  if (sectors[0].n + sectors[1].n == 0)  // empty configuration (tp_accumulator_cpu.hpp:238-239)
    return 0.;
  if (slots_ == max_batch_)
    process();
  stage(sectors, sign, m_f32);
  if (slots_ == max_batch_)
    process();
  return flopEstimate(sectors);
}

void TpAccumulator::flush() {
  process();
}

void TpAccumulator::finalize() {
  if (finalized_)
    return;
  process();
  for (size_t c = 0; c < g4().size(); ++c) {
    if (dims_.half_g4)  // the entries with w1 < Nw / 2 from their mirrors
      launchG4Mirror(g4()[c].get(), dims_, q_mirror_d_.get(), wq_mirror_d_.get(), stream_);
    G4_host_[c].resize(g4_size_);
    DCAACC_CUDA_CHECK(cudaMemcpyAsync(G4_host_[c].data(), g4()[c].get(), g4()[c].bytes(),
                                      cudaMemcpyDeviceToHost, stream_));
  }
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  checkDeviceError();
  finalized_ = true;
  ready_ = false;
}

void TpAccumulator::checkDeviceError() {
  int e = 0;
  DCAACC_CUDA_CHECK(cudaMemcpy(&e, err_d_.get(), sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    DCAACC_CUDA_CHECK(cudaMemset(err_d_.get(), 0, sizeof(int)));
    throw Error(DCAACC_DEVICE_INDEX_ERR, e & 1 ? "a device-side wait timed out; G4 is incomplete"
                                               : "a device-side index check failed; G4 is incomplete");
  }
}

void TpAccumulator::getG4(int channel, double* out, size_t count) const {
  if (!finalized_)
    throw Error(DCAACC_NOT_READY, "G4 is available after finalize().");
  if (channel < 0 || channel >= static_cast<int>(G4_host_.size()))
    invalid("channel index out of range");
  if (count != g4_size_)
    invalid("output size does not match the G4 size");
  std::memcpy(out, G4_host_[channel].data(), 16 * count);
}

void TpAccumulator::sumTo(TpAccumulator& other) {
  if (other.g4().size() != g4().size())
    invalid("Objects accumulate different number of channels.");
  if (!sameG4(other))
    invalid("sumTo between accumulators of different G4 shapes, transfers, channels or beta");
  if (other.device_ != device_)
    invalid("sumTo requires both accumulators on the same device");
  process();
  other.process();
  if (other.g4s_ == g4s_) {  // one shared G4: nothing to add (tp_accumulator_gpu.hpp:487-491)
    // but what other reads of it afterwards (finalize, peek) comes after this handle's updates.
    cudaEvent_t done;
    DCAACC_CUDA_CHECK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    DCAACC_CUDA_CHECK(cudaEventRecord(done, stream_));
    DCAACC_CUDA_CHECK(cudaStreamWaitEvent(other.stream_, done, 0));
    DCAACC_CUDA_CHECK(cudaEventDestroy(done));
    other.sign_sum_ += sign_sum_;
    other.n_meas_ += n_meas_;
    sign_sum_ = 0;
    n_meas_ = 0;
    other.finalized_ = false;
    return;
  }
  cudaEvent_t ev;
  DCAACC_CUDA_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  DCAACC_CUDA_CHECK(cudaEventRecord(ev, other.stream_));
  DCAACC_CUDA_CHECK(cudaStreamWaitEvent(stream_, ev, 0));
  for (size_t c = 0; c < g4().size(); ++c) {
    // A half-G4 source holds only the tiles with w1 >= Nw / 2; a full-G4 target needs the rest
    // too, so the source's lower half is filled from its mirror first.  (A full source adding into
    // a half target is complete already: the target refills its lower half from its upper half.)
    if (dims_.half_g4 && !other.dims_.half_g4) {
      launchG4Mirror(g4()[c].get(), dims_, q_mirror_d_.get(), wq_mirror_d_.get(), stream_);
      ++launches_;
    }
    launchAddAndClear(other.g4()[c].get(), g4()[c].get(), g4_size_, stream_);
    ++launches_;
  }
  DCAACC_CUDA_CHECK(cudaEventRecord(ev, stream_));
  DCAACC_CUDA_CHECK(cudaStreamWaitEvent(other.stream_, ev, 0));
  DCAACC_CUDA_CHECK(cudaEventDestroy(ev));
  other.finalized_ = false;
  other.sign_sum_ += sign_sum_;
  other.n_meas_ += n_meas_;
  sign_sum_ = 0;
  n_meas_ = 0;
}

// The solver's normalisation of the accumulated G4 (ctaux_cluster_solver.hpp:521-525):
// G4 / (accumulated sign * beta^2).
void TpAccumulator::getG4Normalized(int channel, double* out, size_t count) const {
  if (sign_sum_ == 0)
    throw Error(DCAACC_NOT_READY, "the accumulated sign is zero");
  getG4(channel, out, count);
  const double f = 1.0 / (sign_sum_ * dims_.beta * dims_.beta);
  for (size_t i = 0; i < 2 * count; ++i)
    out[i] *= f;
}

void TpAccumulator::signSum(double* sum, uint64_t* count) const {
  if (sum)
    *sum = sign_sum_;
  if (count)
    *count = n_meas_;
}

void TpAccumulator::getG(int spin, double* out, size_t count) const {
  if (mixed_)
    throw Error(DCAACC_UNSUPPORTED, "G is kept for inspection in FP64 mode only");
  if (!have_g_)
    throw Error(DCAACC_NOT_READY, "no measurement has been processed");
  if (spin < 0 || spin > 1)
    invalid("spin must be 0 or 1");
  const int nb = dims_.nb, nc = dims_.nc, nwe = dims_.nw_ext, R = dims_.R;
  const size_t total = size_t(g_sector_stride_);
  if (count != total)
    invalid("output size does not match the G size");
  std::vector<double2> blk(total);
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  DCAACC_CUDA_CHECK(cudaMemcpy(blk.data(), G64_.get() + size_t(spin) * g_sector_stride_,
                               sizeof(double2) * total, cudaMemcpyDeviceToHost));
  // Block layout ((wr nwe + wc) R + r) R + c  ->  (b1, b2, k1, k2, w1, w2).
  for (int wc = 0; wc < nwe; ++wc)
    for (int wr = 0; wr < nwe; ++wr)
      for (int r = 0; r < R; ++r)
        for (int cc = 0; cc < R; ++cc) {
          const int b1 = r % nb, k1 = r / nb, b2 = cc % nb, k2 = cc / nb;
          const size_t o = b1 + nb * (b2 + nb * (k1 + nc * (k2 + size_t(nc) * (wr + size_t(nwe) * wc))));
          const double2 v = blk[((size_t(wr) * nwe + wc) * R + r) * R + cc];
          out[2 * o] = v.x;
          out[2 * o + 1] = v.y;
        }
}

void TpAccumulator::timeBegin(int, cudaEvent_t* b) {
  *b = nullptr;
  if (!timing_)
    return;
  DCAACC_CUDA_CHECK(cudaEventCreate(b));
  DCAACC_CUDA_CHECK(cudaEventRecord(*b, stream_));
}

void TpAccumulator::timeEnd(int stage, cudaEvent_t b, int launches) {
  if (!timing_ || !b)
    return;
  cudaEvent_t e;
  DCAACC_CUDA_CHECK(cudaEventCreate(&e));
  DCAACC_CUDA_CHECK(cudaEventRecord(e, stream_));
  timed_.push_back(Timed{stage, b, e});
  stage_launches_[stage] += launches;
}

void TpAccumulator::collectTimes() {
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  for (auto& t : timed_) {
    float ms = 0;
    DCAACC_CUDA_CHECK(cudaEventElapsedTime(&ms, t.begin, t.end));
    stage_ms_[t.stage] += ms;
    cudaEventDestroy(t.begin);
    cudaEventDestroy(t.end);
  }
  timed_.clear();
}

void TpAccumulator::enableTiming(bool on) {
  collectTimes();
  timing_ = on;
  for (int i = 0; i < DCAACC_N_STAGES; ++i) {
    stage_ms_[i] = 0;
    stage_launches_[i] = 0;
  }
}

void TpAccumulator::stageTimes(double* ms, uint64_t* launches, int n) {
  if (n < 0 || n > DCAACC_N_STAGES)
    invalid("n_stages out of range");
  collectTimes();
  for (int i = 0; i < n; ++i) {
    if (ms)
      ms[i] = stage_ms_[i];
    if (launches)
      launches[i] = stage_launches_[i];
  }
}

void TpAccumulator::peekG4(int channel, size_t offset, size_t count, double* out, bool wait) {
  if (channel < 0 || channel >= static_cast<int>(g4().size()))
    invalid("channel index out of range");
  if (offset > g4_size_ || count > g4_size_ - offset)
    invalid("window outside G4");
  process();
  const double2* src = g4()[channel].get() + offset;
  if (dims_.half_g4) {  // entries with w1 < Nw / 2 come from their mirrors
    if (peek_d_.size() < count) {
      DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));  // earlier reads may still use the window
      peek_d_.alloc(count);
    }
    launchG4Window(g4()[channel].get(), dims_, q_mirror_d_.get(), wq_mirror_d_.get(), offset, count, peek_d_.get(),
                   stream_);
    src = peek_d_.get();
  }
  DCAACC_CUDA_CHECK(cudaMemcpyAsync(out, src, 16 * count, cudaMemcpyDeviceToHost, stream_));
  if (wait)
    DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));
}

void TpAccumulator::setStream(cudaStream_t s) {
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  if (own_stream_)
    DCAACC_CUDA_CHECK(cudaStreamDestroy(stream_));
  own_stream_ = false;
  stream_ = s;
}

void TpAccumulator::synchronize() {
  flushMCopy();
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(copy_stream_));  // host M copies of a pending batch
  DCAACC_CUDA_CHECK(cudaStreamSynchronize(stream_));
  checkDeviceError();
}

size_t TpAccumulator::deviceFingerprint() const {
  size_t b = G0_.bytes() + Fb_.bytes() + k_add_d_.bytes() + k_sub_d_.bytes() + q_d_.bytes() +
             wex_d_.bytes() + G4_ptrs_.bytes() + Tr_d_.bytes() + Tc_d_.bytes() + X64_.bytes() +
             G64_.bytes() + X32_.bytes() + G32_.bytes() + err_d_.bytes();
  for (const auto& g : g4())  // a shared G4 is counted by every handle that shares it
    b += g.bytes();
  for (const auto& d : dstage_)
    b += d.vb_r.bytes() + d.vs_r.bytes() + d.vb_c.bytes() + d.vs_c.bytes() +
         d.sectors.bytes() + d.tau.bytes() + d.M.bytes() + d.perm_r.bytes() + d.perm_c.bytes() +
         d.rstart.bytes() + d.cstart.bytes() + d.signs.bytes() + d.orb_r.bytes() + d.orb_c.bytes();
  return b;
}

}  // namespace dcaacc
