// CPU restatement of the reference's FP64 accumulators — the ORACLE for parity tests.
//
// Test infrastructure only.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
// reference arm load this library, and only as the checker or the timed CPU baseline; the
// product (dca_b200, libdcaacc.so) never calls it.
//
// It restates, in plain loops, the algorithm of:
//   TpAccumulator<Parameters, DistType::NONE, linalg::CPU>
//     accumulate / computeM / computeG   tp_accumulator_cpu.hpp:233-375
//     band transpose in getGMultiband    tp_accumulator_cpu.hpp:389-405
//     updateG4 (all four channels)       tp_accumulator_cpu.hpp:409-757, :761-869
//     G0 slice and extension offset      tp_accumulator_base.hpp:184-221
//   CachedNdft<CPU>                      cached_ndft_base.hpp:89-129, cached_ndft_cpu.hpp:106-252
//   SpaceTransform2D                     space_transform_2D.hpp:60-140
//   exchange domains                     frequency_exchange_domain.cpp:26-48,
//                                        momentum_exchange_domain.cpp:26-50,
//                                        vertex_frequency_domain.hpp:103-185
//   SpAccumulator<CPU>                   sp_accumulator.hpp:161-237
//   Dnfft1D (CUBIC)                      dnfft_1d.hpp:161-489, nfft_time_domain.hpp:112-176,
//                                        kaiser_bessel_function.cpp:28-116
// The FFT of Dnfft1D::transformFTauToFW is evaluated as a direct DFT at the Matsubara indices
// only (the same numbers FFTW returns there).
//
// The C entry points take the same configuration structs as the product's C ABI (include/dcaacc.h).
// Parity is pinned against the reference's own CPU accumulators built by oracle/refbuild.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/dcaacc.h"
#include "casefile.hpp"

namespace oracle {

using cd = std::complex<double>;

static thread_local std::string g_error;

// Runs body(i) for i in [0, n) on a few host threads (ORACLE_THREADS, else the hardware's count).
// Callers split only loops whose iterations write disjoint outputs, so every output is the same
// sum in the same order as in a single-threaded run.
template <class F>
void parallelFor(int n, F&& body) {
  int threads = static_cast<int>(std::thread::hardware_concurrency());
  if (const char* e = std::getenv("ORACLE_THREADS"))
    threads = std::atoi(e);
  threads = std::max(1, std::min(threads, n));
  if (threads == 1) {
    for (int i = 0; i < n; ++i)
      body(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&] {
      for (int i = next++; i < n; i = next++)
        body(i);
    });
  for (auto& th : pool)
    th.join();
}

// ------------------------------------------------------------------------------------------------
// Two-particle accumulator
// ------------------------------------------------------------------------------------------------
class Tp {
public:
  Tp(const dcaacc_tp_config& c, const double* G0in) {
    nb = c.n_bands;
    nc = c.n_sites;
    nw = 2 * c.n_w_half;
    n_sp = c.n_sp_freq;
    beta = c.beta;
    non_density = c.non_density != 0;
    k_ex.assign(c.k_ex, c.k_ex + c.n_k_ex);
    w_ex.assign(c.w_ex, c.w_ex + c.n_w_ex);
    channels.assign(c.channels, c.channels + c.n_channels);
    k_add.assign(c.k_add, c.k_add + nc * nc);
    k_sub.assign(c.k_sub, c.k_sub + nc * nc);
    r_vecs.assign(c.r_vecs, c.r_vecs + 2 * nc);
    k_vecs.assign(c.k_vecs, c.k_vecs + 2 * nc);
    a_vecs.assign(c.a_vecs, c.a_vecs + 2 * nb);

    // Extended mesh: NwExt = 2 (Nw/2 + ext), ext = max |w_ex| (frequency_exchange_domain.cpp:42-45,
    // vertex_frequency_domain.hpp EXTENDED).
    ext = 0;
    for (int w : w_ex)
      ext = std::max(ext, std::abs(w));
    nw_ext = nw + 2 * ext;
    if (2 * n_sp < nw_ext)
      throw std::logic_error("The number of single particle frequencies is too small.");
    w_ext.resize(nw_ext);
    for (int l = 0; l < nw_ext / 2; ++l) {
      w_ext[nw_ext / 2 + l] = M_PI / beta * (1 + 2 * l);
      w_ext[nw_ext / 2 - 1 - l] = -M_PI / beta * (1 + 2 * l);
    }

    // G0_(b1, b2, s, k, w) = G0(b1, s, b2, s, k, w + sp_offset)  (tp_accumulator_base.hpp:210-221).
    const int sp_offset = (2 * n_sp - nw_ext) / 2;
    G0.resize(std::size_t(nb) * nb * 2 * nc * nw_ext);
    for (int w = 0; w < nw_ext; ++w)
      for (int k = 0; k < nc; ++k)
        for (int s = 0; s < 2; ++s)
          for (int b2 = 0; b2 < nb; ++b2)
            for (int b1 = 0; b1 < nb; ++b1) {
              const std::size_t in =
                  b1 + nb * (s + 2 * (b2 + nb * (s + 2 * (k + std::size_t(nc) * (w + sp_offset)))));
              G0[g0idx(b1, b2, s, k, w)] = cd(G0in[2 * in], G0in[2 * in + 1]);
            }

    // Space-transform matrix T(k, r) = exp(i k.r) and phase factors exp(i k.a_b)
    // (space_transform_2D.hpp:93-140).
    Tkr.resize(nc * nc);
    for (int r = 0; r < nc; ++r)
      for (int k = 0; k < nc; ++k)
        Tkr[k + nc * r] = std::exp(cd(0, k_vecs[2 * k] * r_vecs[2 * r] + k_vecs[2 * k + 1] * r_vecs[2 * r + 1]));
    phase.resize(nb * nc);
    for (int k = 0; k < nc; ++k)
      for (int b = 0; b < nb; ++b)
        phase[b + nb * k] =
            std::exp(cd(0, k_vecs[2 * k] * a_vecs[2 * b] + k_vecs[2 * k + 1] * a_vecs[2 * b + 1]));

    g_size = std::size_t(nb) * nb * nc * nc * nw_ext * nw_ext;
    for (int s = 0; s < 2; ++s)
      G[s].assign(g_size, cd(0));
    g4_size = std::size_t(nb) * nb * nb * nb * nc * nc * nw * nw * k_ex.size() * w_ex.size();
    G4.assign(channels.size(), std::vector<cd>(g4_size, cd(0)));
  }

  void reset() {
    for (auto& g : G4)
      std::fill(g.begin(), g.end(), cd(0));
  }

  // accumulate (tp_accumulator_cpu.hpp:233-252).
  void accumulate(const dcaacc_sector* sec, int sign) {
    if (sec[0].n + sec[1].n == 0)  // empty configuration: nothing to add
      return;
    for (int s = 0; s < 2; ++s) {
      std::fill(G[s].begin(), G[s].end(), cd(0));
      if (sec[s].n)
        ndft(sec[s], G[s]);  // M_r_r_w_w, in place in G[s] with the (r1,r2,b1,b2,w1,w2) layout
      spaceTransform(G[s]);
      computeG(s);
    }
    for (std::size_t c = 0; c < channels.size(); ++c)
      updateG4(c, sign);
  }

  int nb, nc, nw, n_sp, nw_ext, ext;
  double beta;
  bool non_density;
  std::vector<int> k_ex, w_ex, channels, k_add, k_sub;
  std::vector<double> r_vecs, k_vecs, a_vecs, w_ext;
  std::vector<cd> G0, Tkr, phase;
  std::vector<cd> G[2];
  std::size_t g_size, g4_size;
  std::vector<std::vector<cd>> G4;

private:
  std::size_t g0idx(int b1, int b2, int s, int k, int w) const {
    return b1 + nb * (b2 + nb * (s + 2 * (k + std::size_t(nc) * w)));
  }
  // G_(b1, b2, k1, k2, w1, w2) of one spin (SpGreensFunction without the spin index).
  std::size_t gidx(int b1, int b2, int k1, int k2, int w1, int w2) const {
    return b1 + nb * (b2 + nb * (k1 + nc * (k2 + std::size_t(nc) * (w1 + std::size_t(nw_ext) * w2))));
  }
  // M_r_r_w_w(r1, r2, b1, b2, w1, w2) of one spin (cached_ndft_cpu.hpp:240-252).
  std::size_t midx(int r1, int r2, int b1, int b2, int w1, int w2) const {
    return r1 + nc * (r2 + nc * (b1 + nb * (b2 + nb * (w1 + std::size_t(nw_ext) * w2))));
  }

  // CachedNdft<CPU>::execute (cached_ndft_cpu.hpp:106-140): for each pair of orbitals,
  // M(w1, w2) = sum_{t1, t2} exp(i (w1 t1 - w2 t2)) M(t1, t2).
  void ndft(const dcaacc_sector& sec, std::vector<cd>& out) {
    const int n = sec.n;
    const int n_orb = nb * nc;
    struct Triple {
      int orbital, idx;
    };
    auto sorted = [&](bool left_side) {
      // Side 0 uses the right band/site, side 1 the left one (cached_ndft_base.hpp:97-103).
      std::vector<Triple> v(n);
      for (int l = 0; l < n; ++l) {
        const int orb = left_side ? sec.left_band[l] + nb * sec.left_site[l]
                                  : sec.right_band[l] + nb * sec.right_site[l];
        v[l] = {orb, l};
      }
      std::sort(v.begin(), v.end(), [](const Triple& a, const Triple& b) {
        return a.orbital == b.orbital ? a.idx < b.idx : a.orbital < b.orbital;
      });
      std::vector<int> start(n_orb + 1, 0);
      for (const auto& t : v)
        start[t.orbital + 1]++;
      std::partial_sum(start.begin(), start.end(), start.begin());
      return std::make_pair(v, start);
    };
    const auto rows = sorted(false);
    const auto cols = non_density ? sorted(true) : rows;

    // T(w, v) = exp(i tau_v w)  (cached_ndft_cpu.hpp:142-158).
    std::vector<cd> T(std::size_t(nw_ext) * n);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < nw_ext; ++i) {
        const double x = sec.tau[j] * w_ext[i];
        T[i + std::size_t(nw_ext) * j] = cd(std::cos(x), std::sin(x));
      }
    auto Mval = [&](int i, int j) { return sec.M[i + std::size_t(sec.ldm) * j]; };

    // Threads split the output blocks (orbital pairs); every entry keeps its own summation order.
    parallelFor(n_orb * n_orb, [&](int pair) {
      const int oj = pair / n_orb, oi = pair % n_orb;
      {
        const int j0 = cols.second[oj], j1 = cols.second[oj + 1];
        std::vector<cd> X;
        const int i0 = rows.second[oi], i1 = rows.second[oi + 1];
        if (i1 == i0 || j1 == j0)
          return;  // setToZero: out is already zero
        // X = T_l * M_ij   (NwExt x n_j)
        X.assign(std::size_t(nw_ext) * (j1 - j0), cd(0));
        for (int jj = j0; jj < j1; ++jj)
          for (int ii = i0; ii < i1; ++ii) {
            const double m = Mval(rows.first[ii].idx, cols.first[jj].idx);
            const cd* t = &T[std::size_t(nw_ext) * rows.first[ii].idx];
            cd* x = &X[std::size_t(nw_ext) * (jj - j0)];
            for (int w = 0; w < nw_ext; ++w)
              x[w] += t[w] * m;
          }
        // Y = X * T_r^H   (NwExt x NwExt)
        const int b1 = oi % nb, r1 = oi / nb, b2 = oj % nb, r2 = oj / nb;
        for (int w2 = 0; w2 < nw_ext; ++w2)
          for (int w1 = 0; w1 < nw_ext; ++w1) {
            cd acc(0);
            for (int jj = j0; jj < j1; ++jj)
              acc += X[w1 + std::size_t(nw_ext) * (jj - j0)] *
                     std::conj(T[w2 + std::size_t(nw_ext) * cols.first[jj].idx]);
            out[midx(r1, r2, b1, b2, w1, w2)] = acc;
          }
      }
    });
  }

  // SpaceTransform2D::execute (space_transform_2D.hpp:60-91): in place, from the
  // (r1,r2,b1,b2,w1,w2) layout to (b1,b2,k1,k2,w1,w2).
  void spaceTransform(std::vector<cd>& f) {
    std::vector<cd> out(g_size);
    const double norm = 1.0 / nc;
    parallelFor(nw_ext * nw_ext, [&](int ww) {
      const int w2 = ww / nw_ext, w1 = ww % nw_ext;
      {
        std::vector<cd> tmp(nc * nc), frr(nc * nc);
        for (int b2 = 0; b2 < nb; ++b2)
          for (int b1 = 0; b1 < nb; ++b1) {
            for (int r2 = 0; r2 < nc; ++r2)
              for (int r1 = 0; r1 < nc; ++r1)
                frr[r1 + nc * r2] = f[midx(r1, r2, b1, b2, w1, w2)];
            // tmp = T * f
            for (int r2 = 0; r2 < nc; ++r2)
              for (int k1 = 0; k1 < nc; ++k1) {
                cd acc(0);
                for (int r1 = 0; r1 < nc; ++r1)
                  acc += Tkr[k1 + nc * r1] * frr[r1 + nc * r2];
                tmp[k1 + nc * r2] = acc;
              }
            // f(k1, k2) = norm * tmp * T^H, then the band phase factors.
            for (int k2 = 0; k2 < nc; ++k2)
              for (int k1 = 0; k1 < nc; ++k1) {
                cd acc(0);
                for (int r2 = 0; r2 < nc; ++r2)
                  acc += tmp[k1 + nc * r2] * std::conj(Tkr[k2 + nc * r2]);
                out[gidx(b1, b2, k1, k2, w1, w2)] =
                    norm * acc * phase[b1 + nb * k1] * std::conj(phase[b2 + nb * k2]);
              }
          }
      }
    });
    f.swap(out);
  }

  // computeGSingleband / computeGMultiband (tp_accumulator_cpu.hpp:289-375):
  // G <- -G0(k1,w1) G G0(k2,w2) + beta G0(k1,w1) delta_{k1 k2} delta_{w1 w2}.
  void computeG(int s) {
    auto& g = G[s];
    parallelFor(nw_ext, [&](int w2) {
      for (int w1 = 0; w1 < nw_ext; ++w1)
        for (int k2 = 0; k2 < nc; ++k2)
          for (int k1 = 0; k1 < nc; ++k1) {
            cd blk[64], g0m[64];
            const cd* g01 = &G0[g0idx(0, 0, s, k1, w1)];
            const cd* g02 = &G0[g0idx(0, 0, s, k2, w2)];
            cd* m = &g[gidx(0, 0, k1, k2, w1, w2)];
            if (nb == 1) {
              const cd mv = m[0];
              m[0] = -g01[0] * mv * g02[0];
              if (k1 == k2 && w1 == w2)
                m[0] += g01[0] * beta;
              continue;
            }
            // G0_M = G0_w1 * M ; M = -G0_M * G0_w2   (column-major nb x nb blocks)
            for (int b2 = 0; b2 < nb; ++b2)
              for (int b1 = 0; b1 < nb; ++b1) {
                cd acc(0);
                for (int c = 0; c < nb; ++c)
                  acc += g01[b1 + nb * c] * m[c + nb * b2];
                g0m[b1 + nb * b2] = acc;
              }
            for (int b2 = 0; b2 < nb; ++b2)
              for (int b1 = 0; b1 < nb; ++b1) {
                cd acc(0);
                for (int c = 0; c < nb; ++c)
                  acc += g0m[b1 + nb * c] * g02[c + nb * b2];
                blk[b1 + nb * b2] = -acc;
              }
            if (k1 == k2 && w1 == w2)
              for (int b2 = 0; b2 < nb; ++b2)
                for (int b1 = 0; b1 < nb; ++b1)
                  blk[b1 + nb * b2] += g01[b1 + nb * b2] * beta;
            std::copy(blk, blk + nb * nb, m);
          }
    });
  }

  // getGMultiband (tp_accumulator_cpu.hpp:389-405): G_a(b1, b2) = G_(b2, b1, s, k1, k2, w1e, w2e)
  // with compact frequencies shifted onto the extended mesh.
  cd Gm(int s, int k1, int k2, int w1, int w2, int b1, int b2) const {
    return G[s][gidx(b2, b1, k1, k2, w1 + ext, w2 + ext)];
  }

  // updateG4 (tp_accumulator_cpu.hpp:409-757), spin-symmetric branch.
  void updateG4(std::size_t channel_id, int sign) {
    auto& g4 = G4[channel_id];
    const int channel = channels[channel_id];
    const double sign_over_2 = 0.5 * sign;
    auto add = [&](int k, int q) { return k_add[k + nc * q]; };
    auto q_minus_k = [&](int k, int q) { return k_sub[k + nc * q]; };  // index of q - k
    const int nq = k_ex.size(), nwq = w_ex.size();
    if (channel < DCAACC_PH_TRANSVERSE || channel > DCAACC_PP_UP_DOWN)
      throw std::logic_error("Specified four point type not implemented.");
    // Threads split (transfer, w2); every G4 entry is written by one thread in the same order.
    parallelFor(nwq * nq * nw, [&](int job) {
      const int w2 = job % nw, iq = (job / nw) % nq, iwq = job / (nw * nq);
      {
        const int wex = w_ex[iwq];
        const int q = k_ex[iq];
          for (int k2 = 0; k2 < nc; ++k2)
            for (int w1 = 0; w1 < nw; ++w1)
              for (int k1 = 0; k1 < nc; ++k1) {
                cd* out = &g4[std::size_t(nb * nb * nb * nb) *
                              (k1 + nc * (w1 + std::size_t(nw) *
                                               (k2 + nc * (w2 + std::size_t(nw) * (iq + std::size_t(nq) * iwq)))))];
                auto at = [&](int b1, int b2, int b3, int b4) -> cd& {
                  return out[b1 + nb * (b2 + nb * (b3 + nb * b4))];
                };
                switch (channel) {
                  case DCAACC_PH_TRANSVERSE:
                    // -1/2 sum_s G(k2+q, k1+q, s) G(k1, k2, -s) (tp_accumulator_cpu.hpp:454-489)
                    for (int s = 0; s < 2; ++s)
                      for (int b4 = 0; b4 < nb; ++b4)
                        for (int b3 = 0; b3 < nb; ++b3)
                          for (int b2 = 0; b2 < nb; ++b2)
                            for (int b1 = 0; b1 < nb; ++b1)
                              at(b1, b2, b3, b4) +=
                                  -sign_over_2 * Gm(s, k1, k2, w1, w2, b2, b4) *
                                  Gm(!s, add(k2, q), add(k1, q), w2 + wex, w1 + wex, b3, b1);
                    break;
                  case DCAACC_PH_MAGNETIC:
                    // (tp_accumulator_cpu.hpp:491-546)
                    for (int s1 = 0; s1 < 2; ++s1)
                      for (int s2 = 0; s2 < 2; ++s2) {
                        const double spin_factor = (s1 == s2) ? 1 : -1;
                        for (int b4 = 0; b4 < nb; ++b4)
                          for (int b3 = 0; b3 < nb; ++b3)
                            for (int b2 = 0; b2 < nb; ++b2)
                              for (int b1 = 0; b1 < nb; ++b1)
                                at(b1, b2, b3, b4) +=
                                    sign_over_2 * Gm(s1, k1, add(k1, q), w1, w1 + wex, b2, b1) *
                                    Gm(s2, add(k2, q), k2, w2 + wex, w2, b3, b4) * spin_factor;
                      }
                    for (int s = 0; s < 2; ++s)
                      for (int b4 = 0; b4 < nb; ++b4)
                        for (int b3 = 0; b3 < nb; ++b3)
                          for (int b2 = 0; b2 < nb; ++b2)
                            for (int b1 = 0; b1 < nb; ++b1)
                              at(b1, b2, b3, b4) +=
                                  -sign_over_2 * Gm(s, k1, k2, w1, w2, b3, b1) *
                                  Gm(s, add(k2, q), add(k1, q), w2 + wex, w1 + wex, b2, b4);
                    break;
                  case DCAACC_PH_CHARGE:
                    // updateG4SpinDifference(+1) then updateG4Atomic x2, cross legs
                    // (tp_accumulator_cpu.hpp:548-575, :761-869)
                    for (int b4 = 0; b4 < nb; ++b4)
                      for (int b3 = 0; b3 < nb; ++b3)
                        for (int b2 = 0; b2 < nb; ++b2)
                          for (int b1 = 0; b1 < nb; ++b1) {
                            const cd ga = Gm(0, k1, add(k1, q), w1, w1 + wex, b2, b1) +
                                          Gm(1, k1, add(k1, q), w1, w1 + wex, b2, b1);
                            const cd gb = Gm(0, add(k2, q), k2, w2 + wex, w2, b3, b4) +
                                          Gm(1, add(k2, q), k2, w2 + wex, w2, b3, b4);
                            at(b1, b2, b3, b4) += sign_over_2 * ga * gb;
                          }
                    for (int s = 0; s < 2; ++s)
                      for (int b4 = 0; b4 < nb; ++b4)
                        for (int b3 = 0; b3 < nb; ++b3)
                          for (int b2 = 0; b2 < nb; ++b2)
                            for (int b1 = 0; b1 < nb; ++b1)
                              at(b1, b2, b3, b4) +=
                                  -sign_over_2 * Gm(s, k1, k2, w1, w2, b1, b4) *
                                  Gm(s, add(k2, q), add(k1, q), w2 + wex, w1 + wex, b2, b3);
                    break;
                  case DCAACC_PP_UP_DOWN: {
                    // 1/2 sum_s G(k1, k2, s) G(q-k1, q-k2, -s) with w -> wex + Nw - 1 - w
                    // (tp_accumulator_cpu.hpp:628-661)
                    const int wm1 = wex + nw - 1 - w1, wm2 = wex + nw - 1 - w2;
                    for (int s = 0; s < 2; ++s)
                      for (int b4 = 0; b4 < nb; ++b4)
                        for (int b3 = 0; b3 < nb; ++b3)
                          for (int b2 = 0; b2 < nb; ++b2)
                            for (int b1 = 0; b1 < nb; ++b1)
                              at(b1, b2, b3, b4) +=
                                  sign_over_2 * Gm(s, k1, k2, w1, w2, b1, b3) *
                                  Gm(!s, q_minus_k(k1, q), q_minus_k(k2, q), wm1, wm2, b2, b4);
                    break;
                  }
                  default:  // rejected before the loops
                    break;
                }
              }
      }
    });
  }
};

// ------------------------------------------------------------------------------------------------
// Single-particle accumulator: Dnfft1D (CUBIC, oversampling 8, window sampling 32) + SpAccumulator
// ------------------------------------------------------------------------------------------------
namespace kb {
// kaiser_bessel_function (kaiser_bessel_function.cpp:28-116), n = padded time size, m = 8, sigma = 2.
struct Window {
  int n;
  int m;
  double sigma;
  double b_val() const {
    return M_PI * (2. - 1. / sigma);
  }
  double renorm() const {
    return 1. / (M_PI * m) * std::sinh(M_PI * m * (2. * sigma - 1.) / sigma);
  }
  double phi_t(double x) const {
    double result = 0;
    const double val = double(m) * m - double(n) * n * x * x;
    if (val > 1.e-12)
      result = 1. / M_PI * std::sinh(b_val() * std::sqrt(val)) / std::sqrt(val);
    if (val < -1.e-12)
      result = 1. / M_PI * std::sin(b_val() * std::sqrt(-val)) / std::sqrt(-val);
    if (val >= -1.e-12 && val < 1.e-12)
      result = b_val() / M_PI;
    return result / renorm();
  }
  double d_phi_t(double x) const {
    double result = 0;
    const double val = double(m) * m - double(n) * n * x * x;
    const double b = b_val();
    if (val > 1.e-12)
      result = 1. / M_PI * (double(n) * n * x) *
               ((-b * std::cosh(b * std::sqrt(val))) / val + std::sinh(b * std::sqrt(val)) / std::pow(val, 1.5));
    if (val < -1.e-12)
      result = 1. / M_PI * (double(n) * n * x) *
               ((b * std::cos(b * std::sqrt(-val))) / (-val) - std::sin(b * std::sqrt(-val)) / std::pow(-val, 1.5));
    if (val >= -1.e-12 && val < 1.e-12)
      return 0;
    return result / renorm();
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
             besselI0(m * std::sqrt(std::pow(b_val(), 2) - std::pow((2. * M_PI * double(wn) / double(n)), 2))) /
             renorm();
    throw std::logic_error("phi_wn out of range");
  }
};
}  // namespace kb

class Sp {
public:
  static constexpr int oversampling = 8;
  static constexpr int window_sampling = 32;

  Sp(const dcaacc_sp_config& c) {
    nb = c.n_bands;
    nc = c.n_sites;
    n_sp = c.n_sp_freq;
    beta = c.beta;
    sqr = c.accumulate_m_sqr != 0;
    r_sub.assign(c.r_sub, c.r_sub + nc * nc);
    // nfft_time_domain (nfft_time_domain.hpp:112-176) with MAX_FREQUENCY = n_sp.
    const int max_freq = n_sp;
    Delta = 1. / double(oversampling * max_freq);
    delta = 1. / double(oversampling * max_freq * window_sampling);
    n_left = oversampling * max_freq;
    n_padded = oversampling * max_freq + 2 * oversampling;
    T0 = -0.5 - oversampling * Delta;
    t0_window = -2. / double(max_freq);
    window = kb::Window{n_padded, oversampling, 2.0};
    // Cubic coefficients (dnfft_1d.hpp:198-250): layout (4, 4*oversampling, window_sampling).
    const int n_os = 4 * oversampling;
    coeff.assign(4 * n_os * window_sampling, 0.0);
    auto fine_tau = [&](int idx) { return t0_window + idx * delta; };
    const double d = fine_tau(1) - fine_tau(0);
    for (int i = 0; i < n_os; ++i)
      for (int j = 0; j < window_sampling; ++j) {
        const double tau = fine_tau(j + i * window_sampling);
        const double f0 = window.phi_t(tau), f1 = window.phi_t(tau + d);
        const double df0 = window.d_phi_t(tau), df1 = window.d_phi_t(tau + d);
        const double a = f0, b = df0;
        const double cc = -(3. * f0 - 3. * f1 + 2. * df0 * d + df1 * d) / std::pow(d, 2);
        const double dd = -(-2. * f0 + 2. * f1 - 1. * df0 * d - df1 * d) / std::pow(d, 3);
        double* cf = &coeff[4 * (i + n_os * j)];
        cf[0] = a;
        cf[1] = b;
        cf[2] = cc;
        cf[3] = dd;
      }
    n_labels = nb * nb * nc;
    for (int s = 0; s < 2; ++s) {
      f_tau[s].assign(std::size_t(n_padded) * n_labels, 0.0);
      f_tau_sqr[s].assign(std::size_t(n_padded) * n_labels, 0.0);
    }
  }

  void reset() {
    for (int s = 0; s < 2; ++s) {
      std::fill(f_tau[s].begin(), f_tau[s].end(), 0.0);
      std::fill(f_tau_sqr[s].begin(), f_tau_sqr[s].end(), 0.0);
    }
    finalized = false;
  }

  // convoluteToFTauFineCubicInterpolation (dnfft_1d.hpp:353-399).
  void convolute(std::vector<double>& f, int index, double t_val, double f_val) const {
    const double one_div_Delta = 1. / Delta, one_div_delta = 1. / delta;
    const int tau_0 = static_cast<int>((t_val - T0) * one_div_Delta);
    const double t0_val_lb = T0 + tau_0 * Delta;
    const int tau_1 = static_cast<int>((t0_val_lb - t_val - t0_window) * one_div_delta);
    const double t1_val_lb = t0_window + tau_1 * delta;
    const double diff_tau = t0_val_lb - t_val - t1_val_lb;
    double y[4];
    y[0] = f_val;
    y[1] = y[0] * diff_tau;
    y[2] = y[1] * diff_tau;
    y[3] = y[2] * diff_tau;
    const int tau_index = tau_0 - oversampling;
    const int delta_tau_index = tau_1 - oversampling * window_sampling;
    const int j = delta_tau_index % window_sampling;
    const int i = (delta_tau_index - j) / window_sampling;
    double* fp = &f[tau_index + std::size_t(n_padded) * index];
    const double* M = &coeff[4 * (i + 4 * oversampling * j)];
    for (int c = 1; c < 2 * oversampling + 1; ++c)
      fp[c] += (M[0 + 4 * c] * y[0] + M[1 + 4 * c] * y[1] + M[2 + 4 * c] * y[2] + M[3 + 4 * c] * y[3]);
  }

  // SpAccumulator<CPU>::accumulate (sp_accumulator.hpp:161-203).
  void accumulate(const dcaacc_sector* sec, double factor) {
    const double one_div_two_beta = 1. / (2. * beta);
    for (int s = 0; s < 2; ++s) {
      const auto& c = sec[s];
      for (int j = 0; j < c.n; j++) {
        const int b_j = c.left_band[j], r_j = c.left_site[j];
        const double t_j = c.tau[j];
        for (int i = 0; i < c.n; i++) {
          const int b_i = c.right_band[i], r_i = c.right_site[i];
          const double t_i = c.tau[i];
          const int delta_r = r_sub[r_j + nc * r_i];  // subtract(r_j, r_i): index of r_i - r_j
          const double scaled_tau = (t_i - t_j) * one_div_two_beta;
          const int index = b_i + nb * (b_j + nb * delta_r);
          const double f_val = c.M[i + std::size_t(c.ldm) * j];
          convolute(f_tau[s], index, scaled_tau, factor * f_val);
          if (sqr)
            convolute(f_tau_sqr[s], index, scaled_tau, factor * f_val * f_val);
        }
      }
    }
  }

  // Dnfft1D::finalize: foldTimeDomainBack + transformFTauToFW (real scalar), then
  // SpAccumulator::finalizeFunction (sp_accumulator.hpp:205-220): out(b1,s,b2,s,r,w) += f_w / Nc.
  void finalizeInto(std::vector<double>* ft, std::vector<cd>& out) const {
    const int nw_sp = 2 * n_sp;
    out.assign(std::size_t(2 * nb) * (2 * nb) * nc * nw_sp, cd(0));
    const int n = n_left, padding = (n_padded - n_left) / 2;
    std::vector<double> cs(n), sn(n);
    for (int m = 0; m < n; ++m) {
      cs[m] = std::cos(2 * M_PI * m / double(n));
      sn[m] = std::sin(2 * M_PI * m / double(n));
    }
    std::vector<int> freq_index(nw_sp);
    std::vector<double> phi(nw_sp);
    for (int l = 0; l < n_sp; ++l) {
      freq_index[n_sp + l] = 2 * l + 1;
      freq_index[n_sp - 1 - l] = -(2 * l + 1);
    }
    for (int w = 0; w < nw_sp; ++w)
      phi[w] = window.phi_wn(freq_index[w]);
    for (int s = 0; s < 2; ++s) {
      std::vector<double> f = ft[s];
      for (int p = 0; p < n_labels; ++p) {
        double* fp = &f[std::size_t(n_padded) * p];
        for (int t = 0; t < padding; ++t)
          fp[t + n] += fp[t];
        for (int t = n_padded - padding; t < n_padded; ++t)
          fp[t - n] += fp[t];
      }
      for (int p = 0; p < n_labels; ++p) {
        const double* fin = &f[std::size_t(n_padded) * p + padding];
        const int b1 = p % nb, b2 = (p / nb) % nb, r = p / (nb * nb);
        for (int w = 0; w < nw_sp; ++w) {
          int tind = freq_index[w];
          if (tind < 0)
            tind += n;
          // f_omega(t) = -sum_x f_in[x] exp(+2 pi i x t / n)  (FFTW r2c then the sign flips)
          double re = 0, im = 0;
          for (int x = 0; x < n; ++x) {
            const int m = static_cast<int>((static_cast<long long>(x) * tind) % n);
            re += fin[x] * cs[m];
            im += fin[x] * sn[m];
          }
          const cd fw = cd(-re, -im) / phi[w] * (1. / n);
          const std::size_t o = b1 + 2 * nb * (b2 + 2 * nb * (r + std::size_t(nc) * w));
          // (b1, s, b2, s, r, w): offsets s for the first spin index, s*nb*2 for the second.
          out[o + s * nb + s * (2 * nb) * nb] += fw * (1. / nc);
        }
      }
    }
  }

  void finalize() {
    finalizeInto(f_tau, mrw);
    if (sqr)
      finalizeInto(f_tau_sqr, mrw_sqr);
    finalized = true;
  }

  int nb, nc, n_sp, n_left, n_padded, n_labels;
  double beta, Delta, delta, T0, t0_window;
  bool sqr, finalized = false;
  kb::Window window;
  std::vector<int> r_sub;
  std::vector<double> coeff;
  std::vector<double> f_tau[2], f_tau_sqr[2];
  std::vector<cd> mrw, mrw_sqr;
};

template <class F>
int guarded(F&& f) {
  try {
    f();
    return DCAACC_OK;
  }
  catch (const std::logic_error& e) {
    g_error = e.what();
    return DCAACC_INVALID_ARG;
  }
  catch (const std::exception& e) {
    g_error = e.what();
    return DCAACC_INVALID_ARG;
  }
}

}  // namespace oracle

extern "C" {

const char* oracle_last_error() {
  return oracle::g_error.c_str();
}

int oracle_tp_create(const dcaacc_tp_config* cfg, const double* G0, void** out) {
  return oracle::guarded([&] { *out = new oracle::Tp(*cfg, G0); });
}
void oracle_tp_destroy(void* h) {
  delete static_cast<oracle::Tp*>(h);
}
int oracle_tp_reset(void* h) {
  return oracle::guarded([&] { static_cast<oracle::Tp*>(h)->reset(); });
}
int oracle_tp_accumulate(void* h, const dcaacc_sector* sectors, int sign) {
  return oracle::guarded([&] { static_cast<oracle::Tp*>(h)->accumulate(sectors, sign); });
}
size_t oracle_tp_g4_size(void* h) {
  return static_cast<oracle::Tp*>(h)->g4_size;
}
int oracle_tp_get_g4(void* h, int channel, double* out, size_t count) {
  auto* t = static_cast<oracle::Tp*>(h);
  if (channel < 0 || channel >= (int)t->G4.size() || count != t->g4_size)
    return DCAACC_INVALID_ARG;
  std::memcpy(out, t->G4[channel].data(), 16 * count);
  return DCAACC_OK;
}
size_t oracle_tp_g_size(void* h) {
  return static_cast<oracle::Tp*>(h)->g_size;
}
int oracle_tp_get_g(void* h, int spin, double* out, size_t count) {
  auto* t = static_cast<oracle::Tp*>(h);
  if (spin < 0 || spin > 1 || count != t->g_size)
    return DCAACC_INVALID_ARG;
  std::memcpy(out, t->G[spin].data(), 16 * count);
  return DCAACC_OK;
}

int oracle_sp_create(const dcaacc_sp_config* cfg, void** out) {
  return oracle::guarded([&] { *out = new oracle::Sp(*cfg); });
}
void oracle_sp_destroy(void* h) {
  delete static_cast<oracle::Sp*>(h);
}
int oracle_sp_reset(void* h) {
  return oracle::guarded([&] { static_cast<oracle::Sp*>(h)->reset(); });
}
int oracle_sp_accumulate(void* h, const dcaacc_sector* sectors, double sign) {
  return oracle::guarded([&] { static_cast<oracle::Sp*>(h)->accumulate(sectors, sign); });
}
int oracle_sp_finalize(void* h) {
  return oracle::guarded([&] { static_cast<oracle::Sp*>(h)->finalize(); });
}
size_t oracle_sp_out_size(void* h) {
  auto* s = static_cast<oracle::Sp*>(h);
  return std::size_t(2 * s->nb) * (2 * s->nb) * s->nc * (2 * s->n_sp);
}
int oracle_sp_get(void* h, int which, double* out, size_t count) {
  auto* s = static_cast<oracle::Sp*>(h);
  const auto& v = which ? s->mrw_sqr : s->mrw;
  if (!s->finalized || count != v.size())
    return DCAACC_INVALID_ARG;
  std::memcpy(out, v.data(), 16 * count);
  return DCAACC_OK;
}
size_t oracle_sp_ftau_size(void* h) {
  auto* s = static_cast<oracle::Sp*>(h);
  return std::size_t(s->n_padded) * s->n_labels;
}
int oracle_sp_get_ftau(void* h, int spin, double* out, size_t count) {
  auto* s = static_cast<oracle::Sp*>(h);
  if (spin < 0 || spin > 1 || count != s->f_tau[spin].size())
    return DCAACC_INVALID_ARG;
  std::memcpy(out, s->f_tau[spin].data(), 8 * count);
  return DCAACC_OK;
}

// Runs a whole case file through the restatement and writes a result file (casefile.hpp).
int oracle_run_case(const char* case_path, const char* out_path, int do_tp, int do_sp) {
  return oracle::guarded([&] {
    const auto c = casefile::readCase(case_path);
    std::vector<int> k_ex, w_ex;
    if (c.all_transfers) {
      for (int k = 0; k < c.nc; ++k)
        k_ex.push_back(k);
      for (int w = 0; w <= c.freq_transfer; ++w)
        w_ex.push_back(w);
    }
    else {
      k_ex.push_back(c.k_transfer);
      w_ex.push_back(c.freq_transfer);
    }
    casefile::Result res;
    std::vector<std::array<dcaacc_sector, 2>> secs(c.meas.size());
    for (std::size_t m = 0; m < c.meas.size(); ++m)
      for (int s = 0; s < 2; ++s) {
        const auto& x = c.meas[m].sector[s];
        secs[m][s] = dcaacc_sector{x.n, x.tau.data(), x.left_band.data(), x.right_band.data(),
                                   x.left_site.data(), x.right_site.data(), x.M.data(),
                                   std::max(x.n, 1), 0};
      }
    if (do_tp) {
      dcaacc_tp_config cfg{};
      cfg.n_bands = c.nb;
      cfg.n_sites = c.nc;
      cfg.n_w_half = c.nw_half;
      cfg.n_sp_freq = c.n_sp_freq;
      cfg.n_k_ex = k_ex.size();
      cfg.k_ex = k_ex.data();
      cfg.n_w_ex = w_ex.size();
      cfg.w_ex = w_ex.data();
      cfg.n_channels = c.channels.size();
      cfg.channels = c.channels.data();
      cfg.beta = c.beta;
      cfg.r_vecs = c.r_vecs.data();
      cfg.k_vecs = c.k_vecs.data();
      cfg.a_vecs = c.a_vecs.data();
      cfg.k_add = c.k_add.data();
      cfg.k_sub = c.k_sub.data();
      oracle::Tp tp(cfg, reinterpret_cast<const double*>(c.G0.data()));
      for (std::size_t m = 0; m < c.meas.size(); ++m)
        tp.accumulate(secs[m].data(), c.meas[m].sign);
      res.G4 = tp.G4;
    }
    if (do_sp) {
      dcaacc_sp_config sc{};
      sc.n_bands = c.nb;
      sc.n_sites = c.nc;
      sc.n_sp_freq = c.n_sp_freq;
      sc.beta = c.beta;
      sc.r_sub = c.r_sub.data();
      sc.accumulate_m_sqr = c.flags & 1;
      oracle::Sp sp(sc);
      for (std::size_t m = 0; m < c.meas.size(); ++m)
        sp.accumulate(secs[m].data(), c.meas[m].sign);
      sp.finalize();
      res.has_sp = true;
      res.MRW = sp.mrw;
      res.has_sqr = sp.sqr;
      res.MRW_sqr = sp.mrw_sqr;
    }
    casefile::writeResult(out_path, res);
  });
}

}  // extern "C"
