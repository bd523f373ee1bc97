// Driver that runs the REFERENCE's own CPU accumulators on a case file.
//
// Test infrastructure only.  Built by oracle/refbuild/Makefile from the reference headers and a
// handful of its .cpp files where they lie (nothing is copied); the binary lands in oracle/_ref/.
// It instantiates, with a mock Parameters type:
//   dca::phys::solver::accumulator::TpAccumulator<Parameters, DistType::NONE, linalg::CPU>
//     (include/dca/phys/dca_step/cluster_solver/shared_tools/accumulation/tp/tp_accumulator_cpu.hpp)
//   dca::phys::solver::accumulator::SpAccumulator<Parameters, linalg::CPU>
//     (include/dca/phys/dca_step/cluster_solver/shared_tools/accumulation/sp/sp_accumulator.hpp)
// and initialises the static domains (frequency, vertex-frequency, exchange, band) the same way
// the reference's parameter setup does, with mock cluster domains that carry the case's
// lattice vectors and add/subtract tables.
//
// Usage: tp_ref <case.bin> <out.bin> [--no-tp] [--no-sp] [--time] [--warmup W]
//   --time prints "tp_seconds=<s> sp_seconds=<s> n_meas=<m>" on stderr, the seconds covering the
//   measurements after the first W.
#include <array>
#include <chrono>
#include <iomanip>
#include <cstdlib>
#include <complex>
#include <cstdint>
#include <iostream>
#include <string>
#include <vector>

#include "dca/function/domains.hpp"
#include "dca/function/function.hpp"
#include "dca/linalg/matrix.hpp"
#include "dca/phys/dca_step/cluster_solver/shared_tools/accumulation/sp/sp_accumulator.hpp"
#include "dca/phys/dca_step/cluster_solver/shared_tools/accumulation/tp/tp_accumulator_cpu.hpp"
#include "dca/phys/domains/cluster/cluster_domain.hpp"
#include "dca/phys/domains/cluster/momentum_exchange_domain.hpp"
#include "dca/phys/domains/quantum/electron_band_domain.hpp"
#include "dca/phys/domains/quantum/electron_spin_domain.hpp"
#include "dca/phys/domains/time_and_frequency/frequency_domain.hpp"
#include "dca/phys/domains/time_and_frequency/frequency_exchange_domain.hpp"
#include "dca/phys/domains/time_and_frequency/vertex_frequency_domain.hpp"
#include "dca/phys/four_point_type.hpp"
#include "dca/profiling/null_profiler.hpp"

#include "../casefile.hpp"

namespace harness {

// Cluster domain whose elements and add/subtract tables come from the case file.
template <int ID>
struct MockCluster {
  using element_type = std::vector<double>;
  using Table = dca::linalg::Matrix<int, dca::linalg::CPU>;

  static int get_size() {
    return static_cast<int>(get_elements().size());
  }
  static std::string get_name() {
    return ID == 0 ? "harness-r-cluster" : "harness-k-cluster";
  }
  static std::vector<element_type>& get_elements() {
    static std::vector<element_type> elements;
    return elements;
  }
  static Table& get_add_matrix() {
    static Table a("add");
    return a;
  }
  static Table& get_subtract_matrix() {
    static Table s("subtract");
    return s;
  }
  static int add(int i, int j) {
    return get_add_matrix()(i, j);
  }
  static int subtract(int i, int j) {
    return get_subtract_matrix()(i, j);
  }
  static void print_2_file(const char*) {}

  static void set(const std::vector<double>& vecs, const std::vector<int>& add,
                  const std::vector<int>& sub, int nc) {
    get_elements().assign(nc, std::vector<double>(2));
    for (int i = 0; i < nc; ++i)
      get_elements()[i] = {vecs[2 * i], vecs[2 * i + 1]};
    get_add_matrix().resizeNoCopy(nc);
    get_subtract_matrix().resizeNoCopy(nc);
    for (int j = 0; j < nc; ++j)
      for (int i = 0; i < nc; ++i) {
        get_add_matrix()(i, j) = add[i + nc * j];
        get_subtract_matrix()(i, j) = sub[i + nc * j];
      }
  }
};

using RCluster = MockCluster<0>;
using KCluster = MockCluster<1>;

struct MockLattice {
  static constexpr bool spin_symmetric = true;
  static std::vector<std::vector<double>>& aVecs() {
    static std::vector<std::vector<double>> v;
    return v;
  }
  static std::vector<int> flavors() {
    std::vector<int> f(aVecs().size());
    for (std::size_t i = 0; i < f.size(); ++i)
      f[i] = static_cast<int>(i);
    return f;
  }
  static std::vector<std::vector<double>> aVectors() {
    return aVecs();
  }
};

template <int NB>
struct MockModel {
  static constexpr int BANDS = NB;
  using lattice_type = MockLattice;
};

struct NoConcurrency {
  int id() const {
    return 0;
  }
  int number_of_processors() const {
    return 1;
  }
};

template <int NB>
struct Params {
  using TPAccumPrec = double;
  using Real = double;
  using Scalar = double;
  using RClusterDmn = dca::func::dmn_0<RCluster>;
  using KClusterDmn = dca::func::dmn_0<KCluster>;
  using model_type = MockModel<NB>;
  using lattice_type = MockLattice;
  using profiler_type = dca::profiling::NullProfiler;
  static constexpr int bands = NB;

  double beta;
  int nw_half;
  bool all_transfers;
  int freq_transfer;
  int k_transfer;
  std::vector<dca::phys::FourPointType> channels;
  NoConcurrency concurrency;

  double get_beta() const {
    return beta;
  }
  int get_accumulators() const {
    return 1;
  }
  const std::vector<dca::phys::FourPointType>& get_four_point_channels() const {
    return channels;
  }
  const NoConcurrency& get_concurrency() const {
    return concurrency;
  }
  int get_four_point_fermionic_frequencies() const {
    return nw_half;
  }
  bool compute_all_transfers() const {
    return all_transfers;
  }
  int get_four_point_frequency_transfer() const {
    return freq_transfer;
  }
  int get_four_point_momentum_transfer_index() const {
    return k_transfer;
  }
  int stamping_period() const {
    return 0;
  }
};

// Vertex exposing the accessors the reference's CachedNdft and SpAccumulator read
// (cached_ndft_base.hpp:97-113, sp_accumulator.hpp:181-187).
struct Vertex {
  double tau;
  int lb, rb, ls, rs;
  double get_tau() const {
    return tau;
  }
  int get_left_band() const {
    return lb;
  }
  int get_right_band() const {
    return rb;
  }
  int get_left_site() const {
    return ls;
  }
  int get_right_site() const {
    return rs;
  }
};

}  // namespace harness

// The momentum exchange domain reads the cluster's symmetry table; the mock cluster has only the
// identity, so "compute all transfers" yields every momentum (as the reference does for a cluster
// without point-group symmetries).
namespace dca {
namespace phys {
namespace domains {
template <>
class cluster_symmetry<harness::KCluster> {
public:
  struct Table {
    int operator[](int i) const {
      return i == 0 ? harness::KCluster::get_size() : 1;
    }
    std::pair<int, int> operator()(int k, int, int) const {
      return {k, 0};
    }
  };
  static const Table& get_symmetry_matrix() {
    static Table t;
    return t;
  }
};
}  // namespace domains
}  // namespace phys
}  // namespace dca

#ifndef DCA_REF_BLAS_NAME
#define DCA_REF_BLAS_NAME "naive-zgemm"
#endif
constexpr const char* kBlasName = DCA_REF_BLAS_NAME;

// Wall-clock seconds since the epoch: comparable across the processes of a parallel timing run.
inline double epochSeconds() {
  return std::chrono::duration<double>(std::chrono::system_clock::now().time_since_epoch()).count();
}

namespace harness {

template <int NB>
int run(const casefile::Case& c, const std::string& out_path, bool do_tp, bool do_sp, bool timing,
        int warmup) {
  using namespace dca;
  using P = Params<NB>;
  P pars;
  pars.beta = c.beta;
  pars.nw_half = c.nw_half;
  pars.all_transfers = c.all_transfers != 0;
  pars.freq_transfer = c.freq_transfer;
  pars.k_transfer = c.k_transfer;
  for (int ch : c.channels)
    pars.channels.push_back(static_cast<phys::FourPointType>(ch));

  RCluster::set(c.r_vecs, c.r_add, c.r_sub, c.nc);
  KCluster::set(c.k_vecs, c.k_add, c.k_sub, c.nc);
  MockLattice::aVecs().clear();
  for (int b = 0; b < NB; ++b)
    MockLattice::aVecs().push_back({c.a_vecs[2 * b], c.a_vecs[2 * b + 1]});

  phys::domains::frequency_domain::initialize(c.beta, c.n_sp_freq);
  phys::domains::electron_band_domain::initialize(pars);
  phys::domains::FrequencyExchangeDomain::initialize(pars);
  phys::domains::MomentumExchangeDomain::initialize(pars);
  phys::domains::vertex_frequency_domain<phys::domains::COMPACT>::initialize(pars);
  phys::domains::vertex_frequency_domain<phys::domains::EXTENDED>::initialize(pars);

  using BDmn = func::dmn_0<phys::domains::electron_band_domain>;
  using SDmn = func::dmn_0<phys::domains::electron_spin_domain>;
  using NuDmn = func::dmn_variadic<BDmn, SDmn>;
  using KDmn = typename P::KClusterDmn;
  using WDmn = func::dmn_0<phys::domains::frequency_domain>;

  casefile::Result res;

  // Measurements: M matrices and configurations per spin sector.
  const int n_meas = static_cast<int>(c.meas.size());
  std::vector<std::array<linalg::Matrix<double, linalg::CPU>, 2>> Ms(n_meas);
  std::vector<std::array<std::vector<Vertex>, 2>> confs(n_meas);
  for (int m = 0; m < n_meas; ++m)
    for (int s = 0; s < 2; ++s) {
      const auto& sec = c.meas[m].sector[s];
      Ms[m][s].resizeNoCopy(sec.n);
      for (int j = 0; j < sec.n; ++j)
        for (int i = 0; i < sec.n; ++i)
          Ms[m][s](i, j) = sec.M[i + std::size_t(sec.n) * j];
      confs[m][s].resize(sec.n);
      for (int i = 0; i < sec.n; ++i)
        confs[m][s][i] = Vertex{sec.tau[i], sec.left_band[i], sec.right_band[i], sec.left_site[i],
                                sec.right_site[i]};
    }

  double tp_seconds = 0, sp_seconds = 0, tp_epoch_start = 0, tp_epoch_end = 0;
  if (do_tp) {
    func::function<std::complex<double>, func::dmn_variadic<NuDmn, NuDmn, KDmn, WDmn>> G0("G0");
    if (G0.size() != c.G0.size())
      throw std::runtime_error("G0 size mismatch");
    for (std::size_t i = 0; i < c.G0.size(); ++i)
      G0(i) = c.G0[i];

    phys::solver::accumulator::TpAccumulator<P, DistType::NONE, linalg::CPU> acc(G0, pars);
    acc.resetAccumulation();
    auto t0 = std::chrono::steady_clock::now();
    tp_epoch_start = epochSeconds();
    for (int m = 0; m < n_meas; ++m) {
      if (m == warmup) {
        t0 = std::chrono::steady_clock::now();
        tp_epoch_start = epochSeconds();
      }
      acc.accumulate(Ms[m], confs[m], static_cast<std::int8_t>(c.meas[m].sign));
    }
    tp_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    tp_epoch_end = epochSeconds();
    for (const auto& g4 : acc.get_G4()) {
      res.G4.emplace_back(g4.size());
      for (std::size_t i = 0; i < g4.size(); ++i)
        res.G4.back()[i] = g4(i);
    }
  }

  if (do_sp) {
    const bool sqr = c.flags & 1;
    phys::solver::accumulator::SpAccumulator<P, linalg::CPU> sp(pars, sqr);
    sp.resetAccumulation();
    auto t0 = std::chrono::steady_clock::now();
    for (int m = 0; m < n_meas; ++m) {
      if (m == warmup)
        t0 = std::chrono::steady_clock::now();
      sp.accumulate(Ms[m], confs[m], static_cast<double>(c.meas[m].sign));
    }
    sp_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    sp.finalize();
    const auto& mrw = sp.get_sign_times_M_r_w();
    res.has_sp = true;
    res.MRW.resize(mrw.size());
    for (std::size_t i = 0; i < mrw.size(); ++i)
      res.MRW[i] = mrw(i);
    if (sqr) {
      const auto& mrw2 = sp.get_sign_times_M_r_w_sqr();
      res.has_sqr = true;
      res.MRW_sqr.resize(mrw2.size());
      for (std::size_t i = 0; i < mrw2.size(); ++i)
        res.MRW_sqr[i] = mrw2(i);
    }
  }

  casefile::writeResult(out_path, res);
  if (timing)
    std::cerr << std::setprecision(17) << "tp_seconds=" << tp_seconds << " sp_seconds=" << sp_seconds
              << " n_meas=" << n_meas << " tp_epoch_start=" << tp_epoch_start << " tp_epoch_end=" << tp_epoch_end
              << " blas=" << kBlasName << "\n";
  return 0;
}

}  // namespace harness

int main(int argc, char** argv) {
  if (argc < 3) {
    std::cerr << "usage: tp_ref <case.bin> <out.bin> [--no-tp] [--no-sp] [--time] [--warmup W]\n";
    return 2;
  }
  bool do_tp = true, do_sp = true, timing = false;
  int warmup = 0;
  for (int i = 3; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--warmup" && i + 1 < argc)
      warmup = std::atoi(argv[++i]);
    if (a == "--no-tp")
      do_tp = false;
    else if (a == "--no-sp")
      do_sp = false;
    else if (a == "--time")
      timing = true;
  }
  try {
    const auto c = casefile::readCase(argv[1]);
    switch (c.nb) {
      case 1:
        return harness::run<1>(c, argv[2], do_tp, do_sp, timing, warmup);
      case 2:
        return harness::run<2>(c, argv[2], do_tp, do_sp, timing, warmup);
      case 3:
        return harness::run<3>(c, argv[2], do_tp, do_sp, timing, warmup);
      default:
        std::cerr << "unsupported band count " << c.nb << "\n";
        return 2;
    }
  }
  catch (const std::exception& e) {
    std::cerr << "tp_ref: " << e.what() << "\n";
    return 1;
  }
}
