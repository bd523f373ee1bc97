// Case files: one binary file holds a synthetic accumulation workload (cluster, G0, a list of
// measurements) so that the reference's own CPU accumulators (oracle/refbuild), the CPU
// restatement (oracle/oracle.cpp) and the tests all read identical inputs.
//
// Test infrastructure only.  Layout (little endian, no padding between fields):
//
//   char    magic[8]       "DCACASE1"
//   int32   nb, nc, nw_half, n_sp_freq, all_transfers, freq_transfer, k_transfer, n_channels
//   int32   channels[4]    FourPointType values (1 PH_TRANSVERSE, 2 PH_MAGNETIC, 3 PH_CHARGE,
//                          4 PP_UP_DOWN), as in the reference's four_point_type.hpp:27-33
//   int32   n_meas, flags  flags bit0: accumulate M^2 in the single-particle accumulator
//   double  beta
//   double  r_vecs[nc][2], k_vecs[nc][2]
//   int32   k_add[nc*nc], k_sub[nc*nc], r_add[nc*nc], r_sub[nc*nc]   A(i,j) at i + nc*j,
//           add(i,j) = index of x_i + x_j, sub(i,j) = index of x_j - x_i (the reference's
//           cluster_domain_initializer.hpp:691-765 convention)
//   double  a_vecs[nb][2]
//   double  G0[2 * (2nb)^2 * nc * 2n_sp]  complex G0(b1,s1,b2,s2,k,w), first index fastest
//   per measurement:
//     int32 sign
//     per spin sector s = 0, 1:
//       int32 n; double tau[n]; int32 left_band[n], right_band[n], left_site[n], right_site[n];
//       double M[n*n] (column major)
//
// Result files ("DCAOUT01"): int32 n_channels; int64 g4_size; complex G4[n_channels][g4_size];
// int32 has_sp; if has_sp: int64 sp_size; complex MRW[sp_size]; int32 has_sqr;
// if has_sqr: complex MRW_sqr[sp_size].  MRW is in the reference layout (b1,s1,b2,s2,r,w).
#ifndef ORACLE_CASEFILE_HPP
#define ORACLE_CASEFILE_HPP

#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace casefile {

struct Sector {
  int n = 0;
  std::vector<double> tau;
  std::vector<int> left_band, right_band, left_site, right_site;
  std::vector<double> M;  // n x n column major
};

struct Measurement {
  int sign = 1;
  Sector sector[2];
};

struct Case {
  int nb = 1, nc = 1, nw_half = 1, n_sp_freq = 1;
  int all_transfers = 0, freq_transfer = 0, k_transfer = 0;
  std::vector<int> channels;
  int flags = 0;
  double beta = 1;
  std::vector<double> r_vecs, k_vecs, a_vecs;
  std::vector<int> k_add, k_sub, r_add, r_sub;
  std::vector<std::complex<double>> G0;
  std::vector<Measurement> meas;
};

class Reader {
public:
  explicit Reader(const std::string& path) : f_(std::fopen(path.c_str(), "rb")) {
    if (!f_)
      throw std::runtime_error("cannot open " + path);
  }
  ~Reader() {
    if (f_)
      std::fclose(f_);
  }
  template <class T>
  void read(T* dst, std::size_t count) {
    if (count && std::fread(dst, sizeof(T), count, f_) != count)
      throw std::runtime_error("truncated case file");
  }
  template <class T>
  T get() {
    T v;
    read(&v, 1);
    return v;
  }

private:
  std::FILE* f_;
};

inline Case readCase(const std::string& path) {
  Reader r(path);
  char magic[8];
  r.read(magic, 8);
  if (std::memcmp(magic, "DCACASE1", 8) != 0)
    throw std::runtime_error("bad case magic");
  Case c;
  int32_t h[8];
  r.read(h, 8);
  c.nb = h[0];
  c.nc = h[1];
  c.nw_half = h[2];
  c.n_sp_freq = h[3];
  c.all_transfers = h[4];
  c.freq_transfer = h[5];
  c.k_transfer = h[6];
  const int n_channels = h[7];
  int32_t ch[4];
  r.read(ch, 4);
  for (int i = 0; i < n_channels; ++i)
    c.channels.push_back(ch[i]);
  const int n_meas = r.get<int32_t>();
  c.flags = r.get<int32_t>();
  c.beta = r.get<double>();
  const int nc = c.nc, nb = c.nb;
  c.r_vecs.resize(2 * nc);
  c.k_vecs.resize(2 * nc);
  r.read(c.r_vecs.data(), 2 * nc);
  r.read(c.k_vecs.data(), 2 * nc);
  for (auto* t : {&c.k_add, &c.k_sub, &c.r_add, &c.r_sub}) {
    t->resize(nc * nc);
    std::vector<int32_t> tmp(nc * nc);
    r.read(tmp.data(), nc * nc);
    for (int i = 0; i < nc * nc; ++i)
      (*t)[i] = tmp[i];
  }
  c.a_vecs.resize(2 * nb);
  r.read(c.a_vecs.data(), 2 * nb);
  const std::size_t g0_size = std::size_t(2 * nb) * (2 * nb) * nc * (2 * c.n_sp_freq);
  c.G0.resize(g0_size);
  r.read(reinterpret_cast<double*>(c.G0.data()), 2 * g0_size);
  c.meas.resize(n_meas);
  for (auto& m : c.meas) {
    m.sign = r.get<int32_t>();
    for (auto& s : m.sector) {
      s.n = r.get<int32_t>();
      const int n = s.n;
      s.tau.resize(n);
      r.read(s.tau.data(), n);
      for (auto* v : {&s.left_band, &s.right_band, &s.left_site, &s.right_site}) {
        std::vector<int32_t> tmp(n);
        r.read(tmp.data(), n);
        v->assign(tmp.begin(), tmp.end());
      }
      s.M.resize(std::size_t(n) * n);
      r.read(s.M.data(), std::size_t(n) * n);
    }
  }
  return c;
}

struct Result {
  std::vector<std::vector<std::complex<double>>> G4;
  std::vector<std::complex<double>> MRW, MRW_sqr;
  bool has_sp = false, has_sqr = false;
};

inline void writeResult(const std::string& path, const Result& res) {
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f)
    throw std::runtime_error("cannot write " + path);
  std::fwrite("DCAOUT01", 1, 8, f);
  const int32_t n_channels = res.G4.size();
  std::fwrite(&n_channels, 4, 1, f);
  const int64_t g4_size = n_channels ? res.G4[0].size() : 0;
  std::fwrite(&g4_size, 8, 1, f);
  for (const auto& g : res.G4)
    std::fwrite(g.data(), 16, g.size(), f);
  const int32_t has_sp = res.has_sp;
  std::fwrite(&has_sp, 4, 1, f);
  if (has_sp) {
    const int64_t sp_size = res.MRW.size();
    std::fwrite(&sp_size, 8, 1, f);
    std::fwrite(res.MRW.data(), 16, res.MRW.size(), f);
    const int32_t has_sqr = res.has_sqr;
    std::fwrite(&has_sqr, 4, 1, f);
    if (has_sqr)
      std::fwrite(res.MRW_sqr.data(), 16, res.MRW_sqr.size(), f);
  }
  std::fclose(f);
}

}  // namespace casefile

#endif  // ORACLE_CASEFILE_HPP
