// Host side of the single-particle accumulator: the object behind a dcaacc_sp handle.
// Mirrors SpAccumulator<Parameters, linalg::GPU> (sp_accumulator_gpu.hpp:42-130).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "../../include/dcaacc.h"
#include "tp_accumulator.hpp"

namespace dcaacc {

// One spin sector as the NFFT kernel reads it.
struct SpSector {
  const double* M;  // device, column major
  int ldm;
  int n;
  int vtx_off;
  int pad;
};

class SpAccumulator {
public:
  explicit SpAccumulator(const dcaacc_sp_config& cfg);
  ~SpAccumulator();

  void reset();
  void accumulate(const dcaacc_sector* sectors, double factor);
  void finalize();
  void get(bool sqr, double* out, size_t count) const;
  void sumTo(SpAccumulator& other) const;
  void setStream(cudaStream_t s);
  void synchronize();
  size_t deviceFingerprint() const;
  uint64_t kernelLaunches() const;
  size_t outputSize() const;
  size_t fTauSize() const;
  void singleMeasurementMrw(double* out, size_t count);
  void singleMeasurementFtau(double* out, size_t count);
  void clearSingleMeasurement();

private:
  struct Impl;
  std::unique_ptr<Impl> d_;
  void finalizeInto(const double* f_tau, std::vector<double2>& host);
};

}  // namespace dcaacc
