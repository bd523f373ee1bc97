// The C ABI (include/dcaacc.h): status codes around the accumulator objects.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <new>
#include <string>

#include "../../include/dcaacc.h"
#include "common.cuh"
#include "sp_accumulator.hpp"
#include "tp_accumulator.hpp"

namespace dcaacc {

namespace {
std::atomic<long> g_alloc_countdown{0};  // > 0: allocations left before the one that fails
}

void setAllocationFailure(long nth) {
  g_alloc_countdown.store(nth > 0 ? nth : 0);
}

void allocationHook() {
  long c = g_alloc_countdown.load();
  while (c > 0 && !g_alloc_countdown.compare_exchange_weak(c, c - 1)) {
  }
  if (c == 1)
    throw Error(DCAACC_OOM, "injected allocation failure (dcaacc_set_allocation_failure)");
}

void computeGNoAlloc(const dcaacc_tp_config& c, const double* G0_dev, const dcaacc_sector* sec,
                     double* G_out, cudaStream_t stream);
size_t staticScratchBytes();
}

struct dcaacc_tp {
  dcaacc::TpAccumulator impl;
  dcaacc_tp(const dcaacc_tp_config& c, const double* g0) : impl(c, g0) {}
};
struct dcaacc_sp {
  dcaacc::SpAccumulator impl;
  explicit dcaacc_sp(const dcaacc_sp_config& c) : impl(c) {}
};

namespace {
thread_local std::string g_last_error;

template <class F>
int guard(F&& f) {
  try {
    f();
    return DCAACC_OK;
  }
  catch (const dcaacc::Error& e) {
    g_last_error = e.what();
    return e.status;
  }
  catch (const std::bad_alloc& e) {
    g_last_error = "host allocation failed";
    return DCAACC_OOM;
  }
  catch (const std::exception& e) {
    g_last_error = e.what();
    return DCAACC_INVALID_ARG;
  }
}

int null_handle() {
  g_last_error = "null handle";
  return DCAACC_INVALID_ARG;
}
}  // namespace

extern "C" {

const char* dcaacc_last_error(void) {
  return g_last_error.c_str();
}

int dcaacc_tp_create(const dcaacc_tp_config* cfg, const double* G0, dcaacc_tp** out) {
  if (!cfg || !out)
    return null_handle();
  *out = nullptr;
  return guard([&] { *out = new dcaacc_tp(*cfg, G0); });
}

void dcaacc_tp_destroy(dcaacc_tp* acc) {
  delete acc;
}

int dcaacc_tp_reset(dcaacc_tp* acc) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.reset(); });
}

int dcaacc_tp_accumulate(dcaacc_tp* acc, const dcaacc_sector* sectors, int32_t sign, double* flops_out) {
  if (!acc)
    return null_handle();
  return guard([&] {
    const double f = acc->impl.accumulate(sectors, sign);
    if (flops_out)
      *flops_out = f;
  });
}

int dcaacc_tp_accumulate_typed(dcaacc_tp* acc, int32_t n_meas, const dcaacc_sector* sectors, int32_t m_scalar,
                               const double* signs_re, const double* signs_im, double* flops_out) {
  if (!acc)
    return null_handle();
  return guard([&] {
    if (n_meas < 0 || (n_meas && (!sectors || !signs_re)))
      throw dcaacc::Error(DCAACC_INVALID_ARG, "invalid batch");
    if (m_scalar == DCAACC_SCALAR_C64 || m_scalar == DCAACC_SCALAR_C128)
      throw dcaacc::Error(DCAACC_UNSUPPORTED, "complex M (complex-valued models) is not implemented");
    if (m_scalar != DCAACC_SCALAR_F64 && m_scalar != DCAACC_SCALAR_F32)
      throw dcaacc::Error(DCAACC_INVALID_ARG, "unknown M scalar type");
    for (int m = 0; m < n_meas; ++m) {
      if (signs_im && signs_im[m] != 0.)
        throw dcaacc::Error(DCAACC_UNSUPPORTED, "complex measurement signs are not implemented");
      if (signs_re[m] != 1. && signs_re[m] != -1.)
        throw dcaacc::Error(DCAACC_INVALID_ARG, "sign must be +1 or -1");
    }
    double f = 0;
    for (int m = 0; m < n_meas; ++m)
      f += acc->impl.accumulate(sectors + 2 * m, signs_re[m] > 0 ? 1 : -1, m_scalar == DCAACC_SCALAR_F32);
    if (flops_out)
      *flops_out = f;
  });
}

int dcaacc_tp_accumulate_batch(dcaacc_tp* acc, int32_t n_meas, const dcaacc_sector* sectors,
                               const int32_t* signs, double* flops_out) {
  if (!acc)
    return null_handle();
  return guard([&] {
    if (n_meas < 0 || (n_meas && (!sectors || !signs)))
      throw dcaacc::Error(DCAACC_INVALID_ARG, "invalid batch");
    double f = 0;
    for (int m = 0; m < n_meas; ++m)
      f += acc->impl.accumulate(sectors + 2 * m, signs[m]);
    if (flops_out)
      *flops_out = f;
  });
}

int dcaacc_tp_flush(dcaacc_tp* acc) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.flush(); });
}

int dcaacc_tp_finalize(dcaacc_tp* acc) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.finalize(); });
}

int dcaacc_tp_get_g4(const dcaacc_tp* acc, int32_t channel, double* out, size_t count) {
  if (!acc || !out)
    return null_handle();
  return guard([&] { acc->impl.getG4(channel, out, count); });
}

size_t dcaacc_tp_g4_size(const dcaacc_tp* acc) {
  return acc ? acc->impl.g4Size() : 0;
}

int dcaacc_tp_sum_to(dcaacc_tp* acc, dcaacc_tp* other) {
  if (!acc || !other)
    return null_handle();
  return guard([&] { acc->impl.sumTo(other->impl); });
}

int dcaacc_tp_get_g(const dcaacc_tp* acc, int32_t spin, double* out, size_t count) {
  if (!acc || !out)
    return null_handle();
  return guard([&] { acc->impl.getG(spin, out, count); });
}

int dcaacc_tp_set_stream(dcaacc_tp* acc, void* stream) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.setStream(static_cast<cudaStream_t>(stream)); });
}

void* dcaacc_tp_get_stream(const dcaacc_tp* acc) {
  return acc ? static_cast<void*>(acc->impl.stream()) : nullptr;
}

int dcaacc_tp_synchronize(dcaacc_tp* acc) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.synchronize(); });
}

size_t dcaacc_tp_device_fingerprint(const dcaacc_tp* acc) {
  return acc ? acc->impl.deviceFingerprint() : 0;
}

int32_t dcaacc_tp_mirror_mode(const dcaacc_tp* acc) {
  return acc ? acc->impl.mirrorMode() : 0;
}

uint64_t dcaacc_tp_kernel_launches(const dcaacc_tp* acc) {
  return acc ? acc->impl.kernelLaunches() : 0;
}

int dcaacc_tp_share_g4(dcaacc_tp* acc, dcaacc_tp* owner) {
  if (!acc || !owner)
    return null_handle();
  return guard([&] { acc->impl.shareG4(owner->impl); });
}

int dcaacc_tp_reset_loop(dcaacc_tp* acc, int32_t dca_loop) {
  if (!acc)
    return null_handle();
  if (dca_loop < 0)
    return guard([&] { throw dcaacc::Error(DCAACC_INVALID_ARG, "dca_loop must be non-negative"); });
  return guard([&] { acc->impl.reset(dca_loop); });
}

int dcaacc_tp_sign_sum(const dcaacc_tp* acc, double* sum, uint64_t* count) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.signSum(sum, count); });
}

int dcaacc_tp_get_g4_normalized(const dcaacc_tp* acc, int32_t channel, double* out, size_t count) {
  if (!acc || !out)
    return null_handle();
  return guard([&] { acc->impl.getG4Normalized(channel, out, count); });
}

size_t dcaacc_tp_static_device_fingerprint(void) {
  return dcaacc::staticScratchBytes();
}

int dcaacc_tp_enable_timing(dcaacc_tp* acc, int32_t on) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.enableTiming(on != 0); });
}

int dcaacc_tp_stage_times(dcaacc_tp* acc, double* ms, uint64_t* launches, int32_t n_stages) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.stageTimes(ms, launches, n_stages); });
}

int dcaacc_tp_set_graphs(dcaacc_tp* acc, int32_t on) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.setGraphs(on != 0); });
}

int dcaacc_tp_graph_stats(const dcaacc_tp* acc, uint64_t* captures, uint64_t* replays) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.graphStats(captures, replays); });
}

int32_t dcaacc_tp_tuning_settled(const dcaacc_tp* acc) {
  return acc ? acc->impl.tuningSettled() : 0;
}

int dcaacc_tp_tuning_report(dcaacc_tp* acc, char* buf, size_t cap, size_t* len) {
  if (!acc)
    return null_handle();
  return guard([&] {
    const std::string r = acc->impl.tuningReport();
    if (len)
      *len = r.size();
    if (buf && cap) {
      const size_t n = std::min(cap - 1, r.size());
      std::memcpy(buf, r.data(), n);
      buf[n] = '\0';
    }
  });
}

int dcaacc_tp_peek_g4(dcaacc_tp* acc, int32_t channel, size_t offset, size_t count, double* out) {
  if (!acc || !out)
    return null_handle();
  return guard([&] { acc->impl.peekG4(channel, offset, count, out); });
}

int dcaacc_tp_peek_g4_async(dcaacc_tp* acc, int32_t channel, size_t offset, size_t count, double* out) {
  if (!acc || !out)
    return null_handle();
  return guard([&] { acc->impl.peekG4(channel, offset, count, out, false); });
}

int dcaacc_tp_compute_g_noalloc(const dcaacc_tp_config* cfg, const double* G0,
                                const dcaacc_sector* sectors, double* G_out, void* stream) {
  if (!cfg)
    return null_handle();
  return guard([&] { dcaacc::computeGNoAlloc(*cfg, G0, sectors, G_out, static_cast<cudaStream_t>(stream)); });
}

int dcaacc_tp_g4_shard(int32_t n_k_ex, int32_t rank, int32_t n_ranks, int32_t* first, int32_t* count) {
  return guard([&] {
    if (!first || !count)
      throw dcaacc::Error(DCAACC_INVALID_ARG, "g4_shard: null output");
    if (n_ranks < 1 || n_ranks > n_k_ex || rank < 0 || rank >= n_ranks)
      throw dcaacc::Error(DCAACC_INVALID_ARG, "g4_shard: need 0 <= rank < n_ranks <= number of momentum transfers");
    const int32_t base = n_k_ex / n_ranks, extra = n_k_ex % n_ranks;
    *count = base + (rank < extra ? 1 : 0);
    *first = rank * base + std::min(rank, extra);
  });
}

int dcaacc_tp_g4_place_shard(const dcaacc_tp_config* cfg, int32_t rank, int32_t n_ranks, const double* shard,
                             size_t shard_count, double* full, size_t full_count) {
  if (!cfg)
    return null_handle();
  return guard([&] {
    if (!shard || !full)
      throw dcaacc::Error(DCAACC_INVALID_ARG, "g4_place_shard: null buffer");
    if (cfg->n_bands < 1 || cfg->n_sites < 1 || cfg->n_w_half < 1 || cfg->n_w_ex < 1)
      throw dcaacc::Error(DCAACC_INVALID_ARG, "g4_place_shard: bad sizes");
    int32_t first = 0, count = 0;
    if (dcaacc_tp_g4_shard(cfg->n_k_ex, rank, n_ranks, &first, &count) != DCAACC_OK)
      throw dcaacc::Error(DCAACC_INVALID_ARG, g_last_error);
    // One (q, wq) slab: every entry with fixed transfers, contiguous since q and wq are the slowest indices.
    const size_t nb = cfg->n_bands, nc = cfg->n_sites, nw = 2 * size_t(cfg->n_w_half);
    const size_t slab = nb * nb * nb * nb * nc * nc * nw * nw;
    const size_t nq = cfg->n_k_ex, nwq = cfg->n_w_ex;
    if (full_count != slab * nq * nwq || shard_count != slab * size_t(count) * nwq)
      throw dcaacc::Error(DCAACC_INVALID_ARG, "g4_place_shard: buffer sizes do not match the configuration");
    for (size_t wq = 0; wq < nwq; ++wq)
      std::memcpy(full + 2 * slab * (wq * nq + first), shard + 2 * slab * (wq * count),
                  2 * slab * count * sizeof(double));
  });
}

int dcaacc_tp_set_fault_injection(dcaacc_tp* acc, int32_t stop_step, uint32_t wait_polls) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.setFaultInjection(stop_step, wait_polls); });
}

int dcaacc_set_allocation_failure(int64_t nth) {
  dcaacc::setAllocationFailure(static_cast<long>(nth));
  return DCAACC_OK;
}

int dcaacc_sp_create(const dcaacc_sp_config* cfg, dcaacc_sp** out) {
  if (!cfg || !out)
    return null_handle();
  *out = nullptr;
  return guard([&] { *out = new dcaacc_sp(*cfg); });
}

void dcaacc_sp_destroy(dcaacc_sp* acc) {
  delete acc;
}

int dcaacc_sp_reset(dcaacc_sp* acc) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.reset(); });
}

int dcaacc_sp_accumulate(dcaacc_sp* acc, const dcaacc_sector* sectors, double sign) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.accumulate(sectors, sign); });
}

int dcaacc_sp_finalize(dcaacc_sp* acc) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.finalize(); });
}

int dcaacc_sp_get_m_r_w(const dcaacc_sp* acc, double* out, size_t count) {
  if (!acc || !out)
    return null_handle();
  return guard([&] { acc->impl.get(false, out, count); });
}

int dcaacc_sp_get_m_r_w_sqr(const dcaacc_sp* acc, double* out, size_t count) {
  if (!acc || !out)
    return null_handle();
  return guard([&] { acc->impl.get(true, out, count); });
}

int dcaacc_sp_get_single_measurement_m_r_w(dcaacc_sp* acc, double* out, size_t count) {
  if (!acc || !out)
    return null_handle();
  return guard([&] { acc->impl.singleMeasurementMrw(out, count); });
}

int dcaacc_sp_get_single_measurement_f_tau(dcaacc_sp* acc, double* out, size_t count) {
  if (!acc || !out)
    return null_handle();
  return guard([&] { acc->impl.singleMeasurementFtau(out, count); });
}

int dcaacc_sp_clear_single_measurement(dcaacc_sp* acc) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.clearSingleMeasurement(); });
}

size_t dcaacc_sp_f_tau_size(const dcaacc_sp* acc) {
  return acc ? acc->impl.fTauSize() : 0;
}

int dcaacc_sp_sum_to(const dcaacc_sp* acc, dcaacc_sp* other) {
  if (!acc || !other)
    return null_handle();
  return guard([&] { acc->impl.sumTo(other->impl); });
}

int dcaacc_sp_set_stream(dcaacc_sp* acc, void* stream) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.setStream(static_cast<cudaStream_t>(stream)); });
}

int dcaacc_sp_synchronize(dcaacc_sp* acc) {
  if (!acc)
    return null_handle();
  return guard([&] { acc->impl.synchronize(); });
}

size_t dcaacc_sp_device_fingerprint(const dcaacc_sp* acc) {
  return acc ? acc->impl.deviceFingerprint() : 0;
}

uint64_t dcaacc_sp_kernel_launches(const dcaacc_sp* acc) {
  return acc ? acc->impl.kernelLaunches() : 0;
}

}  // extern "C"
