// Host side of the two-particle accumulator: the object behind a dcaacc_tp handle.
//
// Mirrors TpAccumulator<Parameters, DistType::NONE, linalg::GPU>
// (tp_accumulator_gpu.hpp:59-263): resetAccumulation, accumulate, finalize, sumTo, get_G4,
// get_stream / synchronizeCopy / deviceFingerprint.  Differences by design:
//   * each handle owns its G4 (the reference keeps one process-wide static device G4,
//     tp_accumulator_gpu.hpp:493-497); several accumulator threads combine with sumTo;
//   * in mixed precision, measurements are queued and processed in batches of max_batch.
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dcaacc.h"
#include "common.cuh"
#include "tp_frontend.hpp"
#include "tp_g4.hpp"
#include "tp_layout.hpp"

namespace dcaacc {

// Owning device buffer.
template <typename T>
class DevBuf {
public:
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p_)
      cudaFree(p_);
  }
  void alloc(size_t n) {
    if (p_)
      cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
    if (n) {
      allocationHook();
      DCAACC_CUDA_CHECK(cudaMalloc(&p_, n * sizeof(T)));
    }
    n_ = n;
  }
  T* get() const {
    return p_;
  }
  size_t size() const {
    return n_;
  }
  size_t bytes() const {
    return n_ * sizeof(T);
  }

private:
  T* p_ = nullptr;
  size_t n_ = 0;
};

// Owning pinned host buffer.
template <typename T>
class PinBuf {
public:
  PinBuf() = default;
  PinBuf(const PinBuf&) = delete;
  PinBuf& operator=(const PinBuf&) = delete;
  ~PinBuf() {
    if (p_)
      cudaFreeHost(p_);
  }
  void alloc(size_t n) {
    if (p_)
      cudaFreeHost(p_);
    p_ = nullptr;
    n_ = 0;
    if (n) {
      allocationHook();
      DCAACC_CUDA_CHECK(cudaMallocHost(&p_, n * sizeof(T)));
    }
    n_ = n;
  }
  T* get() const {
    return p_;
  }
  T& operator[](size_t i) {
    return p_[i];
  }
  size_t size() const {
    return n_;
  }

private:
  T* p_ = nullptr;
  size_t n_ = 0;
};

class TpAccumulator {
public:
  TpAccumulator(const dcaacc_tp_config& cfg, const double* G0);
  ~TpAccumulator();

  void reset(long dca_loop = -1);
  void shareG4(TpAccumulator& owner);
  // m_f32: the sectors' M hold float elements (else double).
  double accumulate(const dcaacc_sector* sectors, int sign, bool m_f32 = false);
  void flush();
  void finalize();
  void getG4(int channel, double* out, size_t count) const;
  void getG4Normalized(int channel, double* out, size_t count) const;
  void signSum(double* sum, uint64_t* count) const;
  void sumTo(TpAccumulator& other);
  void getG(int spin, double* out, size_t count) const;
  void setStream(cudaStream_t s);
  cudaStream_t stream() const {
    return stream_;
  }
  void synchronize();
  size_t deviceFingerprint() const;
  int mirrorMode() const {
    return (dims_.half_g ? 1 : 0) | (dims_.half_g4 ? 2 : 0);
  }
  uint64_t kernelLaunches() const {
    return launches_;
  }
  size_t g4Size() const {
    return g4_size_;
  }
  void enableTiming(bool on);
  void stageTimes(double* ms, uint64_t* launches, int n);
  void setGraphs(bool on);
  void graphStats(uint64_t* captures, uint64_t* replays) const;
  bool tuningSettled() const {
    return tuner_.settled();
  }
  std::string tuningReport() {
    return tuner_.report();
  }
  void peekG4(int channel, size_t offset, size_t count, double* out, bool wait = true);
  void setFaultInjection(int stop_step, uint32_t wait_polls);

private:
  void init(const dcaacc_tp_config& cfg, const double* G0);
  void releaseStreamsAndEvents();
  int fault_stop_step_ = -1;  // error-path tests (G4Args::fault_stop_step)
  uint32_t wait_limit_ = 0;   // error-path tests (G4Args::wait_limit)
  void validateSector(const dcaacc_sector& s) const;
  bool sameG4(const TpAccumulator& o) const;
  void stage(const dcaacc_sector* sectors, int sign, bool m_f32);
  void process();
  double flopEstimate(const dcaacc_sector* sectors) const;

  // Configuration.
  TpDims dims_{};
  bool mixed_ = false;
  bool non_density_ = false;
  bool atomic_ = false;
  int max_batch_ = 1, max_order_ = 1;
  int n_sp_ = 0;
  std::vector<int> k_add_, k_sub_, q_list_, wex_list_;
  size_t g4_size_ = 0;
  long g_sector_stride_ = 0;  // complex elements of one (slot, spin) G

  // Device state.
  int device_ = 0;
  int n_sm_ = 0;  // multiprocessors of the device (persistent grids)
  cudaStream_t stream_ = nullptr;
  bool own_stream_ = false;
  DevBuf<double2> G0_, Fb_;
  DevBuf<int> k_add_d_, k_sub_d_, q_d_, wex_d_;
  // The running G4 per channel.  Usually this handle's own; several handles may share one
  // (shareG4), as the reference's accumulator threads share their static device G4.
  struct SharedG4 {
    std::vector<DevBuf<double2>> bufs;
    std::mutex m;
    long last_loop = -1;  // dca_loop of the last once-per-loop reset
    std::vector<TpAccumulator*> users;  // handles accumulating into it (guarded by m)
  };
  std::shared_ptr<SharedG4> g4s_;
  std::vector<DevBuf<double2>>& g4() {
    return g4s_->bufs;
  }
  const std::vector<DevBuf<double2>>& g4() const {
    return g4s_->bufs;
  }
  bool g4Shared() const {
    return g4s_.use_count() > 1;
  }
  void uploadG4Ptrs();
  DevBuf<double2*> G4_ptrs_;
  DevBuf<int> err_d_;  // kernels' error word (async_copy.cuh kErr* bits)
  // Batch workspace.
  // Per-batch device inputs, double-buffered like the pinned staging below: batch k + 1 is uploaded
  // on copy_stream_ while batch k's kernels run on stream_ (events order the reuse of a set).
  struct DevStage {
    DevBuf<SectorDesc> sectors;
    DevBuf<double> tau, M;  // M: host-resident sectors' matrices, copied in
    DevBuf<int> vb_r, vs_r, vb_c, vs_c;  // per-vertex band and site of the row / column side (uploaded)
    DevBuf<int> perm_r, perm_c, rstart, cstart, signs, orb_r, orb_c;  // sorted on the device
    cudaEvent_t consumed = nullptr;  // the kernels that read this set have completed
  };
  DevStage dstage_[2];
  cudaStream_t copy_stream_ = nullptr;
  int launchBatch(const FrontendArgs& fa, const G4Args& ga, DevStage& ds);
  int launchBatchGraph(int set, const FrontendArgs& fa, const G4Args& ga, DevStage& ds);
  // CUDA graphs of the tensor-core path's batch sequence (launchBatchGraph).
  struct BatchGraph {
    int set, slots, n_max;  // key: device input set, batch size, order bound
    bool clean;             // a batch of this key ran eagerly without launch-shape probes
    cudaGraphExec_t exec;   // instantiated on the batch after the first clean one
    int launches;           // kernels in the graph
    uint64_t last;          // least-recently-used stamp
  };
  std::vector<BatchGraph> graphs_;
  LaunchTuner tuner_;
  bool graphs_on_ = true;
  uint64_t graph_stamp_ = 0, graph_captures_ = 0, graph_replays_ = 0;
  void releaseGraphs();
  DevBuf<double2> Tr_d_, Tc_d_;
  DevBuf<double2> X64_, G64_;  // FP64 mode
  DevBuf<float2> X32_, G32_;   // mixed mode
  DevBuf<unsigned char> disc_;  // mixed mode, one band: tensor-core disconnected-term workspace
  DiscWorkspace disc_ws_{};
  bool have_disc_ = false;
  // Mixed mode: tensor-core front-end (operand planes + TMA descriptors) and the orbital of each
  // vertex in row / column order.
  bool tc_front_ = false;
  DevBuf<unsigned char> ftc_mem_;
  DevBuf<unsigned char> col_tp_;  // factored column step, FFT form: FP16 planes of the column twiddles
  FrontTcWorkspace ftc_{};
  DevBuf<int> gmax_d_;  // [2 slot + spin] largest |G| per sector (column step -> G4 kernel)
  // Half G4 (dims_.half_g4): positions of -q / -wq in the transfer lists, the tiles the update
  // runs, and a device window for peeks.
  DevBuf<int> q_mirror_d_, wq_mirror_d_;
  DevBuf<unsigned> tile_order_d_;
  DevBuf<double2> peek_d_;
  static constexpr size_t kPeekWindow = size_t(1) << 16;  // entries allocated with a half-G4 handle
  // Pinned staging of the batch being assembled, double-buffered: the host fills one set while the
  // uploads from the other (queued behind the previous batch's kernels) are still pending.
  struct HostStage {
    PinBuf<SectorDesc> sectors;
    PinBuf<double> tau;
    PinBuf<int> vb_r, vs_r, vb_c, vs_c, signs;
    cudaEvent_t uploaded = nullptr;  // the uploads from this set have completed
  };
  HostStage hstage_[2];
  int hset_ = 0;  // set being filled
  HostStage& hs() {
    return hstage_[hset_];
  }

  // Batch bookkeeping.
  int slots_ = 0;         // measurements staged
  int vtx_used_ = 0;      // packed vertices staged
  long x_used_ = 0;       // X' elements reserved
  size_t m_used_ = 0;     // host-resident M copied into the device set, packed n x n per sector
  // Host -> device M copy being extended: a sector whose host M directly follows the previous
  // one's (a caller keeping a batch's matrices in one pinned buffer) joins the same copy.
  const double* mcopy_src_ = nullptr;
  double* mcopy_dst_ = nullptr;
  size_t mcopy_bytes_ = 0;
  void flushMCopy();
  int n_max_batch_ = 0;   // largest order staged
  double sign_sum_ = 0;   // signs of the measurements accumulated since reset (sumTo moves them)
  uint64_t n_meas_ = 0;
  bool ready_ = false;    // reset() called since the last finalize
  bool finalized_ = false;
  bool have_g_ = false;   // FP64 mode: G of the last measurement is in G64_
  uint64_t launches_ = 0;
  std::vector<std::vector<std::complex<double>>> G4_host_;

  // Stage timing: pairs of events per recorded launch group.
  struct Timed {
    int stage;
    cudaEvent_t begin, end;
  };
  bool timing_ = false;
  std::vector<Timed> timed_;
  double stage_ms_[4] = {0, 0, 0, 0};
  uint64_t stage_launches_[4] = {0, 0, 0, 0};
  void timeBegin(int stage, cudaEvent_t* b);
  void timeEnd(int stage, cudaEvent_t b, int launches);
  void collectTimes();
  void checkDeviceError();
};

}  // namespace dcaacc
