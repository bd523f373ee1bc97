/*
 * dcaacc.h — C ABI of the B200 QMC measurement accumulators (libdcaacc.so).
 *
 * Two accumulators, each behind an opaque handle, with the method set of the reference's
 * accumulator classes that the CT-AUX / CT-INT solvers call:
 *
 *   two-particle (G4):   TpAccumulator<Parameters, DistType::NONE, linalg::GPU>
 *     include/dca/phys/dca_step/cluster_solver/shared_tools/accumulation/tp/tp_accumulator_gpu.hpp:59-263
 *   single-particle:     SpAccumulator<Parameters, linalg::GPU>
 *     include/dca/phys/dca_step/cluster_solver/shared_tools/accumulation/sp/sp_accumulator_gpu.hpp:42-130
 *
 * Conventions shared by every entry point:
 *   - Every function returns a dcaacc_status (0 = success).  On failure,
 *     dcaacc_last_error() returns a thread-local, human readable message.
 *   - Complex numbers are interleaved (re, im) doubles.
 *   - Matrices are column major with an explicit leading dimension, as linalg::Matrix is.
 *   - Multidimensional outputs use the reference's func::function layout: first index fastest.
 *   - A handle is bound to the CUDA device that was current when it was created, and is used by
 *     one host thread at a time (one accumulator object per accumulator thread, as in
 *     stdthread_qmci_cluster_solver.hpp:523-580).
 */
#ifndef DCAACC_H
#define DCAACC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference throws std::logic_error for misuse (tp_accumulator_gpu.hpp:329-330,
 * :456-468), std::runtime_error for a failed launch (tp_accumulator_kernels.cu:695-699) and rethrows
 * std::bad_alloc (tp_accumulator_gpu.hpp:314-317); the C++ wrapper maps these codes back. */
typedef enum dcaacc_status {
  DCAACC_OK = 0,
  DCAACC_INVALID_ARG = 1,    /* bad shape, index table or configuration (logic_error) */
  DCAACC_NOT_READY = 2,      /* call order violated, e.g. accumulate before reset (logic_error) */
  DCAACC_OOM = 3,            /* device or host allocation failed (bad_alloc) */
  DCAACC_CUDA_ERR = 4,       /* a CUDA call or kernel launch failed (runtime_error) */
  DCAACC_DEVICE_INDEX_ERR = 5, /* a kernel's own bounds check tripped; no memory was touched */
  DCAACC_UNSUPPORTED = 6     /* valid request that this build does not implement (logic_error) */
} dcaacc_status;

/* Four-point channels: the reference's FourPointType values (include/dca/phys/four_point_type.hpp:27-33). */
enum {
  DCAACC_PH_TRANSVERSE = 1,
  DCAACC_PH_MAGNETIC = 2,
  DCAACC_PH_CHARGE = 3,
  DCAACC_PP_UP_DOWN = 4
};

/* Arithmetic of the two-particle pipeline. */
enum {
  /* FP64 everywhere (the reference's double TP accumulation, mc_options.hpp.in TPAccumulationPrecision). */
  DCAACC_PRECISION_FP64 = 0,
  /* Mixed: the NDFT and cluster transform on the tensor cores in split-BF16 with FP32 accumulation,
   * G in FP32, per-batch G4 partial sums in FP32, running G4 in FP64. */
  DCAACC_PRECISION_MIXED = 1
};

/* One spin sector of one measurement: the walker configuration and its M matrix.
 * Mirrors what CachedNdft::sortConfiguration (cached_ndft_base.hpp:89-129) and
 * SpAccumulator::accumulate (sp_accumulator.hpp:178-201) read from a Configuration. */
typedef struct dcaacc_sector {
  int32_t n;                  /* expansion order (number of vertices); 0 is allowed */
  const double* tau;          /* [n] imaginary times in [0, beta) (host memory) */
  const int32_t* left_band;   /* [n] (host memory) */
  const int32_t* right_band;  /* [n] */
  const int32_t* left_site;   /* [n] */
  const int32_t* right_site;  /* [n] */
  const double* M;            /* n x n, column major (host or device memory, see m_on_device) */
  int32_t ldm;                /* leading dimension of M, >= n */
  int32_t m_on_device;        /* 1: M is a device pointer on the handle's device */
} dcaacc_sector;

/* Static description of the two-particle accumulation: the data the reference reads from
 * Parameters and its static domains in TpAccumulatorBase's constructor (tp_accumulator_base.hpp:184-208)
 * and G4Helper::set (g4_helper.cu:34-87). */
typedef struct dcaacc_tp_config {
  int32_t n_bands;            /* nb  (BDmn) */
  int32_t n_sites;            /* Nc  (RClusterDmn = KClusterDmn size) */
  int32_t n_w_half;           /* four-point fermionic frequencies; Nw = 2 * n_w_half (WTpDmn) */
  int32_t n_sp_freq;          /* positive single-particle frequencies of the G0 mesh (WDmn = 2 * n_sp_freq) */
  int32_t n_k_ex;             /* number of momentum transfers (KExchangeDmn) */
  const int32_t* k_ex;        /* [n_k_ex] cluster-momentum indices of the transfers */
  int32_t n_w_ex;             /* number of frequency transfers (WExchangeDmn) */
  const int32_t* w_ex;        /* [n_w_ex] transfers as index shifts (frequency_exchange_domain.cpp:26-48) */
  int32_t n_channels;
  const int32_t* channels;    /* [n_channels] DCAACC_PH_* / DCAACC_PP_* */
  double beta;
  const double* r_vecs;       /* [n_sites][2] real-space cluster sites */
  const double* k_vecs;       /* [n_sites][2] cluster momenta */
  const double* a_vecs;       /* [n_bands][2] intra-cell band positions (electron_band_domain a_vec) */
  const int32_t* k_add;       /* [n_sites * n_sites], (i,j) at i + Nc*j: index of k_i + k_j */
  const int32_t* k_sub;       /* [n_sites * n_sites], (i,j) at i + Nc*j: index of k_j - k_i */
  int32_t non_density;        /* 1: columns of M use the vertex's left band/site (cached_ndft_base.hpp:74-78) */
  int32_t precision;          /* DCAACC_PRECISION_* */
  int32_t max_batch;          /* measurements buffered before one fused G4 update (>= 1) */
  int32_t max_order;          /* upper bound on any sector's n (device buffers are sized for it) */
  int32_t accumulators;       /* > 1: several handles may add into one G4 (atomic updates) */
} dcaacc_tp_config;

typedef struct dcaacc_tp dcaacc_tp;

const char* dcaacc_last_error(void);

/* TpAccumulator(G0, parameters) — tp_accumulator_gpu.hpp:265-269.
 * G0: complex FP64, layout (b1, s1, b2, s2, k, w) over the full single-particle mesh
 * (2 * n_sp_freq frequencies), i.e. func::function<TpComplex, dmn_variadic<NuDmn, NuDmn, KDmn, WDmn>>.
 * The handle allocates all device memory it will use (sized by max_order and max_batch). */
int dcaacc_tp_create(const dcaacc_tp_config* cfg, const double* G0, dcaacc_tp** out);

/* ~TpAccumulator. Null is accepted. */
void dcaacc_tp_destroy(dcaacc_tp* acc);

/* resetAccumulation(dca_loop) — tp_accumulator_gpu.hpp:285-296: zeroes G4, re-slices G0, arms accumulate. */
int dcaacc_tp_reset(dcaacc_tp* acc);

/* The reference's accumulator threads share one static device G4 (get_G4Dev,
 * tp_accumulator_gpu.hpp:493-497), updated atomically when there are several
 * (tp_accumulator_kernels.cu:677-680), zeroed once per DCA loop (callOncePerLoop,
 * tp_accumulator_gpu.hpp:271-296), and sumTo has nothing to add for it (:487-491).  Here each handle
 * owns its G4 unless share_g4 makes acc accumulate into owner's (same G4 shape, transfer lists,
 * channels, beta, mirror mode and device, else DCAACC_INVALID_ARG; what acc has accumulated so
 * far is added into owner's G4 and acc's own is released; both switch to atomic updates).
 * reset_loop is resetAccumulation(dca_loop): a shared G4 is zeroed only by the first handle that
 * resets for a given dca_loop, after the updates already launched on every sharing handle's
 * stream and before any later one (measurements a handle has queued but not launched, see flush,
 * count toward the new loop); a private G4 is zeroed on every call.  sum_to between handles
 * sharing G4 moves only the sign sums and orders the target's later reads (finalize, peek) after
 * the source's updates; without it, a handle's reads of a shared G4 see another handle's updates
 * once that handle has synchronized. */
int dcaacc_tp_share_g4(dcaacc_tp* acc, dcaacc_tp* owner);
int dcaacc_tp_reset_loop(dcaacc_tp* acc, int32_t dca_loop);

/* accumulate(M, configs, sign) — tp_accumulator_gpu.hpp:322-367.
 * sectors: [2] (spin 0, spin 1).  sign: +1 / -1.  flops_out (may be null) receives the
 * reference's flop estimate for the call.  In FP64 mode the measurement is processed
 * immediately; in mixed mode it is queued and processed with its batch (see flush). */
int dcaacc_tp_accumulate(dcaacc_tp* acc, const dcaacc_sector* sectors, int32_t sign, double* flops_out);

/* accumulate for the reference's other instantiations, accumulate<Configuration, SpScalar, SignType>
 * (tp_accumulator_gpu.hpp:118-125, 322-325), for n_meas measurements (sectors [2 n_meas]): M of
 * element type m_scalar (DCAACC_SCALAR_*) in every sector, each M pointer read as that type, and
 * measurement m's sign as (signs_re[m], signs_im[m]) for a SignType that may be std::complex
 * (signs_im may be null).  Real M in float or double with real signs +1 / -1 is accumulated (float
 * M is widened to double as it is read, and a host float M crosses PCIe at half the bytes); complex
 * M, which only complex-valued (e.g. spin-orbit) models produce, and a sign with a non-zero
 * imaginary part return DCAACC_UNSUPPORTED before anything is staged. */
enum { DCAACC_SCALAR_F64 = 0, DCAACC_SCALAR_F32 = 1, DCAACC_SCALAR_C128 = 2, DCAACC_SCALAR_C64 = 3 };
int dcaacc_tp_accumulate_typed(dcaacc_tp* acc, int32_t n_meas, const dcaacc_sector* sectors, int32_t m_scalar,
                               const double* signs_re, const double* signs_im, double* flops_out);

/* Batched form: n_meas measurements, sectors [2 * n_meas], signs [n_meas]. */
int dcaacc_tp_accumulate_batch(dcaacc_tp* acc, int32_t n_meas, const dcaacc_sector* sectors,
                               const int32_t* signs, double* flops_out);

/* Processes queued measurements now (mixed mode).  No-op when nothing is queued. */
int dcaacc_tp_flush(dcaacc_tp* acc);

/* finalize() — tp_accumulator_gpu.hpp:471-484: flushes, then copies G4 to the host side of the handle. */
int dcaacc_tp_finalize(dcaacc_tp* acc);

/* get_G4()[channel] — tp_accumulator_gpu.hpp:503-510.  Copies G4 of one channel (complex FP64,
 * layout (b1,b2,b3,b4,k1,w1,k2,w2,q,wq)) into out, which holds count complex numbers.
 * Valid after finalize. */
int dcaacc_tp_get_g4(const dcaacc_tp* acc, int32_t channel, double* out, size_t count);

/* Number of complex entries of one channel's G4: nb^4 Nc^2 Nw^2 Nq Nwq (dca_data.hpp:108-112). */
size_t dcaacc_tp_g4_size(const dcaacc_tp* acc);

/* sumTo(other) — the CPU accumulator adds its G4 into other's and clears its own
 * (tp_accumulator_cpu.hpp:896-904).  Here: other.G4 += this.G4 on the device, this.G4 = 0.  Both
 * handles must accumulate the same G4 (sizes, transfer lists, channels, beta), else
 * DCAACC_INVALID_ARG; their precisions and mirror modes may differ (a half-G4 source is completed
 * from its mirror before it is added into a full-G4 target). */
int dcaacc_tp_sum_to(dcaacc_tp* acc, dcaacc_tp* other);

/* Debug / parity: copies the last measurement's G for one spin (complex, layout
 * (b1,b2,k1,k2,w1,w2) over the extended frequency mesh; the reference's G_ without the spin
 * index, tp_accumulator_base.hpp:79-80).  FP64 mode only. */
int dcaacc_tp_get_g(const dcaacc_tp* acc, int32_t spin, double* out, size_t count);

/* get_stream() / syncStreams(): the CUDA stream the handle enqueues on (cudaStream_t as void*).
 * set_stream makes the handle use the caller's stream instead of its own. */
int dcaacc_tp_set_stream(dcaacc_tp* acc, void* stream);
void* dcaacc_tp_get_stream(const dcaacc_tp* acc);

/* synchronizeCopy(): returns once host inputs of earlier accumulate calls may be reused. */
int dcaacc_tp_synchronize(dcaacc_tp* acc);

/* deviceFingerprint() — tp_accumulator_gpu.hpp:148-156: device bytes held by the handle. */
size_t dcaacc_tp_device_fingerprint(const dcaacc_tp* acc);

/* Number of this library's kernels launched by the handle since creation. */
uint64_t dcaacc_tp_kernel_launches(const dcaacc_tp* acc);

/* The solver's normalisation of G4 (ctaux_cluster_solver.hpp:521-525): G4 / (accumulated sign *
 * beta^2).  The handle sums the signs passed to accumulate since resetAccumulation (every
 * measurement counts, empty configurations included; sum_to moves the sum with G4).  sign_sum
 * returns that sum and the number of measurements; get_g4_normalized is get_g4 divided by
 * sum * beta^2 (DCAACC_NOT_READY while the sum is zero). */
int dcaacc_tp_sign_sum(const dcaacc_tp* acc, double* sum, uint64_t* count);
int dcaacc_tp_get_g4_normalized(const dcaacc_tp* acc, int32_t channel, double* out, size_t count);

/* staticDeviceFingerprint() — tp_accumulator_gpu.hpp:158-167: device bytes held process-wide, not
 * by a handle.  The reference counts its static shared G4 and G0 there; here G4 and G0 belong to
 * their handle (dcaacc_tp_device_fingerprint), and the process-wide device state is the
 * allocation-free entry point's static scratch array. */
size_t dcaacc_tp_static_device_fingerprint(void);

/* Which mirror symmetries the mixed path uses (no reference counterpart; monitoring): bit 0, only
 * the upper frequency half of G is computed (real M and G0(-k,-w) = conj G0(k,w)); bit 1, only
 * the G4 tiles with w1 >= Nw/2 are accumulated and the rest is their conjugated mirror. */
int32_t dcaacc_tp_mirror_mode(const dcaacc_tp* acc);

/* Stage timers, the counterpart of the reference's Profiler scopes in the accumulator
 * ("Frequency FT", "Space FT", "ComputeG", "updateG4": tp_accumulator_cpu.hpp:236-280,
 * tp_accumulator_gpu_base.hpp:214-219).  When enabled, CUDA events bracket each launch on the
 * handle's stream.  stage_times writes the cumulative milliseconds and launch counts of
 * DCAACC_N_STAGES stages (twiddles, row transform, column transform + G, G4 update) since the
 * last enable, synchronizing the stream first. */
enum { DCAACC_STAGE_TWIDDLE = 0, DCAACC_STAGE_ROW = 1, DCAACC_STAGE_COL = 2, DCAACC_STAGE_G4 = 3,
       DCAACC_N_STAGES = 4 };
int dcaacc_tp_enable_timing(dcaacc_tp* acc, int32_t on);
int dcaacc_tp_stage_times(dcaacc_tp* acc, double* ms, uint64_t* launches, int32_t n_stages);

/* CUDA graphs of the mixed path's per-batch kernel sequence (no reference counterpart; the
 * reference launches each kernel from the host per measurement).  On by default (environment
 * DCAACC_TP_GRAPHS=0 turns them off at creation); used only on a non-default stream and while
 * stage timing is off.  A batch shape's first batch runs eagerly, its second is captured, later
 * ones replay the graph; the results are the same either way.  graph_stats reports the graphs
 * captured and the batches replayed from one since creation (either pointer may be null). */
int dcaacc_tp_set_graphs(dcaacc_tp* acc, int32_t on);
int dcaacc_tp_graph_stats(const dcaacc_tp* acc, uint64_t* captures, uint64_t* replays);

/* Launch-shape tuner (no reference counterpart).  Kernels with several launch shapes that give
 * bit-identical results (tile widths, threads or warps per block) run each shape a few times on the
 * handle's first batches of a given problem shape, timed with CUDA events, and keep the fastest.
 * On by default; environment DCAACC_TUNE=0 keeps the built-in shapes.  tuning_settled is 1 when
 * no problem shape is still being explored (graphs are captured only then).  tuning_report writes
 * one line per tuned launch ("key n=<candidates> choice=<c> ms=<median per candidate>") as a
 * NUL-terminated string of at most cap bytes into buf (which may be null) and the full length
 * (without the NUL) into *len. */
int32_t dcaacc_tp_tuning_settled(const dcaacc_tp* acc);
int dcaacc_tp_tuning_report(dcaacc_tp* acc, char* buf, size_t cap, size_t* len);

/* Reads count complex entries of one channel's running G4 starting at offset, without finalizing
 * (processes queued measurements first, then a synchronous device-to-host copy).  For monitoring
 * an accumulation in progress. */
int dcaacc_tp_peek_g4(dcaacc_tp* acc, int32_t channel, size_t offset, size_t count, double* out);

/* The same read enqueued on the handle's stream without waiting: out (pinned host memory for an
 * asynchronous copy) holds the entries once the stream has reached this point, e.g. after
 * dcaacc_tp_synchronize; it must stay valid until then.  Lets a caller read every batch's result
 * while the next batch is being staged and copied. */
int dcaacc_tp_peek_g4_async(dcaacc_tp* acc, int32_t channel, size_t offset, size_t count, double* out);

/* Allocation-free G of one measurement.  No counterpart in the reference: it exists for callers
 * that cannot allocate device memory while they run -- applications whose device memory is fully
 * reserved by their own pool allocator, and per-measurement loops that must not pay the
 * device-wide synchronisation of cudaMalloc / cudaFree.  It runs the same three front-end kernels
 * as a handle in FP64 mode (twiddles, row NDFT + cluster transform, column NDFT + cluster
 * transform + G0 epilogue) but takes its scratch from a 48 MiB array compiled into the library,
 * which every GPU that loads the library keeps until the process exits; it calls no cudaMalloc,
 * cudaFree or other allocating routine.
 *
 *   cfg       sizes, transfers (only their extent matters here), beta, vectors as for
 *             dcaacc_tp_create; precision, max_batch, max_order and channels are ignored
 *   G0        DEVICE pointer, complex FP64 G0(b1, s1, b2, s2, k, w) over the full single-particle mesh
 *   sectors   [2]; vertex arrays in host memory, M in device memory (m_on_device must be 1)
 *   G_out     DEVICE pointer to 2 * D * D complex FP64 (D = nb Nc NwExt): spin s at offset s D^2,
 *             frequency-block layout -- block (w_r, w_c) of R x R entries (R = nb Nc, row-major,
 *             index b + nb k) at ((w_r NwExt + w_c) R^2); entry (r, c) of block (w_r, w_c) is the
 *             reference's G_(b_r, b_c, s, k_r, k_c, w_r, w_c)
 *   stream    cudaStream_t (as void*), may be null
 * Limits: n <= 512 per spin sector, nb Nc <= 64 with the FP64 front-end's shared-memory tiles
 * within 227 KB per block (for one band: Nc <= 43), and all scratch (about 16 R NwExt (n_0 + n_1)
 * bytes plus small tables) within 48 MiB; larger problems return DCAACC_INVALID_ARG before any
 * GPU work is enqueued.
 * The scratch's device address is looked up on the first call made on each device (with that
 * device current).  Each call uploads its sorted vertex tables from host stack memory, so it must
 * not be called while its stream is being captured into a CUDA graph; such a call returns
 * DCAACC_INVALID_ARG.  All calls share the one scratch array: calls whose GPU work overlaps
 * (different streams, or host threads without ordering) race on it.  Work is enqueued on the
 * stream; synchronise it before reading G_out. */
int dcaacc_tp_compute_g_noalloc(const dcaacc_tp_config* cfg, const double* G0,
                                const dcaacc_sector* sectors, double* G_out, void* stream);

/* Distributed G4: TpAccumulator<Parameters, DistType::LINEAR, GPU> (tp_accumulator_gpu.hpp:350-352,
 * ringG :534-581; the slice bounds G4_[0].get_start() / get_end(), :421-423).  The reference gives
 * each MPI rank one contiguous range of G4's linear index and passes every measurement's G around
 * a ring of ranks so that each rank adds all of them into its range.  Here the ranges are whole
 * momentum transfers: rank r of n_ranks owns the consecutive transfers [first, first + count) of
 * the full transfer list (the first n_k_ex % n_ranks ranks one more), so that its slice is the G4
 * of a handle created with k_ex = that sub-list (all frequency transfers, same channels); its
 * entries are the full G4's with the same (q, wq) bit for bit, since no entry mixes transfers.  A
 * rank feeds its handle every rank's measurements (the walkers' M and configurations are
 * exchanged instead of G: an n x n M crosses the links in place of a D x D G, and recomputing a
 * measurement's G costs less than moving it).  n_ranks must be in 1..n_k_ex.
 *
 * g4_shard writes rank's first transfer position and count.  g4_place_shard copies one channel of
 * that rank's G4 slice (host memory, shard_count complex entries = the sub-list handle's
 * dcaacc_tp_g4_size) into its place in the full G4 of cfg (host memory, full_count complex
 * entries), layout (b1,b2,b3,b4,k1,w1,k2,w2,q,wq) on both sides; only cfg's sizes and transfer
 * counts are read.  Host code only: neither touches a GPU. */
int dcaacc_tp_g4_shard(int32_t n_k_ex, int32_t rank, int32_t n_ranks, int32_t* first, int32_t* count);
int dcaacc_tp_g4_place_shard(const dcaacc_tp_config* cfg, int32_t rank, int32_t n_ranks, const double* shard,
                             size_t shard_count, double* full, size_t full_count);

/* Error-path testing (no reference counterpart; the reference has no device-side failure
 * detection on this path).  Every device wait of the library's kernels is bounded and, when it
 * runs out, sets an error word that the next synchronize / finalize turns into
 * DCAACC_DEVICE_INDEX_ERR while the CUDA context stays usable.
 *
 * set_fault_injection: from the handle's next batch on, the mixed path's tensor-core direct G4
 * term (one band, Nc = 16, all momentum transfers) stops feeding its consumers in its first
 * thread block before pipeline step stop_step (-1: never), and the bounded waits give up after
 * wait_polls polls of up to 2 microseconds each (0: the built-in limit of 2^20 polls).  Drops the
 * handle's CUDA graphs.  G4 is then incomplete: resetAccumulation before measuring again.
 *
 * set_allocation_failure: process-wide; the nth device or pinned-host buffer allocation from now
 * on fails as if memory were exhausted (0 turns it off).  A create call that meets it returns
 * DCAACC_OOM and leaves nothing allocated. */
int dcaacc_tp_set_fault_injection(dcaacc_tp* acc, int32_t stop_step, uint32_t wait_polls);
int dcaacc_set_allocation_failure(int64_t nth);

/* ---------------------------------------------------------------------------------------------
 * Single-particle accumulator (delayed NFFT): SpAccumulator / Dnfft1DGpu.
 * ------------------------------------------------------------------------------------------- */
typedef struct dcaacc_sp_config {
  int32_t n_bands;
  int32_t n_sites;
  int32_t n_sp_freq;          /* positive frequencies of the output mesh (WDmn = 2 * n_sp_freq) */
  double beta;
  const int32_t* r_sub;       /* [n_sites * n_sites], (i,j) at i + Nc*j: index of r_j - r_i */
  int32_t accumulate_m_sqr;   /* also accumulate sign * M^2 (sp_accumulator.hpp:195-196) */
  int32_t max_order;
  int32_t stamping;           /* keep the last measurement's own f(tau) as well, the reference's
                                 stamping_period() > 0 (sp_accumulator_gpu.hpp:160-183) */
} dcaacc_sp_config;

typedef struct dcaacc_sp dcaacc_sp;

/* SpAccumulator(parameters, accumulate_m_sqr) — sp_accumulator_gpu.hpp:134-144. */
int dcaacc_sp_create(const dcaacc_sp_config* cfg, dcaacc_sp** out);
void dcaacc_sp_destroy(dcaacc_sp* acc);

/* resetAccumulation() — sp_accumulator_gpu.hpp:146-158. */
int dcaacc_sp_reset(dcaacc_sp* acc);

/* accumulate(Ms, configs, factor) — sp_accumulator_gpu.hpp:160-195.  sectors: [2]. */
int dcaacc_sp_accumulate(dcaacc_sp* acc, const dcaacc_sector* sectors, double sign);

/* finalize() — sp_accumulator_gpu.hpp:215-229, with the fold / DFT / window division of
 * Dnfft1D::finalize (dnfft_1d.hpp:292-298, :401-489) on the device. */
int dcaacc_sp_finalize(dcaacc_sp* acc);

/* get_sign_times_M_r_w() / get_sign_times_M_r_w_sqr(): complex FP64, layout (b1,s1,b2,s2,r,w),
 * count = (2 nb)^2 Nc (2 n_sp_freq) complex numbers.  Valid after finalize. */
int dcaacc_sp_get_m_r_w(const dcaacc_sp* acc, double* out, size_t count);
int dcaacc_sp_get_m_r_w_sqr(const dcaacc_sp* acc, double* out, size_t count);

/* sumTo(other) — sp_accumulator_gpu.hpp:231-236: other.f_tau += this.f_tau (time domain). */
int dcaacc_sp_sum_to(const dcaacc_sp* acc, dcaacc_sp* other);

/* Single measurement (config.stamping != 0): each accumulate replaces it with that measurement's
 * own f(tau).  get_single_measurement_sign_times_MFunction() — sp_accumulator_gpu.hpp:251-259: the
 * finalize (fold, DFT, window division) of that f(tau), same layout and count as get_m_r_w, computed
 * on each call.  get_single_measurement_sign_times_MFunction_time() — :264-271: the f(tau) itself,
 * FP64 [spin][label = b_i + nb (b_j + nb dr)][8 n_sp_freq + 16 padded times], count =
 * dcaacc_sp_f_tau_size(acc).  clearSingleMeasurement() — sp_accumulator.hpp:286-288: zeroes it.
 * Without stamping these return DCAACC_NOT_READY. */
int dcaacc_sp_get_single_measurement_m_r_w(dcaacc_sp* acc, double* out, size_t count);
int dcaacc_sp_get_single_measurement_f_tau(dcaacc_sp* acc, double* out, size_t count);
int dcaacc_sp_clear_single_measurement(dcaacc_sp* acc);
size_t dcaacc_sp_f_tau_size(const dcaacc_sp* acc);

int dcaacc_sp_set_stream(dcaacc_sp* acc, void* stream);
int dcaacc_sp_synchronize(dcaacc_sp* acc);
size_t dcaacc_sp_device_fingerprint(const dcaacc_sp* acc);
uint64_t dcaacc_sp_kernel_launches(const dcaacc_sp* acc);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* DCAACC_H */
