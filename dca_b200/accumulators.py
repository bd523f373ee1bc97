"""Python mirror of the reference's accumulator interface, over libdcaacc.so.

Method names, argument meaning and error behaviour follow the classes the CT-AUX / CT-INT
solvers call:

* ``TpAccumulator`` -- ``TpAccumulator<Parameters, DistType::NONE, linalg::GPU>``
  (tp_accumulator_gpu.hpp:59-263): ``resetAccumulation``, ``accumulate(M, configs, sign)``,
  ``finalize``, ``sumTo``, ``get_G4``, ``synchronizeCopy``, ``get_stream``, ``deviceFingerprint``.
* ``SpAccumulator`` -- ``SpAccumulator<Parameters, linalg::GPU>`` (sp_accumulator_gpu.hpp:42-130):
  ``resetAccumulation``, ``accumulate``, ``finalize``, ``sumTo``, ``get_sign_times_M_r_w``,
  ``get_sign_times_M_r_w_sqr``, ``synchronizeCopy``, ``deviceFingerprint``.

Misuse raises ``LogicError`` (the reference's ``std::logic_error``), CUDA failures raise
``RuntimeError`` (``std::runtime_error``), allocation failures ``MemoryError`` (``std::bad_alloc``).

Inputs: ``M_pair`` is two column-major ``(n, n)`` float64 matrices, either numpy arrays (host) or
CUDA tensors (device, on the accumulator's device); ``configs`` is two objects with numpy
attributes ``tau``, ``left_band``, ``right_band``, ``left_site``, ``right_site``
(``workloads.Sector`` has them).  G4 is returned per channel as complex128 in the reference layout
(b1, b2, b3, b4, k1, w1, k2, w2, q, wq), first index fastest.
"""

from __future__ import annotations

import ctypes
import dataclasses
import sys
from typing import List, Optional, Sequence

import numpy as np

from . import _native as N
from . import workloads as W


class LogicError(ValueError):
    """Misuse of an accumulator (the reference throws std::logic_error)."""


def _raise(status: int):
    msg = N.lib.dcaacc_last_error().decode(errors="replace")
    if status in (1, 2, 6):
        raise LogicError(f"{N.STATUS_NAMES[status]}: {msg}")
    if status == 3:
        raise MemoryError(msg)
    raise RuntimeError(f"{N.STATUS_NAMES.get(status, status)}: {msg}")


def _check(status: int):
    if status != N.OK:
        _raise(status)


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@dataclasses.dataclass
class TpParameters:
    """What TpAccumulatorBase reads from Parameters and the static domains
    (tp_accumulator_base.hpp:184-208, g4_helper.cu:34-87)."""

    n_bands: int
    n_sites: int
    n_w_half: int
    n_sp_freq: int
    beta: float
    channels: Sequence[int]
    k_ex: Sequence[int]
    w_ex: Sequence[int]
    r_vecs: np.ndarray
    k_vecs: np.ndarray
    a_vecs: np.ndarray
    k_add: np.ndarray  # [i, j] = index of k_i + k_j
    k_sub: np.ndarray  # [i, j] = index of k_j - k_i
    r_sub: Optional[np.ndarray] = None
    precision: int = N.PRECISION_FP64
    max_batch: int = 1
    max_order: int = 512
    accumulators: int = 1
    non_density: bool = False

    @classmethod
    def from_workload(cls, w: W.Workload, cluster: Optional[W.Cluster] = None, **kw) -> "TpParameters":
        cl = cluster if cluster is not None else w.cluster()
        args = dict(
            n_bands=w.nb, n_sites=cl.nc, n_w_half=w.nw_half, n_sp_freq=w.n_sp, beta=w.beta,
            channels=list(w.channels), k_ex=w.exchange_momenta(cl.nc), w_ex=w.exchange_frequencies(),
            r_vecs=cl.r_vecs, k_vecs=cl.k_vecs, a_vecs=w.model.a_vecs(), k_add=cl.k_add,
            k_sub=cl.k_sub, r_sub=cl.r_sub, max_order=w.n_range[1], max_batch=w.batch)
        args.update(kw)
        return cls(**args)

    def g4_shape(self):
        nb, nc, nw = self.n_bands, self.n_sites, 2 * self.n_w_half
        # Fortran-order shape of (b1, b2, b3, b4, k1, w1, k2, w2, q, wq).
        return (nb, nb, nb, nb, nc, nw, nc, nw, len(self.k_ex), len(self.w_ex))


def write_G4(path: str, acc: "TpAccumulator", normalized: bool = True) -> None:
    """Writes each channel's G4 as the dataset "G4_<channel name>" (the names DcaData gives them,
    dca_data.hpp:329-336), shaped (b1, b2, b3, b4, k1, w1, k2, w2, q, wq) in Fortran order like the
    reference's function, into an .npz file (no HDF5 library in this environment).  normalized:
    divided by accumulated sign * beta^2 as the solver does before writing
    (ctaux_cluster_solver.hpp:521-525)."""
    shape = acc.parameters.g4_shape()
    g4 = acc.get_G4_normalized() if normalized else acc.get_G4()
    arrays = {"G4_" + W.CHANNEL_NAMES[ch]: g.reshape(shape, order="F")
              for ch, g in zip(acc.parameters.channels, g4)}
    np.savez(path, **arrays)


# dcaacc_sector as a numpy record (same layout as the C struct and _native.Sector), so that the
# descriptors of a whole batch are filled with a few vectorised assignments.
_SECTOR_FIELDS = ("n", "tau", "left_band", "right_band", "left_site", "right_site", "M", "ldm", "m_on_device")
_SECTOR_DTYPE = np.dtype({
    "names": list(_SECTOR_FIELDS),
    "formats": ["<i4", "<u8", "<u8", "<u8", "<u8", "<u8", "<u8", "<i4", "<i4"],
    "offsets": [getattr(N.Sector, f).offset for f in _SECTOR_FIELDS],
    "itemsize": ctypes.sizeof(N.Sector),
})
_VERTEX_INTS = ("left_band", "right_band", "left_site", "right_site")


def _device_matrix(M, n: int, keep: list, m_dtype=np.float64):
    """(pointer, ldm) of a device matrix of element type m_dtype, made column major if needed."""
    import torch

    want = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
            np.dtype(np.complex128): torch.complex128, np.dtype(np.complex64): torch.complex64}[np.dtype(m_dtype)]
    if M.dtype != want:
        raise LogicError(f"device M must be {want}")
    if n and not (M.stride(0) == 1 and M.stride(1) >= max(n, 1)):
        M = M.t().contiguous().t()  # column major
        keep.append(M)
    return M.data_ptr(), (max(M.stride(1), 1) if n else 1)


def _make_sectors(M_pair, configs, keep: list, count: int = 1, m_dtype=np.float64):
    """Sector descriptors for `count` measurements (M_pair / configs hold 2 * count entries), as a
    pointer to dcaacc_sector records.  The vertex arrays of all sectors are packed into one
    float64 and one int32 buffer; everything the pointers refer to is appended to `keep`."""
    ns = 2 * count
    taus = [c.tau for c in configs]
    lens = np.fromiter((len(t) for t in taus), np.int64, ns)
    offs = np.zeros(ns, np.int64)
    np.cumsum(lens[:-1], out=offs[1:])
    total = int(lens.sum())
    width = max(total, 1)
    tau_all = np.zeros(width, np.float64)
    ints = np.zeros((len(_VERTEX_INTS), width), np.int32)
    if total:
        np.concatenate(taus, out=tau_all[:total], casting="unsafe")
        for k, name in enumerate(_VERTEX_INTS):
            np.concatenate([getattr(c, name) for c in configs], out=ints[k, :total], casting="unsafe")
    rec = np.zeros(ns, _SECTOR_DTYPE)
    rec["n"] = lens
    rec["tau"] = tau_all.ctypes.data + 8 * offs
    for k, name in enumerate(_VERTEX_INTS):
        rec[name] = ints.ctypes.data + 4 * (k * width + offs)
    torch = sys.modules.get("torch")
    if torch is not None and all(type(M) is torch.Tensor and M.is_cuda for M in M_pair):
        # Device matrices (the walkers' M): one pass of attribute reads; a matrix that is not
        # column major float64 goes through _device_matrix.
        f64 = torch.float64 if np.dtype(m_dtype) == np.float64 else None
        ptrs, lds = [], []
        for M, n in zip(M_pair, lens.tolist()):
            st = M.stride()
            if M.dtype is f64 and (n == 0 or (st[0] == 1 and st[1] >= n)):
                ptrs.append(M.data_ptr())
                lds.append(max(st[1], 1) if n else 1)
            else:
                p_, l_ = _device_matrix(M, n, keep, m_dtype)
                ptrs.append(p_)
                lds.append(l_)
        rec["M"] = ptrs
        rec["ldm"] = lds
        rec["m_on_device"] = 1
    else:
        ptr = np.zeros(ns, np.uint64)
        ldm = np.ones(ns, np.int32)
        dev = np.zeros(ns, np.int32)
        for s in range(ns):
            M, n = M_pair[s], int(lens[s])
            if hasattr(M, "is_cuda") and M.is_cuda:
                ptr[s], ldm[s] = _device_matrix(M, n, keep, m_dtype)
                dev[s] = 1
            else:
                Mh = np.asfortranarray(np.asarray(M, m_dtype)) if n else np.zeros((1, 1), m_dtype, order="F")
                keep.append(Mh)
                ptr[s] = Mh.ctypes.data
                ldm[s] = max(n, 1)
        rec["M"] = ptr
        rec["ldm"] = ldm
        rec["m_on_device"] = dev
    keep.extend((tau_all, ints, rec, M_pair))
    return rec.ctypes.data_as(ctypes.POINTER(N.Sector))


class TpAccumulator:
    """Two-particle accumulator (see module docstring)."""

    def __init__(self, G0: np.ndarray, parameters: TpParameters, thread_id: int = 0):
        p = parameters
        self.parameters = p
        self.thread_id = thread_id
        self._keep = [
            np.ascontiguousarray(p.k_ex, np.int32), np.ascontiguousarray(p.w_ex, np.int32),
            np.ascontiguousarray(p.channels, np.int32),
            np.ascontiguousarray(p.r_vecs, np.float64), np.ascontiguousarray(p.k_vecs, np.float64),
            np.ascontiguousarray(p.a_vecs, np.float64),
            # Tables are column major: element (i, j) at i + Nc j.
            np.ascontiguousarray(np.asarray(p.k_add, np.int32).T),
            np.ascontiguousarray(np.asarray(p.k_sub, np.int32).T),
        ]
        k_ex, w_ex, ch, rv, kv, av, kadd, ksub = self._keep
        cfg = N.TpConfig(
            p.n_bands, p.n_sites, p.n_w_half, p.n_sp_freq, len(k_ex), _iptr(k_ex), len(w_ex),
            _iptr(w_ex), len(ch), _iptr(ch), p.beta, _dptr(rv), _dptr(kv), _dptr(av), _iptr(kadd),
            _iptr(ksub), int(p.non_density), p.precision, p.max_batch, p.max_order, p.accumulators)
        g0 = np.ascontiguousarray(G0, np.complex128).reshape(-1)
        expect = (2 * p.n_bands) ** 2 * p.n_sites * 2 * p.n_sp_freq
        if g0.size != expect:
            raise LogicError(f"G0 has {g0.size} entries, expected {expect}")
        self._h = ctypes.c_void_p()
        _check(N.lib.dcaacc_tp_create(ctypes.byref(cfg), g0.view(np.float64).ctypes.data_as(
            ctypes.POINTER(ctypes.c_double)), ctypes.byref(self._h)))
        self._g4: Optional[List[np.ndarray]] = None

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(N, "lib", None)  # None while the interpreter shuts down
        if h and lib is not None:
            lib.dcaacc_tp_destroy(h)
            self._h = None

    # -- reference method set ----------------------------------------------------------------
    def resetAccumulation(self, dca_loop: int = 0):
        """Zeroes G4 (a G4 shared with share_G4_with: once per dca_loop) and arms accumulate."""
        _check(N.lib.dcaacc_tp_reset_loop(self._h, int(dca_loop)))
        self._g4 = None

    def share_G4_with(self, owner: "TpAccumulator"):
        """Accumulate into owner's G4 (the reference's accumulator threads share one device G4)."""
        _check(N.lib.dcaacc_tp_share_g4(self._h, owner._h))

    def accumulate(self, M_pair, configs, sign: int) -> float:
        keep: list = []
        secs = _make_sectors(M_pair, configs, keep)
        flops = ctypes.c_double(0)
        _check(N.lib.dcaacc_tp_accumulate(self._h, secs, int(sign), ctypes.byref(flops)))
        self._last_inputs = keep  # device M must outlive the queued work
        return flops.value

    _SCALARS = {np.dtype(np.float64): 0, np.dtype(np.float32): 1, np.dtype(np.complex128): 2,
                np.dtype(np.complex64): 3}

    @staticmethod
    def _m_dtype(M0):
        return np.dtype(str(M0.dtype).replace("torch.", "")) if hasattr(M0, "is_cuda") else np.asarray(M0).dtype

    def accumulate_typed(self, M_pair, configs, sign, m_dtype=None) -> float:
        """accumulate for the reference's other SpScalar / SignType instantiations
        (dcaacc_tp_accumulate_typed): M of element type m_dtype (by default that of M_pair[0]:
        float64, float32, complex128 or complex64) and a sign that may be complex.  Complex M or a
        sign with an imaginary part raise LogicError (DCAACC_UNSUPPORTED)."""
        return self.accumulate_batch_typed([M_pair], [configs], [sign], m_dtype)

    def accumulate_batch_typed(self, Ms, configs, signs, m_dtype=None) -> float:
        """accumulate_typed for several measurements in one call (Ms[m], configs[m]: measurement m's
        pairs, signs[m] its sign)."""
        count = len(signs)
        m_dtype = np.dtype(m_dtype if m_dtype is not None else self._m_dtype(Ms[0][0]))
        keep: list = []
        secs = _make_sectors([M for pair in Ms for M in pair], [c for pair in configs for c in pair], keep, count,
                             m_dtype=m_dtype)
        sg = np.asarray(signs, np.complex128)
        sr, si = np.ascontiguousarray(sg.real), np.ascontiguousarray(sg.imag)
        flops = ctypes.c_double(0)
        _check(N.lib.dcaacc_tp_accumulate_typed(self._h, count, secs, self._SCALARS[m_dtype], _dptr(sr), _dptr(si),
                                                ctypes.byref(flops)))
        self._last_inputs = keep
        return flops.value

    def accumulate_batch(self, Ms, configs, signs) -> float:
        """Several measurements in one call (dcaacc_tp_accumulate_batch): Ms[m] and configs[m] are
        measurement m's pairs, signs[m] its sign.  Same result as calling accumulate per
        measurement."""
        count = len(signs)
        keep: list = []
        secs = _make_sectors([M for pair in Ms for M in pair], [c for pair in configs for c in pair], keep,
                             count)
        sg = np.ascontiguousarray(signs, np.int32)
        flops = ctypes.c_double(0)
        _check(N.lib.dcaacc_tp_accumulate_batch(self._h, count, secs, _iptr(sg), ctypes.byref(flops)))
        self._last_inputs = keep
        return flops.value

    def flush(self):
        _check(N.lib.dcaacc_tp_flush(self._h))

    def finalize(self):
        _check(N.lib.dcaacc_tp_finalize(self._h))
        size = N.lib.dcaacc_tp_g4_size(self._h)
        out = []
        for c in range(len(self.parameters.channels)):
            g = np.empty(size, np.complex128)
            _check(N.lib.dcaacc_tp_get_g4(self._h, c, g.view(np.float64).ctypes.data_as(
                ctypes.POINTER(ctypes.c_double)), size))
            out.append(g)
        self._g4 = out

    def get_G4(self) -> List[np.ndarray]:
        if self._g4 is None:
            raise LogicError("There is no G4 stored in this class.")
        return self._g4

    def sign_sum(self):
        """(sum of the measurement signs since resetAccumulation, number of measurements)."""
        s, n = ctypes.c_double(), ctypes.c_uint64()
        _check(N.lib.dcaacc_tp_sign_sum(self._h, ctypes.byref(s), ctypes.byref(n)))
        return s.value, n.value

    def get_G4_normalized(self) -> List[np.ndarray]:
        """G4 / (accumulated sign * beta^2), the solver's normalisation (after finalize)."""
        size = N.lib.dcaacc_tp_g4_size(self._h)
        out = []
        for c in range(len(self.parameters.channels)):
            g = np.empty(size, np.complex128)
            _check(N.lib.dcaacc_tp_get_g4_normalized(self._h, c, g.view(np.float64).ctypes.data_as(
                ctypes.POINTER(ctypes.c_double)), size))
            out.append(g)
        return out

    def sumTo(self, other: "TpAccumulator"):
        _check(N.lib.dcaacc_tp_sum_to(self._h, other._h))
        self._g4 = None

    def get_G(self, spin: int) -> np.ndarray:
        """G of the last processed measurement (FP64 mode), layout (b1, b2, k1, k2, w1, w2)."""
        p = self.parameters
        ext = max(abs(w) for w in p.w_ex)
        nwe = 2 * p.n_w_half + 2 * ext
        size = (p.n_bands * p.n_sites * nwe) ** 2
        g = np.empty(size, np.complex128)
        _check(N.lib.dcaacc_tp_get_g(self._h, spin, g.view(np.float64).ctypes.data_as(
            ctypes.POINTER(ctypes.c_double)), size))
        return g

    def synchronizeCopy(self):
        _check(N.lib.dcaacc_tp_synchronize(self._h))

    def syncStreams(self, event=None):
        self.synchronizeCopy()

    def get_stream(self) -> int:
        return N.lib.dcaacc_tp_get_stream(self._h) or 0

    def set_stream(self, stream_handle: int):
        _check(N.lib.dcaacc_tp_set_stream(self._h, ctypes.c_void_p(stream_handle)))

    def deviceFingerprint(self) -> int:
        return N.lib.dcaacc_tp_device_fingerprint(self._h)

    @staticmethod
    def staticDeviceFingerprint() -> int:
        """Device bytes held process-wide (the allocation-free entry point's static scratch)."""
        return N.lib.dcaacc_tp_static_device_fingerprint()

    def kernel_launches(self) -> int:
        return N.lib.dcaacc_tp_kernel_launches(self._h)

    def mirror_mode(self) -> int:
        """Bit 0: half of G computed (mirror symmetry); bit 1: half of the G4 tiles accumulated."""
        return N.lib.dcaacc_tp_mirror_mode(self._h)

    STAGES = ("twiddle", "row_transform", "col_transform", "update_g4")

    def enable_timing(self, on: bool = True):
        _check(N.lib.dcaacc_tp_enable_timing(self._h, int(on)))

    def stage_times(self):
        """{stage: (cumulative ms, launches)} since enable_timing."""
        ms = (ctypes.c_double * 4)()
        cnt = (ctypes.c_uint64 * 4)()
        _check(N.lib.dcaacc_tp_stage_times(self._h, ms, cnt, 4))
        return {name: (ms[i], cnt[i]) for i, name in enumerate(self.STAGES)}

    def set_graphs(self, on: bool = True):
        """Replay each batch shape's kernel sequence from a CUDA graph (mixed path; on by default)."""
        _check(N.lib.dcaacc_tp_set_graphs(self._h, int(on)))

    def graph_stats(self):
        """(graphs captured, batches replayed from a graph) since creation."""
        cap, rep = ctypes.c_uint64(), ctypes.c_uint64()
        _check(N.lib.dcaacc_tp_graph_stats(self._h, ctypes.byref(cap), ctypes.byref(rep)))
        return cap.value, rep.value

    def tuning_settled(self) -> bool:
        """No problem shape is still being explored by the launch-shape tuner."""
        return bool(N.lib.dcaacc_tp_tuning_settled(self._h))

    def tuning_report(self) -> str:
        """One line per tuned launch: key, candidates, choice, median ms per candidate."""
        n = ctypes.c_size_t()
        _check(N.lib.dcaacc_tp_tuning_report(self._h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        _check(N.lib.dcaacc_tp_tuning_report(self._h, buf, n.value + 1, ctypes.byref(n)))
        return buf.value.decode()

    def peek_G4(self, channel: int, offset: int, count: int) -> np.ndarray:
        out = np.empty(count, np.complex128)
        _check(N.lib.dcaacc_tp_peek_g4(self._h, channel, offset, count, _dptr(out.view(np.float64))))
        return out

    def peek_G4_async(self, channel: int, offset: int, out: np.ndarray):
        """Enqueues the read of len(out) entries into out (complex128, ideally pinned); they are
        there after synchronizeCopy().  The caller keeps out alive until then."""
        if out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous complex128 array")
        _check(N.lib.dcaacc_tp_peek_g4_async(self._h, channel, offset, out.size, _dptr(out.view(np.float64))))

    def set_fault_injection(self, stop_step: int = -1, wait_polls: int = 0):
        """Error-path tests: the tensor-core direct G4 term's first block stops feeding its
        consumers before pipeline step stop_step (-1: never), and bounded device waits give up after
        wait_polls polls (0: built-in limit); the next synchronizeCopy / finalize raises."""
        _check(N.lib.dcaacc_tp_set_fault_injection(self._h, stop_step, wait_polls))

    def num_channels(self) -> int:
        return len(self.parameters.channels)


@dataclasses.dataclass
class SpParameters:
    n_bands: int
    n_sites: int
    n_sp_freq: int
    beta: float
    r_sub: np.ndarray  # [i, j] = index of r_j - r_i
    max_order: int = 512
    stamping: bool = False  # keep the last measurement's own f(tau) (stamping_period() > 0)

    @classmethod
    def from_workload(cls, w: W.Workload, cluster: Optional[W.Cluster] = None, **kw):
        cl = cluster if cluster is not None else w.cluster()
        args = dict(n_bands=w.nb, n_sites=cl.nc, n_sp_freq=w.n_sp, beta=w.beta, r_sub=cl.r_sub,
                    max_order=w.n_range[1])
        args.update(kw)
        return cls(**args)


class SpAccumulator:
    """Single-particle accumulator (see module docstring)."""

    def __init__(self, parameters: SpParameters, accumulate_m_squared: bool = False):
        p = parameters
        self.parameters = p
        self._rsub = np.ascontiguousarray(np.asarray(p.r_sub, np.int32).T)
        cfg = N.SpConfig(p.n_bands, p.n_sites, p.n_sp_freq, p.beta, _iptr(self._rsub),
                         int(accumulate_m_squared), p.max_order, int(p.stamping))
        self._sqr = bool(accumulate_m_squared)
        self._h = ctypes.c_void_p()
        _check(N.lib.dcaacc_sp_create(ctypes.byref(cfg), ctypes.byref(self._h)))

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(N, "lib", None)  # None while the interpreter shuts down
        if h and lib is not None:
            lib.dcaacc_sp_destroy(h)
            self._h = None

    def resetAccumulation(self):
        _check(N.lib.dcaacc_sp_reset(self._h))

    def accumulate(self, M_pair, configs, factor: float):
        keep: list = []
        secs = _make_sectors(M_pair, configs, keep)
        _check(N.lib.dcaacc_sp_accumulate(self._h, secs, float(factor)))
        self._last_inputs = keep

    def finalize(self):
        _check(N.lib.dcaacc_sp_finalize(self._h))

    def _get(self, sqr: bool) -> np.ndarray:
        p = self.parameters
        size = (2 * p.n_bands) ** 2 * p.n_sites * 2 * p.n_sp_freq
        out = np.empty(size, np.complex128)
        fn = N.lib.dcaacc_sp_get_m_r_w_sqr if sqr else N.lib.dcaacc_sp_get_m_r_w
        _check(fn(self._h, out.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)), size))
        return out

    def get_sign_times_M_r_w(self) -> np.ndarray:
        return self._get(False)

    def get_sign_times_M_r_w_sqr(self) -> np.ndarray:
        return self._get(True)

    def get_single_measurement_sign_times_MFunction(self) -> np.ndarray:
        """M(r, w) of the last measurement alone (stamping), computed on each call."""
        p = self.parameters
        size = (2 * p.n_bands) ** 2 * p.n_sites * 2 * p.n_sp_freq
        out = np.empty(size, np.complex128)
        _check(N.lib.dcaacc_sp_get_single_measurement_m_r_w(
            self._h, out.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)), size))
        return out

    def get_single_measurement_sign_times_MFunction_time(self) -> np.ndarray:
        """The last measurement's f(tau): [spin][label][padded time], FP64."""
        size = N.lib.dcaacc_sp_f_tau_size(self._h)
        out = np.empty(size, np.float64)
        _check(N.lib.dcaacc_sp_get_single_measurement_f_tau(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), size))
        p = self.parameters
        return out.reshape(2, p.n_bands ** 2 * p.n_sites, -1)

    def clearSingleMeasurement(self):
        _check(N.lib.dcaacc_sp_clear_single_measurement(self._h))

    def sumTo(self, other: "SpAccumulator"):
        _check(N.lib.dcaacc_sp_sum_to(self._h, other._h))

    def synchronizeCopy(self):
        _check(N.lib.dcaacc_sp_synchronize(self._h))

    def deviceFingerprint(self) -> int:
        return N.lib.dcaacc_sp_device_fingerprint(self._h)

    def kernel_launches(self) -> int:
        return N.lib.dcaacc_sp_kernel_launches(self._h)
