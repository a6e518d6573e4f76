"""empi_b200: Matching Pursuit with optimal Gabor dictionaries on NVIDIA B200.

The compute path is the sm_100a library ``libempi_b200.so`` (built in-tree by
``empi_b200.build``), reached through its C ABI (include/empi_b200.h) with
ctypes.  There is no CPU fallback: if the library or a CUDA device is
missing, calls raise.

The Python surface mirrors the reference's decomposition seam
(inc/classes.hpp, inc/gabor.hpp, inc/mmp.hpp of empi) so callers can switch
over one class at a time:

* ``GaborWorkspaceBuilder(energyError, scaleMin, scaleMax, freqMax)
  .prepareWorkspace(freqSampling, channelCount, sampleCount, constraint)``
* ``GaborWorkspace.compute / findBestMatch / getAtomCount / subtractAtom`` and
  the static ``subtractAtomFromSignal(atom, signal, fit)``
* ``SmpDecomposition / Mmp1Decomposition / Mmp2Decomposition /
  Mmp3Decomposition .compute(settings, workspace, signal)`` -- the whole MP
  loop of one epoch on the device (``decompose_epochs`` runs many at once)

Atoms carry the reference's six params: modulus, amplitude, t*fs, s*fs,
f*2/fs, phase (src/gabor.cpp:123-130).
"""
from __future__ import annotations

import atexit
import ctypes
import math
import os
import weakref
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libempi_b200.so")

ATOM_GABOR = 13
SMP, MMP1, MMP2, MMP3 = 0, 1, 2, 3
_VARIANTS = {"smp": SMP, "mmp1": MMP1, "mmp2": MMP2, "mmp3": MMP3}


class EngineOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("stream", ctypes.c_void_p), ("transform_cap", ctypes.c_int),
                ("candidate_band", ctypes.c_double), ("candidate_capacity", ctypes.c_int),
                ("iterations_per_graph", ctypes.c_int), ("timing", ctypes.c_int), ("tune_cache", ctypes.c_char_p),
                ("persistent", ctypes.c_int), ("wait_limit_ms", ctypes.c_int), ("test_unreachable_wait", ctypes.c_int)]


class Dictionary(ctypes.Structure):
    _fields_ = [("energy_error", ctypes.c_double), ("scale_min", ctypes.c_double),
                ("scale_max", ctypes.c_double), ("freq_max", ctypes.c_double)]


class Settings(ctypes.Structure):
    _fields_ = [("iteration_max", ctypes.c_int), ("residual_energy", ctypes.c_double)]


class Epoch(ctypes.Structure):
    _fields_ = [("fs", ctypes.c_double), ("channels", ctypes.c_int), ("samples", ctypes.c_int),
                ("data", ctypes.c_void_p)]


class BatchStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("atoms", ctypes.c_int), ("refresh_units", ctypes.c_longlong),
                ("windows", ctypes.c_longlong), ("fft_flops", ctypes.c_double),
                ("algorithmic_bytes", ctypes.c_double), ("refresh_ms", ctypes.c_double),
                ("refresh_launches", ctypes.c_int), ("kernel_launches", ctypes.c_int),
                ("candidate_bins", ctypes.c_int), ("run_ms", ctypes.c_double), ("transform_cap", ctypes.c_int),
                ("iterations_per_graph", ctypes.c_int), ("wide_mask", ctypes.c_int), ("tuned", ctypes.c_int),
                ("sizes_mask", ctypes.c_int), ("probe_dirty_slots", ctypes.c_longlong),
                ("probe_needed_slots", ctypes.c_longlong), ("probe_dirty_work", ctypes.c_double),
                ("probe_needed_work", ctypes.c_double), ("proposal_iterations", ctypes.c_int),
                ("proposal_hits", ctypes.c_int), ("persistent", ctypes.c_int)]


EXPORTS = [
    "empi_last_error", "empi_status_string", "empi_abi_version", "empi_engine_opts_default",
    "empi_engine_create", "empi_engine_destroy", "empi_dictionary_size", "empi_dictionary_scales",
    "empi_workspace_create", "empi_workspace_destroy", "empi_workspace_compute", "empi_workspace_find_best",
    "empi_workspace_atom_count", "empi_workspace_subtract_atom", "empi_workspace_energy_map",
    "empi_subtract_atom_from_signal", "empi_batch_create", "empi_batch_destroy", "empi_batch_load",
    "empi_batch_run", "empi_batch_atoms", "empi_batch_total_energy", "empi_batch_get_stats",
    "empi_decompose", "empi_run_config", "empi_book_write", "empi_subtract_atom_from_signal_noalloc",
    "empi_dictionary_error_bounds", "empi_tune_lookup", "empi_batch_probe_proposal", "empi_batch_set_proposal",
    "empi_batch_collect_pairs", "empi_batch_pairs", "empi_proposal_parameter_count", "empi_proposal_scores",
    "empi_proposal_gradients", "empi_proposal_train", "empi_batch_tree",
]

_lib = None


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Loads libempi_b200.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or os.environ.get("EMPI_B200_LIB") or LIB_PATH
    if not os.path.exists(p):
        raise OSError(f"{p} is missing: build it with `python -m empi_b200.build`")
    L = ctypes.CDLL(p)
    vp, ip, dp, fp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), \
        ctypes.POINTER(ctypes.c_float)
    L.empi_last_error.restype = ctypes.c_char_p
    L.empi_status_string.restype = ctypes.c_char_p
    L.empi_status_string.argtypes = [ctypes.c_int]
    L.empi_engine_opts_default.argtypes = [ctypes.POINTER(EngineOpts)]
    L.empi_engine_create.argtypes = [ctypes.POINTER(EngineOpts), ctypes.POINTER(vp)]
    L.empi_engine_destroy.argtypes = [vp]
    L.empi_engine_destroy.restype = None
    L.empi_dictionary_size.argtypes = [ctypes.POINTER(Dictionary), ctypes.c_double, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_uint64), ip]
    L.empi_dictionary_scales.argtypes = [ctypes.POINTER(Dictionary), ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                         dp, ip, ip, ip, ip]
    L.empi_dictionary_error_bounds.argtypes = [ctypes.POINTER(Dictionary), ctypes.c_double, ctypes.c_int,
                                               ctypes.c_int, fp, fp, fp, ip, ip, ip]
    L.empi_tune_lookup.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_double, ip, ip, ip, ip]
    L.empi_workspace_create.argtypes = [vp, ctypes.POINTER(Dictionary), ctypes.c_double, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.empi_workspace_destroy.argtypes = [vp]
    L.empi_workspace_destroy.restype = None
    L.empi_workspace_compute.argtypes = [vp, dp]
    L.empi_workspace_find_best.argtypes = [vp, dp, ip]
    L.empi_workspace_atom_count.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
    L.empi_workspace_subtract_atom.argtypes = [vp, dp, dp, ctypes.c_int]
    L.empi_workspace_energy_map.argtypes = [vp, ctypes.c_int, fp]
    L.empi_subtract_atom_from_signal.argtypes = [vp, dp, dp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
    L.empi_subtract_atom_from_signal_noalloc.argtypes = [ctypes.c_int, vp, dp, dp, ctypes.c_int, ctypes.c_double,
                                                         ctypes.c_int]
    L.empi_batch_create.argtypes = [vp, ctypes.c_int, ctypes.POINTER(Dictionary), ctypes.POINTER(Settings),
                                    ctypes.POINTER(Epoch), ctypes.c_int, ctypes.POINTER(vp)]
    L.empi_batch_destroy.argtypes = [vp]
    L.empi_batch_destroy.restype = None
    L.empi_batch_load.argtypes = [vp, ctypes.POINTER(Epoch)]
    L.empi_batch_run.argtypes = [vp]
    L.empi_batch_atoms.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ip, dp, ip]
    L.empi_batch_total_energy.argtypes = [vp, ctypes.c_int, dp]
    L.empi_batch_get_stats.argtypes = [vp, ctypes.POINTER(BatchStats)]
    L.empi_batch_probe_proposal.argtypes = [vp, ctypes.c_int]
    L.empi_batch_set_proposal.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
    L.empi_batch_collect_pairs.argtypes = [vp, ctypes.c_int]
    L.empi_batch_pairs.argtypes = [vp, ctypes.c_int, fp, ip, ip]
    u64p = ctypes.POINTER(ctypes.c_uint64)
    L.empi_batch_tree.argtypes = [vp, ctypes.c_int, ctypes.c_longlong, u64p, ctypes.POINTER(ctypes.c_longlong),
                                  ctypes.c_int, u64p, ctypes.POINTER(ctypes.c_uint32), ip]
    L.empi_proposal_parameter_count.restype = ctypes.c_int
    L.empi_proposal_scores.argtypes = [ctypes.c_int, fp, ctypes.c_int, fp, ctypes.c_int, fp]
    L.empi_proposal_gradients.argtypes = [ctypes.c_int, fp, ip, ctypes.c_int, fp, fp, fp]
    L.empi_proposal_train.argtypes = [ctypes.c_int, fp, ip, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_float, ctypes.c_float, ctypes.c_uint, fp, fp]
    L.empi_decompose.argtypes = [vp, ctypes.c_int, ctypes.POINTER(Dictionary), ctypes.POINTER(Settings),
                                 ctypes.POINTER(Epoch), ctypes.c_int, ctypes.c_int, dp, ip]
    L.empi_run_config.argtypes = [ctypes.c_char_p, ctypes.POINTER(EngineOpts)]
    L.empi_book_write.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                  ctypes.c_int, fp, ctypes.c_int, dp, ip]
    _lib = L
    return L


class EmpiError(RuntimeError):
    """A failed C-ABI call; ``message`` is the camelCase text (e.g. energyMapIsEmpty)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status
        self.message = message


def _check(st: int) -> None:
    if st != 0:
        L = load_library()
        msg = (L.empi_last_error() or b"").decode() or L.empi_status_string(st).decode()
        raise EmpiError(st, msg)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


# ---------------------------------------------------------------- engine


class Engine:
    """A device context: CUDA ordinal, stream and tuning options."""

    def __init__(self, device: int = 0, stream: int | None = None, transform_cap: int = 0,
                 candidate_band: float = 0.0, candidate_capacity: int = 0, iterations_per_graph: int = 0,
                 timing: bool = False, tune_cache: str | None = None, persistent: int = -1,
                 wait_limit_ms: int = 0, test_unreachable_wait: bool = False):
        L = load_library()
        o = EngineOpts()
        L.empi_engine_opts_default(ctypes.byref(o))
        o.device = device
        o.stream = stream
        if transform_cap:
            o.transform_cap = transform_cap
        if candidate_band:
            o.candidate_band = candidate_band
        if candidate_capacity:
            o.candidate_capacity = candidate_capacity
        if iterations_per_graph:
            o.iterations_per_graph = iterations_per_graph
        o.timing = int(timing)
        o.tune_cache = os.fsencode(tune_cache) if tune_cache else None
        o.persistent = int(persistent)
        if wait_limit_ms:
            o.wait_limit_ms = int(wait_limit_ms)
        o.test_unreachable_wait = int(bool(test_unreachable_wait))
        h = ctypes.c_void_p()
        _check(L.empi_engine_create(ctypes.byref(o), ctypes.byref(h)))
        self.handle = h
        self.opts = o
        self._children = weakref.WeakSet()
        _live_engines.add(self)

    def _adopt(self, child):
        self._children.add(child)

    def close(self):
        """Destroys the engine after every workspace and batch created on it
        (the C ABI requires children to go first)."""
        if getattr(self, "handle", None):
            for c in list(self._children):
                c.close()
            load_library().empi_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_engine = None
_live_engines = weakref.WeakSet()


@atexit.register
def _close_all():
    # release device objects before the interpreter (and the CUDA runtime) tear down
    for e in list(_live_engines):
        try:
            e.close()
        except Exception:
            pass


def default_engine() -> Engine:
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine()
    return _default_engine


# ---------------------------------------------------------------- data types


@dataclass
class Atom:
    """struct Atom, inc/base.hpp:26-29."""
    params: list
    type: int = ATOM_GABOR


@dataclass
class DecompositionSettings:
    """inc/classes.hpp:84-87."""
    iterationMax: int
    residualEnergy: float


def _dictionary(energyError, scaleMin, scaleMax, freqMax) -> Dictionary:
    return Dictionary(float(energyError), float(scaleMin), float(scaleMax), float(freqMax))


def dictionary_scales(energyError, freqSampling, sampleCount, scaleMin=0.0, scaleMax=math.inf,
                      freqMax=math.inf):
    """(s, Nfft, fCount, tCount) per scale, as GaborWorkspaceBuilder builds them."""
    L = load_library()
    d = _dictionary(energyError, scaleMin, scaleMax, freqMax)
    cap = 4096
    s = np.zeros(cap)
    nf, fc, tc = (np.zeros(cap, np.int32) for _ in range(3))
    n = ctypes.c_int()
    _check(L.empi_dictionary_scales(ctypes.byref(d), freqSampling, int(sampleCount), cap, _dp(s), _ip(nf),
                                    _ip(fc), _ip(tc), ctypes.byref(n)))
    return [(float(s[i]), int(nf[i]), int(fc[i]), int(tc[i])) for i in range(n.value)]


def dictionary_error_bounds(energyError, freqSampling, sampleCount, scaleMin=0.0, scaleMax=math.inf,
                            freqMax=math.inf):
    """Per scale: (bnd_d, rho, tph, klo, khi) of the engine's certified FP32
    error bound (include/empi_b200.h, empi_dictionary_error_bounds)."""
    L = load_library()
    d = _dictionary(energyError, scaleMin, scaleMax, freqMax)
    cap = 4096
    bd, rho, tph = (np.zeros(cap, np.float32) for _ in range(3))
    klo, khi = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
    n = ctypes.c_int()
    fp = ctypes.POINTER(ctypes.c_float)
    _check(L.empi_dictionary_error_bounds(ctypes.byref(d), freqSampling, int(sampleCount), cap,
                                          bd.ctypes.data_as(fp), rho.ctypes.data_as(fp), tph.ctypes.data_as(fp),
                                          _ip(klo), _ip(khi), ctypes.byref(n)))
    return [(float(bd[i]), float(rho[i]), float(tph[i]), int(klo[i]), int(khi[i])) for i in range(n.value)]


def tune_lookup(path, mode, channels, fs, samples, energy_error):
    """(transform_cap, iterations_per_graph, wide_mask, persistent) of the tune
    cache's entry for a workload (persistent -1: not tuned), or None
    (empi_tune_lookup; no GPU needed)."""
    L = load_library()
    cap, k, wide, pers = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    st = L.empi_tune_lookup(os.fsencode(path), int(mode), int(channels), float(fs), int(samples),
                            float(energy_error), ctypes.byref(cap), ctypes.byref(k), ctypes.byref(wide),
                            ctypes.byref(pers))
    if st != 0:
        msg = (L.empi_last_error() or b"").decode()
        if msg == "noTunedEntry":
            return None
        raise EmpiError(st, msg)
    return cap.value, k.value, wide.value, pers.value


# ---------------------------------------------------------------- workspace seam


class GaborWorkspaceBuilder:
    """inc/gabor.hpp:77-88 / src/gabor.cpp:213-252."""

    def __init__(self, energyError, scaleMin=0.0, scaleMax=math.inf, freqMax=math.inf, engine=None):
        self.energyError = float(energyError)
        self.scaleMin = float(scaleMin)
        self.scaleMax = float(scaleMax)
        self.freqMax = float(freqMax)
        self.engine = engine

    def prepareWorkspace(self, freqSampling, channelCount, sampleCount, constraint=None):
        """constraint: None, or MMP1 (the common-phase constraint of Mmp1Decomposition)."""
        return GaborWorkspace(self, float(freqSampling), int(channelCount), int(sampleCount),
                              MMP1 if constraint in (MMP1, "mmp1") else MMP3)


class GaborWorkspace:
    """A C-channel workspace on the device (Workspace, inc/classes.hpp:63-75)."""

    def __init__(self, builder, fs, C, N, variant):
        self.builder = builder
        self.engine = builder.engine or default_engine()
        self.freqSampling, self.channelCount, self.sampleCount = fs, C, N
        self.variant = variant
        L = load_library()
        d = _dictionary(builder.energyError, builder.scaleMin, builder.scaleMax, builder.freqMax)
        h = ctypes.c_void_p()
        _check(L.empi_workspace_create(self.engine.handle, ctypes.byref(d), fs, C, N, variant, ctypes.byref(h)))
        self.handle = h
        self.engine._adopt(self)

    def close(self):
        if getattr(self, "handle", None) and getattr(self.engine, "handle", None):
            load_library().empi_workspace_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compute(self, signal):
        """Workspace::compute(MultiSignal): signal is (C, N) float64 (or a list of channels)."""
        x = np.ascontiguousarray(np.asarray(signal, np.float64).reshape(self.channelCount, self.sampleCount))
        _check(load_library().empi_workspace_compute(self.handle, _dp(x)))

    def findBestMatch(self, with_index=False):
        """Workspace::findBestMatch() -> one Atom per channel."""
        p = np.zeros((self.channelCount, 6))
        idx = np.zeros(3, np.int32)
        _check(load_library().empi_workspace_find_best(self.handle, _dp(p), _ip(idx)))
        atoms = [Atom(list(map(float, p[c]))) for c in range(self.channelCount)]
        return (atoms, tuple(int(v) for v in idx)) if with_index else atoms

    def getAtomCount(self):
        n = ctypes.c_uint64()
        _check(load_library().empi_workspace_atom_count(self.handle, ctypes.byref(n)))
        return n.value

    def subtractAtom(self, atom, signal, channel):
        """Workspace::subtractAtom: signal (N float64 array) is updated in place."""
        p = np.ascontiguousarray(np.asarray(atom.params if isinstance(atom, Atom) else atom, np.float64))
        if not (isinstance(signal, np.ndarray) and signal.dtype == np.float64 and signal.flags.c_contiguous):
            raise TypeError("signal must be a contiguous float64 array (updated in place)")
        _check(load_library().empi_workspace_subtract_atom(self.handle, _dp(p), _dp(signal), int(channel)))

    def energy_map(self, scale):
        """FP32 energies [f, t] the engine ranks for one scale (parity checks)."""
        s = dictionary_scales(self.builder.energyError, self.freqSampling, self.sampleCount,
                              self.builder.scaleMin, self.builder.scaleMax, self.builder.freqMax)[scale]
        e = np.zeros((s[2], s[3]), np.float32)
        _check(load_library().empi_workspace_energy_map(
            self.handle, int(scale), e.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return e

    @staticmethod
    def subtractAtomFromSignal(atom, signal, fit, freqSampling, engine=None):
        """Workspace::subtractAtomFromSignal (src/gabor.cpp:143-187) on the device.
        signal (float64, in place); with fit, atom params 0 and 1 are updated."""
        eng = engine or default_engine()
        p = np.asarray(atom.params if isinstance(atom, Atom) else atom, np.float64).copy()
        if not (isinstance(signal, np.ndarray) and signal.dtype == np.float64 and signal.flags.c_contiguous):
            raise TypeError("signal must be a contiguous float64 array (updated in place)")
        _check(load_library().empi_subtract_atom_from_signal(eng.handle, _dp(p), _dp(signal), signal.size,
                                                             float(freqSampling), int(bool(fit))))
        if isinstance(atom, Atom):
            atom.params[0], atom.params[1] = float(p[0]), float(p[1])
        return p


# ---------------------------------------------------------------- decomposition


@dataclass
class EpochResult:
    atoms: np.ndarray       # [C, iterations, 6]
    counts: np.ndarray      # atoms per channel
    energies: np.ndarray    # residual energy after each iteration ([C, it] for SMP, [it] otherwise)
    indices: np.ndarray     # (scale, t, f) of each atom, same leading shape as energies
    totals: np.ndarray      # total energy per MP loop


class Batch:
    """Device state for many epochs of one variant (empi_batch_*)."""

    def __init__(self, variant, energyError, settings, shapes, fs, scaleMin=0.0, scaleMax=math.inf,
                 freqMax=math.inf, engine=None):
        self.engine = engine or default_engine()
        self.variant = _VARIANTS[variant] if isinstance(variant, str) else int(variant)
        self.settings = settings
        self.shapes = [(int(n), int(c)) for n, c in shapes]
        self.fs = float(fs)
        L = load_library()
        d = _dictionary(energyError, scaleMin, scaleMax, freqMax)
        s = Settings(int(settings.iterationMax), float(settings.residualEnergy))
        eps = (Epoch * len(self.shapes))(*[Epoch(self.fs, c, n, None) for n, c in self.shapes])
        h = ctypes.c_void_p()
        _check(L.empi_batch_create(self.engine.handle, self.variant, ctypes.byref(d), ctypes.byref(s), eps,
                                   len(self.shapes), ctypes.byref(h)))
        self.handle = h
        self.engine._adopt(self)

    def close(self):
        if getattr(self, "handle", None) and getattr(self.engine, "handle", None):
            load_library().empi_batch_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, epochs):
        """epochs: list of float32 arrays shaped (N, C), sample-major."""
        self._keep = [np.ascontiguousarray(e, np.float32) for e in epochs]
        eps = (Epoch * len(self._keep))(*[Epoch(self.fs, e.shape[1], e.shape[0], e.ctypes.data)
                                          for e in self._keep])
        _check(load_library().empi_batch_load(self.handle, eps))

    def run(self):
        _check(load_library().empi_batch_run(self.handle))

    def set_proposal(self, source="net", k=16, weights=None):
        """Block proposal for later runs (empi_batch_set_proposal): source
        "net" (weights file), "last_atom", "none" or None (off)."""
        code = {"net": 0, "last_atom": 1, "none": 2, None: -1}[source]
        _check(load_library().empi_batch_set_proposal(self.handle, code, int(k),
                                                      os.fsencode(weights) if weights else None))

    def collect_pairs(self, enable=True):
        """Keep the residual spectrogram before every selection of later runs
        (empi_batch_collect_pairs)."""
        _check(load_library().empi_batch_collect_pairs(self.handle, int(bool(enable))))

    def pairs(self):
        """(spectrograms [n, 64, 128] float32, blocks [n] int32) of the last run."""
        L = load_library()
        n = ctypes.c_int()
        _check(L.empi_batch_pairs(self.handle, 0, None, None, ctypes.byref(n)))
        spec = np.zeros((n.value, 64, 128), np.float32)
        blocks = np.zeros(n.value, np.int32)
        if n.value:
            _check(L.empi_batch_pairs(self.handle, n.value, spec.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                      _ip(blocks), ctypes.byref(n)))
        return spec, blocks

    def tree(self, instance):
        """(slot keys [S] uint64, leaf-chunk maxima [K] uint64, chunk lower
        bounds [K] uint32) of MP loop `instance` (empi_batch_tree)."""
        L = load_library()
        ns, nc = ctypes.c_longlong(), ctypes.c_int()
        _check(L.empi_batch_tree(self.handle, int(instance), 0, None, ctypes.byref(ns), 0, None, None,
                                 ctypes.byref(nc)))
        slots = np.zeros(ns.value, np.uint64)
        chunks = np.zeros(nc.value, np.uint64)
        chunk_l = np.zeros(nc.value, np.uint32)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        _check(L.empi_batch_tree(self.handle, int(instance), ns.value, slots.ctypes.data_as(u64p), ctypes.byref(ns),
                                 nc.value, chunks.ctypes.data_as(u64p),
                                 chunk_l.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), ctypes.byref(nc)))
        return slots, chunks, chunk_l

    def probe_proposal(self, enable=True):
        """Measure, in later runs, the refresh work no certified block
        proposal could skip (empi_batch_probe_proposal)."""
        _check(load_library().empi_batch_probe_proposal(self.handle, int(bool(enable))))

    def stats(self) -> BatchStats:
        st = BatchStats()
        _check(load_library().empi_batch_get_stats(self.handle, ctypes.byref(st)))
        return st

    def result(self, e) -> EpochResult:
        n, C = self.shapes[e]
        cap = self.settings.iterationMax
        smp = self.variant == SMP or C == 1
        loops = C if smp else 1
        atoms = np.zeros((C, cap, 6))
        counts = np.zeros(C, np.int32)
        energies = np.zeros((loops, cap))
        idx = np.zeros((loops, cap, 3), np.int32)
        totals = np.zeros(loops)
        L = load_library()
        _check(L.empi_batch_atoms(self.handle, e, cap, _dp(atoms), _ip(counts), _dp(energies), _ip(idx)))
        _check(L.empi_batch_total_energy(self.handle, e, _dp(totals)))
        if not smp:
            energies, idx = energies[0], idx[0]
        return EpochResult(atoms, counts, energies, idx, totals)


def decompose_epochs(variant, epochs, fs, energyError, iterationMax, energyPercent=100.0, scaleMin=0.0,
                     scaleMax=math.inf, freqMax=math.inf, engine=None):
    """Decomposes a list of (N, C) float32 epochs in one device batch."""
    settings = DecompositionSettings(int(iterationMax), 1.0 - 0.01 * float(energyPercent))
    b = Batch(variant, energyError, settings, [e.shape for e in epochs], fs, scaleMin, scaleMax, freqMax,
              engine)
    b.load(epochs)
    b.run()
    out = [b.result(i) for i in range(len(epochs))]
    b.close()
    return out


class Decomposition:
    """Decomposition::compute (src/classes.cpp:26-73): the full MP loop of one
    epoch, on the device, for the variant of the subclass."""

    variant = SMP

    def compute(self, settings, workspace, signal):
        x = np.asarray(signal, np.float64).reshape(workspace.channelCount, workspace.sampleCount)
        b = workspace.builder
        epoch = np.ascontiguousarray(x.T.astype(np.float32))
        res = decompose_epochs(self.variant, [epoch], workspace.freqSampling, b.energyError,
                               settings.iterationMax, 100.0 * (1.0 - settings.residualEnergy), b.scaleMin,
                               b.scaleMax, b.freqMax, workspace.engine)[0]
        return [[Atom(list(map(float, res.atoms[c, a]))) for a in range(res.counts[c])]
                for c in range(workspace.channelCount)]


class SmpDecomposition(Decomposition):
    variant = SMP


class Mmp1Decomposition(Decomposition):
    variant = MMP1


class Mmp2Decomposition(Decomposition):
    variant = MMP2


class Mmp3Decomposition(Decomposition):
    variant = MMP3


def run_config(path, device=0):
    """The empi CLI on a config file (src/empi.cpp:49-167)."""
    L = load_library()
    o = EngineOpts()
    L.empi_engine_opts_default(ctypes.byref(o))
    o.device = device
    _check(L.empi_run_config(str(path).encode(), ctypes.byref(o)))


def book_write(path, epoch_number, fs, samples, atoms, counts, append=False):
    """BookWriter::write for one epoch; samples (C, N), atoms [C, cap, 6]."""
    s = np.ascontiguousarray(samples, np.float32)
    a = np.ascontiguousarray(atoms, np.float64)
    c = np.ascontiguousarray(counts, np.int32)
    _check(load_library().empi_book_write(str(path).encode(), int(append), int(epoch_number), float(fs),
                                          s.shape[0], s.shape[1], s.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                          a.shape[1], _dp(a), _ip(c)))
