"""Test infrastructure (oracle), not product code.

ctypes access to the CPU checkers:
  * ``liboracle.so`` -- this project's C restatement of empi's MP path
    (mp_oracle.c), built by ``make -C oracle oracle``;
  * ``_ref/libempiref.so`` -- empi's own sources with a project FFT in place of
    FFTW (ref_glue.cpp), built by ``make -C oracle ref`` where the reference
    sources exist; ``_ref/empi`` is the reference CLI from the same build.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
VARIANTS = {"smp": 0, "mmp1": 1, "mmp2": 2, "mmp3": 3}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class Scale(ctypes.Structure):
    _fields_ = [("s", ctypes.c_double), ("nfft", ctypes.c_int), ("fcount", ctypes.c_int),
                ("tcount", ctypes.c_int)]


def build(ref: bool = True) -> None:
    src = os.environ.get("EMPI_REFERENCE", "/root/reference")
    targets = ["oracle"] + (["ref"] if ref and os.path.isdir(os.path.join(src, "src")) else [])
    subprocess.run(["make", "-s", "-C", HERE, f"REF={src}"] + targets, check=True)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        _lib = ctypes.CDLL(path)
        _lib.or_geometry.restype = ctypes.c_int
        _lib.or_decompose.restype = ctypes.c_int
        _lib.or_energy_map.restype = ctypes.c_int
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libempiref.so"))


def ref():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(os.path.join(HERE, "_ref", "libempiref.so"))
    return _ref


def _d(x):
    return ctypes.c_double(float(x))


def geometry(fs, n, eps, smin=0.0, smax=float("inf"), fmax=float("inf")):
    """List of (s, nfft, fcount, tcount) per scale (restatement)."""
    L = lib()
    count = L.or_geometry(_d(fs), ctypes.c_int(n), _d(eps), _d(smin), _d(smax), _d(fmax), 0, None)
    arr = (Scale * max(count, 1))()
    L.or_geometry(_d(fs), ctypes.c_int(n), _d(eps), _d(smin), _d(smax), _d(fmax), count, arr)
    return [(a.s, a.nfft, a.fcount, a.tcount) for a in arr[:count]]


def ref_geometry(fs, n, eps, smin=0.0, smax=float("inf"), fmax=float("inf")):
    R = ref()
    cap = 4096
    s = np.zeros(cap)
    nf = np.zeros(cap, np.int32)
    fc = np.zeros(cap, np.int32)
    tc = np.zeros(cap, np.int32)
    count = R.empiref_geometry(_d(fs), ctypes.c_int(n), _d(eps), _d(smin), _d(smax), _d(fmax),
                               ctypes.c_int(cap), s.ctypes.data_as(_dp), nf.ctypes.data_as(_ip),
                               fc.ctypes.data_as(_ip), tc.ctypes.data_as(_ip))
    return [(float(s[i]), int(nf[i]), int(fc[i]), int(tc[i])) for i in range(count)]


def _map(fn, fs, x, eps, scale, mmp1, smin, smax, fmax, with_values):
    x = np.ascontiguousarray(np.asarray(x, np.float64))
    if x.ndim == 1:
        x = x[None, :]
    C, N = x.shape
    g = geometry(fs, N, eps, smin, smax, fmax)[scale]
    F, T = g[2], g[3]
    e = np.zeros((F, T))
    v = np.zeros((C, F, T, 2)) if with_values else None
    rc = fn(_d(fs), ctypes.c_int(C), ctypes.c_int(N), _d(eps), _d(smin), _d(smax), _d(fmax),
            ctypes.c_int(int(mmp1)), x.ctypes.data_as(_dp), ctypes.c_int(scale),
            e.ctypes.data_as(_dp), v.ctypes.data_as(_dp) if with_values else None)
    if rc != 0:
        raise RuntimeError(f"energy map failed ({rc})")
    return (e, v[..., 0] + 1j * v[..., 1]) if with_values else e


def energy_map(fs, x, eps, scale, mmp1=False, smin=0.0, smax=float("inf"), fmax=float("inf"),
               values=False):
    """FP64 energy map [f, t] of one scale (restatement); x is (C, N)."""
    return _map(lib().or_energy_map, fs, x, eps, scale, mmp1, smin, smax, fmax, values)


def ref_energy_map(fs, x, eps, scale, mmp1=False, smin=0.0, smax=float("inf"), fmax=float("inf"),
                   values=False):
    """Same map from the reference's own GaborWorkspace code."""
    return _map(ref().empiref_map, fs, x, eps, scale, mmp1, smin, smax, fmax, values)


class Result:
    """Atoms [c][a][6] (modulus, amplitude, t*fs, s*fs, f*2/fs, phase), counts per
    channel, residual energies after each iteration, the (scale, t, f) indices of
    each iteration's argmax and the relative margin to the runner-up."""

    def __init__(self, atoms, natoms, energies, indices=None, margins=None):
        self.atoms = atoms
        self.natoms = natoms
        self.energies = energies
        self.indices = indices
        self.margins = margins


def decompose(variant, fs, x, eps, iterations, energy_percent=100.0, smin=0.0,
              smax=float("inf"), fmax=float("inf")):
    """Restatement decomposition of one epoch x (C, N)."""
    return _decompose(lib().or_decompose, True, variant, fs, x, eps, iterations, energy_percent,
                      smin, smax, fmax)


def ref_decompose(variant, fs, x, eps, iterations, energy_percent=100.0, smin=0.0,
                  smax=float("inf"), fmax=float("inf")):
    """The reference's own decomposition classes on one epoch x (C, N)."""
    return _decompose(ref().empiref_decompose, False, variant, fs, x, eps, iterations,
                      energy_percent, smin, smax, fmax)


def _decompose(fn, restatement, variant, fs, x, eps, iterations, energy_percent, smin, smax, fmax):
    x = np.ascontiguousarray(np.asarray(x, np.float64))
    if x.ndim == 1:
        x = x[None, :]
    C, N = x.shape
    v = VARIANTS[variant] if isinstance(variant, str) else int(variant)
    if C == 1:
        v = 0
    M = iterations
    atoms = np.zeros((C, M, 6))
    nat = np.zeros(C, np.int32)
    ne = C if v == 0 else 1
    energies = np.full((ne, M), np.nan)
    err = ctypes.create_string_buffer(256)
    residual = 1.0 - 0.01 * energy_percent
    args = [ctypes.c_int(v), _d(fs), ctypes.c_int(C), ctypes.c_int(N), _d(eps), _d(smin), _d(smax),
            _d(fmax), ctypes.c_int(iterations), _d(residual), x.ctypes.data_as(_dp), ctypes.c_int(M),
            atoms.ctypes.data_as(_dp), nat.ctypes.data_as(_ip), energies.ctypes.data_as(_dp)]
    indices = margins = None
    if restatement:
        indices = np.zeros((ne, M, 3), np.int32)
        margins = np.full((ne, M), np.nan)
        args += [indices.ctypes.data_as(_ip), margins.ctypes.data_as(_dp)]
    args += [err, ctypes.c_int(256)]
    rc = fn(*args)
    if rc != 0:
        raise RuntimeError(err.value.decode() or f"decomposition failed ({rc})")
    return Result(atoms, nat, energies, indices, margins)


def subtract_atom(params, x, fs, fit):
    """GaborWorkspace::subtractAtomFromSignal restated; returns (params, x) copies."""
    p = np.array(params, np.float64)
    y = np.array(x, np.float64)
    lib().or_subtract_atom(p.ctypes.data_as(_dp), y.ctypes.data_as(_dp), ctypes.c_int(y.size), _d(fs),
                           ctypes.c_int(int(fit)))
    return p, y


def ref_cli() -> str:
    return os.path.join(HERE, "_ref", "empi")
