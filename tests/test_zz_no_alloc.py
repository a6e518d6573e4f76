"""The allocation-free subtraction entry point against the allocating one.

empi_subtract_atom_from_signal_noalloc exists for callers that cannot
allocate device memory (inside CUDA stream capture, or beside a framework
whose memory pool owns the GPU): it stages the signal in a fixed static
device array instead of cudaMalloc'd buffers.  Its results must equal
empi_subtract_atom_from_signal's, call after call, although every call
reuses the same array.  This file is collected last so a run that stops at
the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import empi_b200

pytestmark = pytest.mark.gpu

MAX_SAMPLES = 1 << 20
_dp = ctypes.POINTER(ctypes.c_double)


def noalloc(params, x, fs, fit):
    L = empi_b200.load_library()
    p = np.array(params, np.float64)
    y = np.array(x, np.float64)
    st = L.empi_subtract_atom_from_signal_noalloc(0, None, p.ctypes.data_as(_dp), y.ctypes.data_as(_dp), y.size,
                                                  float(fs), int(fit))
    empi_b200._check(st)
    return p, y


def allocating(engine, params, x, fs, fit):
    y = np.array(x, np.float64)
    p = empi_b200.GaborWorkspace.subtractAtomFromSignal(list(params), y, fit, fs, engine)
    return p, y


@pytest.mark.parametrize("fit", [False, True])
def test_noalloc_matches_allocating_entry_point_twice(fit):
    eng = empi_b200.Engine()
    rng = np.random.default_rng(17)
    fs = 256.0
    # two calls in a row; the second signal is shorter, so leftovers of the
    # first call sit in the shared array past its end
    cases = [(6000, [0.0, 1.7, 2900.0, 1.3 * fs, 9.0 * 2 / fs, 0.4]),
             (2500, [0.0, -0.6, 1200.0, 0.4 * fs, 31.0 * 2 / fs, -2.1])]
    for n, params in cases:
        x = rng.standard_normal(n)
        p1, y1 = noalloc(params, x, fs, fit)
        p2, y2 = allocating(eng, params, x, fs, fit)
        np.testing.assert_allclose(y1, y2, rtol=0, atol=1e-12)
        np.testing.assert_allclose(p1, p2, rtol=1e-12)
        assert not np.array_equal(y1, x)  # the atom was subtracted
    eng.close()


def test_noalloc_rejects_signals_longer_than_its_array():
    with pytest.raises(empi_b200.EmpiError) as ei:
        noalloc([0.0, 1.0, 10.0, 8.0, 0.1, 0.0], np.zeros(MAX_SAMPLES + 1), 256.0, False)
    assert ei.value.message == "signalLongerThanStaticScratch"
