"""The allocation-free subtraction entry point against the allocating one.

empi_subtract_atom_from_signal_noalloc exists for callers that cannot
allocate device memory: a program whose device memory another framework's
pool allocator owns, or one with a fixed device-memory budget.  It stages the
signal in a fixed static device array instead of cudaMalloc'd buffers.  Its
results must equal empi_subtract_atom_from_signal's (and the FP64 oracle's),
call after call, although every call reuses the same array, on the default
stream and on a caller's own stream, and the caller's current device must be
the same after every return, an error return included.  This file is
collected last so a run that stops at the first failure has run every other
test before it.
"""
import ctypes

import numpy as np
import pytest

import empi_b200
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_SAMPLES = 1 << 20
_dp = ctypes.POINTER(ctypes.c_double)


def noalloc(params, x, fs, fit, stream=None):
    L = empi_b200.load_library()
    p = np.array(params, np.float64)
    y = np.array(x, np.float64)
    st = L.empi_subtract_atom_from_signal_noalloc(0, stream, p.ctypes.data_as(_dp), y.ctypes.data_as(_dp), y.size,
                                                  float(fs), int(fit))
    empi_b200._check(st)
    return p, y


def allocating(engine, params, x, fs, fit):
    y = np.array(x, np.float64)
    p = empi_b200.GaborWorkspace.subtractAtomFromSignal(list(params), y, fit, fs, engine)
    return p, y


CASES = [(6000, [0.0, 1.7, 2900.0, 1.3 * 256.0, 9.0 * 2 / 256.0, 0.4]),
         (2500, [0.0, -0.6, 1200.0, 0.4 * 256.0, 31.0 * 2 / 256.0, -2.1])]


@pytest.mark.parametrize("use_stream", [False, True])
@pytest.mark.parametrize("fit", [False, True])
def test_noalloc_matches_allocating_entry_point_twice(fit, use_stream):
    import torch

    eng = empi_b200.Engine()
    rng = np.random.default_rng(17)
    fs = 256.0
    s = torch.cuda.Stream() if use_stream else None
    dev = torch.cuda.current_device()
    # two calls in a row; the second signal is shorter, so leftovers of the
    # first call sit in the shared array past its end
    for n, params in CASES:
        x = rng.standard_normal(n)
        p1, y1 = noalloc(params, x, fs, fit, s.cuda_stream if s is not None else None)
        assert torch.cuda.current_device() == dev
        p2, y2 = allocating(eng, params, x, fs, fit)
        np.testing.assert_allclose(y1, y2, rtol=0, atol=1e-12)
        np.testing.assert_allclose(p1, p2, rtol=1e-12)
        # and the numbers themselves: the FP64 restatement of
        # subtractAtomFromSignal (src/gabor.cpp:143-187)
        p3, y3 = O.subtract_atom(params, x, fs, fit)
        np.testing.assert_allclose(y1, y3, rtol=0, atol=1e-10)
        np.testing.assert_allclose(p1, p3, rtol=1e-10, atol=1e-12)
        assert not np.array_equal(y1, x)  # the atom was subtracted
    eng.close()


def test_noalloc_rejects_bad_sizes_and_keeps_the_current_device():
    import torch

    dev = torch.cuda.current_device()
    with pytest.raises(empi_b200.EmpiError) as ei:
        noalloc([0.0, 1.0, 10.0, 8.0, 0.1, 0.0], np.zeros(MAX_SAMPLES + 1), 256.0, False)
    assert ei.value.message == "signalLongerThanStaticScratch"
    assert torch.cuda.current_device() == dev
    with pytest.raises(empi_b200.EmpiError) as ei:
        noalloc([0.0, 1.0, 10.0, 8.0, 0.1, 0.0], np.zeros(0), 256.0, False)
    assert ei.value.message == "invalidArgument"
    assert torch.cuda.current_device() == dev
