"""Shared-memory and table addressing of the refresh kernel, emulated on the
CPU for every sub-FFT size.  The kernel addresses its padded buffer (one
float2 of padding per 16 points) from one padded base plus compile-time
offsets; that is only right where the run of points it covers stays inside
one 16-point block, or steps by a multiple of 16.  These tests enumerate the
jobs, tasks and points of a full work unit for L = 2^0 .. 2^12 and check each
such offset against the padded index computed directly, and every index
against the buffer and table sizes (empi_b200/csrc/fft.cuh, refresh.cuh,
plan.hpp)."""
import numpy as np
import pytest

UNIT_POINTS = 8192   # kUnitPoints
UNIT_THREADS = 512   # kUnitThreads
MAX_WINDOWS = 1024   # kMaxWindowsPerUnit
TW_N = 8192          # kTwN
BUF = UNIT_POINTS + UNIT_POINTS // 16 + 16   # kBufFloat2
BINS_PER_TASK = 8    # kBinsPerTask


def pad16(i):
    return i + (i >> 4)


def passes(logl):
    """(radix, logNs) of the Stockham passes for L = 2^logl: the odd first
    radix, then radix-16 passes."""
    first = logl & 3
    out = [(1 << first, 0)] if first else []
    out += [(16, ns) for ns in range(first, logl, 4)]
    return out


def unit_points(logl, pair):
    L = 1 << logl
    nwin = max(1, min(MAX_WINDOWS, UNIT_POINTS // (2 * L))) if pair else min(MAX_WINDOWS, UNIT_POINTS // L)
    return nwin, (2 if pair else 1) * nwin * L


SIZES = [(lg, pair) for lg in range(1, 13) for pair in (False, True)]


@pytest.mark.parametrize("logl,pair", SIZES)
def test_stockham_pass_offsets(logl, pair):
    L = 1 << logl
    _, points = unit_points(logl, pair)
    assert points <= UNIT_POINTS
    for radix, logns in passes(logl):
        if logns == 0 and (logl & 3):
            continue  # the odd first pass is fused into the load
        ns = 1 << logns
        logr = radix.bit_length() - 1
        q = L // radix
        jobs = np.arange(points // radix)
        j = jobs & (q - 1)
        base = (jobs >> (logl - logr)) << logl
        k = j & (ns - 1)
        ob = base + (j - k) * radix + k
        for r in range(radix):
            src = base + j + r * q
            assert np.all(pad16(src) < BUF)
            if q % 16 == 0:
                assert np.array_equal(pad16(base + j) + r * (q + (q >> 4)), pad16(src))
            dst = ob + r * ns
            assert np.all(pad16(dst) < BUF)
            assert np.array_equal(pad16(ob) + r * ns + ((r * ns) >> 4), pad16(dst))
        # twiddle W^k of the stage from the table
        tw_shift = TW_N >> (logns + logr)
        assert tw_shift >= 1 and int((k * tw_shift).max()) < TW_N


@pytest.mark.parametrize("logl,pair", [(lg, p) for lg, p in SIZES if lg & 3])
def test_fused_first_pass_stores(logl, pair):
    L = 1 << logl
    first = logl & 3
    r0, lq = 1 << first, logl - first
    nwin, _ = unit_points(logl, pair)
    nf = 2 if pair else 1
    job = np.arange(nwin << lq)
    w, jq = job >> lq, job & ((1 << lq) - 1)
    o = ((w * nf) << logl) + jq * r0
    for rr in range(r0):
        assert np.array_equal(pad16(o) + rr, pad16(o + rr))
        if pair:
            assert np.array_equal(pad16(o) + L + L // 16 + rr, pad16(o + L + rr))
            assert np.all(pad16(o + L + rr) < BUF)
        # the points of a job: jq + rr L / R0, all inside the window's transform
        assert int((jq + (rr << lq)).max()) < L


@pytest.mark.parametrize("pair", [False, True])
def test_large_transform_load_strides(pair):
    # L = 4096 (> threads per CTA): a thread's points np0 + i T of one window
    logl = 12
    L = 1 << logl
    nwin, _ = unit_points(logl, pair)
    nf = 2 if pair else 1
    np0 = np.arange(UNIT_THREADS) & (L - 1)
    for w in range(nwin):
        o = (w * nf) << logl
        pp = pad16(o + np0)
        for i, npt in enumerate(range(0, L, UNIT_THREADS)):
            pts = np0 + npt
            assert np.array_equal(pp + i * (UNIT_THREADS + UNIT_THREADS // 16), pad16(o + pts))
            if pair:
                assert np.array_equal(pad16(o + pts) + L + L // 16, pad16(o + L + pts))
                assert np.all(pad16(o + L + pts) < BUF)


@pytest.mark.parametrize("logl,pair", SIZES)
def test_spectrum_task_runs_stay_in_one_block(logl, pair):
    L = 1 << logl
    ch = min(L, BINS_PER_TASK)
    tpw = L // ch
    nwin, _ = unit_points(logl, pair)
    nf = 2 if pair else 1
    for mirrored in (True, False):
        nq = ch if (pair or not mirrored) else max(ch // 2, 1)
        if mirrored and not pair and ch < 2:
            continue
        for w in (0, nwin - 1):
            o0 = (w * nf) << logl
            obs = [o0 + L] if pair else [o0]
            if not mirrored and pair:
                obs = [o0, o0 + L]
            for tau in range(tpw):
                q0 = tau * nq
                if q0 + nq > L:
                    continue
                qq = np.arange(nq)
                assert np.array_equal(pad16(o0 + q0) + qq, pad16(o0 + q0 + qq))
                for ob in obs:
                    if L - 1 - q0 - (nq - 1) < 0:
                        continue
                    assert np.array_equal(pad16(ob + L - 1 - q0) - qq, pad16(ob + L - 1 - q0 - qq))
                    assert np.all(pad16(ob + L - 1 - q0 - qq) < BUF)
                # W_2L^q from the table at q0
                assert (q0 << (12 - logl)) < TW_N


@pytest.mark.parametrize("logl", range(0, 13))
def test_load_twiddle_indices(logl):
    L = 1 << logl
    n = np.arange(4 * L)
    # W_L^n (pair factor) and W_2L^n (residue M/2) from the 8192-entry table
    assert int(((n & (L - 1)) << (13 - logl)).max()) < TW_N
    assert int(((n & (2 * L - 1)) << (12 - logl)).max()) < TW_N


@pytest.mark.parametrize("logl", range(1, 13))
def test_mmp_channel_sum_indices(logl):
    # MMP per-bin channel sums: acc[w nb + q'] with nb = L + 1 (group 0, the
    # Nyquist bin at q' = L), 2L (pairs) or L (residue M/2), held in
    # kUnitPoints + NW floats per sum
    L = 1 << logl
    nw = min(UNIT_POINTS >> logl, MAX_WINDOWS)
    for g, pair in ((0, False), (1, False), (2, True)):
        nwin, _ = unit_points(logl, pair)
        nb = L + 1 if g == 0 else (2 * L if pair else L)
        q = np.arange(L)
        direct = q
        mirrored_q = np.arange(max(L // 2, 1)) if not pair else q
        mirror = (2 * L - 1 - mirrored_q) if pair else ((L - mirrored_q) if g == 0 else (L - 1 - mirrored_q))
        idx = np.concatenate([direct, mirror, [L] if g == 0 else [], q + L if pair else []]).astype(int)
        assert idx.min() >= 0 and idx.max() < nb
        assert nwin * nb <= UNIT_POINTS + nw
