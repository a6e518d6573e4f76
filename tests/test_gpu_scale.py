"""The engine at BASELINE shapes.

Against the reference's goldens (tests/golden/scale_cases.json): the first
epoch of the bench workload (MMP2, 19 x 5120 @ 256 Hz), a 2-channel MMP3 case
at 512 Hz (Nfft up to 2^18), 16384-sample windows (folded transforms) and
energyError 0.001 (111 scales).  At full size, where no CPU oracle finishes in
test time, size-independent properties: residual energies never increase, the
stop rule holds, parameters stay on the dictionary grid and the first atoms of
the full batch equal the single-epoch golden.
"""
import json
import math
import os

import numpy as np
import pytest

import empi_b200
from helpers import GOLDEN, case_limits, case_signal, compare_sequences

pytestmark = pytest.mark.gpu

with open(os.path.join(GOLDEN, "scale_cases.json")) as f:
    SCALE = json.load(f)["cases"]


@pytest.mark.parametrize("case", SCALE, ids=[c["name"] for c in SCALE])
def test_scale_case_matches_reference_golden(engine, case):
    fs, x = case_signal(case)
    lim = case_limits(case)
    res = empi_b200.decompose_epochs(case["variant"], [x], fs, case["energy_error"], case["iterations"],
                                     case["energy_percent"], lim["smin"], lim["smax"], lim["fmax"], engine)[0]
    smp = case["variant"] == "smp" or x.shape[1] == 1
    for c in range(x.shape[1]):
        margins = case["margins"][c if smp else 0]
        e_ref = case["energies"][c if smp else 0] if (c == 0 or smp) else None
        e_got = res.energies[c] if smp else res.energies
        compare_sequences(case["atoms"][c], res.atoms[c, : res.counts[c]], margins, e_ref, e_got,
                          label=f"{case['name']} ch{c}")


def check_properties(res, fs, geometry, stop_ratio, iters):
    loops = res.energies if res.energies.ndim == 2 else res.energies[None, :]
    totals = np.atleast_1d(res.totals)
    for l, row in enumerate(loops):
        n = int(res.counts[l] if res.energies.ndim == 2 else res.counts[0])
        e = row[: n - 1] if n == iters else row[:n]
        e = e[np.isfinite(e)]
        assert np.all(np.diff(np.concatenate([[totals[l]], e])) <= 1e-9 * totals[l]), "energy increased"
        if n < iters:
            assert e[-1] / totals[l] <= stop_ratio
    scales = {round(g[0] * fs, 9) for g in geometry}
    for c in range(res.atoms.shape[0]):
        for a in range(int(res.counts[c])):
            p = res.atoms[c, a]
            assert np.all(np.isfinite(p))
            assert round(p[3], 9) in scales
            assert 0.0 <= p[4] <= 1.0 + 1e-12       # f * 2 / fs
            assert -math.pi - 1e-12 <= p[5] <= math.pi + 1e-12


def test_bench_workload_full_size(engine):
    from empi_b200 import synth

    w = synth.workload(1)
    res = empi_b200.decompose_epochs("mmp2", w.epochs, w.fs, w.energy_error, w.iterations, w.energy_percent,
                                     engine=engine)
    geo = empi_b200.dictionary_scales(w.energy_error, w.fs, w.samples)
    for r in res:
        check_properties(r, w.fs, geo, 1 - 0.01 * w.energy_percent, w.iterations)
    # the first atoms of epoch 0 equal the single-epoch golden (fits are sequential in atom order)
    g = [c for c in SCALE if c["name"] == "mmp2_bench_epoch0"][0]
    for c in range(w.channels):
        ref = g["atoms"][c]
        compare_sequences(ref, res[0].atoms[c, : len(ref)], g["margins"][0], label=f"epoch0 ch{c}")


def test_mmp3_32ch_16384_full_shape(engine):
    from empi_b200 import synth

    w = synth.workload(2, epochs=1)
    res = empi_b200.decompose_epochs("mmp3", w.epochs, w.fs, w.energy_error, 3, 100.0, engine=engine)[0]
    geo = empi_b200.dictionary_scales(w.energy_error, w.fs, w.samples)
    assert len(geo) == 65 and max(g[1] for g in geo) == 524288
    check_properties(res, w.fs, geo, 0.0, 3)
    assert list(res.counts) == [3] * 32


def test_energy_error_0001_nfft_2_20(engine):
    from empi_b200 import synth

    w = synth.workload(4, epochs=1, channels=1)
    res = empi_b200.decompose_epochs("smp", w.epochs, w.fs, w.energy_error, 2, 100.0, engine=engine)[0]
    geo = empi_b200.dictionary_scales(w.energy_error, w.fs, w.samples)
    assert len(geo) == 144 and max(g[1] for g in geo) == 1048576
    check_properties(res, w.fs, geo, 0.0, 2)


def test_uneven_batch_of_workload3_instances(engine):
    from empi_b200 import synth
    from oracle import oracle as O

    w = synth.workload(3, epochs=40)
    epochs = [e for e in w.epochs if e.shape[0] <= 3000][:8] + [e for e in w.epochs if e.shape[0] > 3000][:4]
    res = empi_b200.decompose_epochs("smp", epochs, w.fs, w.energy_error, 8, w.energy_percent, engine=engine)
    for e, (ep, r) in enumerate(zip(epochs, res)):
        geo = empi_b200.dictionary_scales(w.energy_error, w.fs, ep.shape[0])
        check_properties(r, w.fs, geo, 1 - 0.01 * w.energy_percent, 8)
        if ep.shape[0] <= 3000 and e < 3:
            ora = O.decompose("smp", w.fs, ep[:, :1].T.astype(np.float64), w.energy_error, 8, w.energy_percent)
            compare_sequences(ora.atoms[0, : ora.natoms[0]], r.atoms[0, : r.counts[0]], ora.margins[0],
                              ora.energies[0], r.energies[0], label=f"instance {e}")
