"""The oracle (C restatement, oracle/mp_oracle.c) pinned against the
reference's own code: golden fixtures generated from empi's sources, and the
reference library itself where it has been built (oracle/_ref)."""
import hashlib
import math

import numpy as np
import pytest

from helpers import case_limits, case_signal, compare_sequences, golden
from oracle import oracle as O

CASES = golden()["cases"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_golden_signal_regenerates(case):
    _, x = case_signal(case)
    assert hashlib.sha256(x.tobytes()).hexdigest() == case["signal_sha_f32"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_restatement_matches_reference_golden(case):
    fs, x = case_signal(case)
    r = O.decompose(case["variant"], fs, x.T.astype(np.float64), case["energy_error"], case["iterations"],
                    case["energy_percent"], **case_limits(case))
    assert list(r.natoms) == case["counts"]
    for c in range(x.shape[1]):
        ref = case["atoms"][c]
        got = r.atoms[c, : r.natoms[c]]
        # both sides are FP64; indices must agree everywhere, values to ~1e-9
        m = r.margins[c if case["variant"] == "smp" else 0]
        compare_sequences(ref, got, m, label=f"{case['name']} ch{c}")
        for a in range(len(ref)):
            np.testing.assert_allclose(got[a][:2], ref[a][:2], rtol=1e-9)
    e_ref = case["energies"]
    e_got = r.energies
    for row_r, row_g in zip(e_ref, e_got):
        for a, v in enumerate(row_r):
            if v is not None:
                assert abs(row_g[a] - v) <= 1e-11 * abs(v)


def test_zero_signal_is_empty():
    err = {e["name"]: e["error"] for e in golden()["errors"]}
    with pytest.raises(RuntimeError, match=err["zeros"]):
        O.decompose("smp", 128.0, np.zeros((1, 256)), 0.01, 5, 99.0)


GEOMS = [(128.0, 1280, 0.01, {}), (256.0, 5120, 0.01, {}), (512.0, 16384, 0.005, {}),
         (256.0, 777, 0.03, {}), (100.0, 1000, 0.01, dict(smin=0.05, smax=3.0, fmax=30.0)),
         (512.0, 16384, 0.001, {}), (1000.0, 64, 0.2, {})]


@pytest.mark.parametrize("fs,n,eps,lim", GEOMS)
def test_geometry_matches_reference(fs, n, eps, lim):
    if not O.ref_available():
        pytest.skip("reference library not built here")
    kw = dict(smin=lim.get("smin", 0.0), smax=lim.get("smax", math.inf), fmax=lim.get("fmax", math.inf))
    assert O.geometry(fs, n, eps, **kw) == O.ref_geometry(fs, n, eps, **kw)


@pytest.mark.parametrize("variant", ["smp", "mmp1", "mmp3"])
def test_restatement_maps_match_reference(variant):
    if not O.ref_available():
        pytest.skip("reference library not built here")
    from empi_b200 import synth

    w = synth.workload(1, epochs=1, channels=1 if variant == "smp" else 3, samples=600, seed=5)
    x = w.epochs[0].T.astype(np.float64)
    g = O.geometry(w.fs, x.shape[1], 0.02)
    for j in (0, len(g) // 2, len(g) - 1):
        a = O.energy_map(w.fs, x, 0.02, j, mmp1=variant == "mmp1")
        b = O.ref_energy_map(w.fs, x, 0.02, j, mmp1=variant == "mmp1")
        assert np.max(np.abs(a - b)) <= 1e-11 * b.max()


def test_subtract_fit_matches_reference_values():
    # fit=true projection of MMP2: modulus = <w/|w|, x>, amplitude = modulus/|w|
    fs = 128.0
    x = np.sin(np.arange(512) * 0.3) * np.exp(-((np.arange(512) - 250) / 60.0) ** 2)
    params = [0.0, 1.0, 250.0, 60.0 * math.sqrt(math.pi) / math.sqrt(math.pi), 0.3 * 2 / (2 * math.pi), 0.0]
    p, y = O.subtract_atom(params, x, fs, True)
    w = np.zeros(512)
    sA, fA, tA = p[3] / fs, p[4] * fs / 2, p[2] / fs
    iL, iR = max(0, int(np.rint((tA - 3 * sA) * fs))), min(511, int(np.rint((tA + 3 * sA) * fs)))
    i = np.arange(iL, iR + 1)
    wav = np.cos(2 * math.pi * fA * (i / fs - tA)) * np.exp(-math.pi * ((i / fs - tA) / sA) ** 2)
    nrm = np.sqrt(np.sum(wav ** 2))
    mod = np.sum(wav / nrm * x[iL:iR + 1])
    assert abs(p[0] - mod) < 1e-12 * abs(mod)
    assert abs(p[1] - mod / nrm) < 1e-12 * abs(mod / nrm)


FULL_FIXTURES = ["mmp2_19x8x5120", "mmp3_4x16384_512", "smp_batch_16x2", "smp_16384_512_eps0001"]


@pytest.mark.parametrize("name", FULL_FIXTURES)
def test_full_size_fixture_signals_regenerate(name):
    """The full-size goldens (tests/golden/full/) belong to the seeded signals
    the GPU tests regenerate: same shapes, same float32 bytes."""
    import json
    import os

    from empi_b200 import synth

    path = os.path.join(os.path.dirname(__file__), "golden", "full", name + ".npz")
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    w = synth.workload(meta["workload"], **meta["overrides"])
    for e, sha in enumerate(meta["signal_sha_f32"]):
        x = w.epochs[e] if meta["channels"] is None else w.epochs[e][:, : meta["channels"]]
        assert hashlib.sha256(np.ascontiguousarray(x).tobytes()).hexdigest() == sha, (name, e)
    counts = z["counts"] if "counts" in z.files else np.concatenate([z[f"counts_{e}"] for e in range(meta["epochs"])])
    assert np.all(np.asarray(counts) >= 1)
