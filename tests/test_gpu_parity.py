"""Parity of the sm_100a engine with the oracle and the reference goldens.

Tolerances: FP32 energy maps within 1e-5 of the map maximum, and within
2.5e-5 relative (a quarter of the 1e-4 candidate band that is re-scored in
FP64) on entries above half the maximum, where argmax decisions are made;
atom sequences by the rule in
helpers.py (indices exact unless the oracle margin is < 1e-6; amplitude 1e-5
relative; phase 1e-5 rad; residual energy 1e-6 relative)."""
import math
import os
import subprocess

import numpy as np
import pytest

import empi_b200
from helpers import GOLDEN, case_limits, case_signal, compare_sequences, golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = golden()["cases"]


def workload0():
    from empi_b200 import synth

    w = synth.workload(0)
    return w.fs, w.epochs[0].T.astype(np.float64)


@pytest.mark.parametrize("scale", [0, 1, 4, 12, 20, 27, 33])
def test_energy_map_fp32_matches_fp64_oracle(engine, scale):
    fs, x = workload0()
    ws = empi_b200.GaborWorkspaceBuilder(0.01, engine=engine).prepareWorkspace(fs, 1, x.shape[1])
    ws.compute(x)
    got = ws.energy_map(scale).astype(np.float64)
    ref = O.energy_map(fs, x, 0.01, scale)
    assert got.shape == ref.shape
    top = ref.max()
    assert np.max(np.abs(got - ref)) <= 1e-5 * top
    near = ref > 0.5 * top
    assert np.max(np.abs(got[near] - ref[near]) / ref[near]) <= 2.5e-5
    ws.close()


@pytest.mark.parametrize("variant,mmp1", [("mmp3", False), ("mmp1", True)])
def test_multichannel_energy_maps(engine, variant, mmp1):
    from empi_b200 import synth

    w = synth.workload(1, epochs=1, channels=4, samples=900, seed=3)
    x = w.epochs[0].T.astype(np.float64)
    ws = empi_b200.GaborWorkspaceBuilder(0.01, engine=engine).prepareWorkspace(
        w.fs, 4, 900, constraint=empi_b200.MMP1 if mmp1 else None)
    ws.compute(x)
    g = O.geometry(w.fs, 900, 0.01)
    for j in (0, len(g) // 3, len(g) // 2, len(g) - 1):
        got = ws.energy_map(j).astype(np.float64)
        ref = O.energy_map(w.fs, x, 0.01, j, mmp1=mmp1)
        top = ref.max()
        assert np.max(np.abs(got - ref)) <= 1e-5 * top, (variant, j)
        near = ref > 0.5 * top
        assert np.max(np.abs(got[near] - ref[near]) / ref[near]) <= 2.5e-5, (variant, j)
    ws.close()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_decomposition_matches_reference_golden(engine, case):
    fs, x = case_signal(case)
    lim = case_limits(case)
    res = empi_b200.decompose_epochs(case["variant"], [x], fs, case["energy_error"], case["iterations"],
                                     case["energy_percent"], lim["smin"], lim["smax"], lim["fmax"], engine)[0]
    ora = O.decompose(case["variant"], fs, x.T.astype(np.float64), case["energy_error"], case["iterations"],
                      case["energy_percent"], **lim)
    smp = case["variant"] == "smp" or x.shape[1] == 1
    for c in range(x.shape[1]):
        ref = case["atoms"][c]
        got = res.atoms[c, : res.counts[c]]
        margins = ora.margins[c if smp else 0]
        e_ref = case["energies"][c if smp else 0]
        e_got = res.energies[c] if smp else res.energies
        # MMP2 per-channel fits carry no loop energies of their own
        compare_sequences(ref, got, margins, e_ref if case["variant"] != "mmp2" or c == 0 else None,
                          e_got, label=f"{case['name']} ch{c}")


def test_workspace_seam_step_by_step(engine):
    case = [c for c in CASES if c["name"] == "mmp3_3ch_1024"][0]
    fs, x = case_signal(case)
    C, N = x.shape[1], x.shape[0]
    sig = [np.ascontiguousarray(x[:, c].astype(np.float64)) for c in range(C)]
    ws = empi_b200.GaborWorkspaceBuilder(case["energy_error"], engine=engine).prepareWorkspace(fs, C, N)
    ws.compute(np.stack(sig))
    ora = O.decompose("mmp3", fs, x.T.astype(np.float64), case["energy_error"], 6, 100.0)
    for it in range(5):
        atoms, idx = ws.findBestMatch(with_index=True)
        if ora.margins[0][it] >= 1e-6:
            assert tuple(idx) == tuple(ora.indices[0][it])
        for c in range(C):
            ref = case["atoms"][c][it]
            np.testing.assert_allclose(atoms[c].params[:2], ref[:2], rtol=1e-5)
            np.testing.assert_allclose(atoms[c].params[2:5], ref[2:5], rtol=1e-12)
            before = sig[c].copy()
            ws.subtractAtom(atoms[c], sig[c], c)
            _, expect = O.subtract_atom(atoms[c].params, before, fs, False)
            np.testing.assert_allclose(sig[c], expect, rtol=0, atol=1e-12 * np.max(np.abs(before)))
    ws.close()


def test_atom_count_matches_reference(engine):
    ws = empi_b200.GaborWorkspaceBuilder(0.01, engine=engine).prepareWorkspace(128.0, 1, 1280)
    assert ws.getAtomCount() == 5008073
    ws.close()


@pytest.mark.parametrize("fit", [False, True])
def test_subtract_atom_from_signal(engine, fit):
    rng = np.random.default_rng(4)
    fs = 200.0
    x = rng.standard_normal(1500)
    params = [0.0, 2.5, 700.0, 0.8 * fs, 12.0 * 2 / fs, 0.7]
    p_ref, y_ref = O.subtract_atom(params, x, fs, fit)
    y = x.copy()
    p = empi_b200.GaborWorkspace.subtractAtomFromSignal(list(params), y, fit, fs, engine)
    np.testing.assert_allclose(y, y_ref, rtol=0, atol=1e-12)
    if fit:
        np.testing.assert_allclose(p[:2], p_ref[:2], rtol=1e-12)


def test_uneven_batch_matches_oracle(engine):
    from empi_b200 import synth

    rng = np.random.default_rng(9)
    epochs = []
    for n, c in [(512, 1), (1000, 2), (777, 1), (2048, 3), (600, 2)]:
        epochs.append(np.stack([synth.smp_channel(rng, n, 256.0, 6, 10.0) for _ in range(c)], 1).astype(np.float32))
    settings = empi_b200.DecompositionSettings(12, 0.005)
    b = empi_b200.Batch("smp", 0.01, settings, [e.shape for e in epochs], 256.0, engine=engine)
    b.load(epochs)
    b.run()
    for e, ep in enumerate(epochs):
        res = b.result(e)
        ora = O.decompose("smp", 256.0, ep.T.astype(np.float64), 0.01, 12, 99.5)
        for c in range(ep.shape[1]):
            ref = ora.atoms[c, : ora.natoms[c]]
            compare_sequences(ref, res.atoms[c, : res.counts[c]], ora.margins[c], ora.energies[c],
                              res.energies[c], label=f"epoch {e} ch {c}")
    b.close()


def test_signal_is_empty(engine):
    with pytest.raises(empi_b200.EmpiError) as ei:
        empi_b200.decompose_epochs("smp", [np.zeros((256, 1), np.float32)], 128.0, 0.01, 5, 99.0, engine=engine)
    assert ei.value.message == "signalIsEmpty"


def test_batch_rerun_is_deterministic(engine):
    from empi_b200 import synth

    w = synth.workload(1, epochs=2, channels=3, samples=1024, seed=77)
    settings = empi_b200.DecompositionSettings(15, 0.0)
    b = empi_b200.Batch("mmp2", 0.01, settings, [e.shape for e in w.epochs], w.fs, engine=engine)
    b.load(w.epochs)
    b.run()
    r1 = [b.result(e) for e in range(2)]
    b.run()
    r2 = [b.result(e) for e in range(2)]
    for a, c in zip(r1, r2):
        assert np.array_equal(a.atoms, c.atoms)
        assert np.array_equal(a.counts, c.counts)
    b.close()


@pytest.mark.parametrize("variant", ["smp", "mmp2", "mmp3"])
def test_results_follow_each_load_and_run(engine, variant):
    """A batch's results are read from one host copy per run: after new
    epochs are loaded and run, every read (atoms, energies, indices, totals)
    gives the new run's results, equal to a fresh batch's on those epochs."""
    from empi_b200 import synth

    wa = synth.workload(1, epochs=2, channels=3, samples=1024, seed=91)
    wb = synth.workload(1, epochs=2, channels=3, samples=1024, seed=92)
    settings = empi_b200.DecompositionSettings(12, 0.0)
    shapes = [e.shape for e in wa.epochs]
    b = empi_b200.Batch(variant, 0.01, settings, shapes, wa.fs, engine=engine)
    b.load(wa.epochs)
    b.run()
    ra = [b.result(e) for e in range(2)]
    b.load(wb.epochs)
    b.run()
    rb = [b.result(e) for e in range(2)]
    b.close()
    fresh = empi_b200.Batch(variant, 0.01, settings, shapes, wb.fs, engine=engine)
    fresh.load(wb.epochs)
    fresh.run()
    rf = [fresh.result(e) for e in range(2)]
    fresh.close()
    for x, y, z in zip(ra, rb, rf):
        assert not np.array_equal(x.atoms, y.atoms)
        for field in ("atoms", "counts", "energies", "indices", "totals"):
            assert np.array_equal(getattr(y, field), getattr(z, field), equal_nan=field == "energies"), field


def decode_book(data):
    """Minimal MPv5 decoder (field conversions of the reference's utils/readbook.cpp)."""
    import struct

    pos = 6
    out = {"atoms": []}
    while pos < len(data):
        bid = data[pos]
        ln = struct.unpack(">I", data[pos + 1:pos + 5])[0]
        if bid in (1, 2):
            pos += 5 + ln
        elif bid == 7:
            pos += 11
        elif bid == 8:
            pos += 5 + ln
        elif bid == 9:
            end = pos + 5 + ln
            pos += 7
            while pos < end:
                vals = struct.unpack(">6f", data[pos + 2:pos + 26])
                out["atoms"].append(vals)
                pos += 26
        else:
            raise ValueError(bid)
    return out


def test_cli_book_matches_reference(tmp_path):
    case = [c for c in CASES if c["name"] == "smp0"][0]
    fs, x = case_signal(case)
    x.astype(np.float32).tofile(tmp_path / "smp0.bin")
    (tmp_path / "smp0.cfg").write_text(open(os.path.join(GOLDEN, "smp0.cfg")).read())
    cli = os.path.join(os.path.dirname(empi_b200.LIB_PATH), "empi-gpu")
    p = subprocess.run([cli, "-x", "smp0.cfg"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.splitlines()[:3] == open(os.path.join(GOLDEN, "smp0.stdout")).read().splitlines()[:3]
    assert p.stdout.rstrip().endswith("END")
    got = (tmp_path / "smp0_smp.b").read_bytes()
    ref = open(os.path.join(GOLDEN, "smp0.b"), "rb").read()
    assert len(got) == len(ref)
    head = 6 + 9 + 32 + 11 + 7 + 4 * 1280
    assert got[:head] == ref[:head]
    ga, ra = decode_book(got)["atoms"], decode_book(ref)["atoms"]
    assert len(ga) == len(ra) == 50
    for g, r in zip(ga, ra):
        assert all(abs(a - b) <= 2e-5 * max(1.0, abs(b)) for a, b in zip(g[:5], r[:5]))


def compare_protocol(got, ref):
    """Progress lines (src/empi.cpp:159, src/classes.cpp:41-48, 83): the same
    lines in the same order; ATOM percentages within print precision."""
    g, r = got.splitlines(), ref.splitlines()
    assert len(g) == len(r), (len(g), len(r))
    for a, b in zip(g, r):
        fa, fb = a.split("\t"), b.split("\t")
        assert fa[0] == fb[0] and len(fa) == len(fb), (a, b)
        if fa[0] == "ATOM":
            assert fa[1:3] == fb[1:3], (a, b)
            for x, y in zip(fa[3:], fb[3:]):
                assert abs(float(x) - float(y)) <= 2e-4 * max(1.0, abs(float(y))), (a, b)
        else:
            assert a == b


@pytest.mark.parametrize("variant", ["MMP2", "SMP"])
def test_cli_streams_epochs_in_batches(tmp_path, variant):
    """Epochs stream through the device in batches (gpuEpochsPerBatch), the
    next batch read from the file and copied to the device while the current
    one runs, and the progress lines printed as the device advances.  For a
    5-epoch, 3-channel file and every batch size the protocol lines and the
    book match the reference CLI's own (tests/golden/stream_*), and a
    truncated last epoch still ends the job with fileIsTruncated after the
    complete epochs are written (src/empi.cpp:148-164, src/io.cpp:48-55).
    Sharding every batch across engines (EMPI_DEVICES) changes no byte."""
    from golden.make_golden import STREAM_CONFIG, stream_signal

    data = stream_signal()
    cli = os.path.join(os.path.dirname(empi_b200.LIB_PATH), "empi-gpu")
    name = f"stream_{variant.lower()}"
    ref_out = open(os.path.join(GOLDEN, name + ".stdout")).read()
    ref_book = open(os.path.join(GOLDEN, name + ".b"), "rb").read()
    ref_atoms = decode_book(ref_book)["atoms"]
    outs = {}
    # (batch size, truncated file, EMPI_DEVICES): "0,0" shards every batch
    # across two engines, both on the one GPU these tests get
    runs = ((1, False, None), (2, False, None), (64, False, None), (2, True, None), (2, False, "0,0"),
            (64, False, "0,0"))
    for per, trunc, devs in runs:
        d = tmp_path / f"b{per}{'t' if trunc else ''}{'d' if devs else ''}"
        d.mkdir()
        (data[:-5] if trunc else data).tofile(d / "sig.bin")
        (d / "run.cfg").write_text(STREAM_CONFIG.format(mp=variant) + f"gpuEpochsPerBatch {per}\n")
        env = dict(os.environ, **({"EMPI_DEVICES": devs} if devs else {}))
        p = subprocess.run([cli, "run.cfg"], cwd=d, capture_output=True, text=True, timeout=300, env=env)
        key = (per, trunc) if not devs else (per, "sharded")
        outs[key] = (p.returncode, p.stdout, (d / f"sig_{variant.lower()[:3]}.b").read_bytes())
    for per in (2, 64):
        assert outs[(per, "sharded")] == outs[(64, False)], per  # sharded across engines: the same bytes
    for per in (1, 2, 64):
        rc, out, book = outs[(per, False)]
        assert rc == 0 and out.count("START") == 5
        compare_protocol(out, ref_out)
        assert len(book) == len(ref_book)
        got_atoms = decode_book(book)["atoms"]
        assert len(got_atoms) == len(ref_atoms)
        for g, r in zip(got_atoms, ref_atoms):
            assert all(abs(x - y) <= 2e-5 * max(1.0, abs(y)) for x, y in zip(g[:5], r[:5])), (per, g, r)
        assert outs[(per, False)] == outs[(64, False)]  # whatever the batch size
    rc, out, book = outs[(64, False)]
    rc_t, out_t, book_t = outs[(2, True)]
    assert rc_t != 0 and "ERROR\tfileIsTruncated" in out_t
    assert out_t.count("START") == 4
    # the four complete epochs are written as in the full run
    assert book.startswith(book_t) and len(book_t) < len(book)


@pytest.mark.parametrize("variant", ["mmp1", "mmp3"])
def test_more_than_64_channels(engine, variant):
    """MMP1/MMP3 sum over any channel count (src/gabor.cpp:62-70): 80 channels
    against the restatement."""
    from empi_b200 import synth

    w = synth.workload(1, epochs=1, channels=80, samples=600, seed=19)
    x = w.epochs[0]
    res = empi_b200.decompose_epochs(variant, [x], w.fs, 0.02, 6, 100.0, engine=engine)[0]
    ora = O.decompose(variant, w.fs, x.T.astype(np.float64), 0.02, 6, 100.0)
    for c in range(80):
        compare_sequences(ora.atoms[c, : ora.natoms[c]], res.atoms[c, : res.counts[c]], ora.margins[0],
                          ora.energies[0] if c == 0 else None, res.energies if c == 0 else None,
                          label=f"{variant} 80ch ch{c}")
