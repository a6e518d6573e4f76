"""The certified FP32 error bound and the exact argmax it guarantees.

The engine ranks dictionary values by FP32 energies and re-scores in FP64
every bin whose certified upper bound reaches the best certified lower bound
(include/empi_b200.h, empi_dictionary_error_bounds).  These tests check:

* every FP32 map value lies inside its certified interval around the FP64
  oracle value (oracle/mp_oracle.c), on signals chosen to stress it -- a
  stationary sinusoid, a constant offset with noise, a periodic pulse train --
  and on 2^20-point transforms (energyError 0.001, 16384 samples @ 512 Hz);
  the largest ratio of measured error to bound is printed per scale;
* on the same stress signals every atom the engine picks is an exact argmax
  of the FP64 maps of its residual (within the 1e-6 relative tie margin the
  parity rule allows), each step checked against the oracle's maps after the
  engine's own previous subtractions, and its modulus matches that value;
* a candidate overflow grows the buffers instead of failing, with the same
  atoms as a run that never overflowed.
"""
import math

import numpy as np
import pytest

import empi_b200
from oracle import oracle as O

pytestmark = pytest.mark.gpu

U = 2.0 ** -24


def stress_signal(kind, n=2048, fs=128.0, seed=5):
    rng = np.random.default_rng(seed)
    t = np.arange(n) / fs
    if kind == "sinusoid":
        x = 3.0 * np.cos(2 * math.pi * 11.3 * t + 0.7) + 0.01 * rng.standard_normal(n)
    elif kind == "offset":
        x = 2.5 + 0.3 * rng.standard_normal(n)
    elif kind == "pulses":
        x = np.where(np.arange(n) % 37 == 0, 1.0, 0.0) + 0.01 * rng.standard_normal(n)
    else:
        raise ValueError(kind)
    return fs, x.astype(np.float32).astype(np.float64)


def check_map_bound(fs, x, eps, scales, engine, label):
    """x: (N,) float64 holding float32 values.  Returns max measured/bound."""
    n = x.size
    geo = empi_b200.dictionary_scales(eps, fs, n)
    bnd = empi_b200.dictionary_error_bounds(eps, fs, n)
    ws = empi_b200.GaborWorkspaceBuilder(eps, engine=engine).prepareWorkspace(fs, 1, n)
    ws.compute(x[None, :])
    B = float(np.max(np.abs(x.astype(np.float32))))
    worst = 0.0
    for j in scales:
        s = geo[j][0]
        bd, rho, tph, klo, khi = bnd[j]
        got = ws.energy_map(j).astype(np.float64)
        ref = O.energy_map(fs, x[None, :], eps, j)
        kc = 2.0 * math.sqrt(2.0) / (s * fs)
        k = np.arange(got.shape[0])[:, None]
        phase = (k < klo) | (k > khi)
        d = math.sqrt(kc) * bd * B * np.where(phase, math.sqrt(rho), 1.0)
        tau = np.where(phase, tph, 8 * U) + 2 * (1 + 4) * U
        hi = np.sqrt(got * (1 + tau)) + d
        lo = np.sqrt(np.maximum(got * (1 - tau), 0.0)) - d
        sr = np.sqrt(ref)
        assert np.all(sr <= hi), (label, j, float(np.max(sr - hi)))
        assert np.all(sr >= lo), (label, j, float(np.max(lo - sr)))
        ratio = float(np.max(np.abs(sr - np.sqrt(got)) / np.maximum(hi - np.sqrt(got), 1e-300)))
        worst = max(worst, ratio)
        print(f"{label} scale {j} (Nfft {geo[j][1]}): max |sqrt(E64) - sqrt(E32)| / bound = {ratio:.3e}")
    ws.close()
    return worst


@pytest.mark.parametrize("kind", ["sinusoid", "offset", "pulses"])
def test_stress_maps_within_certified_bound(engine, kind):
    fs, x = stress_signal(kind)
    nsc = len(empi_b200.dictionary_scales(0.01, fs, x.size))
    worst = check_map_bound(fs, x, 0.01, [0, 1, nsc // 4, nsc // 2, 3 * nsc // 4, nsc - 2, nsc - 1], engine, kind)
    assert worst <= 1.0


def test_maps_within_certified_bound_at_2_20_points(engine):
    from empi_b200 import synth

    w = synth.workload(4, epochs=1, channels=1)
    x = w.epochs[0][:, 0].astype(np.float64)
    geo = empi_b200.dictionary_scales(w.energy_error, w.fs, x.size)
    assert max(g[1] for g in geo) == 1 << 20
    nsc = len(geo)
    worst = check_map_bound(w.fs, x, w.energy_error, [nsc - 1, nsc - 2, nsc - 20, nsc // 2], engine, "eps0.001")
    assert worst <= 1.0


def all_maps(fs, x, eps):
    n = x.size
    geo = O.geometry(fs, n, eps)
    return [O.energy_map(fs, x[None, :], eps, j) for j in range(len(geo))], geo


@pytest.mark.parametrize("kind", ["sinusoid", "offset", "pulses"])
def test_stress_atoms_are_exact_argmax(engine, kind):
    fs, x = stress_signal(kind)
    eps, steps = 0.01, 6
    res = empi_b200.decompose_epochs("smp", [x.astype(np.float32)[:, None]], fs, eps, steps, 100.0,
                                     engine=engine)[0]
    assert int(res.counts[0]) == steps
    r = x.copy()
    for a in range(steps):
        maps, geo = all_maps(fs, r, eps)
        best = max(float(m.max()) for m in maps)
        j, t, f = (int(v) for v in res.indices[0, a])
        e = float(maps[j][f, t])
        assert e >= best * (1 - 1e-6), (kind, a, e, best)
        p = res.atoms[0, a]
        assert abs(p[0] ** 2 - e) <= 1e-6 * e, (kind, a, p[0] ** 2, e)  # modulus^2 is the energy (SMP)
        _, r = O.subtract_atom(p, r, fs, False)
    print(f"{kind}: {steps} atoms, each an exact argmax of the FP64 maps")


def test_candidate_overflow_grows_and_matches(engine):
    fs, x = stress_signal("sinusoid")
    eps, steps = 0.01, 10
    x32 = [x.astype(np.float32)[:, None]]
    ref = empi_b200.decompose_epochs("smp", x32, fs, eps, steps, 100.0, engine=engine)[0]
    small = empi_b200.Engine(candidate_capacity=2)
    b = empi_b200.Batch("smp", eps, empi_b200.DecompositionSettings(steps, 0.0), [x32[0].shape], fs, engine=small)
    b.load(x32)
    b.run()
    got = b.result(0)
    b.close()
    small.close()
    assert int(got.counts[0]) == int(ref.counts[0]) == steps
    np.testing.assert_array_equal(got.indices, ref.indices)
    np.testing.assert_allclose(got.atoms, ref.atoms, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", ["smp0", "mmp1_3ch_768", "mmp3_3ch_1024", "mmp2_4ch_1024"])
def test_candidate_flood_gives_the_same_atoms(engine, name):
    """A wide extra margin (candidate_band 0.5) floods the candidate path with
    thousands of slots and bins: the buffers grow, every candidate is re-scored
    in FP64, and the atoms are the ones the certified bound alone selects."""
    from helpers import case_limits, case_signal, golden

    case = [c for c in golden()["cases"] if c["name"] == name][0]
    fs, x = case_signal(case)
    lim = case_limits(case)
    args = (case["variant"], [x], fs, case["energy_error"], case["iterations"], case["energy_percent"],
            lim["smin"], lim["smax"], lim["fmax"])
    ref = empi_b200.decompose_epochs(*args, engine=engine)[0]
    wide = empi_b200.Engine(candidate_band=0.5)
    got = empi_b200.decompose_epochs(*args, engine=wide)[0]
    wide.close()
    np.testing.assert_array_equal(got.counts, ref.counts)
    np.testing.assert_array_equal(got.indices, ref.indices[..., :3] if got.indices.shape != ref.indices.shape
                                  else ref.indices)
    np.testing.assert_allclose(got.atoms, ref.atoms, rtol=1e-12, atol=1e-300)


def test_proposal_probe_leaves_atoms_unchanged(engine):
    """The proposal-ceiling probe (empi_batch_probe_proposal) only measures:
    same atoms, and the refresh work no certified proposal could skip is part
    of the work the refresh rule did."""
    from empi_b200 import synth

    w = synth.workload(1, epochs=2, channels=4, samples=2000, seed=9)
    settings = empi_b200.DecompositionSettings(20, 1.0 - 0.01 * w.energy_percent)
    ref = empi_b200.decompose_epochs("mmp2", w.epochs, w.fs, w.energy_error, 20, w.energy_percent, engine=engine)
    b = empi_b200.Batch("mmp2", w.energy_error, settings, [e.shape for e in w.epochs], w.fs, engine=engine)
    b.probe_proposal(True)
    b.load(w.epochs)
    b.run()
    st = b.stats()
    got = [b.result(e) for e in range(2)]
    b.close()
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g.indices, r.indices)
        np.testing.assert_allclose(g.atoms, r.atoms, rtol=1e-12, atol=0)
    assert st.probe_dirty_slots > 0 and 0 <= st.probe_needed_slots <= st.probe_dirty_slots
    assert 0 < st.probe_needed_work <= st.probe_dirty_work
    print(f"needed {st.probe_needed_work / st.probe_dirty_work:.3f} of the refresh work")
