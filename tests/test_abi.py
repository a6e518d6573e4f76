"""The C ABI library without a GPU: it loads, exports every symbol the header
declares, and its host-side parts (dictionary geometry, config parsing, book
writing) match the reference."""
import math
import os
import re

import numpy as np
import pytest

import empi_b200
from helpers import GOLDEN, case_signal, golden
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "empi_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(empi_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    L = empi_b200.load_library()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(empi_b200.EXPORTS)
    assert L.empi_abi_version() == 3


@pytest.mark.parametrize("fs,n,eps", [(128.0, 1280, 0.01), (256.0, 5120, 0.01), (512.0, 16384, 0.005),
                                      (512.0, 16384, 0.001), (256.0, 513, 0.01)])
def test_dictionary_matches_oracle(fs, n, eps):
    got = empi_b200.dictionary_scales(eps, fs, n)
    ref = O.geometry(fs, n, eps)
    assert len(got) == len(ref)
    for a, b in zip(got, ref):
        assert a[1:] == b[1:]
        assert a[0] == b[0]


def test_dictionary_with_limits():
    got = empi_b200.dictionary_scales(0.01, 100.0, 1000, 0.05, 3.0, 30.0)
    assert got == [tuple(v) for v in O.geometry(100.0, 1000, 0.01, 0.05, 3.0, 30.0)]


def test_book_writer_is_byte_identical_to_reference(tmp_path):
    case = [c for c in golden()["cases"] if c["name"] == "smp0"][0]
    fs, x = case_signal(case)
    atoms = np.array(case["atoms"])  # [1, n, 6]
    path = tmp_path / "book.b"
    empi_b200.book_write(path, 1, fs, x.T, atoms, case["counts"])
    assert path.read_bytes() == open(os.path.join(GOLDEN, "smp0.b"), "rb").read()


def write_cfg(d, **kv):
    base = dict(energyError="0.01", maximalNumberOfIterations="5", energyPercent="99.0", MP="SMP",
                nameOfDataFile=str(d / "sig.bin"), nameOfOutputDirectory=str(d), samplingFrequency="128.0",
                numberOfChannels="2", selectedChannels="1-2")
    base.update(kv)
    p = d / "cfg"
    p.write_text("# comment line\n" + "".join(f"{k} {v}\n" for k, v in base.items() if v is not None))
    return p


@pytest.mark.parametrize("kv,msg", [
    (dict(energyError=None), "missingConfigurationEntry:energyError"),
    (dict(energyError="1.5"), "invalidEnergyErrorValue"),
    (dict(maximalNumberOfIterations="0"), "invalidMaximalNumberOfIterations"),
    (dict(energyPercent="100.5"), "invalidEnergyPercentValue"),
    (dict(nameOfDataFile="/nonexistent/sig.bin"), "couldNotOpenSignalFile"),
    (dict(samplingFrequency="0"), "invalidSamplingFrequency"),
    (dict(numberOfChannels="-1"), "invalidNumberOfChannels"),
    (dict(selectedChannels="1-3"), "invalidSubsetSpecification"),
    (dict(MP="XYZ"), "unsupportedDecompositionType"),
    (dict(numberOfSamplesInEpoch="0"), "invalidNumberOfSamplesInEpoch"),
    (dict(selectedEpochs="1"), "missingConfigurationEntry:numberOfSamplesInEpoch"),
])
def test_config_errors_match_reference_messages(tmp_path, kv, msg):
    np.zeros(256, np.float32).tofile(tmp_path / "sig.bin")
    cfg = write_cfg(tmp_path, **kv)
    with pytest.raises(empi_b200.EmpiError) as ei:
        empi_b200.run_config(cfg)
    assert ei.value.message == msg


def test_synth_workloads_are_seeded():
    from empi_b200 import synth

    a = synth.workload(1, epochs=1, channels=2, samples=300)
    b = synth.workload(1, epochs=1, channels=2, samples=300)
    assert np.array_equal(a.epochs[0], b.epochs[0])
    w = synth.workload(3, epochs=5)
    assert len(w.epochs) == 5 and all(512 <= e.shape[0] <= 16384 for e in w.epochs)


@pytest.mark.parametrize("fs,n,eps", [(128.0, 1280, 0.01), (256.0, 5120, 0.01), (512.0, 16384, 0.001)])
def test_error_bound_constants(fs, n, eps):
    """The certified FP32 bound per scale: a positive FFT error constant that
    grows with the transform's passes and the Gaussian's width, and
    rho = 1 / (1 - expFactor) of the worst phase-dependent bin (other than
    k = 0 and the Nyquist bin, which are real), recomputed here in FP64."""
    geo = empi_b200.dictionary_scales(eps, fs, n)
    bnd = empi_b200.dictionary_error_bounds(eps, fs, n)
    assert len(bnd) == len(geo)
    u = 2.0 ** -24
    for (s, nfft, fcount, tcount), (bd, rho, tph, klo, khi) in zip(geo, bnd):
        assert 0 < klo <= khi + 1 <= fcount
        # at least the rounding of the samples and of the Gaussian (2 * 9 u per
        # unit of the Gaussian's sum s fs + 1), at most a few thousand u per unit
        assert 18 * u * (s * fs + 1) <= bd <= 4000 * u * (s * fs + 2)
        nh = nfft // 2
        others = klo > 1 or min(fcount - 1, nh - 1) > khi
        x = s * fs / nfft
        want = 1.0 / (1.0 - math.exp(-2 * math.pi * x * x)) if others else 1.0
        assert rho == pytest.approx(want, rel=1e-5)
        assert tph >= 7 * u + rho * 68 * u


def test_tune_cache_lookup(tmp_path):
    """The engine's reader of the autotuner's cache (empi_tune_lookup):
    entries match on (mode, channels, fs, samples, energyError); samples 0 is
    the entry of uneven batches; unknown keys and string values are skipped."""
    from empi_b200 import autotune

    path = tmp_path / "cache.json"
    e1 = dict(mode=0, channels=1, fs=256.0, samples=5120, energy_error=0.01, transform_cap=2048,
              iterations_per_graph=16, wide_mask=5, gpu="NVIDIA B200", tuned_ms=1.5)
    e2 = dict(mode=0, channels=1, fs=256.0, samples=0, energy_error=0.01, transform_cap=1024,
              iterations_per_graph=4, wide_mask=0, variant="smp")
    autotune.write_cache(str(path), e1)
    autotune.write_cache(str(path), e2)
    autotune.write_cache(str(path), dict(e1, wide_mask=4))  # replaces e1
    assert empi_b200.tune_lookup(str(path), 0, 1, 256.0, 5120, 0.01) == (2048, 16, 4, -1)
    assert empi_b200.tune_lookup(str(path), 0, 1, 256.0, 0, 0.01) == (1024, 4, 0, -1)
    autotune.write_cache(str(path), dict(e2, persistent=1))
    assert empi_b200.tune_lookup(str(path), 0, 1, 256.0, 0, 0.01) == (1024, 4, 0, 1)
    assert empi_b200.tune_lookup(str(path), 3, 1, 256.0, 5120, 0.01) is None
    assert empi_b200.tune_lookup(str(path), 0, 1, 256.0, 5120, 0.02) is None
    bad = tmp_path / "bad.json"
    bad.write_text('{"entries": [{"mode": 0,, }]}')
    with pytest.raises(empi_b200.EmpiError) as ei:
        empi_b200.tune_lookup(str(bad), 0, 1, 256.0, 5120, 0.01)
    assert ei.value.message == "invalidTuneCache"
    with pytest.raises(empi_b200.EmpiError):
        empi_b200.tune_lookup(str(tmp_path / "missing.json"), 0, 1, 256.0, 5120, 0.01)


def test_tune_workload_key():
    from empi_b200 import autotune, synth

    w = synth.workload(1, epochs=2, channels=3, samples=700, seed=1)
    assert autotune.workload_key("mmp2", w.epochs, w.fs, 0.01) == dict(mode=0, channels=1, fs=256.0, samples=700,
                                                                     energy_error=0.01)
    assert autotune.workload_key("mmp3", w.epochs, w.fs, 0.01)["mode"] == 3
    u = synth.workload(3, epochs=3)
    assert autotune.workload_key("smp", u.epochs, u.fs, 0.01)["samples"] == 0


def test_proposal_weights_format(tmp_path):
    """The proposer's weights file: "EMPIPN01", int32 count, float32 parameters
    in the layout the engine reads (empi_proposal_parameter_count)."""
    from empi_b200 import proposal as P

    assert P.parameter_count() == sum(int(np.prod(s)) for _, s in P.LAYOUT) == 22256
    w = P.init_weights(4)
    path = tmp_path / "w.bin"
    P.save_weights(str(path), w)
    data = path.read_bytes()
    assert data[:8] == b"EMPIPN01" and len(data) == 12 + 4 * w.size
    np.testing.assert_array_equal(P.load_weights(str(path)), w)
    path.write_bytes(b"EMPIPN00" + data[8:])
    with pytest.raises(ValueError):
        P.load_weights(str(path))
    parts = P.unpack(w)
    assert parts["w2"].shape == (32, 16, 3, 3) and parts["b4"].shape == (16,)
