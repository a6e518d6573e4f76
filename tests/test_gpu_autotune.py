"""The autotuner (empi_b200/autotune.py) on the device: it searches the launch
shape of a small workload, every shape it tries gives the default shape's
atoms exactly (tune() asserts it), and a batch created with the resulting
cache runs with the tuned shape."""
import numpy as np
import pytest

import empi_b200
from empi_b200 import autotune, synth

pytestmark = pytest.mark.gpu


def test_autotune_small_workload(tmp_path):
    w = synth.workload(1, epochs=2, channels=4, samples=1500, seed=5)
    lines = []
    entry = autotune.tune("mmp2", w.epochs, w.fs, w.energy_error, 12, w.energy_percent, reps=1, log=lines.append)
    assert entry["transform_cap"] in autotune.CAPS
    assert entry["iterations_per_graph"] in autotune.GRAPH_ITERS
    assert entry["tuned_ms"] <= entry["default_ms"]
    assert len(lines) >= 6  # default, two caps, two graph sizes, one or more sizes
    path = str(tmp_path / "cache.json")
    autotune.write_cache(path, entry)
    eng = empi_b200.Engine(tune_cache=path)
    settings = empi_b200.DecompositionSettings(12, 1.0 - 0.01 * w.energy_percent)
    b = empi_b200.Batch("mmp2", w.energy_error, settings, [e.shape for e in w.epochs], w.fs, engine=eng)
    b.load(w.epochs)
    b.run()
    st = b.stats()
    assert st.tuned == 1
    assert (st.transform_cap, st.iterations_per_graph, st.wide_mask) == (
        entry["transform_cap"], entry["iterations_per_graph"], entry["wide_mask"])
    got = b.result(0)
    b.close()
    eng.close()
    ref = empi_b200.decompose_epochs("mmp2", w.epochs, w.fs, w.energy_error, 12, w.energy_percent)[0]
    np.testing.assert_array_equal(got.indices, ref.indices)
    np.testing.assert_allclose(got.atoms, ref.atoms, rtol=1e-12, atol=0)
