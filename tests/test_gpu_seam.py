"""The drop-in proof for empi's Workspace seam (inc/classes.hpp:63-80): the
reference's own Decomposition, SmpDecomposition, Mmp1/Mmp2/Mmp3Decomposition
loops (src/classes.cpp, src/mmp.cpp, compiled unmodified by oracle/Makefile's
`seam` target) run on the GPU workspace through the adapter a maintainer
would add (empi_b200/adapter/gpu_workspace.hpp), and their atoms match the
reference goldens.  This is the per-iteration host path (one host round trip
per MP iteration); the batched engine is the fast path."""
import os
import subprocess

import numpy as np
import pytest

from helpers import case_limits, case_signal, compare_sequences, golden

pytestmark = pytest.mark.gpu

SEAM = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "seam")
NAMES = ["smp0", "smp_2ch_512", "mmp1_3ch_768", "mmp2_4ch_1024", "mmp3_3ch_1024", "smp_limits"]


@pytest.mark.parametrize("name", NAMES)
def test_reference_loops_on_the_gpu_workspace(tmp_path, name):
    assert os.path.exists(SEAM), "oracle/_ref/seam is built by `make -C oracle seam` where the reference is"
    case = [c for c in golden()["cases"] if c["name"] == name][0]
    fs, x = case_signal(case)
    lim = case_limits(case)
    C, N = x.shape[1], x.shape[0]
    xin = np.ascontiguousarray(x.T.astype(np.float64))
    xin.tofile(tmp_path / "in.f64")
    args = [SEAM, case["variant"], repr(fs), str(C), str(N), repr(case["energy_error"]), str(case["iterations"]),
            repr(case["energy_percent"]), repr(lim["smin"]), repr(lim["smax"] if np.isfinite(lim["smax"]) else 0.0),
            repr(lim["fmax"] if np.isfinite(lim["fmax"]) else 0.0), str(tmp_path / "in.f64"), str(tmp_path / "out.f64")]
    p = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    # the reference's loop printed its own progress protocol (src/classes.cpp:41-48)
    assert p.stdout.count("ATOM") == sum(case["counts"][:1] if case["variant"] != "smp" else case["counts"])
    out = np.fromfile(tmp_path / "out.f64")
    pos, compared = 0, 0
    from oracle import oracle as O

    ora = O.decompose(case["variant"], fs, xin, case["energy_error"], case["iterations"], case["energy_percent"],
                      **lim)
    smp = case["variant"] == "smp" or C == 1
    for c in range(C):
        n = int(out[pos])
        atoms = out[pos + 1: pos + 1 + 6 * n].reshape(n, 6)
        pos += 1 + 6 * n
        compared += compare_sequences(case["atoms"][c], atoms, ora.margins[c if smp else 0],
                                      label=f"{name} seam ch{c}")
    print(f"{name}: {compared} atoms of the reference's own loop on the GPU workspace match the golden")
