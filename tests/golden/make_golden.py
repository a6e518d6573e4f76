"""Regenerates the golden fixtures in this directory from the reference's own
code (empi's src/*.cpp compiled by oracle/Makefile against the project's FFT
shim).  Runs in a container that has the reference sources:

    make -C oracle ref && python tests/golden/make_golden.py

Writes:
  cases.json      per case: inputs (seeded), reference atoms (FP64 params per
                  channel), residual-energy trajectory, error text if any
  smp0.b          the reference CLI's book for workload 0 (SMP 1x1280 @128 Hz)
  smp0.cfg        the config that produced it (signal: smp0.bin, regenerated
                  from the seed by the tests)
  scale_cases.json  larger cases at BASELINE shapes (the bench workload's first
                  epoch, 16384-sample windows that need folded transforms,
                  energyError 0.001 with Nfft up to 2^17), with the
                  restatement's best-to-second margins for the tie rule
"""
from __future__ import annotations

import json
import math
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from empi_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

# name, variant, workload index, overrides, energyError, iterations, energyPercent, limits
CASES = [
    ("smp0", "smp", 0, {}, 0.01, 50, 99.0, {}),
    ("smp_2ch_512", "smp", 0, {"channels": 2, "samples": 512, "seed": 7}, 0.02, 20, 99.0, {}),
    ("mmp1_3ch_768", "mmp1", 1, {"epochs": 1, "channels": 3, "samples": 768, "seed": 11}, 0.02, 15, 99.0, {}),
    ("mmp2_4ch_1024", "mmp2", 1, {"epochs": 1, "channels": 4, "samples": 1024, "seed": 12}, 0.01, 20, 99.0, {}),
    ("mmp3_3ch_1024", "mmp3", 2, {"epochs": 1, "channels": 3, "samples": 1024, "seed": 13}, 0.01, 20, 100.0, {}),
    ("smp_limits", "smp", 0, {"samples": 1000, "seed": 21}, 0.01, 25, 99.0,
     {"smin": 0.05, "smax": 3.0, "fmax": 30.0}),
    ("smp_tiny_64", "smp", 0, {"samples": 64, "seed": 31}, 0.01, 10, 99.0, {}),
    ("smp_stop_early", "smp", 0, {"samples": 800, "seed": 41}, 0.05, 40, 80.0, {}),
]


def case_signal(wl, ov):
    w = synth.workload(wl, **ov)
    return w.fs, w.epochs[0]


SCALE_CASES = [
    ("mmp2_bench_epoch0", "mmp2", 1, {"epochs": 1}, 0.01, 15, 99.0, {}),
    ("mmp3_2x8192_512", "mmp3", 2, {"epochs": 1, "channels": 2, "samples": 8192}, 0.005, 6, 100.0, {}),
    ("smp_16384_512_fold", "smp", 2, {"epochs": 1, "channels": 1, "samples": 16384}, 0.005, 4, 100.0, {}),
    ("smp_2048_128_eps001", "smp", 0, {"samples": 2048, "seed": 44}, 0.001, 5, 100.0, {}),
]


def scale_main():
    out = []
    for name, variant, wl, ov, eps, iters, pct, lim in SCALE_CASES:
        fs, x = case_signal(wl, ov)
        xs = x.T.astype(np.float64)
        kw = dict(smin=lim.get("smin", 0.0), smax=lim.get("smax", math.inf), fmax=lim.get("fmax", math.inf))
        r = O.ref_decompose(variant, fs, xs, eps, iters, pct, **kw)
        m = O.decompose(variant, fs, xs, eps, iters, pct, **kw)
        rec = {"name": name, "variant": variant, "workload": wl, "overrides": ov, "fs": fs, "energy_error": eps,
               "iterations": iters, "energy_percent": pct, "limits": lim, "channels": int(x.shape[1]),
               "samples": int(x.shape[0]),
               "signal_sha_f32": __import__("hashlib").sha256(x.tobytes()).hexdigest(),
               "counts": [int(v) for v in r.natoms],
               "atoms": [[list(map(float, r.atoms[c, a])) for a in range(r.natoms[c])] for c in range(xs.shape[0])],
               "energies": [[None if not np.isfinite(v) else float(v) for v in row] for row in r.energies],
               "margins": [[None if not np.isfinite(v) else float(v) for v in row] for row in m.margins]}
        out.append(rec)
        print(name, rec["counts"], flush=True)
    with open(os.path.join(HERE, "scale_cases.json"), "w") as f:
        json.dump({"cases": out}, f, indent=1)


def main():
    if "--scale" in sys.argv:
        return scale_main()
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libempiref.so missing: run `make -C oracle ref` first")
    out = []
    for name, variant, wl, ov, eps, iters, pct, lim in CASES:
        fs, x = case_signal(wl, ov)
        xs = x.T.astype(np.float64)
        kw = dict(smin=lim.get("smin", 0.0), smax=lim.get("smax", math.inf), fmax=lim.get("fmax", math.inf))
        rec = {"name": name, "variant": variant, "workload": wl, "overrides": ov, "fs": fs,
               "energy_error": eps, "iterations": iters, "energy_percent": pct, "limits": lim,
               "channels": int(x.shape[1]), "samples": int(x.shape[0]),
               "signal_sha_f32": __import__("hashlib").sha256(x.tobytes()).hexdigest()}
        r = O.ref_decompose(variant, fs, xs, eps, iters, pct, **kw)
        rec["counts"] = [int(v) for v in r.natoms]
        rec["atoms"] = [[list(map(float, r.atoms[c, a])) for a in range(r.natoms[c])] for c in range(xs.shape[0])]
        rec["energies"] = [[None if not np.isfinite(v) else float(v) for v in row] for row in r.energies]
        out.append(rec)
        print(name, rec["counts"])
    # error cases from the reference
    errs = []
    z = np.zeros((1, 256))
    try:
        O.ref_decompose("smp", 128.0, z, 0.01, 5, 99.0)
        errs.append({"name": "zeros", "error": None})
    except RuntimeError as e:
        errs.append({"name": "zeros", "error": str(e)})
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump({"cases": out, "errors": errs}, f, indent=1)

    # reference CLI book for workload 0
    fs, x = case_signal(0, {})
    with tempfile.TemporaryDirectory() as d:
        x.astype(np.float32).tofile(os.path.join(d, "smp0.bin"))
        cfg = ("energyError 0.01\nmaximalNumberOfIterations 50\nenergyPercent 99.0\nMP SMP\n"
               "nameOfDataFile smp0.bin\nnameOfOutputDirectory .\nsamplingFrequency 128.0\n"
               "numberOfChannels 1\nselectedChannels 1\n")
        with open(os.path.join(d, "smp0.cfg"), "w") as f:
            f.write(cfg)
        proc = subprocess.run([O.ref_cli(), "smp0.cfg"], cwd=d, capture_output=True, text=True, check=True)
        shutil.copy(os.path.join(d, "smp0_smp.b"), os.path.join(HERE, "smp0.b"))
        shutil.copy(os.path.join(d, "smp0.cfg"), os.path.join(HERE, "smp0.cfg"))
        with open(os.path.join(HERE, "smp0.stdout"), "w") as f:
            f.write(proc.stdout)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
