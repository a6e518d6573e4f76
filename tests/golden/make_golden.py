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
  stream_*.b/.stdout  (--cli) the reference CLI's book and progress lines
                  for a 5-epoch, 3-channel file, MMP2 and SMP
  full/*.npz      (--full) the benchmark configurations at full size: every
                  atom of the 8-epoch MMP2 workload, 4 channels of the 32-channel
                  MMP3 epoch, 16 of the 512 batched SMP instances, and a
                  2^20-point energyError 0.001 case (FULL_CASES)
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


# Full-size cases at the benchmark configurations, stored compactly as .npz
# under full/ (atoms, counts, residual-energy trajectory, restatement margins).
# name, variant, workload, workload overrides, channel subset per epoch (None =
# all), epochs/instances, energyError, iterations, energyPercent, pinned by
# ("reference": empi's own classes; "restatement": mp_oracle.c, used where the
# reference's workspace does not fit in host memory)
FULL_CASES = [
    # MMP2 19 ch x 8 epochs x 5120 @256 Hz, 100 iterations: the bench workload, every atom
    ("mmp2_19x8x5120", "mmp2", 1, {}, None, 8, 0.01, 100, 99.0, "reference"),
    # MMP3 32 ch x 16384 @512 Hz, energyError 0.005: 4 channels of epoch 0 (the
    # reference's workspace for all 32 needs ~131 GB of host memory)
    ("mmp3_4x16384_512", "mmp3", 2, {"epochs": 1}, 4, 1, 0.005, 50, 100.0, "reference"),
    # batched SMP: the first 16 seeded instances of the 512, first two channels each
    ("smp_batch_16x2", "smp", 3, {"epochs": 16}, 2, 16, 0.01, 150, 99.5, "reference"),
    # energyError 0.001 at 16384 samples @512 Hz (Nfft up to 2^20, 144 scales):
    # 2.7e9 dictionary values per channel, ~108 GB in the reference's workspace,
    # 22 GB in the restatement's
    ("smp_16384_512_eps0001", "smp", 4, {"epochs": 1}, 1, 1, 0.001, 20, 100.0, "restatement"),
]


def full_main(names):
    os.makedirs(os.path.join(HERE, "full"), exist_ok=True)
    for name, variant, wl, ov, csub, nep, eps, iters, pct, pin in FULL_CASES:
        if names and name not in names:
            continue
        w = synth.workload(wl, **ov)
        rec = {"atoms": [], "counts": [], "energies": [], "margins": [], "indices": []}
        shas = []
        t0 = __import__("time").time()
        for e in range(nep):
            x = w.epochs[e] if csub is None else w.epochs[e][:, :csub]
            x = np.ascontiguousarray(x)
            shas.append(__import__("hashlib").sha256(x.tobytes()).hexdigest())
            xs = x.T.astype(np.float64)
            m = O.decompose(variant, w.fs, xs, eps, iters, pct)
            r = O.ref_decompose(variant, w.fs, xs, eps, iters, pct) if pin == "reference" else m
            rec["atoms"].append(r.atoms)
            rec["counts"].append(r.natoms)
            rec["energies"].append(r.energies)
            rec["margins"].append(m.margins)
            rec["indices"].append(m.indices)
            print(name, e, list(r.natoms), f"{__import__('time').time() - t0:.0f}s", flush=True)
        ragged = len({a.shape for a in rec["atoms"]}) > 1
        out = {"meta": json.dumps({"name": name, "variant": variant, "workload": wl, "overrides": ov,
                                   "channels": csub, "epochs": nep, "fs": w.fs, "energy_error": eps,
                                   "iterations": iters, "energy_percent": pct, "pinned_by": pin,
                                   "signal_sha_f32": shas})}
        for k, v in rec.items():
            if ragged:
                for e, a in enumerate(v):
                    out[f"{k}_{e}"] = a
            else:
                out[k] = np.stack(v)
        np.savez_compressed(os.path.join(HERE, "full", name + ".npz"), **out)


STREAM_CONFIG = ("energyError 0.01\nmaximalNumberOfIterations 12\nenergyPercent 99.0\nMP {mp}\n"
                 "nameOfDataFile sig.bin\nnameOfOutputDirectory .\nsamplingFrequency 256.0\n"
                 "numberOfChannels 3\nselectedChannels 1-3\nnumberOfSamplesInEpoch 700\n")


def stream_signal():
    """Five 3-channel epochs of 700 samples (workload 1, seed 11), as one file."""
    w = synth.workload(1, epochs=5, channels=3, samples=700, seed=11)
    return np.concatenate([e.reshape(-1) for e in w.epochs]).astype(np.float32)


def cli_main():
    """The reference CLI on a multi-epoch file (MMP2 and SMP): its book and
    stdout, for the streaming tests of the GPU CLI."""
    data = stream_signal()
    for mp in ("MMP2", "SMP"):
        with tempfile.TemporaryDirectory() as d:
            data.tofile(os.path.join(d, "sig.bin"))
            with open(os.path.join(d, "run.cfg"), "w") as f:
                f.write(STREAM_CONFIG.format(mp=mp))
            proc = subprocess.run([O.ref_cli(), "run.cfg"], cwd=d, capture_output=True, text=True, check=True)
            name = f"stream_{mp.lower()}"
            shutil.copy(os.path.join(d, f"sig_{mp.lower()[:3]}.b"), os.path.join(HERE, name + ".b"))
            with open(os.path.join(HERE, name + ".stdout"), "w") as f:
                f.write(proc.stdout)
        print(name, proc.stdout.count("ATOM"), "atom lines")


def main():
    if "--cli" in sys.argv:
        return cli_main()
    if "--scale" in sys.argv:
        return scale_main()
    if "--full" in sys.argv:
        return full_main([a for a in sys.argv[1:] if not a.startswith("--")])
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
