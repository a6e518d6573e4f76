"""Autotuner of the engine's launch shape, per workload.

    python -m empi_b200.autotune --workload 1 [--epochs E] [--iterations I]
                                 [--cache empi_b200/tuned_b200.json]

The reference runs its scales with OpenMP's dynamic schedule
(src/gabor.cpp:77-82) and has no launch shape to choose.  On the B200 the
refresh kernels' shape decides throughput, and the best one depends on the
dictionary (Nfft range, sub-FFT sizes L, fold counts), the channels per MP loop
and the variant.  The tuner searches, on the device and by device time of
whole batch runs (CUDA events, stats.run_ms), over:

* transform_cap -- the largest shared-memory sub-FFT (4096, 2048, 1024): a
  smaller cap splits large transforms into more residues and folds;
* iterations_per_graph -- MP iterations per CUDA-graph launch (4, 8, 16);
* per sub-FFT size present in the workload, the refresh variant: two CTAs per
  SM at 64 registers (the default) or one at 128 registers without spills
  (wide_mask bit log2 L);
* persistent -- the MP loop as one persistent cooperative kernel per chunk of
  iterations (1) or as the multi-kernel CUDA graph (0); the engine's own
  choice, without a tuned entry, is by batch size.

The search is coordinate descent from the default shape, keeping a change only
when it is faster by more than 1 %, and every candidate shape is checked to
give exactly the default shape's atoms (the certified FP32 bound makes the
argmax independent of the FFT decomposition).  Results go to a JSON cache keyed
by (mode, channels per MP loop, fs, samples -- 0 for uneven batches --,
energyError) that the engine reads through empi_engine_opts.tune_cache (the
CLI's gpuTuneCache key), together with default and tuned atoms/s.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile

import numpy as np

import empi_b200
from empi_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_CACHE = os.path.join(HERE, "tuned_b200.json")
CAPS = (4096, 2048, 1024)
GRAPH_ITERS = (8, 4, 16)
MODES = {"smp": 0, "mmp2": 0, "mmp1": 1, "mmp3": 3}


def workload_key(variant, epochs, fs, energy_error):
    """The cache key of a list of (N, C) epochs (empi_tune_lookup's)."""
    multi = variant in ("mmp1", "mmp3") and any(e.shape[1] > 1 for e in epochs)
    mode = MODES[variant] if multi else 0
    loop_c = {e.shape[1] if multi else 1 for e in epochs}
    samples = {e.shape[0] for e in epochs}
    return {"mode": mode, "channels": loop_c.pop() if len(loop_c) == 1 else 0, "fs": float(fs),
            "samples": samples.pop() if len(samples) == 1 else 0, "energy_error": float(energy_error)}


def _same_key(a, b):
    return all(abs(float(a[k]) - float(b[k])) <= 1e-9 * max(1.0, abs(float(b[k])))
               for k in ("mode", "channels", "fs", "samples", "energy_error"))


def read_cache(path):
    try:
        with open(path) as f:
            return json.load(f)
    except OSError:
        return {"version": 1, "entries": []}


def write_cache(path, entry):
    """Adds or replaces the entry of entry's key."""
    cache = read_cache(path)
    cache["entries"] = [e for e in cache["entries"] if not _same_key(e, entry)] + [entry]
    with open(path, "w") as f:
        json.dump(cache, f, indent=1)
        f.write("\n")


class _Trial:
    """Runs a workload with one launch shape, through a one-entry tune cache."""

    def __init__(self, variant, epochs, fs, energy_error, settings, key, device):
        self.variant, self.epochs, self.fs, self.eps = variant, epochs, fs, energy_error
        self.settings, self.key, self.device = settings, key, device
        self.dir = tempfile.TemporaryDirectory()

    def run(self, shape, reps):
        path = os.path.join(self.dir.name, "trial.json")
        with open(path, "w") as f:
            json.dump({"version": 1, "entries": [dict(self.key, **shape)]}, f)
        eng = empi_b200.Engine(device=self.device, tune_cache=path)
        b = empi_b200.Batch(self.variant, self.eps, self.settings, [e.shape for e in self.epochs], self.fs,
                            engine=eng)
        b.load(self.epochs)
        b.run()  # warm-up (graph capture, first touch)
        times = []
        for _ in range(reps):
            b.run()
            times.append(b.stats().run_ms)
        st = b.stats()
        assert st.tuned == 1 and st.transform_cap == shape["transform_cap"]
        atoms = [b.result(e) for e in range(len(self.epochs))]
        b.close()
        eng.close()
        return min(times), st, atoms


def _same_atoms(a, b):
    return all(np.array_equal(x.counts, y.counts) and np.array_equal(x.indices, y.indices) and
               np.allclose(x.atoms, y.atoms, rtol=1e-12, atol=0.0) for x, y in zip(a, b))


def tune(variant, epochs, fs, energy_error, iterations, energy_percent, device=0, reps=3, log=print):
    """Tunes one workload; returns its cache entry."""
    settings = empi_b200.DecompositionSettings(int(iterations), 1.0 - 0.01 * float(energy_percent))
    key = workload_key(variant, epochs, fs, energy_error)
    trial = _Trial(variant, epochs, fs, energy_error, settings, key, device)
    shape = {"transform_cap": CAPS[0], "iterations_per_graph": GRAPH_ITERS[0], "wide_mask": 0}
    t0, st0, ref_atoms = trial.run(shape, reps)
    atoms_per_run = st0.atoms
    log(f"default {shape}: {t0:.2f} ms")
    best_t, best = t0, dict(shape)

    def consider(cand):
        nonlocal best_t, best
        t, st, atoms = trial.run(cand, reps)
        if cand.get("persistent") == 1 and not st.persistent:
            log(f"  {cand}: the persistent kernel does not fit this workload's layout")
            return
        if not _same_atoms(atoms, ref_atoms):
            raise AssertionError(f"shape {cand} changed the atoms")
        better = t < best_t * 0.99
        log(f"  {cand}: {t:.2f} ms{'  <- better' if better else ''}")
        if better:
            best_t, best = t, dict(cand)

    for cap in CAPS[1:]:
        consider(dict(best, transform_cap=cap))
    for k in GRAPH_ITERS[1:]:
        consider(dict(best, iterations_per_graph=k))
    # the loop's form: graph or persistent kernel, against the engine's default
    # by batch size (what the default shape above ran)
    consider(dict(best, persistent=0 if st0.persistent else 1))
    # the sizes present depend on the cap: read them from a run with the best one
    _, st, _ = trial.run(best, 1)
    for lg in range(13):
        if (st.sizes_mask >> lg) & 1:
            consider(dict(best, wide_mask=best["wide_mask"] ^ (1 << lg)))
    entry = dict(key, **best)
    entry.update({"default_ms": round(t0, 3), "tuned_ms": round(best_t, 3),
                  "default_atoms_per_s": round(atoms_per_run / (t0 * 1e-3), 1),
                  "tuned_atoms_per_s": round(atoms_per_run / (best_t * 1e-3), 1),
                  "atoms_per_run": atoms_per_run, "iterations": int(iterations), "epochs": len(epochs),
                  "variant": variant})
    log(f"tuned {best}: {best_t:.2f} ms ({t0 / best_t:.3f}x)")
    return entry


def main():
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--workload", type=int, required=True, help="empi_b200.synth workload index")
    p.add_argument("--epochs", type=int, default=0)
    p.add_argument("--iterations", type=int, default=0, help="MP iterations per run (default: the workload's)")
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--cache", default=DEFAULT_CACHE)
    a = p.parse_args()
    w = synth.workload(a.workload, epochs=a.epochs or None)
    entry = tune(w.variant, w.epochs, w.fs, w.energy_error, a.iterations or w.iterations, w.energy_percent,
                 a.device, a.reps)
    entry["workload"] = w.name
    entry["gpu"] = _gpu_name(a.device)
    write_cache(a.cache, entry)
    print(json.dumps(entry))


def _gpu_name(device):
    try:
        import torch

        return torch.cuda.get_device_name(device)
    except Exception:
        return None


if __name__ == "__main__":
    main()
