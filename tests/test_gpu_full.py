"""Atom-sequence parity at the benchmark configurations, at full size.

The fixtures under tests/golden/full/ were generated by
tests/golden/make_golden.py --full from the reference's own decomposition
classes (empi's src/*.cpp built by oracle/Makefile), except the energyError
0.001 case, whose reference workspace (~108 GB) does not fit the generating
host: that one is pinned to the restatement (oracle/mp_oracle.c), itself
pinned to the reference on every smaller golden.

  mmp2_19x8x5120        every atom of the 8-epoch MMP2 bench workload
  mmp3_4x16384_512      MMP3 at 16384 samples @ 512 Hz, 4 channels, 50 atoms
  smp_batch_16x2        16 of the 512 batched SMP instances (two channels each),
                        150 iterations, decomposed in one uneven batch
  smp_16384_512_eps0001 energyError 0.001, Nfft up to 2^20 (144 scales)

Each test reports how many atoms it compared; the parity rule is
helpers.compare_sequences' (at least 95 % compared, indices exact outside
near-ties, amplitudes 1e-5 relative, phases 1e-5 rad, residual energies 1e-6
relative).
"""
import json
import os

import numpy as np
import pytest

import empi_b200
from helpers import GOLDEN, compare_sequences

pytestmark = pytest.mark.gpu

FULL = os.path.join(GOLDEN, "full")


def load(name):
    z = np.load(os.path.join(FULL, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    keys = ("atoms", "counts", "energies", "margins")
    if "atoms" in z.files:
        per = [{k: z[k][e] for k in keys} for e in range(meta["epochs"])]
    else:
        per = [{k: z[f"{k}_{e}"] for k in keys} for e in range(meta["epochs"])]
    return meta, per


def signals(meta):
    from empi_b200 import synth

    w = synth.workload(meta["workload"], **meta["overrides"])
    out = []
    for e in range(meta["epochs"]):
        x = w.epochs[e] if meta["channels"] is None else w.epochs[e][:, : meta["channels"]]
        out.append(np.ascontiguousarray(x))
    return w.fs, out


def run_and_compare(engine, name):
    meta, ref = load(name)
    fs, xs = signals(meta)
    res = empi_b200.decompose_epochs(meta["variant"], xs, fs, meta["energy_error"], meta["iterations"],
                                     meta["energy_percent"], engine=engine)
    compared = total = 0
    for e, (x, r, g) in enumerate(zip(xs, res, ref)):
        C = x.shape[1]
        smp = meta["variant"] == "smp" or C == 1
        loops = C if smp else 1
        for c in range(C):
            l = c if smp else 0
            n_ref = int(g["counts"][c])
            e_got = r.energies[c] if smp else r.energies
            # residual energies belong to the MP loop: per channel for SMP, once otherwise
            check_e = smp or c == 0
            # the 95 % rule is asserted over the test's atoms below: a genuine
            # near-tie in one channel exempts the rest of that channel only
            n = compare_sequences(g["atoms"][c, :n_ref], r.atoms[c, : r.counts[c]], g["margins"][l],
                                  g["energies"][l] if check_e else None, e_got if check_e else None,
                                  label=f"{name} epoch {e} ch{c}", min_fraction=0.0)
            if c < loops:  # an MMP atom counts once, an SMP channel is its own loop
                compared += n
                total += n_ref
    print(f"{name}: {compared} of {total} atoms compared against {meta['pinned_by']}")
    assert compared >= 0.95 * total
    return compared, total


def test_mmp2_19x8x5120_every_atom(engine):
    compared, total = run_and_compare(engine, "mmp2_19x8x5120")
    assert total == 800


def test_mmp3_4x16384_512(engine):
    run_and_compare(engine, "mmp3_4x16384_512")


def test_smp_batch_16_instances(engine):
    run_and_compare(engine, "smp_batch_16x2")


def test_energy_error_0001_nfft_2_20_against_restatement(engine):
    run_and_compare(engine, "smp_16384_512_eps0001")
