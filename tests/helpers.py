"""Shared test helpers: golden fixtures and the parity rule.

Parity rule (atom sequences): the (scale, position, frequency) of each atom
must match the reference exactly unless the oracle's relative margin between
the best and second-best energy at that iteration is below 1e-6 (a near-tie,
whose order the reference itself leaves to heap/OpenMP order); after an
exempt divergence the sequences are not compared further.  Amplitude and
modulus must agree within 1e-5 relative, phase within 1e-5 rad, residual
energies within 1e-6 relative.  Every comparison reports how many atoms it
actually compared and, by default, fails if a near-tie exemption left fewer
than 95 % of the reference's atoms compared.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

TIE_MARGIN = 1e-6
AMP_RTOL = 1e-5
PHASE_ATOL = 1e-5
ENERGY_RTOL = 1e-6


def golden():
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        return json.load(f)


def case_signal(case):
    from empi_b200 import synth

    w = synth.workload(case["workload"], **case["overrides"])
    return w.fs, w.epochs[0]


def case_limits(case):
    lim = case.get("limits", {})
    return dict(smin=lim.get("smin", 0.0), smax=lim.get("smax", math.inf), fmax=lim.get("fmax", math.inf))


def phase_diff(a, b):
    d = (a - b + math.pi) % (2 * math.pi) - math.pi
    return abs(d)


MIN_COMPARED = 0.95


def compare_sequences(ref_atoms, got_atoms, margins, ref_energies=None, got_energies=None, label="",
                      min_fraction=MIN_COMPARED):
    """ref_atoms/got_atoms: [n][6] for one channel.  margins: oracle margins per
    iteration.  Returns the number of atoms compared (all of them unless a
    near-tie exemption stopped the comparison) and asserts that it is at least
    min_fraction of the reference's atoms; raises AssertionError."""
    n = min(len(ref_atoms), len(got_atoms))
    total = len(ref_atoms)
    for a in range(n):
        r, g = np.asarray(ref_atoms[a]), np.asarray(got_atoms[a])
        same = all(abs(r[p] - g[p]) <= 1e-9 * max(1.0, abs(r[p])) for p in (2, 3, 4))
        if not same:
            m = margins[a] if margins is not None and a < len(margins) else 0.0
            assert m < TIE_MARGIN, f"{label} atom {a}: index mismatch with margin {m:.3e}: ref {r[2:5]} got {g[2:5]}"
            assert a >= min_fraction * total, \
                f"{label}: near-tie at atom {a} left only {a} of {total} atoms compared"
            return a
        for p in (0, 1):
            assert abs(r[p] - g[p]) <= AMP_RTOL * abs(r[p]) + 1e-300, \
                f"{label} atom {a} param {p}: {r[p]} vs {g[p]}"
        assert phase_diff(r[5], g[5]) <= PHASE_ATOL, f"{label} atom {a} phase {r[5]} vs {g[5]}"
        if ref_energies is not None and got_energies is not None and a < len(ref_energies):
            re_, ge = ref_energies[a], got_energies[a]
            if re_ is not None and np.isfinite(re_):
                assert abs(re_ - ge) <= ENERGY_RTOL * abs(re_), f"{label} energy {a}: {re_} vs {ge}"
    if len(ref_atoms) != len(got_atoms):
        # a count difference is only allowed after an exempt divergence (handled above)
        raise AssertionError(f"{label}: atom counts differ {len(ref_atoms)} vs {len(got_atoms)}")
    return n
