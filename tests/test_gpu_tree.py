"""The device tournament tree, the counterpart of the reference's Heap
(inc/heap.hpp:13-94) and of its one test (tests/test-heap.cpp:13-48, peek
order under random updates).

Every MP iteration updates the slot keys of the dirty windows only (the
refresh rule of src/gabor.cpp:189-209) and re-reduces the leaf chunks those
windows fall in.  After runs of different lengths -- so after different
sequences of partial updates, on several instances, variants and with the
block proposal's bound propagation -- every leaf chunk must hold the largest
upper bound of its slots (ties to the highest slot index, the tree's rule) and
its largest lower bound, and the root (the maximum over chunks) must be the
largest upper bound of all slots, as a CPU scan finds them.
"""
import numpy as np
import pytest

import empi_b200
from empi_b200 import synth

pytestmark = pytest.mark.gpu

CHUNK = 1024  # slots per leaf chunk (common.cuh kChunk)


def cpu_tree(slots):
    """Leaf chunks of a slot-key array as k_tree defines them: (upper bits <<
    32 | slot index) maximised over the chunk, and the largest lower bits."""
    n = len(slots)
    idx = np.arange(n, dtype=np.uint64)
    keyed = (slots & np.uint64(0xFFFFFFFF00000000)) | idx
    nch = (n + CHUNK - 1) // CHUNK
    pad = nch * CHUNK - n
    k = np.concatenate([keyed, np.zeros(pad, np.uint64)]).reshape(nch, CHUNK)
    low = np.concatenate([slots & np.uint64(0xFFFFFFFF), np.zeros(pad, np.uint64)]).reshape(nch, CHUNK)
    return k.max(axis=1), low.max(axis=1).astype(np.uint32)


def check_tree(b, instances):
    checked = 0
    for i in range(instances):
        slots, chunks, chunk_l = b.tree(i)
        want, want_l = cpu_tree(slots)
        assert len(chunks) == len(want)
        bad = np.nonzero(chunks != want)[0]
        assert bad.size == 0, f"instance {i}: {bad.size} leaf chunks differ from the CPU max, first {bad[:5]}"
        np.testing.assert_array_equal(chunk_l, want_l)
        root = chunks.max()
        assert (int(root) >> 32) == int((slots >> np.uint64(32)).max())
        # the root's slot holds the largest upper bound of all slots
        s = int(root) & 0xFFFFFFFF
        assert int(slots[s]) >> 32 == int(root) >> 32
        assert np.count_nonzero(slots) > 0.5 * len(slots)
        checked += len(chunks)
    return checked


@pytest.mark.parametrize("variant", ["smp", "mmp2", "mmp3"])
@pytest.mark.parametrize("iterations", [1, 4, 13])
def test_tree_matches_cpu_max_after_partial_updates(engine, variant, iterations):
    w = synth.workload(1, epochs=2, channels=3, samples=2500, seed=5 + iterations)
    settings = empi_b200.DecompositionSettings(iterations, 0.0)
    b = empi_b200.Batch(variant, w.energy_error, settings, [e.shape for e in w.epochs], w.fs, engine=engine)
    b.load(w.epochs)
    b.run()
    loops = 2 * 3 if variant == "smp" else 2
    n = check_tree(b, loops)
    b.close()
    print(f"{variant}, {iterations} iterations: {n} leaf chunks over {loops} MP loops match")


def test_tree_matches_cpu_max_with_bound_propagation(engine):
    """The proposal path rewrites stale slots' keys by propagated bounds
    (k_propagate_stale) between the two refresh rounds of an iteration."""
    w = synth.workload(1, epochs=2, channels=3, samples=2500, seed=31)
    settings = empi_b200.DecompositionSettings(9, 0.0)
    b = empi_b200.Batch("mmp2", w.energy_error, settings, [e.shape for e in w.epochs], w.fs, engine=engine)
    b.set_proposal("none")
    b.load(w.epochs)
    b.run()
    check_tree(b, 2)
    b.close()
