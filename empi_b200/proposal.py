"""The learned block proposal: training pairs, training, weights files.

    python -m empi_b200.proposal --out weights.bin [--instances 96] [--iterations 60]
                                 [--epochs 4] [--device 0]

The proposer (empi_b200/csrc/proposal.cu) reads a normalised 64 x 128
log-spectrogram of an MP loop's residual and scores 16 scale bands x 32 time
tiles; the engine refreshes the dirty windows of the top-k blocks first and
certifies the rest (empi_batch_set_proposal), so the atoms never change.  It
is trained on (residual spectrogram, block of the atom chosen next) pairs that
plain MP on the GPU produces from seeded batched-SMP signals (the batched
workload's instance model), with the project's FP32 training kernels, and
stored in the "EMPIPN01" weights format: 8-byte magic, int32 parameter count,
float32 parameters.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import struct
import time

import numpy as np

import empi_b200
from empi_b200 import synth

MAGIC = b"EMPIPN01"
BANDS, TILES = 16, 32
# (offset, shape) of the parameters, in the engine's order (proposal.hpp)
LAYOUT = [("w1", (16, 1, 3, 3)), ("b1", (16,)), ("w2", (32, 16, 3, 3)), ("b2", (32,)), ("w3", (32, 32, 3, 3)),
          ("b3", (32,)), ("w4", (16, 32 * 16)), ("b4", (16,))]


def parameter_count():
    return int(empi_b200.load_library().empi_proposal_parameter_count())


def unpack(w):
    """Flat parameter vector -> dict of arrays (views)."""
    out, off = {}, 0
    for name, shape in LAYOUT:
        n = int(np.prod(shape))
        out[name] = w[off:off + n].reshape(shape)
        off += n
    assert off == len(w)
    return out


def init_weights(seed=0):
    """He-normal weights, zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in LAYOUT:
        if name.startswith("b"):
            parts.append(np.zeros(shape, np.float32))
        else:
            fan_in = int(np.prod(shape[1:]))
            parts.append((rng.standard_normal(shape) * np.sqrt(2.0 / fan_in)).astype(np.float32))
    w = np.concatenate([p.reshape(-1) for p in parts])
    assert w.size == parameter_count()
    return w


def save_weights(path, w):
    w = np.ascontiguousarray(w, np.float32)
    with open(path, "wb") as f:
        f.write(MAGIC + struct.pack("<i", w.size) + w.tobytes())


def load_weights(path):
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != MAGIC:
        raise ValueError("invalidProposalWeights")
    (n,) = struct.unpack("<i", data[8:12])
    w = np.frombuffer(data[12:], np.float32)
    if n != parameter_count() or w.size != n:
        raise ValueError("invalidProposalWeights")
    return w.copy()


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def scores(spec, w, bf16=True, device=0):
    """Block scores [n, 512] of spectrograms [n, 64, 128]."""
    spec = np.ascontiguousarray(spec, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    out = np.zeros((spec.shape[0], BANDS * TILES), np.float32)
    empi_b200._check(empi_b200.load_library().empi_proposal_scores(device, _fp(spec), spec.shape[0], _fp(w),
                                                                   int(bf16), _fp(out)))
    return out


def gradients(spec, labels, w, device=0):
    """(gradient of the mean cross-entropy, loss) from the FP32 kernels."""
    spec = np.ascontiguousarray(spec, np.float32)
    labels = np.ascontiguousarray(labels, np.int32)
    w = np.ascontiguousarray(w, np.float32)
    g = np.zeros_like(w)
    loss = np.zeros(1, np.float32)
    empi_b200._check(empi_b200.load_library().empi_proposal_gradients(device, _fp(spec), empi_b200._ip(labels),
                                                                      spec.shape[0], _fp(w), _fp(g), _fp(loss)))
    return g, float(loss[0])


def train(spec, labels, w0, epochs=4, batch=64, lr=0.05, momentum=0.9, seed=0, device=0):
    """SGD on the device; returns (weights, mean loss per epoch)."""
    spec = np.ascontiguousarray(spec, np.float32)
    labels = np.ascontiguousarray(labels, np.int32)
    w = np.array(w0, np.float32)
    losses = np.zeros(epochs, np.float32)
    empi_b200._check(empi_b200.load_library().empi_proposal_train(
        device, _fp(spec), empi_b200._ip(labels), spec.shape[0], epochs, batch, lr, momentum, seed, _fp(w),
        _fp(losses)))
    return w, losses


def collect_pairs(instances=96, iterations=60, seed=2024, engine=None):
    """(spectrograms, blocks) from plain GPU MP on `instances` seeded
    batched-SMP signals (the batched workload's instance model, seeds apart
    from the benchmark's)."""
    w = synth.workload(3, seed=seed, epochs=instances, iterations=iterations)
    settings = empi_b200.DecompositionSettings(iterations, 1.0 - 0.01 * w.energy_percent)
    b = empi_b200.Batch("smp", w.energy_error, settings, [e.shape for e in w.epochs], w.fs, engine=engine)
    b.collect_pairs(True)
    b.load(w.epochs)
    b.run()
    spec, blocks = b.pairs()
    b.close()
    return spec, blocks


def top_k_hit_rate(spec, blocks, w, k=16):
    """Share of pairs whose block is among the k best-scored blocks."""
    s = scores(spec, w)
    top = np.argsort(-s, axis=1)[:, :k]
    return float(np.mean([blocks[i] in top[i] for i in range(len(blocks))]))


def main():
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--out", required=True)
    p.add_argument("--instances", type=int, default=96)
    p.add_argument("--iterations", type=int, default=60)
    p.add_argument("--epochs", type=int, default=4)
    p.add_argument("--batch", type=int, default=64)
    p.add_argument("--lr", type=float, default=0.05)
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--pairs-out", help="also write the pairs (npz)")
    a = p.parse_args()
    eng = empi_b200.Engine(device=a.device)
    t0 = time.time()
    spec, blocks = collect_pairs(a.instances, a.iterations, engine=eng)
    t1 = time.time()
    print(f"{len(blocks)} pairs from {a.instances} instances x {a.iterations} iterations in {t1 - t0:.1f} s")
    if a.pairs_out:
        np.savez_compressed(a.pairs_out, spec=spec, blocks=blocks)
    n_val = max(1, len(blocks) // 10)
    rng = np.random.default_rng(0)
    perm = rng.permutation(len(blocks))
    val, tr = perm[:n_val], perm[n_val:]
    w0 = init_weights(0)
    print(f"untrained: validation top-16 hit rate {top_k_hit_rate(spec[val], blocks[val], w0):.3f}")
    w, losses = train(spec[tr], blocks[tr], w0, a.epochs, a.batch, a.lr, device=a.device)
    print(f"trained in {time.time() - t1:.1f} s, loss per epoch {[round(float(x), 3) for x in losses]}")
    print(f"trained: validation top-16 hit rate {top_k_hit_rate(spec[val], blocks[val], w):.3f}")
    save_weights(a.out, w)
    eng.close()


if __name__ == "__main__":
    main()
