"""The learned block proposal on the device.

* BF16 tensor-core inference and FP32 inference against a NumPy FP64
  restatement of the network (proposal.hpp);
* the FP32 training kernels' gradients against FP64 central finite
  differences of that restatement's loss;
* training on pairs that plain GPU MP produced lowers the loss, and the trained
  network ranks the chosen block better than the untrained one (what it gains
  over the method without it);
* with every proposer -- the trained network, the last-atom heuristic, none
  (only the certified second round) -- the atoms are the plain decomposition's.
"""
import numpy as np
import pytest

import empi_b200
from empi_b200 import proposal as P
from empi_b200 import synth

pytestmark = pytest.mark.gpu


def np_forward(spec, w):
    """FP64 restatement of the network: scores [n, 512]."""
    p = {k: v.astype(np.float64) for k, v in P.unpack(np.asarray(w, np.float64)).items()}

    def conv(x, wt, bias, stride):
        n, c, h, wd = x.shape
        ho, wo = h // stride, wd // stride
        xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
        out = np.zeros((n, wt.shape[0], ho, wo))
        for ky in range(3):
            for kx in range(3):
                xs = xp[:, :, ky:ky + stride * ho:stride, kx:kx + stride * wo:stride]
                out += np.einsum("nchw,oc->nohw", xs, wt[:, :, ky, kx])
        return np.maximum(out + bias[None, :, None, None], 0.0)

    x = np.asarray(spec, np.float64)[:, None]
    x1 = conv(x, p["w1"], p["b1"], 1)
    x2 = conv(x1, p["w2"], p["b2"], 2)
    x3 = conv(x2, p["w3"], p["b3"], 2)
    s = np.einsum("nkt,bk->nbt", x3.reshape(x3.shape[0], 32 * 16, 32), p["w4"]) + p["b4"][None, :, None]
    return s.reshape(s.shape[0], -1)


def np_loss(spec, labels, w):
    z = np_forward(spec, w)
    m = z.max(axis=1, keepdims=True)
    lse = m[:, 0] + np.log(np.exp(z - m).sum(axis=1))
    return float(np.mean(lse - z[np.arange(len(labels)), labels]))


def random_spec(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, 64, 128)).astype(np.float32)


def test_inference_bf16_and_fp32_match_fp64():
    spec = random_spec(3, 1)
    w = P.init_weights(3)
    ref = np_forward(spec, w)
    f32 = P.scores(spec, w, bf16=False)
    bf = P.scores(spec, w, bf16=True)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(f32 - ref)) <= 1e-4 * scale
    # BF16 inputs and weights (8-bit mantissa), FP32 accumulation
    err = np.max(np.abs(bf - ref)) / scale
    print(f"BF16 scores: max error {err:.2e} of the largest score")
    assert err <= 3e-2
    assert np.mean(np.argsort(-bf, axis=1)[:, :16] == np.argsort(-ref, axis=1)[:, :16]) > 0.5


def test_gradients_match_fp64_finite_differences():
    spec = random_spec(2, 2)
    labels = np.array([37, 400], np.int32)
    w = P.init_weights(5) * 0.5
    g, loss = P.gradients(spec, labels, w)
    assert abs(loss - np_loss(spec, labels, w)) <= 1e-4 * max(1.0, loss)
    rng = np.random.default_rng(7)
    # parameters of every layer, biases included
    idx = np.concatenate([rng.choice(np.arange(a, b), 8, replace=False) for a, b in
                          ((0, 144), (144, 160), (160, 4768), (4768, 4800), (4800, 14016), (14016, 14048),
                           (14048, 22240), (22240, 22256))])
    w64 = w.astype(np.float64)
    h = 1e-5
    scale = np.max(np.abs(g))
    for i in idx:
        wp, wm = w64.copy(), w64.copy()
        wp[i] += h
        wm[i] -= h
        fd = (np_loss(spec, labels, wp) - np_loss(spec, labels, wm)) / (2 * h)
        assert abs(g[i] - fd) <= 2e-3 * scale + 1e-3 * abs(fd), (int(i), float(g[i]), fd)


def test_training_on_mp_pairs_lowers_loss_and_ranks_better():
    spec, blocks = P.collect_pairs(instances=24, iterations=30)
    assert len(blocks) > 300 and np.all((blocks >= 0) & (blocks < 512))
    n_val = len(blocks) // 5
    val, tr = np.arange(n_val), np.arange(n_val, len(blocks))
    w0 = P.init_weights(0)
    w, losses = P.train(spec[tr], blocks[tr], w0, epochs=6, batch=32, lr=0.02)
    print(f"losses {losses}")
    assert np.min(losses[1:]) < losses[0]
    before = P.top_k_hit_rate(spec[val], blocks[val], w0)
    after = P.top_k_hit_rate(spec[val], blocks[val], w)
    print(f"validation top-16 hit rate: untrained {before:.3f}, trained {after:.3f}")
    assert after > before


@pytest.mark.parametrize("variant", ["smp", "mmp2", "mmp3"])
def test_every_proposer_gives_the_plain_atoms(engine, tmp_path, variant):
    w = synth.workload(1, epochs=2, channels=3, samples=2500, seed=21)
    iters = 25
    settings = empi_b200.DecompositionSettings(iters, 1.0 - 0.01 * w.energy_percent)
    ref = empi_b200.decompose_epochs(variant, w.epochs, w.fs, w.energy_error, iters, w.energy_percent,
                                     engine=engine)
    wpath = str(tmp_path / "w.bin")
    P.save_weights(wpath, P.init_weights(11))
    for source in ("net", "last_atom", "none"):
        b = empi_b200.Batch(variant, w.energy_error, settings, [e.shape for e in w.epochs], w.fs, engine=engine)
        b.set_proposal(source, 16, wpath if source == "net" else None)
        b.load(w.epochs)
        b.run()
        st = b.stats()
        got = [b.result(e) for e in range(len(w.epochs))]
        b.close()
        for g, r in zip(got, ref):
            np.testing.assert_array_equal(g.counts, r.counts)
            np.testing.assert_array_equal(g.indices, r.indices)
            np.testing.assert_allclose(g.atoms, r.atoms, rtol=1e-12, atol=0)
        assert st.proposal_iterations > 0 and 0 <= st.proposal_hits <= st.proposal_iterations
        print(f"{variant} {source}: hits {st.proposal_hits}/{st.proposal_iterations}, "
              f"refresh flops {st.fft_flops:.3e}")


def test_mmp1_rejects_a_proposal(engine):
    w = synth.workload(1, epochs=1, channels=3, samples=800, seed=1)
    b = empi_b200.Batch("mmp1", 0.02, empi_b200.DecompositionSettings(5, 0.0), [w.epochs[0].shape], w.fs,
                        engine=engine)
    with pytest.raises(empi_b200.EmpiError) as ei:
        b.set_proposal("none")
    assert ei.value.message == "proposalUnsupportedForMmp1"
    b.close()
