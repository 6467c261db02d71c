"""Learned warm start through the C ABI: features, the training kernels'
forward pass and gradient, and the tensor-core inference, each against the
numpy oracle (oracle/warm_oracle.py); then training on the GPU and what the trained
network gains over the uniform start at the same residual.

Tolerances: features rtol 2e-5 (the device sums in FP32 in chunk order, the
oracle in FP64; the network sees the features rounded to BF16, 4e-3 relative);
forward |dy| <= 2e-3 (FP32 sums in another order can move a hidden value across
a BF16 rounding boundary); gradient relative L2 error <= 1e-2 per parameter block
(same cause); PageRank answers from the two starts within normalised L1 1e-6."""
import numpy as np
import pytest

import gcgpu
import oracle as O
import warm_oracle as W

pytestmark = pytest.mark.gpu


def graph_and_oracle_features(scale=11, seed=3):
    s, d = O.rmat_numpy(scale, 16 << scale, seed=seed)
    g = gcgpu.Graph.from_edges(s, d, dedup=True)
    rp, col = g.csr(gcgpu.CSR_IN)
    deg = g.degrees()
    f_ref = W.features(g.num_vertices, rp, col, deg[:, 1])
    return g, f_ref


def random_model(seed=2):
    m = gcgpu.Mlp(seed=seed)
    p, _ = m.get()
    rng = np.random.default_rng(seed)
    p[W.OB1:W.OW2] = rng.normal(0, 0.1, W.NH)
    p[W.OB2:W.OW3] = rng.normal(0, 0.1, W.NH)
    p[W.OB3] = 0.5
    return m, p


def test_features_vs_oracle():
    g, f_ref = graph_and_oracle_features()
    with g:
        f = g.warm_features()
    assert f.shape == f_ref.shape
    assert np.allclose(f, f_ref, rtol=2e-5, atol=1e-6)
    # an Erdos-Renyi graph with isolated vertices, and a tiny graph
    s, d = O.er_numpy(3000, 6000, seed=4)
    with gcgpu.Graph.from_edges(s, d, dedup=True) as g2:
        rp, col = g2.csr(gcgpu.CSR_IN)
        ref = W.features(g2.num_vertices, rp, col, g2.degrees()[:, 1])
        assert np.allclose(g2.warm_features(), ref, rtol=2e-5, atol=1e-6)


def test_forward_and_gradient_vs_oracle():
    g, f = graph_and_oracle_features()
    g.free()
    m, p = random_model()
    with m:
        m.set(p)
        m.fit_normalisation(f)
        p, norm = m.get()
        rng = np.random.default_rng(5)
        t = (rng.normal(1.0, 1.0, f.shape[0])).astype(np.float32)
        y = m.forward(f)
        y_ref = W.forward(p, norm, f)
        assert np.abs(y - y_ref).max() <= 2e-3
        g_dev, loss = m.gradient(f, t)
        g_ref, loss_ref = W.gradient(p, norm, f, t)
        assert abs(loss - loss_ref) <= 1e-3 * loss_ref
        for lo, hi in [(W.OW1, W.OB1), (W.OB1, W.OW2), (W.OW2, W.OB2), (W.OB2, W.OW3), (W.OW3, W.OB3),
                       (W.OB3, W.NP)]:
            err = np.linalg.norm(g_dev[lo:hi] - g_ref[lo:hi]) / max(np.linalg.norm(g_ref[lo:hi]), 1e-12)
            assert err <= 1e-2, (lo, hi, err)


def test_tensor_core_inference_vs_oracle():
    g, f = graph_and_oracle_features(scale=12, seed=6)
    m, p = random_model(seed=3)
    with g, m:
        m.set(p)
        m.fit_normalisation(f)
        p, norm = m.get()
        init, ms = g.warm_start_rank(m, teleport=0.15, damping=0.85)
        y_ref = np.clip(W.forward(p, norm, f), -30, 30)
        has_in = f[:, 0] > 0
        # vertices without in-edges start at their exact rank
        assert np.all(init[~has_in] == np.float32(0.15))
        deg = g.degrees()
        pred = np.where(has_in, 0.15 * np.exp(y_ref), 0.15)
        alpha = W.mass_alpha(pred, deg[:, 0], deg[:, 1])
        assert 0.2 < alpha < 5.0
        y = np.log(init[has_in].astype(np.float64) / (0.15 * alpha))
        assert np.abs(y - y_ref[has_in]).max() <= 2e-3
        # one Jacobi sweep keeps the total rank of the warm start
        rp, col = g.csr(gcgpu.CSR_IN)
        r = init.astype(np.float64)
        c = np.where(deg[:, 1] > 0, r / np.maximum(deg[:, 1], 1), 0.0)
        dst = np.repeat(np.arange(g.num_vertices), np.diff(rp.astype(np.int64)))
        nxt = 0.15 + 0.85 * np.bincount(dst, weights=c[col], minlength=g.num_vertices)
        assert abs(nxt.sum() - r.sum()) <= 1e-5 * r.sum()


def _train_small():
    import gcgpu.warm as gw
    x, t = gw.build_training_set(ngraphs=12, scales=(12, 14), per_graph=None, seed=7)
    m, losses = gw.train(x, t, epochs=30, batch=1024, lr=3e-3)
    return m, losses


def test_training_lowers_loss_and_warm_start_saves_sweeps():
    import gcgpu.warm as gw
    m, losses = _train_small()
    with m:
        assert losses[-1] < 0.5 * losses[0]
        rng = np.random.default_rng(11)
        saved = []
        for i in range(3):
            with gw.rmat_graph(15, int(rng.integers(1 << 40)), gw.jittered_abc(rng)) as g:
                rec = gw.evaluate(g, m)
            # the same stopping rule, so the same answer
            assert rec["residual_warm"] <= 1e-8 and rec["residual_plain"] <= 1e-8
            assert rec["l1_between"] <= 1e-6
            assert rec["init_l1_error"] < 0.25 * rec["uniform_l1_error"]
            saved.append(rec["sweeps_plain"] - rec["sweeps_warm"])
        # fewer sweeps on every held-out graph, about 10 % or more in total
        assert min(saved) >= 1 and sum(saved) >= 20, saved


def test_model_roundtrip_and_invalid_arguments(tmp_path):
    m, p = random_model()
    with m:
        m.set(p)
        path = str(tmp_path / "m.npz")
        m.save(path)
        m2 = gcgpu.Mlp.load(path)
        with m2:
            p2, n2 = m2.get()
            assert np.array_equal(p2, m.get()[0]) and np.array_equal(n2, m.get()[1])
        with pytest.raises(gcgpu.GcgError):
            m.train(np.zeros((10, 8), np.float32), np.zeros(10, np.float32), batch=100)
