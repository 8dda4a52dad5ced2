"""The surrogate's GPU MLP ensemble (fdtd_mlp_*) against the CPU FP64 oracle (oracle/mlp.py).

* gradients of every member (BF16 tensor-core GEMMs, FP32 accumulation) against the oracle
  with the same BF16 roundings (tight) and against exact FP64 backprop (loose), for both GEMM
  paths (tcgen05 with a TMEM accumulator, and warp-level mma.sync), and the two paths against
  each other on odd shapes;
* forward outputs of every member and the ensemble mean / standard deviation;
* one Adam step against the oracle's Adam on the oracle's gradient;
* training on a smooth function lowers the loss and generalises; invalid arguments fail.
"""
import numpy as np
import pytest

import gdiamond_b200 as gd
from oracle import mlp as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def data(n, dims, seed):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-1, 1, (n, dims[0])).astype(np.float32),
            rng.normal(0, 1, (n, dims[-1])).astype(np.float32))


@pytest.mark.parametrize("dims,members,n", [((6, 37, 19, 3), 2, 70), ((7, 200, 130, 72), 3, 333),
                                            ((6, 256, 256, 256, 64), 4, 1000)])
def test_gemm_paths_agree(dims, members, n):
    x, y = data(n, dims, 9)
    out = {}
    for gemm in ("mma_sync", "tcgen05"):
        net = gd.MLP(dims, members=members, seed=5, gemm=gemm)
        mean, sd, per = net.predict(x, members=True)
        loss, g = net.grad(x, y)
        out[gemm] = (per, loss, g)
        net.close()
    (p0, l0, g0), (p1, l1, g1) = out["mma_sync"], out["tcgen05"]
    assert rel(p1, p0) <= 1e-4, rel(p1, p0)
    assert np.allclose(l1, l0, rtol=1e-4)
    for e in range(members):
        assert rel(g1[e], g0[e]) <= 2e-3, (e, rel(g1[e], g0[e]))


@pytest.mark.parametrize("gemm", ["tcgen05", "mma_sync"])
@pytest.mark.parametrize("dims,members,n", [((6, 256, 256, 256, 64), 4, 200),
                                            ((5, 37, 19, 3), 2, 70)])
def test_gradients_match_oracle(dims, members, n, gemm):
    net = gd.MLP(dims, members=members, seed=7, gemm=gemm)
    x, y = data(n, dims, 1)
    loss, g = net.grad(x, y)
    P = net.get_params()
    for e in range(members):
        L = [(W.astype(np.float64), b.astype(np.float64)) for W, b in net.unpack(P[e])]
        lq, gq = O.loss_and_grad(L, x, y, bf16=True)
        lx, gx = O.loss_and_grad(L, x, y, bf16=False)
        assert abs(loss[e] - lq) <= 1e-4 * lq
        assert abs(loss[e] - lx) <= 2e-2 * lx
        got = net.unpack(g[e])
        for n_, ((dW, db), (qW, qb), (xW, xb)) in enumerate(zip(got, gq, gx)):
            assert rel(dW, qW) <= 2e-3, (e, n_, "W", rel(dW, qW))
            assert rel(db, qb) <= 2e-3, (e, n_, "b", rel(db, qb))
            assert rel(dW, xW) <= 5e-2, (e, n_, "W exact", rel(dW, xW))
            assert rel(db, xb) <= 5e-2, (e, n_, "b exact", rel(db, xb))
    net.close()


@pytest.mark.parametrize("gemm", ["tcgen05", "mma_sync"])
def test_forward_and_ensemble_statistics_match_oracle(gemm):
    dims = (6, 256, 256, 256, 64)
    net = gd.MLP(dims, members=4, seed=3, gemm=gemm)
    x, _ = data(333, dims, 2)
    mean, sd, per = net.predict(x, members=True)
    P = net.get_params()
    outs = []
    for e in range(4):
        L = [(W.astype(np.float64), b.astype(np.float64)) for W, b in net.unpack(P[e])]
        ref, _ = O.forward(L, x, bf16=True)
        assert rel(per[e], ref) <= 1e-3, (e, rel(per[e], ref))
        outs.append(per[e].astype(np.float64))
    outs = np.array(outs)
    assert np.allclose(mean, outs.mean(0), rtol=1e-5, atol=1e-5)
    assert np.allclose(sd, outs.std(0), rtol=1e-4, atol=1e-5)
    assert sd.mean() > 0  # members start from different seeds
    net.close()


def test_layout_and_param_roundtrip():
    dims = (6, 256, 256, 256, 64)
    net = gd.MLP(dims, members=2, seed=0)
    for w, (o, i), b in net.layout():
        assert w % 8 == 0 and b % 8 == 0 and b >= w + o * i
    assert net.n_params >= sum(o * i + o for _, (o, i), _ in net.layout())
    P = net.get_params()
    P2 = P * np.float32(0.5)
    net.set_params(P2)
    assert np.array_equal(net.get_params(), P2)
    net.close()


def test_first_adam_step_matches_oracle():
    dims = (6, 64, 64, 8)
    net = gd.MLP(dims, members=2, seed=11)
    x, y = data(96, dims, 4)
    P0 = net.get_params()
    net.set_data(x, y)
    net.train(epochs=1, batch=96, lr=1e-3, seed=0)  # one full-batch step per member
    P1 = net.get_params()
    for e in range(2):
        L = [(W.astype(np.float64), b.astype(np.float64)) for W, b in net.unpack(P0[e])]
        _, gq = O.loss_and_grad(L, x, y, bf16=True)
        flat = np.zeros(net.n_params)
        for (w, (o, i), b), (dW, db) in zip(net.layout(), gq):
            flat[w:w + o * i] = dW.reshape(-1)
            flat[b:b + o] = db
        want, _, _ = O.adam(P0[e].astype(np.float64), flat, 0.0, 0.0, t=1, lr=1e-3)
        used = np.zeros(net.n_params, bool)
        for w, (o, i), b in net.layout():
            used[w:w + o * i] = True
            used[b:b + o] = True
        d_got = (P1[e] - P0[e])[used].astype(np.float64)
        d_want = (want - P0[e])[used]
        # the first Adam step moves every parameter by ~lr * sign(gradient)
        close = np.abs(d_got - d_want) <= 2e-6 + 1e-3 * np.abs(d_want)
        assert close.mean() >= 0.99, close.mean()
        assert np.array_equal(P1[e][~used], P0[e][~used])
    net.close()


def test_training_fits_a_smooth_function():
    dims = (6, 256, 256, 256, 64)
    rng = np.random.default_rng(0)
    A = rng.normal(0, 1, (6, 64))
    f = lambda x: np.sin(x @ A * 0.7) + 0.3 * np.cos(x @ A * 0.3)  # noqa: E731
    x = rng.uniform(-1, 1, (2048, 6)).astype(np.float32)
    xt = rng.uniform(-1, 1, (256, 6)).astype(np.float32)
    net = gd.MLP(dims, members=4, seed=1)
    net.set_data(x, f(x))
    losses = net.train(epochs=60, batch=64, lr=1e-3, seed=2)
    assert losses.shape == (60, 4) and np.all(np.isfinite(losses))
    assert np.all(losses[-1] < 0.05 * losses[0])
    mean, sd = net.predict(xt)
    err = rel(mean, f(xt))
    assert err < 0.1, err
    # the ensemble spread tracks the error: larger off the training range
    _, sd_far = net.predict(xt * 3)
    assert sd_far.mean() > sd.mean()
    net.close()


def test_invalid_arguments():
    with pytest.raises(gd.FdtdError):
        gd.MLP((6,), members=1)
    with pytest.raises(gd.FdtdError):
        gd.MLP((6, 0, 4), members=1)
    net = gd.MLP((4, 8, 2), members=1)
    with pytest.raises(gd.FdtdError):
        net.train(epochs=1)  # no data
    with pytest.raises(KeyError):
        net.set_gemm("wmma")
    with pytest.raises(ValueError):
        net.set_data(np.zeros((3, 4)), np.zeros((2, 2)))
    net.close()


@pytest.mark.parametrize("n", [1, 127, 129, 70000])
def test_fused_inference_matches_layer_by_layer(n):
    """predict() on the tcgen05 path runs every layer in one kernel (activations kept in shared
    memory); the warp-level path runs the layers one GEMM at a time."""
    dims = (6, 256, 256, 256, 64)
    x, _ = data(n, dims, 11)
    out = {}
    for gemm in ("tcgen05", "mma_sync"):
        net = gd.MLP(dims, members=4, seed=8, gemm=gemm)
        out[gemm] = net.predict(x, members=True)
        net.close()
    (m1, s1, p1), (m0, s0, p0) = out["tcgen05"], out["mma_sync"]
    assert np.all(np.isfinite(p1))
    assert rel(p1, p0) <= 1e-3, rel(p1, p0)
    assert rel(m1, m0) <= 1e-3
