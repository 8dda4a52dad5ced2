"""The CPU MLP oracle (oracle/mlp.py) pinned without a GPU.

* its exact gradient against central finite differences of its own loss (float64);
* its BF16 rounding against torch's float32 -> bfloat16 conversion (round to nearest even);
* its BF16-emulating gradient stays close to the exact one (the roundings are small);
* its Adam step against the textbook update written out here.
"""
import numpy as np
import torch

from oracle import mlp as O


def layers(dims, seed):
    rng = np.random.default_rng(seed)
    return [(rng.normal(0, np.sqrt(2.0 / i), (o, i)), rng.normal(0, 0.1, o))
            for i, o in zip(dims[:-1], dims[1:])]


def test_exact_gradient_matches_finite_differences():
    dims = (3, 7, 5, 2)
    L = layers(dims, 0)
    rng = np.random.default_rng(1)
    x, y = rng.normal(size=(9, 3)), rng.normal(size=(9, 2))
    _, grads = O.loss_and_grad(L, x, y)
    h = 1e-6
    for n, (W, b) in enumerate(L):
        for arr, g in ((W, grads[n][0]), (b, grads[n][1])):
            flat, gf = arr.reshape(-1), g.reshape(-1)
            for q in range(0, flat.size, max(1, flat.size // 7)):
                old = flat[q]
                flat[q] = old + h
                lp, _ = O.loss_and_grad(L, x, y)
                flat[q] = old - h
                lm, _ = O.loss_and_grad(L, x, y)
                flat[q] = old
                fd = (lp - lm) / (2 * h)
                assert abs(fd - gf[q]) <= 1e-7 + 1e-6 * abs(fd), (n, q, fd, gf[q])


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.normal(0, 10, 5000), rng.normal(0, 1e-30, 500),
                        np.array([0.0, -0.0, 1.0, 3.0e38, -3.0e38, 1.00390625, 1.01171875])])
    x = x.astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy().astype(np.float64)
    assert np.array_equal(O.round_bf16(x), ref)


def test_bf16_gradient_close_to_exact():
    dims = (6, 64, 64, 16)
    L = layers(dims, 3)
    rng = np.random.default_rng(4)
    x, y = rng.uniform(-1, 1, (50, 6)), rng.normal(size=(50, 16))
    _, ge = O.loss_and_grad(L, x, y)
    _, gq = O.loss_and_grad(L, x, y, bf16=True)
    for (a, b), (c, d) in zip(ge, gq):
        assert np.linalg.norm(a - c) <= 3e-2 * np.linalg.norm(a)
        assert np.linalg.norm(b - d) <= 3e-2 * np.linalg.norm(b)


def test_adam_step():
    rng = np.random.default_rng(5)
    p, g = rng.normal(size=100), rng.normal(size=100)
    m, v = rng.normal(size=100) * 0.1, rng.uniform(0, 0.1, 100)
    p1, m1, v1 = O.adam(p, g, m, v, t=3, lr=1e-3)
    mm = 0.9 * m + 0.1 * g
    vv = 0.999 * v + 0.001 * g * g
    want = p - 1e-3 * (mm / (1 - 0.9 ** 3)) / (np.sqrt(vv / (1 - 0.999 ** 3)) + 1e-8)
    assert np.allclose(p1, want, rtol=0, atol=1e-15)
    assert np.allclose(m1, mm) and np.allclose(v1, vv)
