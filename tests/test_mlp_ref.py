"""The CPU reference of the warm-start network (oracle/mlp_ref.py): its
gradient agrees with central finite differences of its own loss, so the
GPU gradient check (tests/test_gpu_learned.py) compares against a checked
reference."""
import numpy as np


def test_reference_gradient_matches_finite_differences():
    import mlp_ref as M
    rng = np.random.default_rng(3)
    dims = (16, 8, 8, 24)
    P = sum(a * b + a for a, b in ((dims[1], dims[0]), (dims[2], dims[1]), (dims[3], dims[2])))
    flat = rng.standard_normal(P) * 0.3
    x = rng.standard_normal((5, dims[0]))
    t = rng.standard_normal((5, dims[3]))
    g, _ = M.gradient(flat, dims, x, t)

    def loss(f):
        y, _ = M.forward(f, dims, x)
        return float(((y - t) ** 2).mean())

    h = 1e-6
    idx = rng.choice(P, size=60, replace=False)
    for i in idx:
        e = np.zeros(P)
        e[i] = h
        fd = (loss(flat + e) - loss(flat - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    import mlp_ref as M
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 2.0 ** -7, 1.0 + 3 * 2.0 ** -8, -2.5, 3.14159265])
    r = M.to_bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0                  # tie to even
    assert r[2] == 1.0 + 2.0 ** -7
    assert r[3] == 1.0 + 2.0 ** -6                      # tie to even (upwards)
    assert r[4] == -2.5
    assert abs(r[5] - 3.140625) < 1e-12


def test_reference_adam_step():
    import mlp_ref as M
    w = np.array([1.0, -2.0])
    g = np.array([0.5, -0.25])
    m, v = np.zeros(2), np.zeros(2)
    w1 = M.adam(w, g, m, v, 1, 0.1)
    # first step: m_hat = g, v_hat = g^2, update lr * sign(g)
    assert np.allclose(w1, w - 0.1 * np.sign(g), atol=1e-6)
