"""The learned-cache oracle checks itself (CPU): hash indices against the
published hash, the analytic gradients against central differences of the
loss, and Adam's bias correction against a hand-worked step."""

import numpy as np
import pytest


@pytest.fixture()
def lrc(monkeypatch):
    from oracle import lrc as m

    return m


def test_resolutions_and_hash_follow_the_published_encoding(lrc):
    cfg = lrc.CacheConfig(log2_table=19, base_resolution=16, max_resolution=2048)
    res = cfg.resolutions()
    assert res[0] == 16 and res[-1] == 2048 and np.all(np.diff(res.astype(np.int64)) > 0)
    # a hashed level: index = (x ^ y*2654435761 ^ z*805459861) mod 2^19
    pos = np.array([[0.31, 0.72, 0.05]], np.float32)
    idx, w = lrc.corner_lookup(cfg, pos)
    l = 15
    r = np.float32(res[l])
    c = np.floor(pos[0] * r).astype(np.uint64)
    expect = int((c[0] * 1) ^ ((c[1] * 2654435761) & 0xFFFFFFFF) ^ ((c[2] * 805459861) & 0xFFFFFFFF)) & ((1 << 19) - 1)
    assert idx[0, l, 0] == expect
    # a dense level: (16+1)^3 <= 2^19
    c0 = np.floor(pos[0] * np.float32(16)).astype(np.int64)
    assert idx[0, 0, 7] == (c0[0] + 1) + (c0[1] + 1) * 17 + (c0[2] + 1) * 17 * 17
    # trilinear weights sum to one
    assert np.allclose(w.sum(axis=2), 1.0, atol=1e-6)


def test_gradients_match_central_differences(lrc, monkeypatch):
    # exact arithmetic (no bf16 rounding) so the loss is smooth in the parameters
    monkeypatch.setattr(lrc, "bf16", lambda x: np.asarray(x, np.float32))
    cfg = lrc.CacheConfig(log2_table=10, base_resolution=2, max_resolution=16)
    params, table = lrc.init_params(cfg, seed=3)
    params *= 4.0
    table = (np.random.default_rng(1).uniform(-0.5, 0.5, table.size)).astype(np.float16)
    rng = np.random.default_rng(2)
    n = 24
    q = np.zeros((n, 8), np.float32)
    q[:, 0:3] = rng.uniform(0.05, 0.95, (n, 3))
    nrm = rng.normal(size=(n, 3))
    q[:, 4:7] = nrm / np.linalg.norm(nrm, axis=1, keepdims=True)
    y = rng.uniform(0.1, 2.0, (n, 4)).astype(np.float32)
    loss, gp, gt = lrc.loss_and_grads(cfg, table, params, q, y)

    def loss_at(p):
        o = lrc.forward(cfg, table, p, q).astype(np.float64)
        # the denominator is held constant in the relative L2 loss
        return np.sum((o - y[:, :3]) ** 2 / (o0 * o0 + cfg.loss_eps)) / n

    o0 = lrc.forward(cfg, table, params, q).astype(np.float32).astype(np.float64)
    # float32 parameters: a step of 1e-2 keeps the central difference accurate
    for k in rng.choice(lrc.MLP_PARAMS - 13 * 64, 12, replace=False):
        p1, p2 = params.copy(), params.copy()
        h = 1e-2
        p1[k] += h
        p2[k] -= h
        fd = (loss_at(p1) - loss_at(p2)) / (2 * h)
        assert abs(fd - gp[k]) <= 2e-3 * max(1.0, abs(gp[k])) + 1e-5, (k, fd, gp[k])


def test_adam_step(lrc):
    cfg = lrc.CacheConfig(lr=0.1, beta1=0.9, beta2=0.99, eps=1e-8)
    p, m, v = lrc.adam(cfg, np.array([1.0]), np.array([0.0]), np.array([0.0]), np.array([2.0]), 1)
    # first step: m_hat = g, v_hat = g^2, so the update is lr * sign(g)
    assert np.allclose(p, 1.0 - 0.1 * 2.0 / (2.0 + 1e-8)) and np.allclose(m, 0.2) and np.allclose(v, 0.04)
