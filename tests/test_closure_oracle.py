"""The closure oracle's hand-written backward pass against finite differences (CPU)."""
import numpy as np

from oracle import closure_oracle as co


def _net(seed):
    rng = np.random.default_rng(seed)
    net = co.init_net(seed)
    net[co.oB1:co.oW2] = rng.normal(0, 0.1, co.HID)
    net[co.oB2:co.oW3] = rng.normal(0, 0.1, co.HID)
    net[co.oB3:co.PARAMS] = rng.normal(0, 0.1, co.OUT)
    net[co.oMean:co.oInvStd] = rng.normal(0, 0.5, co.IN)
    net[co.oInvStd:co.oScale] = rng.uniform(0.5, 2.0, co.IN)
    net[co.oScale:co.oOffset] = [0.01, 2.0]
    net[co.oOffset:co.NET] = [0.0, 1.0]
    return net


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    net = _net(1)
    feat = rng.normal(0, 1, (40, co.IN)).astype(np.float32)
    tgt = np.stack([rng.uniform(0, 0.02, 40), rng.uniform(0.5, 2, 40)], 1).astype(np.float32)
    w = rng.uniform(0.1, 1.0, (40, 2)).astype(np.float32)
    _, g = co.loss_and_grad(net, feat, tgt, w, emulate_bf16=False)
    idx = np.concatenate([rng.choice(np.arange(co.oW1, co.oB1).reshape(co.HID, co.K1)[:, :co.IN].reshape(-1), 20),
                          rng.choice(np.arange(co.oB1, co.PARAMS), 60, replace=False)])
    for i in idx:
        h = np.float32(1e-2) * max(1.0, abs(float(net[i])))
        p, m = net.copy(), net.copy()
        p[i] += h
        m[i] -= h
        lp, _ = co.loss_and_grad(p, feat, tgt, w, emulate_bf16=False)
        lm, _ = co.loss_and_grad(m, feat, tgt, w, emulate_bf16=False)
        fd = (lp - lm) / (float(p[i]) - float(m[i]))
        assert abs(fd - g[i]) <= 2e-3 * max(1e-3, abs(g[i])) + 1e-6, (i, fd, g[i])
    # padded input columns never receive gradient
    assert np.all(g[co.oW1:co.oB1].reshape(co.HID, co.K1)[:, co.IN:] == 0)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-20], np.float32)
    r = co.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] - x[3]) <= abs(x[3]) * 2 ** -8
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)


def test_filter_and_targets_shapes():
    rng = np.random.default_rng(0)
    shape = (8, 6, 4)
    f = [rng.normal(0, 0.01, shape).astype(np.float32) for _ in range(3)]
    phi = rng.uniform(0, 1, shape).astype(np.float32)
    rho = (1 + rng.normal(0, 1e-3, shape)).astype(np.float32)
    coarse, tau, area = co.box_filter(rho, *f, phi, (True, True, False))
    assert coarse[0].shape == (4, 3, 2) and len(tau) == 6 and area.shape == (4, 3, 2)
    assert np.all(tau[0] >= -1e-9) and np.all(area >= 0)
    tg, w = co.targets(coarse, tau, area, (True, True, False), 0.05)
    assert tg.shape == (24, 2) and np.all((tg[:, 0] >= -0.05) & (tg[:, 0] <= 0.05))
    assert np.all((tg[:, 1] >= 0.25) & (tg[:, 1] <= 4.0))
    feats = co.features(rho, *f, phi, (True, True, False), 0.01, 0.02)
    assert feats.shape == (phi.size, 12) and np.all(np.isfinite(feats))
