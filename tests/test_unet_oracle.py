"""The FP64 numpy oracle of the warm-start network, pinned by central finite
differences (CPU).  A step of 1e-7 stays clear of the ReLU kinks for this
seed; larger steps cross some of them and show O(step) errors."""
import numpy as np
import pytest

from oracle import unet_oracle as U


@pytest.fixture(scope="module")
def net():
    C, H, W = 16, 16, 16
    rng = np.random.default_rng(0)
    table, n = U.layer_table(C)
    p = np.zeros(n)
    for cin, cout, wo, bo in table:
        p[wo:bo] = rng.normal(0.0, np.sqrt(2.0 / (9 * cin)), bo - wo)
        p[bo:bo + cout] = rng.normal(0.0, 0.05, cout)
    x = U.cavity_inputs([150.0, 2000.0], H, W, 256)
    tgt = rng.normal(0.0, 1.0, (2, 3, H, W))
    return dict(C=C, p=p, x=x, tgt=tgt, sc=[50.0, 10.0, 10.0], off=[1.0, 0.0, 0.0], table=table)


def test_layer_table_matches_channel_plan(net):
    table = net["table"]
    C = net["C"]
    cins = [t[0] for t in table]
    couts = [t[1] for t in table]
    assert cins == [8, C, C, 2 * C, 2 * C, 4 * C, 4 * C, 8 * C, 12 * C, 4 * C, 6 * C, 2 * C, 3 * C, C, C]
    assert couts == [C, C, 2 * C, 2 * C, 4 * C, 4 * C, 8 * C, 8 * C, 4 * C, 4 * C, 2 * C, 2 * C, C, C, 16]
    assert U.layer_table(32)[1] == 1952912  # parameters of the 32-channel network


@pytest.mark.parametrize("gw", [0.0, 5.0])
def test_gradient_matches_central_differences_per_layer(net, gw):
    p, x, tgt, sc, off, C = net["p"], net["x"], net["tgt"], net["sc"], net["off"], net["C"]
    _, g = U.loss_and_grad(p, x, tgt, sc, off, C, grad_weight=gw)
    rng = np.random.default_rng(1)
    eps = 1e-7
    for li, (cin, cout, wo, bo) in enumerate(net["table"]):
        v = np.zeros_like(p)
        v[wo:bo + cout] = rng.normal(0.0, 1.0, bo + cout - wo)
        lp, _ = U.loss_and_grad(p + eps * v, x, tgt, sc, off, C, grad_weight=gw)
        lm, _ = U.loss_and_grad(p - eps * v, x, tgt, sc, off, C, grad_weight=gw)
        fd = (lp - lm) / (2 * eps)
        an = float(g @ v)
        assert abs(fd - an) <= 1e-5 * max(abs(an), 1e-3), (li, fd, an)


def test_pool_and_upsample_adjoints():
    rng = np.random.default_rng(2)
    a = rng.normal(size=(2, 8, 8, 16))
    b = rng.normal(size=(2, 4, 4, 16))
    # <pool(a), b> == <a, pool_grad(b)>; <up(b), a> == <b, up_grad(a)>
    assert np.isclose(np.sum(U._pool(a) * b), np.sum(a * U._pool_grad(b)))
    assert np.isclose(np.sum(U._up(b) * a), np.sum(b * U._up_grad(a)))
    c = rng.normal(size=(1, 6, 5, 8))
    d = rng.normal(size=(1, 6, 5, 72))
    assert np.isclose(np.sum(U._im2col(c) * d), np.sum(c * U._col2im(d, 8)))
