"""The learned correction of the CG preconditioner (crt_gnn_*): the CPU
restatement's backward pass against finite differences, the device's loss
and weight gradients against the restatement, deterministic training, and
the learned form of the inner solve against the plain one, whose update it
must reproduce."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import gnn_oracle as go  # noqa: E402


def _tiny_graph(M=12, seed=0):
    rng = np.random.default_rng(seed)
    nbr = -np.ones((M, 4), np.int64)
    for i in range(M):
        for j in (i - 1, i + 1, i + 4, i - 4):
            if 0 <= j < M:
                nbr[i, int((nbr[i] >= 0).sum())] = j
    a = np.where(nbr >= 0, rng.uniform(-0.4, -0.1, (M, 4)), 0.0)
    return nbr, a, rng


def test_oracle_backward_matches_finite_differences():
    nbr, a, rng = _tiny_graph()
    x = rng.standard_normal((12, 4))
    t = rng.standard_normal((12, 2))
    w = rng.standard_normal(go.NPARAM) * 0.3
    _, g = go.loss_grad(w, x, t, nbr, a, 3.0, bf16=False)
    for p in rng.choice(go.NPARAM, 40, replace=False):
        e = np.zeros(go.NPARAM)
        e[p] = 1e-6
        fd = (go.loss_grad(w + e, x, t, nbr, a, 3.0, bf16=False)[0] -
              go.loss_grad(w - e, x, t, nbr, a, 3.0, bf16=False)[0]) / 2e-6
        assert abs(fd - g[p]) <= 1e-5 * (abs(g[p]) + 1e-3)


def test_oracle_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.1415927, 1e-20], np.float32)
    r = go.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125    # ties to even, then up
    assert abs(r[3] + 3.140625) < 1e-12
    assert (go.bf16_round(r) == r).all()


def _c2_context():
    import bench
    from crtomo_stable_b200 import synth
    from crtomo_stable_b200.lib import PREC_FP64
    s = synth.config2()
    ctx, dat, wmatd, par0, lam0, nb, sm = bench.setup_context(s, 0, PREC_FP64)
    ctx.set_model(par0)
    _, sa0 = ctx.forward(np.exp(par0))
    ctx.jacobian(mode=0, copy=False)
    return ctx, par0, sa0, lam0


@pytest.mark.gpu
def test_device_gradient_matches_oracle():
    """Loss and weight gradient of recorded (residual, error) pairs: device
    (bf16 weights, FP32 sums) against the FP64 restatement with the same
    bf16-rounded weights."""
    from crtomo_stable_b200.lib import Context
    ctx, par0, sa0, lam0 = _c2_context()
    n = ctx.gnn_collect(Context.params(lam0, eps=1e-12, ncgmax=20000), stride=16, nmax=6)
    assert n >= 2
    ctx.gnn_init(3)
    w, form = ctx.gnn_get_weights()
    assert form == 0 and w.size == go.NPARAM
    for idx in (0, n - 1):
        r = ctx.gnn_record(idx)
        gd, ld = ctx.gnn_record_grad(idx)
        lo, gref = go.loss_grad(w, r["x"], r["t"], r["nbr"], r["a"], r["tnorm2"])
        assert abs(ld - lo) <= 1e-5 * abs(lo)
        assert np.linalg.norm(gd - gref) <= 1e-5 * np.linalg.norm(gref)
    ctx.close()


@pytest.mark.gpu
def test_training_is_deterministic_and_reduces_the_loss():
    from crtomo_stable_b200.lib import Context
    ctx, par0, sa0, lam0 = _c2_context()
    for f in (2.0, 0.5):
        ctx.gnn_collect(Context.params(lam0 * f, eps=1e-12, ncgmax=20000), stride=16, nmax=64)
    ctx.gnn_init(7)
    h1 = ctx.gnn_train(epochs=4, batch=8, lr=1e-3, seed=5)
    w1, _ = ctx.gnn_get_weights()
    ctx.gnn_init(7)
    h2 = ctx.gnn_train(epochs=4, batch=8, lr=1e-3, seed=5)
    w2, _ = ctx.gnn_get_weights()
    assert np.array_equal(w1, w2) and np.array_equal(h1, h2)
    assert h1[-1] < h1[0]
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("base", ["identity", "block"])
def test_learned_preconditioner_against_the_plain_form(base):
    """Trained on records of the plain CG at other lam values, the learned
    form solves a held-out system to the same relative residual: its update
    matches the plain form's, and the guard bounds the iterations when the
    network does not help.  The iteration counts of both forms are printed
    (the measured gain of the network, which may be negative)."""
    from crtomo_stable_b200.lib import (PRECOND_BLOCK, PRECOND_BLOCK_GNN, PRECOND_GNN, PRECOND_JACOBI,
                                        Context)
    ctx, par0, sa0, lam0 = _c2_context()
    block = base == "block"
    for f in (4.0, 1.0, 0.25):
        ctx.gnn_collect(Context.params(lam0 * f, eps=1e-12, ncgmax=20000), base_block=block, stride=8,
                        nmax=128)
    ctx.gnn_init(7)
    ctx.gnn_train(epochs=10, batch=8, lr=1e-3, seed=5)
    lam = lam0 * 0.7
    plain, learned = (PRECOND_BLOCK, PRECOND_BLOCK_GNN) if block else (PRECOND_JACOBI, PRECOND_GNN)
    ref = ctx.update(Context.params(lam, eps=1e-12, ncgmax=20000, precond=plain), par0, sigmaa=sa0)
    got = ctx.update(Context.params(lam, eps=1e-12, ncgmax=20000, precond=learned), par0, sigmaa=sa0)
    st = ctx.gnn_status()
    assert ctx.cg_info()[0] == learned and st["trained"] == 1
    print(f"\n{base}: plain {ref['ncg']} iterations, learned {got['ncg']} "
          f"(guard {'fired' if st['guard_fired'] else 'quiet'})")
    assert got["ncg"] < 20000
    assert got["ncg"] <= 2 * ref["ncg"] + 2 * 50
    np.testing.assert_allclose(got["dpar"], ref["dpar"], rtol=1e-4, atol=1e-4 * np.abs(ref["dpar"]).max())
    ctx.close()
