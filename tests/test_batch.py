"""Batches of independent instances (crt_batch_*: forward + Jacobian of many
contexts as one captured CUDA graph) and the autotuned panel width of the
blocked band factorisation.  The instances are the uneven synthetic ones of
the batched configuration (synth.config4), at reduced sizes so the oracle
finishes in seconds."""
import ctypes as C

import numpy as np
import pytest

TOL_MIXED = 1e-6     # complex64 factor + two FP64 refinement steps vs the FP64 oracle
RTOL_SAME = 1e-12    # the same kernels on the same inputs (graph replay vs eager calls)


def _instances(count=5, emin=1200, emax=4000):
    from crtomo_stable_b200 import synth
    return synth.config4(count=count, emin=emin, emax=emax)


def test_config4_instances_are_uneven_and_in_range():
    from crtomo_stable_b200 import lib, synth
    S = synth.config4(count=24)
    E = np.array([s.mesh.elanz for s in S])
    L = np.array([len(s.enr) for s in S])
    mb = np.array([s.mesh.mb for s in S])
    assert E.min() >= 1900 and E.max() <= 31000 and E.max() > 4 * E.min()
    assert L.min() >= 24 and L.max() <= 96 and len(set(L.tolist())) > 10
    assert mb.max() <= 65
    K = [len(lib.rwaven(s.mesh, s.enr, s.strnr, s.vnr)[0]) for s in S]
    assert 8 <= min(K) and max(K) <= 15 and len(set(K)) >= 3
    for s in S:
        rho = 1.0 / np.abs(s.sigma)
        assert rho.min() >= 9.99 and rho.max() <= 1000.01
        pha = np.angle(s.sigma) * 1e3     # conductivity phase = -(resistivity phase)
        assert pha.min() >= 0.999 and pha.max() <= 30.001
    again = synth.config4(count=3)
    for a, b in zip(S[:3], again):
        assert np.array_equal(a.sigma, b.sigma) and np.array_equal(a.strnr, b.strnr)


def test_batch_create_rejects_bad_arguments():
    from crtomo_stable_b200 import lib
    L = lib.load()
    err = C.c_int32()
    assert not L.crt_batch_create(None, 3, 0, 0, C.byref(err)) and err.value == 3
    arr = (C.c_void_p * 1)(None)
    assert not L.crt_batch_create(arr, 1, 0, 0, C.byref(err)) and err.value == 3
    assert L.crt_batch_status(None, 0) == 3


@pytest.mark.gpu
def test_batch_graph_matches_eager_calls_and_oracle():
    """Five uneven instances in complex64 with FP64 refinement, forward and
    Jacobian in one graph, each context's workspace capped so the forward
    runs in several chunks: the replayed results equal those of separate
    eager calls, and the smallest instance's voltages and Jacobian are within
    1e-6 of the FP64 oracle."""
    from crtomo_stable_b200.lib import PREC_MIXED, Batch, Context
    from oracle.oracle import OracleProblem
    S = _instances()
    ctxs = [Context(s.mesh, s.enr, s.strnr, s.vnr, precision=PREC_MIXED) for s in S]
    for c in ctxs:
        c.set_workspace_limit(32 << 20)
    b = Batch(ctxs, jacobian_mode=0)
    b.set_models([s.sigma for s in S])
    ms1 = b.run()
    ms2 = b.run()
    assert ms1 > 0 and ms2 > 0
    for i, s in enumerate(S):
        assert b.status(i) == 0
        v, sa, J = b.results(i, sens=True)
        e = Context(s.mesh, s.enr, s.strnr, s.vnr, precision=PREC_MIXED)
        e.set_workspace_limit(32 << 20)   # the same forward form as the batch's context
        ve, sae = e.forward(s.sigma)
        Je = e.jacobian(0)
        np.testing.assert_allclose(v, ve, rtol=RTOL_SAME, atol=RTOL_SAME * np.abs(ve).max())
        np.testing.assert_allclose(sa, sae, rtol=RTOL_SAME, atol=RTOL_SAME * np.abs(sae).max())
        assert np.abs(J - Je).max() <= RTOL_SAME * np.abs(Je).max()
        e.close()
    i0 = int(np.argmin([s.mesh.elanz for s in S]))
    s = S[i0]
    op = OracleProblem(s.mesh, s.enr, s.strnr, s.vnr)
    kp = op.forward(s.sigma, nthreads=4)
    vo, sao = op.bvolti(op.rtrafo(kp))
    v, sa, J = b.results(i0, sens=True)
    assert np.abs(v - vo).max() <= TOL_MIXED * np.abs(vo).max()
    Jo = op.bsensi(kp, s.sigma, vo, nthreads=4)
    colmax = np.abs(Jo).max(axis=0)
    assert (np.abs(J - Jo).max(axis=0) <= TOL_MIXED * colmax + 1e-300).all()
    b.close()
    for c in ctxs:
        c.close()


@pytest.mark.gpu
def test_batch_replay_follows_new_models():
    from crtomo_stable_b200.lib import PREC_MIXED, Batch, Context
    S = _instances(count=3, emin=1500, emax=3000)
    ctxs = [Context(s.mesh, s.enr, s.strnr, s.vnr, precision=PREC_MIXED) for s in S]
    b = Batch(ctxs, jacobian_mode=-1)
    b.set_models([s.sigma for s in S])
    b.run()
    new = [s.sigma * np.exp(np.random.default_rng(i).normal(0, 0.2, s.sigma.size)) for i, s in enumerate(S)]
    b.set_models(new)
    b.run()
    for i, s in enumerate(S):
        v, sa = b.results(i)
        e = Context(s.mesh, s.enr, s.strnr, s.vnr, precision=PREC_MIXED)
        ve, _ = e.forward(new[i])
        np.testing.assert_allclose(v, ve, rtol=RTOL_SAME, atol=RTOL_SAME * np.abs(ve).max())
        e.close()
    b.close()
    for c in ctxs:
        c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("panel", [4, 8, 16])
def test_panel_widths_match_oracle(panel, precision, monkeypatch):
    """Each panel width the autotuner may choose (forced here) gives the
    oracle's potentials: FP64 to 1e-10, complex64 with refinement to 1e-6."""
    from crtomo_stable_b200 import synth
    from crtomo_stable_b200.lib import Context
    from oracle.oracle import OracleProblem
    s = synth.small_triangles(nx=30, nz=14)
    monkeypatch.setenv("CRT_B200_PANEL", str(panel))
    ctx = Context(s.mesh, s.enr, s.strnr, s.vnr, precision=precision)
    _, _, kp = ctx.forward(s.sigma, want_kpot=True)
    assert ctx.timings()["panel"] == panel
    kp_o = OracleProblem(s.mesh, s.enr, s.strnr, s.vnr).forward(s.sigma)
    tol = 1e-10 if precision == 0 else TOL_MIXED
    assert np.abs(kp - kp_o).max() <= tol * np.abs(kp_o).max()
    ctx.close()


@pytest.mark.gpu
def test_autotuned_panel_is_a_candidate():
    from crtomo_stable_b200 import synth
    from crtomo_stable_b200.lib import PREC_MIXED, Context
    s = synth.small_triangles(nx=40, nz=20)
    ctx = Context(s.mesh, s.enr, s.strnr, s.vnr, precision=PREC_MIXED)
    ctx.forward(s.sigma)
    assert ctx.timings()["panel"] in (4, 8, 16)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("cta", [128, 512])
def test_factor_cta_shapes_match_oracle(cta, precision, monkeypatch):
    """The CTA shapes the autotuner may choose besides two 256-thread CTAs per
    SM (forced here): four of 128 threads for small windows, one of 512."""
    from crtomo_stable_b200 import synth
    from crtomo_stable_b200.lib import Context
    from oracle.oracle import OracleProblem
    s = synth.small_triangles(nx=30, nz=14)
    monkeypatch.setenv("CRT_B200_PANEL", "8")
    monkeypatch.setenv("CRT_B200_FACTOR_CTA", str(cta))
    ctx = Context(s.mesh, s.enr, s.strnr, s.vnr, precision=precision)
    _, _, kp = ctx.forward(s.sigma, want_kpot=True)
    kp_o = OracleProblem(s.mesh, s.enr, s.strnr, s.vnr).forward(s.sigma)
    tol = 1e-10 if precision == 0 else TOL_MIXED
    assert np.abs(kp - kp_o).max() <= tol * np.abs(kp_o).max()
    ctx.close()
