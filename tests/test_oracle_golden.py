"""The FP64 oracle against the reference's own recorded outputs (CPU)."""
import os

import numpy as np
import pytest

from fixtures import (FORWARD_CASES, GOLDEN, load_forward_case, read_eps_ctr_first_block, read_inv_ctr_rows,
                      wdatm_phase)


def _oracle(case, **kw):
    from oracle.oracle import OracleProblem
    c = case["cfg"]
    return OracleProblem(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr, swrtr=c.swrtr,
                         lsink=c.lsink, nsink=c.nsink, **kw)


@pytest.mark.parametrize("name", sorted(FORWARD_CASES))
def test_oracle_forward_matches_recorded_voltages(name):
    case = load_forward_case(name)
    op = _oracle(case)
    kp = op.forward(case["sigma"], nthreads=4)
    _, sa = op.bvolt(op.rtrafo(kp))
    mag, pha = wdatm_phase(sa)
    d = case["volt"]
    assert np.abs(mag / d.bet - 1).max() <= FORWARD_CASES[name]
    assert np.abs(pha - d.pha).max() <= 1e-3


def test_oracle_detects_a_planted_model_error():
    """Negative control: a 0.1 % change of one cell's conductivity moves the
    voltages beyond the tolerance the forward test uses."""
    case = load_forward_case("minimal")
    op = _oracle(case)
    sig = case["sigma"].copy()
    sig[150] *= 1.001
    _, sa = op.bvolt(op.rtrafo(op.forward(sig)))
    mag, _ = wdatm_phase(sa)
    assert np.abs(mag / case["volt"].bet - 1).max() > FORWARD_CASES["minimal"]


def test_geometric_factors_match_tmp_kfak():
    case = load_forward_case("Lambda_search")
    op = _oracle(case)
    kf = op.bkfak()
    rec = np.loadtxt(os.path.join(case["base"], "exe", "tmp.kfak"))
    assert rec.shape[0] == len(kf)
    np.testing.assert_allclose(kf, rec[:, 1], rtol=6e-4)   # written as G12.4


@pytest.mark.parametrize("name,k", [("minimal", 8), ("dc_problem_complex", 14)])
def test_wavenumber_count_matches_inv_ctr(name, k):
    from crtomo_stable_b200 import io
    from oracle.oracle import OracleProblem
    base = os.path.join(GOLDEN, name)
    m = io.read_elem(os.path.join(base, "grid", "elem.dat"))
    e = io.read_elec(os.path.join(base, "grid", "elec.dat"))
    d = io.read_volt(os.path.join(base, "mod", "volt.dat"))
    op = OracleProblem(m, e, d.strnr, d.vnr)
    assert len(op.kwn) == k
    # weights of the Gauss-Legendre part integrate sqrt-substituted k exactly:
    assert np.all(op.kwnwi > 0) and np.all(np.diff(op.kwn) > 0)


def _first_step(name):
    from crtomo_stable_b200 import inversion, io, regularization
    from oracle.oracle import OracleCG, OracleProblem, dmisft
    base = os.path.join(GOLDEN, name)
    cfg = inversion.read_crtomo_cfg(os.path.join(base, "exe", "crtomo.cfg"))
    m = io.read_elem(os.path.join(base, "grid", "elem.dat"))
    e = io.read_elec(os.path.join(base, "grid", "elec.dat"))
    d = io.read_volt(os.path.join(base, "mod", "volt.dat"))
    ds = inversion.error_model(d, cfg)
    op = OracleProblem(m, e, d.strnr, d.vnr)
    E = m.elanz
    sig = np.full(E, complex(np.cos(cfg.pha0 / 1e3) / cfg.bet0, -np.sin(cfg.pha0 / 1e3) / cfg.bet0))
    kp = op.forward(sig, ldc=cfg.ldc, nthreads=4)
    volt, sa = op.bvolti(op.rtrafo(kp))
    dat, sa, vnr, wdfak = inversion.chkpol(ds.dat, sa, d.vnr, True)
    r0 = dmisft(dat, sa, ds.wmatd, ds.wmatdr, ds.wmatdp)[0]
    J = op.bsensi(kp, sig, volt, nthreads=4)
    nb = regularization.nachbar(m)
    sm = regularization.smatm_tri(m, nb, cfg.alfx, cfg.alfz)
    lam = inversion.lam0_preset(cfg, E, len(d.bet))
    cg = OracleCG(E, len(dat), cfg.ltri, sm, nachbar=nb, nnb=m.maxnodes, wmatd=ds.wmatd, wdfak=wdfak, lam=lam,
                  eps=1e-4)
    res = cg.update(J, dat, sa, np.log(sig), 1.0)
    rough = cg.brough(res["par"])
    op2 = OracleProblem(m, e, d.strnr, vnr)
    _, sa1 = op2.bvolti(op2.rtrafo(op2.forward(np.exp(res["par"]), nthreads=4)))
    r1 = dmisft(dat, sa1, ds.wmatd, ds.wmatdr, ds.wmatdp)[0]
    rows = read_inv_ctr_rows(os.path.join(base, "inv", "inv.ctr"))
    return dict(r0=r0, r1=r1, bdpar=res["bdpar"], rough=rough, ncg=res["ncg"], lam=lam, sa0=sa), rows


@pytest.mark.parametrize("name", ["minimal", "dc_problem_complex"])
def test_oracle_first_gn_step_matches_inv_ctr(name):
    got, rows = _first_step(name)
    it0 = [r for r in rows if r["kind"] == "IT"][0]
    up1 = [r for r in rows if r["kind"] == "UP"][0]
    assert abs(got["r0"] / it0["rms"] - 1) < 5e-4
    assert abs(got["r1"] / up1["rms"] - 1) < 5e-4
    assert abs(got["bdpar"] / up1["step"] - 1) < 5e-3
    assert abs(got["rough"] / up1["rough"] - 1) < 5e-4
    assert got["ncg"] == up1["ncg"]
    assert got["lam"] == up1["lam"]


def test_oracle_it0_response_matches_eps_ctr():
    got, _ = _first_step("minimal")
    f0 = read_eps_ctr_first_block(os.path.join(GOLDEN, "minimal", "inv", "eps.ctr"))
    np.testing.assert_allclose(got["sa0"].real, f0.real, rtol=2e-6)


def test_oracle_dc_path_on_triangles_matches_eps_ctr():
    from crtomo_stable_b200 import inversion, io
    from oracle.oracle import OracleProblem
    base = os.path.join(GOLDEN, "dc_problem")
    cfg = inversion.read_crtomo_cfg(os.path.join(base, "exe", "crtomo.cfg"))
    m = io.read_elem(os.path.join(base, "grid", "elem.dat"))
    e = io.read_elec(os.path.join(base, "grid", "elec.dat"))
    d = io.read_volt(os.path.join(base, "mod", "volt.dat"))
    op = OracleProblem(m, e, d.strnr, d.vnr)
    sig = np.full(m.elanz, 1.0 / cfg.bet0 + 0j)
    _, sa = op.bvolti(op.rtrafo(op.forward(sig, ldc=True, nthreads=4)))
    f0 = read_eps_ctr_first_block(os.path.join(base, "inv", "eps.ctr"))
    np.testing.assert_allclose(sa.real, f0.real, rtol=2e-6, atol=1e-6)


def test_oracle_analytic_half_space_converges():
    """Homogeneous half-space: K * V -> rho under mesh refinement (within the
    quadrature's 0.5 % plus discretisation error)."""
    from crtomo_stable_b200 import synth
    from oracle.oracle import OracleProblem
    errs = []
    for h in (0.5, 0.25):
        nx, nz = int(60 / h), int(10 / h)
        xs = np.arange(nx + 1) * h
        m = synth.structured_mesh(xs, np.arange(nz + 1) * h, triangles=False)
        enr = synth.surface_electrodes(m, xs, 10.0 + np.arange(40), nz)
        s, v = synth.encode(synth.dipole_dipole(40, (1,), 8))
        op = OracleProblem(m, enr, s, v)
        _, sa = op.bvolt(op.rtrafo(op.forward(np.full(m.elanz, 0.01 + 0j), nthreads=8)), op.bkfak())
        n = v % 10000 - s // 10000
        errs.append(np.abs(np.abs(sa[n >= 4]) / 100.0 - 1).max())
    assert errs[1] < errs[0] and errs[1] < 0.01
