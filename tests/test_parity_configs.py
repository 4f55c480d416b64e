"""Parity of the device path with the FP64 oracle on the benchmark
configurations and on the boundary options the golden tomodirs do not
exercise:

* the 60 x 20 quadrilateral survey (C1) in FP64: all 400 band systems,
  268 readings and the Jacobian against the oracle;
* the 8,000-triangle topography survey (C2) in the mixed form (complex64
  factorisation with FP64 refinement, Jacobian stored complex64) against
  the complex128 oracle, to the 1e-6 the precision form promises;
* Dirichlet nodes: type-13 boundary elements (src/randb.f90:40-82,
  src/randdc.f90) and prescribed non-zero boundary.dat values
  (src/randb2.f90:39-79, src/randbdc2.f90), with and without mixed
  boundaries, complex and real;
* the five-point regulariser (ltri = 0, src/bsmatm_mod.f90:190-362) inside
  the reference's Jacobi-form CG (bp, src/cg_mod.f90:547-577);
* the 60k-triangle benchmark survey (C5): the mixed form's Jacobian and
  one-step model against the FP64 form, and a slice of readings against the
  oracle itself.

Tolerances are stated per test.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-10      # device FP64 vs oracle FP64 (potentials, voltages)
RTOL_SENS = 1e-9       # Jacobian entries relative to the column's largest entry
RTOL_MIXED = 1e-6      # the mixed form's stated accuracy (north of FP32 rounding)


def _threads():
    return max(1, min(16, os.cpu_count() or 1))


def _oracle_forward_jacobian(s, sigma, mode=0, ldc=False, **kw):
    from oracle.oracle import OracleProblem
    op = OracleProblem(s.mesh, s.enr, s.strnr, s.vnr, **kw)
    kp = op.forward(sigma, ldc=ldc, nthreads=_threads())
    hp = op.rtrafo(kp)
    volt, sa = op.bvolti(hp) if mode != 2 else op.bvolt(hp)
    J = None
    if mode == 0:
        J = op.bsensi(kp, sigma, volt, nthreads=_threads())
    elif mode == 1:
        J = op.bsendc(kp, sigma, volt, nthreads=_threads())
    return op, kp, volt, sa, J


def test_c1_fp64_matches_oracle():
    """C1 (60 x 20 quadrilaterals, 40 electrodes, K = 10, 268 readings,
    mixed boundaries: 400 assemble + factor + solve systems) in FP64:
    potentials and voltages to 1e-10, Jacobian to 1e-9 of its column
    maximum."""
    from crtomo_stable_b200 import synth
    from crtomo_stable_b200.lib import PREC_FP64, Context
    s = synth.config1()
    ctx = Context(s.mesh, s.enr, s.strnr, s.vnr, precision=PREC_FP64)
    assert len(ctx.kwn) == 10 and len(s.enr) == 40 and len(s.strnr) == 268
    volt_g, sa_g, kp_g = ctx.forward(s.sigma, want_kpot=True)
    J_g = ctx.jacobian(mode=0)
    op, kp_o, volt_o, sa_o, J_o = _oracle_forward_jacobian(s, s.sigma, kwn=ctx.kwn, kwnwi=ctx.kwnwi)
    assert np.abs(kp_g - kp_o).max() <= RTOL_FP64 * np.abs(kp_o).max()
    np.testing.assert_allclose(volt_g, volt_o, rtol=RTOL_FP64, atol=0)
    np.testing.assert_allclose(sa_g, sa_o, rtol=RTOL_FP64, atol=RTOL_FP64)
    colmax = np.abs(J_o).max(axis=0, keepdims=True) + 1e-300
    assert (np.abs(J_g - J_o) / colmax).max() <= RTOL_SENS
    ctx.close()


def test_c2_mixed_form_matches_complex128_oracle():
    """C2 (~8,000 triangles under sinusoidal topography, 48 electrodes,
    dipole-dipole + Wenner) in the mixed form against the complex128 oracle:
    potentials to 1e-6 of their maximum, every reading's voltage to 1e-6
    relative, and every Jacobian entry above 1e-2 of its column maximum to
    1e-6 relative (all entries to 1e-6 of the column maximum)."""
    from crtomo_stable_b200 import synth
    from crtomo_stable_b200.lib import PREC_MIXED, Context
    s = synth.config2()
    ctx = Context(s.mesh, s.enr, s.strnr, s.vnr, precision=PREC_MIXED)
    volt_g, sa_g, kp_g = ctx.forward(s.sigma, want_kpot=True)
    J_g = ctx.jacobian(mode=0)
    op, kp_o, volt_o, sa_o, J_o = _oracle_forward_jacobian(s, s.sigma, kwn=ctx.kwn, kwnwi=ctx.kwnwi)
    ek = np.abs(kp_g - kp_o).max() / np.abs(kp_o).max()
    ev = (np.abs(volt_g - volt_o) / np.abs(volt_o)).max()
    colmax = np.abs(J_o).max(axis=0, keepdims=True) + 1e-300
    err = np.abs(J_g - J_o)
    big = np.abs(J_o) >= 1e-2 * colmax
    ej = (err[big] / np.abs(J_o[big])).max()
    ec = (err / colmax).max()
    print(f"\nC2 mixed vs complex128 oracle: potentials {ek:.1e}, voltages {ev:.1e}, "
          f"Jacobian (large entries) {ej:.1e}, Jacobian / column max {ec:.1e}")
    assert ek <= RTOL_MIXED and ev <= RTOL_MIXED and ej <= RTOL_MIXED and ec <= RTOL_MIXED
    ctx.close()


# ---------------------------------------------------------------------------
# Dirichlet nodes
def _dirichlet_survey(side_type, nx=30, nz=12, nel=14, seed=11):
    from crtomo_stable_b200 import synth
    xs = np.arange(nx + 1, dtype=np.float64) - 8.0
    depths = synth.graded_depths(nz, 0.5, 1.1)
    mesh = synth.structured_mesh(xs, depths, triangles=True, topo=lambda x: 0.2 * np.sin(x / 4.0),
                                 side_type=side_type)
    rng = np.random.default_rng(seed)
    enr = synth.surface_electrodes(mesh, xs, np.arange(nel, dtype=np.float64), nz)
    strnr, vnr = synth.encode(synth.dipole_dipole(nel, (1, 2), 5))
    sigma = synth.sigma_from(np.exp(rng.uniform(np.log(10), np.log(500), mesh.elanz)),
                             -rng.uniform(1, 25, mesh.elanz))
    return synth.Survey(mesh, enr, strnr, vnr, sigma, f"dirichlet{side_type}", nx, nz)


def _boundary_dat(s, count, seed, up=0):
    """Prescribed values at `count` nodes of the row `up` cells above the
    bottom (node numbers column by column, depth fastest: the bottom node of
    column ix is (ix + 1)(nz + 1)), complex and non-zero."""
    rng = np.random.default_rng(seed)
    cols = np.sort(rng.choice(np.arange(2, s.nx - 1), size=count, replace=False))
    nodes = ((cols + 1) * (s.nz + 1) - up).astype(np.int32)
    vals = rng.uniform(-2e-3, 2e-3, count) + 1j * rng.uniform(-2e-5, 2e-5, count)
    return nodes, vals


@pytest.mark.parametrize("side_type,rwd,ldc", [(13, 0, False), (13, 0, True), (11, 6, False), (11, 6, True),
                                               (13, 6, False), (13, 6, True)])
@pytest.mark.parametrize("precision", [0, 1])
def test_dirichlet_edits_match_oracle(side_type, rwd, ldc, precision):
    """Type-13 Dirichlet elements (randb / randdc: unit row, zero couplings)
    without mixed boundaries -- one factorisation per wavenumber, the other
    electrodes through kompb -- and prescribed boundary.dat values (randb2 /
    randbdc2: couplings moved to the right-hand side) alone with mixed
    boundaries (a factorisation per wavenumber and electrode) or together
    with type-13 elements.  As in the reference, only the refactored
    systems' right-hand sides carry the boundary.dat values; the kompb
    right-hand sides of the other electrodes do not.  Potentials and
    voltages against the oracle: 1e-10 in FP64, 1e-9 in the mixed form
    (complex64 factorisation with FP64 refinement; the real DC systems stay
    FP64)."""
    from crtomo_stable_b200.lib import Context
    s = _dirichlet_survey(side_type)
    kw = {}
    if rwd:
        # with type-13 sides the prescribed nodes sit one row above the
        # (Dirichlet) bottom, so that their couplings are not zeroed by randb
        kw = dict(zip(("rwdnr", "rwd"), _boundary_dat(s, rwd, seed=side_type, up=1 if side_type == 13 else 0)))
    ctx = Context(s.mesh, s.enr, s.strnr, s.vnr, precision=precision, **kw)
    lbeta, lrandb = ctx.precal()[3:]
    assert lbeta == (side_type == 11) and lrandb == (side_type == 13)
    volt_g, sa_g, kp_g = ctx.forward(s.sigma, ldc=ldc, want_kpot=True)
    op, kp_o, volt_o, sa_o, _ = _oracle_forward_jacobian(s, s.sigma, mode=-1, ldc=ldc, kwn=ctx.kwn, kwnwi=ctx.kwnwi,
                                                         **kw)
    tol = RTOL_FP64 if precision == 0 or ldc else 1e-9
    assert np.abs(kp_g - kp_o).max() <= tol * np.abs(kp_o).max()
    np.testing.assert_allclose(volt_g, volt_o, rtol=tol, atol=tol * np.abs(volt_o).max())
    if rwd:
        # the prescribed values themselves, in the refactored systems
        nodes, vals = kw["rwdnr"], kw["rwd"]
        want = vals.real if ldc else vals
        for l in ([0] if side_type == 13 else range(len(s.enr))):
            np.testing.assert_allclose(kp_g[nodes - 1, l, :], np.repeat(want[:, None], len(ctx.kwn), 1),
                                       rtol=tol, atol=tol * np.abs(kp_o).max())
    ctx.close()


# ---------------------------------------------------------------------------
def _true_relres_5pt(J, wmatd, cgfac, lam, sm, nx, rhs, dpar):
    """|b - A x| / |b| of the scaled system A = C (J^H W J + lam R) C with the
    five-point R of src/cg_mod.f90:547-577 (bp), x = dpar / cgfac, in FP64."""
    import scipy.sparse as sp
    M = sm.shape[0]
    i = np.arange(M)
    rows = [i, i[1:], i[:-1], i[nx:], i[:-nx]]
    cols = [i, i[:-1], i[1:], i[:-nx], i[nx:]]
    vals = [sm[:, 0], sm[:-1, 1], sm[:-1, 1], sm[:-nx, 2], sm[:-nx, 2]]
    R = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(M, M))
    x = dpar / cgfac
    Js = J * cgfac[None, :]
    Ax = Js.conj().T @ (wmatd * (Js @ x)) + lam * cgfac * (R @ (cgfac * x))
    return np.linalg.norm(rhs - Ax) / np.linalg.norm(rhs)


@pytest.mark.parametrize("eps,ncgmax", [(1e-4, None), (1e-12, 3000)])
def test_five_point_regulariser_cg_matches_oracle(eps, ncgmax):
    """ltri = 0: the five-point smoothing operator of bsmatmreg
    (smatm(manz, 3): diagonal, x and z couplings, nx cells per row) inside
    the reference's Jacobi-form cjggra (bp, src/cg_mod.f90:547-577), on the
    C1 grid (60 x 20 cells) with its device Jacobian.  At the reference's
    stop rule and iteration cap (1e-4, manz/10): equal iteration counts,
    cgfac to 1e-11, dpar to 1e-7 of its maximum, the float32 residual
    history to 1e-5; at rel-res 1e-6: iteration counts within 2, the true
    relative residual of the device update in the oracle's system below
    2e-6, dpar to 1e-4 of its maximum."""
    from crtomo_stable_b200 import regularization, synth
    from crtomo_stable_b200.lib import Context
    from oracle.oracle import OracleCG, OracleProblem
    s = synth.config1()
    m = s.mesh
    ctx = Context(m, s.enr, s.strnr, s.vnr)
    _, sa_true = ctx.forward(s.sigma)
    rng = np.random.default_rng(3)
    dat = sa_true + 0.02 * rng.standard_normal(len(sa_true)) + 1e-3j * rng.standard_normal(len(sa_true))
    wmatd = np.full(len(dat), 1.0 / 0.02 ** 2)
    sig0 = np.full(m.elanz, 0.01 + 0j)
    _, sa0 = ctx.forward(sig0)
    ctx.jacobian(mode=0, copy=False)
    op = OracleProblem(m, s.enr, s.strnr, s.vnr, kwn=ctx.kwn, kwnwi=ctx.kwnwi)
    kp = op.forward(sig0, nthreads=_threads())
    volt_o, sa_o = op.bvolti(op.rtrafo(kp))
    J_o = op.bsensi(kp, sig0, volt_o, nthreads=_threads())
    sm = regularization.smatm_reg(m, s.nx, s.nz, 1.0, 1.0)
    np.testing.assert_allclose(sm, op.bsmatmreg(s.nx, s.nz, 1.0, 1.0), rtol=1e-14)
    ctx.set_regularizer(0, sm, nx=s.nx)
    ctx.set_data(dat, wmatd)
    lam = 200.0
    ncg_cap = ncgmax if ncgmax else m.elanz // 10
    cg = OracleCG(m.elanz, len(dat), 0, sm, nx=s.nx, wmatd=wmatd, lam=lam, eps=eps, ncgmax=ncg_cap)
    par = np.log(sig0)
    ref = cg.update(J_o, dat, sa_o, par, 1.0)
    got = ctx.update(Context.params(lam, eps=eps, ncgmax=ncg_cap), par, sigmaa=sa_o)
    assert ctx.cg_info()[0] == 0
    np.testing.assert_allclose(got["cgfac"], ref["cgfac"], rtol=1e-11)
    if ncgmax is None:
        assert got["ncg"] == ref["ncg"]
        np.testing.assert_allclose(got["dpar"], ref["dpar"], rtol=1e-7, atol=1e-7 * np.abs(ref["dpar"]).max())
        np.testing.assert_allclose(got["cgres"][1:], ref["cgres"][1:], rtol=1e-5)
        np.testing.assert_allclose(got["bdpar"], ref["bdpar"], rtol=1e-8)
    else:
        # hundreds of iterations in a different summation order: the
        # iteration count within 2, the device update's true relative
        # residual in the oracle's FP64 system below 2e-6 (the stop rule is
        # 1e-6), the update to 1e-4 of its maximum
        assert got["ncg"] < ncg_cap and abs(got["ncg"] - ref["ncg"]) <= 2
        assert _true_relres_5pt(J_o, wmatd, ref["cgfac"], lam, sm, s.nx, ref["rhs"], got["dpar"]) < 2e-6
        np.testing.assert_allclose(got["dpar"], ref["dpar"], rtol=1e-4, atol=1e-4 * np.abs(ref["dpar"]).max())
    ctx.close()


# ---------------------------------------------------------------------------
def _observed(sa_true, seed=20261203):
    """3 % magnitude + 0.1 mrad Gaussian noise on a forward response, with
    the matching data weights (the benchmark's data)."""
    rng = np.random.default_rng(seed)
    mag = np.exp(-sa_true.real)
    pha = -sa_true.imag
    mag = mag * (1.0 + 0.03 * rng.standard_normal(len(mag)))
    pha = pha + 1e-4 * rng.standard_normal(len(pha))
    dat = -np.log(np.abs(mag)) - 1j * pha
    wmatd = 1.0 / (0.03 + 1e-4 / np.abs(mag)) ** 2
    return dat, wmatd


def test_c5_mixed_form_against_fp64_form_and_oracle_slice():
    """The benchmark survey C5 (60,160 triangles, n = 30,444, mb = 129, 128
    electrodes, 12,027 readings, K = 16), one Gauss-Newton step from the
    homogeneous model, as the benchmark runs it:
      * mixed form (complex64 factorisation, adaptive FP64 refinement,
        Jacobian stored complex64, block-preconditioned CG to rel-res 1e-6)
        against the FP64 form (complex128 throughout, the reference's
        Jacobi-form CG to rel-res 1e-6): every Jacobian entry above 1e-2 of
        its column maximum within 1e-6 relative, all entries within 1e-6 of
        their column maximum, the model after the step within 1e-3 in
        log-resistivity and in phase;
      * a slice against the FP64 oracle itself: the readings of one current
        dipole (electrodes 60, 61; the potential dipoles of n = 1..10), their
        voltages and Jacobian rows from the oracle's forward of those
        electrodes' systems: FP64 form to 1e-10 (voltages) and 1e-9 of the
        row maximum (Jacobian), mixed form to 1e-6."""
    from crtomo_stable_b200 import regularization, synth
    from crtomo_stable_b200.lib import PREC_FP64, PREC_MIXED, PRECOND_BLOCK, Context
    from oracle.oracle import OracleProblem
    s = synth.config5()
    m = s.mesh
    E, N = m.elanz, len(s.strnr)
    rho0 = float(np.exp(np.mean(np.log(np.abs(1.0 / s.sigma)))))
    par0 = np.full(E, np.log(1.0 / rho0) + 0j)
    sig0 = np.exp(par0)
    lam = float(max(E, N))
    nb = regularization.nachbar(m)
    sm = regularization.smatm_tri(m, nb, 1.0, 1.0)
    out = {}
    dat = wmatd = None
    for prec in (PREC_FP64, PREC_MIXED):
        ctx = Context(m, s.enr, s.strnr, s.vnr, precision=prec)
        if dat is None:
            _, sa_true = ctx.forward(s.sigma)
            dat, wmatd = _observed(sa_true)
        ctx.set_regularizer(1, sm, nachbar=nb)
        ctx.set_data(dat, wmatd)
        volt, sa = ctx.forward(sig0)
        J = ctx.jacobian(mode=0)
        precond = PRECOND_BLOCK if prec == PREC_MIXED else 0
        upd = ctx.update(Context.params(lam, eps=1e-12, ncgmax=20000, precond=precond), par0, sigmaa=sa)
        out[prec] = dict(volt=volt, sa=sa, J=J, par=upd["par"], ncg=upd["ncg"], kwn=ctx.kwn.copy(),
                         kwnwi=ctx.kwnwi.copy())
        ctx.close()
        del J
    J64, J32 = out[PREC_FP64]["J"], out[PREC_MIXED]["J"]
    worst_big = worst_col = 0.0
    for c0 in range(0, E, 4096):
        a, b = J64[:, c0:c0 + 4096], J32[:, c0:c0 + 4096]
        colmax = np.abs(a).max(axis=0, keepdims=True) + 1e-300
        err = np.abs(b - a)
        big = np.abs(a) >= 1e-2 * colmax
        worst_big = max(worst_big, float((err[big] / np.abs(a[big])).max()))
        worst_col = max(worst_col, float((err / colmax).max()))
    dm = out[PREC_MIXED]["par"] - out[PREC_FP64]["par"]
    dre, dim = np.abs(dm.real).max(), np.abs(dm.imag).max()
    ev = (np.abs(out[PREC_MIXED]["volt"] - out[PREC_FP64]["volt"]) / np.abs(out[PREC_FP64]["volt"])).max()
    print(f"\nC5 mixed vs FP64: voltages {ev:.1e}, Jacobian large entries {worst_big:.1e}, "
          f"Jacobian / column max {worst_col:.1e}, model after the step: log-resistivity {dre:.1e}, "
          f"phase {dim:.1e} (CG iterations {out[PREC_MIXED]['ncg']} block vs {out[PREC_FP64]['ncg']} Jacobi)")
    assert ev <= RTOL_MIXED and worst_big <= RTOL_MIXED and worst_col <= RTOL_MIXED
    assert dre <= 1e-3 and dim <= 1e-3
    # oracle slice: the readings of current dipole (60, 61)
    c1, c2 = s.strnr % 10000, s.strnr // 10000
    rows = np.nonzero((c1 == 60) & (c2 == 61))[0]
    assert len(rows) >= 8
    els = sorted({int(e) for i in rows for e in (c1[i], c2[i], s.vnr[i] % 10000, s.vnr[i] // 10000) if e > 0})
    remap = {e: j + 1 for j, e in enumerate(els)}
    rn = lambda a, b: np.array([remap[int(x)] + 10000 * remap[int(y)] for x, y in zip(a, b)], np.int32)  # noqa: E731
    st = rn(c1[rows], c2[rows])
    vn = rn(s.vnr[rows] % 10000, s.vnr[rows] // 10000)
    op = OracleProblem(m, s.enr[np.array(els) - 1], st, vn, kwn=out[PREC_FP64]["kwn"], kwnwi=out[PREC_FP64]["kwnwi"])
    kp = op.forward(sig0, nthreads=_threads())
    volt_o, _ = op.bvolti(op.rtrafo(kp))
    J_o = op.bsensi(kp, sig0, volt_o, nthreads=_threads())
    rmax = np.abs(J_o).max(axis=1, keepdims=True)
    for prec, tv, tj in ((PREC_FP64, RTOL_FP64, RTOL_SENS), (PREC_MIXED, RTOL_MIXED, RTOL_MIXED)):
        v = out[prec]["volt"][rows]
        Jr = out[prec]["J"][rows, :]
        evr = (np.abs(v - volt_o) / np.abs(volt_o)).max()
        ejr = (np.abs(Jr - J_o) / rmax).max()
        print(f"C5 oracle slice ({len(rows)} readings, {len(els)} electrodes), precision {prec}: "
              f"voltages {evr:.1e}, Jacobian rows / row max {ejr:.1e}")
        assert evr <= tv and ejr <= tj


# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name,ldc,precision", [("minimal", False, 0), ("TestModInv", False, 0), ("TestModInv", True, 0),
                                                ("mixed_surf", False, 1), ("non_ordered", False, 0),
                                                ("Lambda_search", False, 1)])
def test_schur_form_matches_direct_form_and_oracle(name, ldc, precision):
    """The forward by elimination of the mixed-boundary nodes (one interior
    factorisation per wavenumber, dense Schur complement per electrode)
    against the reference's per-system loop on the device and against the
    oracle: potentials and voltages to 1e-10 (both forms FP64 here; the
    Schur form is FP64 in the mixed precision form too)."""
    from fixtures import load_forward_case
    from crtomo_stable_b200.lib import FORWARD_DIRECT, FORWARD_SCHUR, Context
    case = load_forward_case(name)
    c = case["cfg"]
    ctx = Context(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr, swrtr=c.swrtr, lsink=c.lsink,
                  nsink=c.nsink, precision=precision)
    form, m, nI, mbI = ctx.forward_info()
    assert m > 0 and nI + m == case["mesh"].sanz and 0 < mbI <= case["mesh"].mb
    ctx.set_forward_form(FORWARD_SCHUR)
    v_s, sa_s, kp_s = ctx.forward(case["sigma"], ldc=ldc, want_kpot=True)
    assert ctx.forward_info()[0] == FORWARD_SCHUR
    ctx.set_forward_form(FORWARD_DIRECT)
    v_d, sa_d, kp_d = ctx.forward(case["sigma"], ldc=ldc, want_kpot=True)
    assert ctx.forward_info()[0] == FORWARD_DIRECT
    from oracle.oracle import OracleProblem
    op = OracleProblem(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr, swrtr=c.swrtr,
                       lsink=c.lsink, nsink=c.nsink, kwn=ctx.kwn, kwnwi=ctx.kwnwi)
    kp_o = op.forward(case["sigma"], ldc=ldc, nthreads=_threads())
    volt_o, _ = op.bvolti(op.rtrafo(kp_o))
    scale = np.abs(kp_o).max()
    assert np.abs(kp_s - kp_o).max() <= RTOL_FP64 * scale
    assert np.abs(kp_s - kp_d).max() <= (RTOL_FP64 if precision == 0 or ldc else 1e-9) * scale
    np.testing.assert_allclose(v_s, volt_o, rtol=RTOL_FP64, atol=RTOL_FP64 * np.abs(volt_o).max())
    if ldc:
        assert np.abs(kp_s.imag).max() == 0.0
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,ldc", [("minimal", False), ("mixed_surf", False), ("TestModInv", True)])
def test_schur_iteration_matches_schur_cholesky(name, ldc, monkeypatch):
    """The electrode systems S_l solved by the iteration preconditioned with
    one factor per group of electrodes (the default) and by their own
    Cholesky each: the same potentials to 1e-11 of their maximum, and the
    iteration ran (its mean count is reported) and converged (on
    TestModInv's DC systems in about 20 steps, on the 60k-triangle
    benchmark mesh in fewer than 10)."""
    from fixtures import load_forward_case
    from crtomo_stable_b200.lib import FORWARD_SCHUR, Context
    case = load_forward_case(name)
    c = case["cfg"]
    out = {}
    for form in ("iter", "direct"):
        # small meshes take the Cholesky by default (too few systems to fill
        # the GPU with the iteration's CTAs): force each form
        monkeypatch.setenv("CRT_B200_SCHUR_SOLVE", form)
        ctx = Context(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr, swrtr=c.swrtr,
                      lsink=c.lsink, nsink=c.nsink)
        ctx.set_forward_form(FORWARD_SCHUR)
        _, _, kp = ctx.forward(case["sigma"], ldc=ldc, want_kpot=True)
        out[form] = (kp, ctx.timings()["schur_iter"])
        ctx.close()
    assert 1.0 <= out["iter"][1] < 40.0 and out["direct"][1] == 0.0   # 40: the iteration limit
    scale = np.abs(out["direct"][0]).max()
    assert np.abs(out["iter"][0] - out["direct"][0]).max() <= 1e-11 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("name,ldc", [("mixed_surf", False), ("TestModInv", True)])
def test_schur_sweep_beside_the_factor_is_the_sequential_sweep(name, ldc, monkeypatch):
    """The forward sweep run on a second stream, each column block waiting
    for the interior factor's published progress, does the arithmetic of
    the sweep run after the factor: potentials bit for bit equal, and no
    wait gave up (the forward reports no error)."""
    from fixtures import load_forward_case
    from crtomo_stable_b200.lib import FORWARD_SCHUR, Context
    case = load_forward_case(name)
    c = case["cfg"]
    out = {}
    for ov in ("1", "0"):
        monkeypatch.setenv("CRT_B200_SCHUR_OVERLAP", ov)
        ctx = Context(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr, swrtr=c.swrtr,
                      lsink=c.lsink, nsink=c.nsink)
        ctx.set_forward_form(FORWARD_SCHUR)
        for _ in range(2):
            _, sa, kp = ctx.forward(case["sigma"], ldc=ldc, want_kpot=True)
        out[ov] = (kp, sa)
        ctx.close()
    assert np.array_equal(out["1"][0], out["0"][0])
    assert np.array_equal(out["1"][1], out["0"][1])


@pytest.mark.gpu
@pytest.mark.parametrize("name,ldc", [("mixed_surf", False), ("TestModInv", True)])
def test_schur_back_sweep_pipelined_is_the_sequential_sweep(name, ldc, monkeypatch):
    """The back sweep with the block triangles beside the update of the
    rows below (warp groups in two phases, three factor buffers) applies
    every row's contributions in the sequential sweep's order: potentials
    and voltages bit for bit equal."""
    from fixtures import load_forward_case
    from crtomo_stable_b200.lib import FORWARD_SCHUR, Context
    case = load_forward_case(name)
    c = case["cfg"]
    out = {}
    for pp in ("1", "0"):
        monkeypatch.setenv("CRT_B200_SCHUR_BACK_PP", pp)
        ctx = Context(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr, swrtr=c.swrtr,
                      lsink=c.lsink, nsink=c.nsink)
        ctx.set_forward_form(FORWARD_SCHUR)
        _, sa, kp = ctx.forward(case["sigma"], ldc=ldc, want_kpot=True)
        out[pp] = (kp, sa)
        ctx.close()
    assert np.array_equal(out["1"][0], out["0"][0])
    assert np.array_equal(out["1"][1], out["0"][1])


@pytest.mark.gpu
@pytest.mark.parametrize("name,ldc", [("mixed_surf", False), ("TestModInv", True)])
def test_schur_iteration_four_systems_per_cta_is_eight(name, ldc, monkeypatch):
    """The electrode iteration with 4 systems per CTA (two CTAs per SM)
    against 8: each system's steps are the same, but a CTA iterates until
    all its systems have converged, so the other grouping may add a step to
    some systems; the potentials agree to the iteration's tolerance."""
    from fixtures import load_forward_case
    from crtomo_stable_b200.lib import FORWARD_SCHUR, Context
    case = load_forward_case(name)
    c = case["cfg"]
    monkeypatch.setenv("CRT_B200_SCHUR_SOLVE", "iter")
    out = {}
    for ns in ("4", "8"):
        monkeypatch.setenv("CRT_B200_SCHUR_IT_NS", ns)
        ctx = Context(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr, swrtr=c.swrtr,
                      lsink=c.lsink, nsink=c.nsink)
        ctx.set_forward_form(FORWARD_SCHUR)
        _, sa, kp = ctx.forward(case["sigma"], ldc=ldc, want_kpot=True)
        out[ns] = (kp, sa, ctx.timings()["schur_iter"])
        ctx.close()
    assert out["4"][2] >= 1.0
    scale = np.abs(out["8"][0]).max()
    assert np.abs(out["4"][0] - out["8"][0]).max() <= 1e-12 * scale
    np.testing.assert_allclose(out["4"][1], out["8"][1], rtol=1e-11, atol=0)


def test_schur_form_is_refused_where_it_does_not_apply():
    """No mixed boundary (the 2D decoupling grid): the Schur form does not
    apply, the setter says so (errnr 201) and the direct form runs."""
    from fixtures import load_forward_case
    from crtomo_stable_b200.lib import FORWARD_DIRECT, FORWARD_SCHUR, CRTError, Context
    case = load_forward_case("grid_decoupling")
    c = case["cfg"]
    ctx = Context(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr, swrtr=c.swrtr, lsink=c.lsink,
                  nsink=c.nsink)
    with pytest.raises(CRTError) as ei:
        ctx.set_forward_form(FORWARD_SCHUR)
    assert ei.value.errnr == 201
    ctx.forward(case["sigma"])
    assert ctx.forward_info()[:2] == (FORWARD_DIRECT, 0)
    ctx.close()
