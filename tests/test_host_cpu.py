"""Host-side pieces on the CPU: readers/writers, regulariser set-up,
polarity check and the synthetic configurations."""
import os

import numpy as np
import pytest

from fixtures import GOLDEN, load_forward_case


def test_readers_parse_all_fixtures(tmp_path):
    from crtomo_stable_b200 import io
    for name in ("minimal", "TestModInv", "mixed_surf", "grid_decoupling", "dc_problem"):
        base = os.path.join(GOLDEN, name)
        m = io.read_elem(os.path.join(base, "grid", "elem.dat"))
        e = io.read_elec(os.path.join(base, "grid", "elec.dat"))
        assert m.nrel.shape == (m.elanz + m.relanz, m.maxnodes)
        assert e.min() >= 1 and e.max() <= m.sanz
        io.write_elem(str(tmp_path / "elem.dat"), m)
        m2 = io.read_elem(str(tmp_path / "elem.dat"))
        assert np.array_equal(m.nrel, m2.nrel) and np.array_equal(m.rnr, m2.rnr)
        np.testing.assert_allclose(m.sx, m2.sx, rtol=1e-9)
    s = io.read_rho(os.path.join(GOLDEN, "TestModInv", "rho", "rho.dat"))
    io.write_rho(str(tmp_path / "rho.dat"), s)
    np.testing.assert_allclose(io.read_rho(str(tmp_path / "rho.dat")), s, rtol=1e-8)


def test_config_roundtrip_and_checks(tmp_path):
    from crtomo_stable_b200 import io
    d = io.read_volt(os.path.join(GOLDEN, "minimal", "mod", "volt.dat"))
    io.write_config(str(tmp_path / "config.dat"), d.strnr, d.vnr)
    s, v = io.read_config(str(tmp_path / "config.dat"))
    assert np.array_equal(s, d.strnr) and np.array_equal(v, d.vnr)
    io.check_configs(s, v, 6)
    with pytest.raises(ValueError):
        io.check_configs(np.array([10001]), np.array([30002]), 6)   # C1 == C2


def test_write_volt_flips_negative_readings(tmp_path):
    from crtomo_stable_b200 import io
    z = np.array([0.05 + 0j, -0.02 + 1e-6j])
    vnr = io.write_volt(str(tmp_path / "v.dat"), np.array([10002, 10002]), np.array([40003, 50004]), z)
    assert list(vnr) == [40003, 40005]
    d = io.read_volt(str(tmp_path / "v.dat"))
    np.testing.assert_allclose(d.bet, [0.05, 0.02], rtol=1e-7)


def test_crtomo_cfg_parser():
    from crtomo_stable_b200 import inversion
    c = inversion.read_crtomo_cfg(os.path.join(GOLDEN, "minimal", "exe", "crtomo.cfg"))
    assert (c.mswitch, c.nx, c.nz, c.alfx, c.alfz, c.itmax) == (15, 0, -1, 10.0, 1.0, 20)
    assert (c.ldc, c.lfphai, c.stabw0, c.stabm0, c.stabp0) == (False, True, 1.0, 1e-3, -0.5)
    assert (c.lrho0, c.bet0, c.swrtr, c.ltri) == (True, 100.0, 1, 1)
    d = inversion.read_crtomo_cfg(os.path.join(GOLDEN, "dc_problem", "exe", "crtomo.cfg"))
    assert d.ldc and d.bet0 == 20.0 and d.stabw0 == 3.0


@pytest.mark.parametrize("name", ["minimal", "dc_problem", "grid_decoupling"])
def test_regulariser_setup_matches_oracle(name):
    from crtomo_stable_b200 import io, regularization
    from oracle.oracle import OracleProblem
    base = os.path.join(GOLDEN, name)
    m = io.read_elem(os.path.join(base, "grid", "elem.dat"))
    e = io.read_elec(os.path.join(base, "grid", "elec.dat"))
    d = io.read_volt(os.path.join(base, "mod", "volt.dat"))
    op = OracleProblem(m, e, d.strnr, d.vnr, swrtr=1)
    nb_o = op.bnachbar()
    nb = regularization.nachbar(m)
    assert np.array_equal(nb, nb_o)
    np.testing.assert_allclose(regularization.smatm_tri(m, nb, 3.0, 1.0), op.bsmatmtri(nb_o, 3.0, 1.0),
                               rtol=1e-14, atol=1e-14)


def test_regular_grid_regulariser_matches_oracle():
    from crtomo_stable_b200 import regularization, synth
    from oracle.oracle import OracleProblem
    s = synth.config1()
    op = OracleProblem(s.mesh, s.enr, s.strnr, s.vnr)
    np.testing.assert_allclose(regularization.smatm_reg(s.mesh, 60, 20, 10.0, 1.0),
                               op.bsmatmreg(60, 20, 10.0, 1.0), rtol=1e-14)


def test_chkpol_swaps_and_excludes():
    from crtomo_stable_b200 import inversion
    dat = np.array([1.0 + 0.0j, 1.0 + 0.01j])
    sa = np.array([1.0 + np.pi - 0.01j, 1.0 + 0.0j])
    sa[0] = complex(1.0, np.pi - 0.01)
    vnr = np.array([30004, 30004])
    d2, s2, v2, w = inversion.chkpol(dat, sa, vnr, lsetup=True)
    assert v2[0] == 40003 and v2[1] == 30004
    assert list(w) == [0, 1]
    assert abs(s2[0].imag) < 0.1


def test_synthetic_configurations_have_the_stated_sizes():
    from crtomo_stable_b200 import synth
    s1 = synth.config1()
    assert (s1.mesh.sanz, s1.mesh.elanz, s1.mesh.mb, len(s1.enr), len(s1.strnr)) == (1281, 1200, 22, 40, 268)
    s5 = synth.config5()
    assert s5.mesh.elanz == 60160 and len(s5.enr) == 128 and 11000 <= len(s5.strnr) <= 13000
    assert s5.mesh.mb >= 128


def test_synthetic_meshes_are_valid_for_precal():
    from crtomo_stable_b200 import synth
    from oracle.oracle import OracleProblem
    for s in (synth.config1(), synth.config2(), synth.small_triangles()):
        OracleProblem(s.mesh, s.enr, s.strnr, s.vnr)   # raises on a bad orientation (errnr 26)


def test_crmod_geometric_factors_match_oracle_and_recording():
    from crtomo_stable_b200 import crmod
    from oracle.oracle import OracleProblem
    case = load_forward_case("Lambda_search")
    d = case["volt"]
    kf = crmod.bkfak(case["mesh"], case["enr"], d.strnr, d.vnr)
    op = OracleProblem(case["mesh"], case["enr"], d.strnr, d.vnr)
    np.testing.assert_allclose(kf, op.bkfak(), rtol=1e-13)
    rec = np.loadtxt(os.path.join(case["base"], "exe", "tmp.kfak"))
    np.testing.assert_allclose(kf, rec[:, 1], rtol=6e-4)


def test_rcm_order_bandwidth_and_permutation():
    """crt_rcm_order (host code of the block preconditioner): a permutation
    whose bandwidth is no worse than scipy's reverse Cuthill-McKee on the
    element graph of a triangle mesh, and argument checks."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    from crtomo_stable_b200 import regularization, synth
    from crtomo_stable_b200.lib import CRTError, rcm_order
    s = synth.small_triangles(nx=30, nz=12)
    E = s.mesh.elanz
    nb = regularization.nachbar(s.mesh)
    rows, cols = [], []
    for k in range(3):
        h = nb[:, k] > 0
        rows.append(np.arange(E)[h])
        cols.append(nb[h, k] - 1)
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    A = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(E, E))
    A = (A + A.T).tocsr()
    order, bw = rcm_order(A.indptr, A.indices)
    assert np.array_equal(np.sort(order), np.arange(E))
    pos = np.empty(E, int)
    pos[order] = np.arange(E)
    c = A.tocoo()
    assert bw == np.abs(pos[c.row] - pos[c.col]).max()
    p = reverse_cuthill_mckee(A, symmetric_mode=True)
    q = np.empty(E, int)
    q[p] = np.arange(E)
    assert bw <= np.abs(q[c.row] - q[c.col]).max()
    # two components and an isolated vertex
    xadj = np.array([0, 1, 2, 3, 4, 4])
    adj = np.array([1, 0, 3, 2])
    order, bw = rcm_order(xadj, adj)
    assert sorted(order) == [0, 1, 2, 3, 4] and bw == 1
    with pytest.raises(CRTError):
        rcm_order(np.array([0, 1]), np.array([5]))
