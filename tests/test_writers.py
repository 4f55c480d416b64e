"""Output formats of crtomo_stable_b200.writers against the reference's
recorded files (host only)."""
import os

import numpy as np

from fixtures import GOLDEN


def test_fortran_g_editing_matches_recorded_inv_ctr_tokens():
    from crtomo_stable_b200.writers import fortran_g
    # (value, w, d, token as the recorded inv.ctr prints it)
    cases = [(9.006, 10, 4, "9.006"), (1356.568, 9, 3, "0.136E+04"), (300.0, 10, 4, "300.0"),
             (233640.1, 10, 4, "0.2336E+06"), (1567.3, 10, 4, "1567."), (0.0, 9, 3, "0.00"),
             (0.98, 10, 4, "0.9800"), (22.7, 9, 3, "22.7"), (88.6176, 10, 4, "88.62"), (-0.0, 12, 4, "-0.000")]
    for v, w, d, tok in cases:
        s = fortran_g(v, w, d)
        assert len(s) == w and s.split() == [tok], (v, s)


def test_kont2_rows_read_back_and_match_recorded_layout(tmp_path):
    from crtomo_stable_b200.writers import write_inv_ctr_rows
    from fixtures import compare_trajectory, read_inv_ctr_trajectory
    gold = read_inv_ctr_trajectory(os.path.join(GOLDEN, "minimal", "inv", "inv.ctr"))
    rows, events = [], {}
    for g in gold:
        if g["kind"] == "RESET":
            events.setdefault(len(rows), []).append("RESET")
            continue
        rows.append({k: v for k, v in g.items() if k not in ("tol", "setup")})
    p = str(tmp_path / "inv.ctr")
    write_inv_ctr_rows(p, rows, events)
    back = read_inv_ctr_trajectory(p)
    assert compare_trajectory(rows, back, slack=1.01) == []
    assert sum(1 for b in back if b["kind"] == "RESET") == 1


def test_list_directed_items_parse_to_float32_values():
    from crtomo_stable_b200.writers import ld_r4, ld_r8
    for v in (-2.25, -0.25, 0.0510120392, 1234567.8, 3.1e-9, 0.0, -7.25):
        assert np.float32(float(ld_r4(v))) == np.float32(v)
        assert float(ld_r8(v)) == v


def test_wsens_and_wpot_file_names_and_values(tmp_path):
    from crtomo_stable_b200.writers import write_potentials, write_sensitivities
    rng = np.random.default_rng(1)
    J = rng.standard_normal((12, 5)) + 1j * rng.standard_normal((12, 5))
    x, y = np.arange(5.0), -np.arange(5.0)
    os.makedirs(tmp_path / "sens")
    ps = write_sensitivities(str(tmp_path / "sens" / "sens.dat"), J, x, y)
    assert [os.path.basename(p) for p in ps[:2]] == ["sens01.dat", "sens02.dat"]
    rows = np.loadtxt(ps[3], skiprows=1)
    np.testing.assert_allclose(rows[:, 2] + 1j * rows[:, 3], J[3], rtol=1e-6)
    head = np.loadtxt(ps[3], max_rows=1)
    s = J[3].sum()
    np.testing.assert_allclose(head, [abs(s), 1e3 * np.angle(s)], rtol=1e-6)
    hp = rng.standard_normal((7, 4)) + 1j * rng.standard_normal((7, 4))
    strnr = np.array([10002, 30004, 20001] + [10003] * 9)
    pp = write_potentials(str(tmp_path / "pot.dat"), hp, strnr, np.arange(7.0), np.zeros(7))
    assert os.path.basename(pp[11]) == "pot12.dat"
    v = np.loadtxt(pp[1])
    np.testing.assert_allclose(v[:, 2] + 1j * v[:, 3], hp[:, 2] - hp[:, 3], rtol=1e-6, atol=1e-7)
