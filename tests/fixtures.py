"""Shared loaders for the golden tomodirs (tests only)."""
import os

import numpy as np

from crtomo_stable_b200 import io

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# forward fixtures: case -> tolerance on |V| relative to the recorded volt.dat
# (float32 text, 7-9 significant digits)
FORWARD_CASES = {
    "minimal": 2e-7,
    "TestModInv": 2e-7,
    "Lambda_search": 2e-7,
    "mixed_surf": 1e-6,
    "grid_decoupling": 2e-7,
    # recorded by a binary whose output differs from the current source by
    # ~6e-6 (its Test twin agrees with it, not with the source)
    "non_ordered": 1e-5,
}


def load_forward_case(name):
    base = os.path.join(GOLDEN, name)
    cfg = io.read_crmod_cfg(os.path.join(base, "exe", "crmod.cfg"))
    mesh = io.read_elem(os.path.join(base, "grid", "elem.dat"))
    enr = io.read_elec(os.path.join(base, "grid", "elec.dat"))
    sigma = io.read_rho(os.path.join(base, "rho", "rho.dat"), mesh.elanz)
    volt = io.read_volt(os.path.join(base, "mod", "volt.dat"))
    return dict(cfg=cfg, mesh=mesh, enr=enr, sigma=sigma, volt=volt, base=base)


def wdatm_phase(sigmaa):
    """Magnitude and wdatm phase (mrad, folded by +-pi) of responses."""
    pha = np.angle(sigmaa)
    npi = np.sign(pha) * np.floor(np.abs(pha / np.pi) + 0.5) * np.pi
    return np.abs(sigmaa), 1e3 * (pha - npi)


def read_inv_ctr_rows(path):
    """IT / UP rows of inv.ctr as dicts."""
    rows = []
    with open(path) as fh:
        for ln in fh:
            t = ln.split()
            if not t:
                continue
            if t[0] == "IT" and len(t) >= 3:
                rows.append(dict(kind="IT", it=int(t[1]), rms=float(t[2])))
            elif t[0] == "UP" and len(t) >= 8:
                rows.append(dict(kind="UP", it=int(t[1]), rms=float(t[2]), step=float(t[3]),
                                 lam=float(t[4]), rough=float(t[5]), ncg=int(t[6])))
    return rows


def read_eps_ctr_first_block(path):
    """Model response Re/Im(f(m)) of the IT 0 block of eps.ctr."""
    out = []
    with open(path) as fh:
        lines = fh.read().splitlines()
    for i, ln in enumerate(lines):
        if ln.strip().startswith("IT#") or ln.strip().startswith("PIT#"):
            j = i + 2
            while j < len(lines) and lines[j].strip():
                t = lines[j].split()
                out.append(complex(float(t[3]), float(t[4])))
                j += 1
            break
    return np.array(out)


def _printed_tol(tok):
    """Half a unit in the last printed digit of an inv.ctr number."""
    t = tok.upper()
    mant, _, ex = t.partition("E")
    dec = len(mant.split(".")[1]) if "." in mant else 0
    return 0.5 * 10.0 ** (-dec) * 10.0 ** (int(ex) if ex else 0)


def read_inv_ctr_trajectory(path):
    """Every control row of inv.ctr (src/kont2.f90): starting rows (IT / PIT
    with rms, betrms, pharms, npol), lambda / step trials (UP / PUP with rms,
    stepsize, lambda, roughness, CG steps, steplength) and accepted iterates
    (IT / PIT with all of them), each value with its print tolerance, and the
    marker of a phase-model reset."""
    rows = []
    names_setup = ("rms", "betrms", "pharms", "npol")
    names_up = ("rms", "step", "lam", "rough", "ncg", "steplength")
    names_it = ("rms", "step", "lam", "rough", "ncg", "betrms", "pharms", "npol", "steplength")
    with open(path) as fh:
        for ln in fh:
            t = ln.split()
            if "Resetting phase model" in ln:
                rows.append(dict(kind="RESET"))
                continue
            if not t or t[0] not in ("IT", "UP", "PIT", "PUP") or len(t) < 3:
                continue
            vals = t[2:]
            if t[0] in ("UP", "PUP"):
                names = names_up
            elif len(vals) == len(names_it):
                names = names_it
            else:
                names = names_setup
            r = dict(kind=t[0], it=int(t[1]), setup=names is names_setup, tol={})
            for n, v in zip(names, vals):
                if v.upper() == "NAN":
                    continue
                r[n] = int(v) if n in ("ncg", "npol") else float(v)
                r["tol"][n] = _printed_tol(v)
            rows.append(r)
    return rows


def compare_trajectory(got, gold, slack=1.5, rel_extra=0.0):
    """Mismatches between Inversion.run rows and recorded rows, value by
    value within `slack` times the print tolerance (plus rel_extra relative);
    CG steps and excluded-reading counts exactly."""
    bad = []
    gold = [g for g in gold if g["kind"] != "RESET"]
    for i, (a, g) in enumerate(zip(got, gold)):
        if a["kind"] != g["kind"] or a["it"] != g["it"]:
            bad.append((i, "kind/it", (a["kind"], a["it"]), (g["kind"], g["it"])))
            continue
        for n, tol in g["tol"].items():
            if n not in a:
                continue
            if n in ("ncg", "npol"):
                if int(a[n]) != g[n]:
                    bad.append((i, n, a[n], g[n]))
            elif abs(a[n] - g[n]) > slack * tol + rel_extra * abs(g[n]):
                bad.append((i, n, a[n], g[n]))
    return bad
