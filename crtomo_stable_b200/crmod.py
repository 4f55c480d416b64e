"""CRMod-compatible forward driver on the device path.

    python -m crtomo_stable_b200.crmod EXE_DIR
        reads EXE_DIR/crmod.cfg (src/fem.f90:163-184) and the files it names,
        runs the forward model through the C ABI and writes volt.dat in the
        format of src/wdatm.f90 (|R| * K and phase in mrad, float32 text);
    python -m crtomo_stable_b200.crmod --synthetic C3 OUT_DIR
        writes the seeded synthetic configuration as a tomodir
        (grid/, rho/, config/, exe/crmod.cfg) and runs it.

Geometric factors (src/bkfak.f90) are applied when mswitch bit 1 is set and
the mesh has mixed boundaries, as CRMod does.
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import time

import numpy as np

from . import io, writers


def bkfak(mesh, enr, strnr, vnr) -> np.ndarray:
    """Half-space geometric factors with image terms (src/bkfak.f90:46-136)."""
    pi = math.acos(-1.0)
    kf = np.zeros(len(strnr))
    xk = np.zeros(4)
    yk = np.zeros(4)
    for i, (s, v) in enumerate(zip(strnr, vnr)):
        e = [int(s) % 10000, int(s) // 10000, int(v) % 10000, int(v) // 10000]
        for q in range(4):
            if e[q] > 0:
                x, y = mesh.node_xy(np.array([enr[e[q] - 1]]))
                xk[q], yk[q] = x[0], y[0]

        def r(u, w):
            if e[u] > 0 and e[w] > 0:
                dx = xk[u] - xk[w]
                dym = 1.0 / math.sqrt(dx * dx + (yk[u] - yk[w]) ** 2)
                dyp = 1.0 / math.sqrt(dx * dx + (yk[u] + yk[w]) ** 2)
                return dym + dyp
            return 0.0

        dum = (r(3, 1) - r(3, 0)) - (r(2, 1) - r(2, 0))
        if dum == 0.0:
            raise ValueError(f"zero geometric factor for reading {i + 1} (errnr 93)")
        kf[i] = 4.0 * pi / dum
    return kf


def run(exe_dir: str, device: int = 0, verbose: bool = True) -> dict:
    from .lib import Context
    cfg = io.read_crmod_cfg(os.path.join(exe_dir, "crmod.cfg"))
    mesh = io.read_elem(io.resolve(exe_dir, cfg.elem))
    enr = io.read_elec(io.resolve(exe_dir, cfg.elec))
    sigma = io.read_rho(io.resolve(exe_dir, cfg.rho), mesh.elanz)
    strnr, vnr = io.read_config(io.resolve(exe_dir, cfg.config))
    io.check_configs(strnr, vnr, len(enr))
    if cfg.lrandb2:
        raise NotImplementedError("boundary.dat values are not supported by this driver")
    t0 = time.perf_counter()
    ctx = Context(mesh, enr, strnr, vnr, swrtr=cfg.swrtr, lsink=cfg.lsink, nsink=cfg.nsink, device=device)
    kfak = None
    wkfak = bool(cfg.mswitch & 2)
    lbeta = bool(np.any(mesh.typ == 11))
    if wkfak and lbeta:
        kfak = bkfak(mesh, enr, strnr, vnr)
    volt, sigmaa = ctx.forward(sigma, mode=1, kfak=kfak)
    t1 = time.perf_counter()
    out = {}
    if cfg.lvolt:
        path = io.resolve(exe_dir, cfg.volt)
        os.makedirs(os.path.dirname(path), exist_ok=True)
        io.write_volt(path, strnr, vnr, sigmaa)
        out["volt"] = path
    if cfg.lpot:
        # bpot / wpot (src/bpot.f90, src/wpot.f90): one file per reading
        hpot = ctx.potentials()
        path = io.resolve(exe_dir, cfg.pot)
        os.makedirs(os.path.dirname(path), exist_ok=True)
        nx, ny = mesh.node_xy(np.arange(1, mesh.sanz + 1))
        out["pot"] = writers.write_potentials(path, hpot, strnr, nx, ny)
    if cfg.lsens:
        # bsens + wsens (src/bsens.f90, src/wsens.f90): one file per reading
        sens = ctx.jacobian(mode=2)
        path = io.resolve(exe_dir, cfg.sens)
        os.makedirs(os.path.dirname(path), exist_ok=True)
        espx, espy = mesh.midpoints()
        out["sens"] = writers.write_sensitivities(path, sens, espx, espy)
    tm = ctx.timings()
    ctx.close()
    if verbose:
        print(f"crmod: n={mesh.sanz} E={mesh.elanz} mb={mesh.mb} electrodes={len(enr)} readings={len(strnr)} "
              f"K={len(ctx.kwn)} forward {1e3 * (t1 - t0):.1f} ms (factor {tm['factor']:.1f} ms, solve "
              f"{tm['solve']:.1f} ms)", file=sys.stderr)
    out["sigmaa"] = sigmaa
    return out


CRMOD_CFG = """***FILES***
../grid/elem.dat
../grid/elec.dat
../rho/rho.dat
../config/config.dat
F                ! potentials ?
../mod/pot/pot.dat
T                ! measurements ?
../mod/volt.dat
F                ! sensitivities ?
../mod/sens/sens.dat
F                ! another dataset ?
1                ! 2D (=0) or 2.5D (=1)
F                ! fictitious sink ?
1                ! fictitious sink node number
F                ! boundary values ?
boundary.dat
2
"""


def write_synthetic_tomodir(name: str, out_dir: str) -> str:
    from . import synth
    s = synth.CONFIGS[name]()
    for d in ("grid", "rho", "config", "exe", "mod"):
        os.makedirs(os.path.join(out_dir, d), exist_ok=True)
    io.write_elem(os.path.join(out_dir, "grid", "elem.dat"), s.mesh)
    io.write_elec(os.path.join(out_dir, "grid", "elec.dat"), s.enr)
    io.write_rho(os.path.join(out_dir, "rho", "rho.dat"), s.sigma)
    io.write_config(os.path.join(out_dir, "config", "config.dat"), s.strnr, s.vnr)
    with open(os.path.join(out_dir, "exe", "crmod.cfg"), "w") as fh:
        fh.write(CRMOD_CFG)
    return os.path.join(out_dir, "exe")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("exe_dir", nargs="?")
    ap.add_argument("--synthetic", default=None, help="C1, C2, C3 or C5")
    ap.add_argument("--out", default=None, help="tomodir for --synthetic")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    exe = a.exe_dir
    if a.synthetic:
        exe = write_synthetic_tomodir(a.synthetic, a.out or ("tomodir_" + a.synthetic))
    if not exe:
        ap.error("EXE_DIR or --synthetic required")
    run(exe, device=a.device)


if __name__ == "__main__":
    main()
