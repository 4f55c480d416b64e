"""Small cases of single kernels, sized for an ncu capture.

    python -m crtomo_stable_b200.cases schur [N]    N Schur-form forwards
    python -m crtomo_stable_b200.cases sens [N]     N forwards + Jacobians
    python -m crtomo_stable_b200.cases <case> check  the case's sizes (host only)

schur: a 60 x 128 strip of split quadrilaterals with mixed sides and bottom
(interior band 129 like the 60k-triangle benchmark mesh), 32 surface
electrodes: m = 317 boundary nodes, 12 wavenumbers, 384 Schur systems.
sens: a 140 x 30 strip (8,400 triangles) with 128 surface electrodes and
3,576 dipole-dipole readings, the benchmark's electrode count for the
Gram-form Jacobian.
"""
from __future__ import annotations

import sys

import numpy as np

from . import synth


def strip(nx: int, nz: int, nel: int, dz0: float, growth: float, spacings, nmax: int):
    xs = -(nx - nel) / 2.0 + np.arange(nx + 1, dtype=np.float64)
    mesh = synth.structured_mesh(xs, synth.graded_depths(nz, dz0, growth), triangles=True)
    enr = synth.surface_electrodes(mesh, xs, np.arange(nel, dtype=np.float64), nz)
    strnr, vnr = synth.encode(synth.dipole_dipole(nel, spacings, nmax))
    return mesh, enr, strnr, vnr


CASES = {
    "schur": dict(nx=60, nz=128, nel=32, dz0=0.25, growth=1.03, spacings=(1, 2, 3, 4, 5), nmax=8),
    "sens": dict(nx=140, nz=30, nel=128, dz0=0.25, growth=1.06, spacings=(1, 2, 3, 4), nmax=8),
}


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    name = argv[0] if argv else "schur"
    mesh, enr, strnr, vnr = strip(**CASES[name])
    if len(argv) > 1 and argv[1] == "check":
        from .lib import rwaven
        print(name, "nodes", mesh.sanz, "elements", mesh.elanz, "mb", mesh.mb, "electrodes", len(set(enr.tolist())),
              "readings", len(strnr), "K", len(rwaven(mesh, enr, strnr, vnr)[0]))
        return
    reps = int(argv[1]) if len(argv) > 1 else 1
    from .lib import FORWARD_SCHUR, PREC_MIXED, Context
    if name == "schur":
        ctx = Context(mesh, enr, strnr, vnr)
        ctx.set_forward_form(FORWARD_SCHUR)
    else:
        ctx = Context(mesh, enr, strnr, vnr, precision=PREC_MIXED)
    sig = np.full(mesh.elanz, 0.01 + 0j)
    for _ in range(reps):
        ctx.forward(sig)
        if name == "sens":
            ctx.jacobian(mode=0, copy=False)
    print(name, "form", ctx.forward_info(), {k: round(v, 3) for k, v in ctx.timings().items() if v})
    ctx.close()


if __name__ == "__main__":
    main()
