"""A stand-in for crtomo_stable_b200.lib.Context built on the CPU oracle
(tests only).

It lets the Gauss-Newton loop's host logic (inversion.Inversion.run) run on
a machine without a GPU, so that its lambda search, step-length control,
stop tests and final phase improvement are checked against the reference's
recorded inv.ctr files by the CPU suite.  Every numerical step is the
oracle's restatement of the reference (forward, bvolti, bsensi / bsendc,
update + cjggra / cjggdc, blam0).
"""
import numpy as np

from crtomo_stable_b200.lib import CRTError
from oracle.oracle import OracleCG, OracleProblem


class OracleContext:
    def __init__(self, mesh, enr, strnr, vnr, swrtr=1, lsink=False, nsink=0, nthreads=4):
        self.mesh = mesh
        self.op = OracleProblem(mesh, enr, strnr, vnr, swrtr=swrtr, lsink=lsink, nsink=nsink)
        self.nthreads = nthreads
        self.elanz = mesh.elanz
        self.nanz = len(strnr)
        self.kpot = self.sigma = self.volt = self.sigmaa = None
        self.sens = self.sensdc = None
        self.calls = dict(forward=0, jacobian=0, update=0, blam0=0)

    # -- set-up ---------------------------------------------------------------
    def set_regularizer(self, ltri, smatm, nx=0, nachbar=None):
        self.ltri, self.smatm, self.nx = ltri, smatm, nx
        self.nachbar = nachbar
        self.nnb = 0 if nachbar is None else nachbar.shape[1] - 1

    def set_data(self, dat, wmatd, wdfak=None):
        self.dat = np.array(dat, np.complex128)
        self.wmatd = np.array(wmatd, np.float64)
        self.wdfak = np.ones(self.nanz, np.int32) if wdfak is None else np.array(wdfak, np.int32)

    def set_configs(self, strnr, vnr):
        """Same contract as crt_set_configs: readings whose potential
        electrodes were swapped get the stored response flipped."""
        old = self.op.vnr.copy()
        v = np.asarray(vnr, np.int32)
        if self.volt is not None:
            sw = (old != v) & (old % 10000 == v // 10000) & (old // 10000 == v % 10000)
            self.volt[sw] = -self.volt[sw]
            im = self.sigmaa[sw].imag
            self.sigmaa[sw] = self.sigmaa[sw].real + 1j * np.where(im > 0, im - np.pi, im + np.pi)
        np.copyto(self.op.vnr, v)        # the oracle's problem points at this array
        np.copyto(self.op.strnr, np.asarray(strnr, np.int32))

    # -- device path stand-ins --------------------------------------------------
    def forward(self, sigma, ldc=False, mode=0):
        self.calls["forward"] += 1
        self.sigma = np.array(sigma, np.complex128)
        try:
            self.kpot = self.op.forward(self.sigma, ldc=ldc, nthreads=self.nthreads)
            volt, sa = self.op.bvolti(self.op.rtrafo(self.kpot))
        except RuntimeError as exc:
            msg = str(exc)
            errnr = int(msg.split()[-1]) if msg.split()[-1].isdigit() else 1
            raise CRTError(errnr, msg) from exc
        self.volt, self.sigmaa = volt.copy(), sa.copy()
        return volt, sa

    def jacobian(self, mode=0, strom=None, copy=True):
        self.calls["jacobian"] += 1
        if mode == 1:
            self.sensdc = self.op.bsendc(self.kpot, self.sigma, self.volt, nthreads=self.nthreads)
            self.sens = None
            return self.sensdc.copy() if copy else None
        self.sens = self.op.bsensi(self.kpot, self.sigma, self.volt, nthreads=self.nthreads)
        self.sensdc = None
        return self.sens.copy() if copy else None

    def _cg(self, prm):
        return OracleCG(self.elanz, self.nanz, self.ltri, self.smatm, nachbar=self.nachbar, nx=self.nx,
                        nnb=self.nnb, wmatd=self.wmatd, wdfak=self.wdfak, lam=prm.lam, eps=prm.eps,
                        ncgmax=prm.ncgmax, ldc=bool(prm.ldc), lfpi=bool(prm.lfpi))

    def update(self, prm, par, sigmaa=None):
        self.calls["update"] += 1
        sa = self.sigmaa if sigmaa is None else sigmaa
        r = self._cg(prm).update(self.sens, self.dat, sa, par, step=prm.step, sensdc=self.sensdc)
        return dict(par=r["par"], dpar=r["dpar"], cgfac=r["cgfac"], cgres=r["cgres"], ncg=r["ncg"],
                    bdpar=r["bdpar"])

    def blam0(self, alfx, alfz, ldc=False, lfpi=False):
        self.calls["blam0"] += 1

        class _P:
            lam, eps, ncgmax, step = 1.0, 1e-4, 1, 1.0
        _P.ldc, _P.lfpi = ldc, lfpi
        return self._cg(_P).blam0(sens=self.sens, sensdc=self.sensdc, alfx=alfx, alfz=alfz)

    def coverage(self, part=0, weight=None):
        """bbsens's column sums (src/bbsens.f90:52-70) of the resident
        Jacobian in numpy."""
        w = np.sqrt(self.wmatd * self.wdfak) if weight is None else np.asarray(weight)
        J = self.sensdc if self.sens is None else self.sens
        a = np.abs(J.real) if (part == 1 and self.sens is not None) else np.abs(J)
        return (a * w[:, None]).sum(axis=0)

    def close(self):
        pass
