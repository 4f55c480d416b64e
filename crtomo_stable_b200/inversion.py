"""Host driver of the CRTomo inversion around the device path.

Mirrors the set-up of src/rall.f90 (crtomo.cfg), src/rdati.f90 (data and
error model), src/bsigm0.f90 (starting model) and the first pass of the
Gauss-Newton loop of src/inv.f90:332-956 (forward, dmisft, bsensi/bsendc,
bsmatm, blam0 presets, bpar, update, bsigma, brough), calling the C ABI for
every hot-path step.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Optional

import numpy as np

from . import io, regularization, writers
from .lib import Context, CRTError, dmisft


def _quot(a: float, b: float) -> float:
    """a / b with IEEE semantics (0 / 0 = NaN, which fails every comparison,
    as in the reference's Fortran)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return float(np.float64(a) / np.float64(b))


@dataclasses.dataclass
class CRTomoConfig:
    """crtomo.cfg (src/rall.f90:234-472)."""

    mswitch: int
    elem: str
    elec: str
    volt: str
    ramd: str
    ldiff: bool
    nx: int
    nz: int
    alfx: float
    alfz: float
    itmax: int
    ldc: bool
    lrobust: bool
    lfphai: bool
    stabw0: float
    stabm0: float
    stabpA1: float
    stabpB: float
    stabpA2: float
    stabp0: float
    lrho0: bool
    bet0: float
    pha0: float
    lagain: bool
    swrtr: int
    lsink: bool
    nsink: int
    lrandb2: bool
    randb: str
    ltri: int = 0
    lamfix: float = 0.0
    llamf: int = 0
    iseedpri: int = 0
    modl_stdn: float = 0.0


def _lines_no_comments(path):
    with open(path) as fh:
        raw = fh.read().splitlines()
    return raw


def read_crtomo_cfg(path: str) -> CRTomoConfig:
    lines = _lines_no_comments(path)
    pos = 0

    def nxt():
        # read_comments (src/get_unit.f90): skip lines whose first non-blank
        # character is '#', then return the next record
        nonlocal pos
        while pos < len(lines) and lines[pos].strip().startswith("#"):
            pos += 1
        if pos >= len(lines):
            raise EOFError(path)
        ln = lines[pos]
        pos += 1
        return ln

    def val(ln):
        return ln.split("!")[0].strip()

    def first_tok(ln):
        t = val(ln).split()
        return t[0] if t else ""

    ln = nxt()
    try:
        mswitch = int(first_tok(ln))
    except ValueError:
        mswitch = 0
    elem = val(nxt())
    elec = val(nxt())
    volt = val(nxt())
    ramd = val(nxt())
    ldiff = io._fortran_bool(first_tok(nxt()))
    nxt(); nxt(); nxt()          # dd0, dm0, dfm0
    iseedpri, modl_stdn = 0, 0.0
    save = pos
    ln = nxt()
    toks = val(ln).split()
    try:
        iseedpri, modl_stdn = int(toks[0]), float(toks[1])
    except (ValueError, IndexError):
        pass  # a non-numeric line is consumed (err= branch of rall)
    del save
    nx = int(first_tok(nxt()))
    nz = int(first_tok(nxt()))
    alfx = float(first_tok(nxt()))
    alfz = float(first_tok(nxt()))
    itmax = int(first_tok(nxt()))
    ldc = io._fortran_bool(first_tok(nxt()))
    lrobust = io._fortran_bool(first_tok(nxt()))
    lfphai = io._fortran_bool(first_tok(nxt()))
    stabw0 = io._ffloat(first_tok(nxt()))
    stabm0 = io._ffloat(first_tok(nxt()))
    stabpA1 = io._ffloat(first_tok(nxt()))
    stabpB = io._ffloat(first_tok(nxt()))
    stabpA2 = io._ffloat(first_tok(nxt()))
    stabp0 = io._ffloat(first_tok(nxt()))
    lrho0 = io._fortran_bool(first_tok(nxt()))
    bet0 = io._ffloat(first_tok(nxt()))
    pha0 = io._ffloat(first_tok(nxt()))
    lagain = io._fortran_bool(first_tok(nxt()))
    swrtr = int(first_tok(nxt()))
    lsink = io._fortran_bool(first_tok(nxt()))
    nsink = int(first_tok(nxt()))
    lrandb2 = io._fortran_bool(first_tok(nxt()))
    randb = val(nxt())
    ltri = 0
    lamfix = 0.0
    llamf = 0
    try:
        ln = nxt()
        s = ln[:2].strip()   # READ '(I2)'
        ltri = int(s) if s else 0
        if ltri & (1 << 5):
            llamf = 1
            try:
                lamfix = float(first_tok(nxt()))
            except (ValueError, EOFError):
                lamfix = 1.0
            ltri -= 1 << 5
            if ltri & (1 << 6):
                llamf += 2
                ltri -= 1 << 6
    except (ValueError, EOFError):
        ltri = 0
    if (nx <= 0 or nz <= 0) and ltri == 0:
        ltri = 1
    return CRTomoConfig(mswitch, elem, elec, volt, ramd, ldiff, nx, nz, alfx, alfz, itmax, ldc, lrobust,
                        lfphai, stabw0, stabm0, stabpA1, stabpB, stabpA2, stabp0, lrho0, bet0, pha0, lagain,
                        swrtr, lsink, nsink, lrandb2, randb, ltri, lamfix, llamf, iseedpri, modl_stdn)


@dataclasses.dataclass
class DataSet:
    """datmod / invmod arrays after rdati."""

    strnr: np.ndarray
    vnr: np.ndarray
    dat: np.ndarray        # complex (-ln|R|, -phase/1000)
    wmatdr: np.ndarray
    wmatdp: np.ndarray
    wmatd_cri: np.ndarray
    wmatd: np.ndarray
    wdfak: np.ndarray


def error_model(d: io.Data, cfg: CRTomoConfig) -> DataSet:
    """src/rdati.f90:133-231 without synthetic noise (lnse = .false.), and
    the wmatd choice of src/rall.f90:802-817."""
    stabp0 = abs(cfg.stabp0)      # lffhom: negative A3 flags a phase restart
    bet = np.asarray(d.bet, np.float64)
    pha = np.asarray(d.pha, np.float64)
    if d.stabw is not None:
        stabw = d.stabw / bet
        stabwp = 1e-3 * d.stabwp if not cfg.ldc else np.zeros_like(bet)
    else:
        stabw = 1e-2 * cfg.stabw0 + cfg.stabm0 / bet
        if cfg.ldc:
            stabwp = np.zeros_like(bet)
        else:
            stabwp = (cfg.stabpA1 * bet ** cfg.stabpB + 1e-2 * cfg.stabpA2 * np.abs(pha) + stabp0) * 1e-3
    if np.any(bet <= 0):
        raise ValueError("non-positive resistance (errnr 94)")
    if cfg.ldc:
        pha = np.zeros_like(pha)
    dat = -np.log(bet) - 1j * pha / 1e3
    wmatdr = 1.0 / stabw ** 2
    with np.errstate(divide="ignore"):
        wmatdp = np.where(stabwp > 0, 1.0 / stabwp ** 2, 0.0) if not cfg.ldc else np.zeros_like(bet)
    wmatd_cri = 1.0 / (stabw ** 2 + stabwp ** 2) if not cfg.ldc else np.zeros_like(bet)
    lelerr = (not cfg.lfphai and not cfg.ldc) or bool(cfg.mswitch & (1 << 5))
    if cfg.ldc:
        wmatd = wmatdr
    elif lelerr:
        wmatd = wmatd_cri
    else:
        wmatd = wmatdr
    return DataSet(d.strnr, d.vnr, dat, wmatdr, wmatdp, wmatd_cri, wmatd.copy(), np.ones(len(bet), np.int32))


def lam0_preset(cfg: CRTomoConfig, manz: int, nanz: int, lamnull_file: Optional[str] = None) -> Optional[float]:
    """blam0 presets (src/blam0.f90:45-77 with src/rall.f90:763-800).
    Returns None when lam0 has to be computed from the Jacobian."""
    lamnull_cri = 0.0
    if lamnull_file and os.path.exists(lamnull_file):
        with open(lamnull_file) as fh:
            try:
                lamnull_cri = float(fh.read().split()[0])
            except (ValueError, IndexError):
                lamnull_cri = 0.0
    elif cfg.llamf & 1:
        lamnull_cri = cfg.lamfix
    elif cfg.nz == -1:
        lamnull_cri = float(max(manz, nanz))
    elif cfg.nz < 0:
        lamnull_cri = float(abs(cfg.nz))
    if (cfg.llamf & 1) or lamnull_cri > np.finfo(float).eps:
        if cfg.nz == -1:
            return float(np.float32(max(manz, nanz)))
        return lamnull_cri
    return None


class Inversion:
    """Device-backed CRTomo state for one tomodir-like problem."""

    def __init__(self, mesh: io.Mesh, enr, data: DataSet, cfg: CRTomoConfig, device: int = 0,
                 lam0: Optional[float] = None, ctx=None):
        """ctx: the problem's device context; default a new Context on
        `device`.  Any object with Context's set_regularizer / set_data /
        set_configs / forward / jacobian / update / blam0 / close methods
        can stand in (the loop's host logic is independent of it)."""
        self.mesh = mesh
        self.cfg = cfg
        self.data = data
        if ctx is None:
            ctx = Context(mesh, enr, data.strnr, data.vnr, swrtr=cfg.swrtr, lsink=cfg.lsink,
                          nsink=cfg.nsink, device=device)
        self.ctx = ctx
        self.manz = mesh.elanz
        self.nanz = len(data.dat)
        if cfg.ltri == 0:
            self.smatm = regularization.smatm_reg(mesh, cfg.nx, cfg.nz, cfg.alfx, cfg.alfz)
            self.ctx.set_regularizer(0, self.smatm, nx=cfg.nx)
            self.nachbar = None
        elif cfg.ltri in (1, 2):
            self.nachbar = regularization.nachbar(mesh)
            self.smatm = regularization.smatm_tri(mesh, self.nachbar, cfg.alfx, cfg.alfz)
            self.ctx.set_regularizer(1, self.smatm, nachbar=self.nachbar)
        else:
            raise NotImplementedError(f"regulariser ltri={cfg.ltri} is outside the implemented path")
        self.ctx.set_data(data.dat, data.wmatd, data.wdfak)
        self.lam0 = lam0 if lam0 is not None else lam0_preset(cfg, self.manz, self.nanz)
        self.ncgmax = self.manz // 10 if cfg.ltri < 5 else self.manz

    def start_model(self) -> np.ndarray:
        """bsigm0 with a homogeneous background (src/bsigm0.f90:55-61)."""
        c = self.cfg
        if not c.lrho0:
            raise NotImplementedError("only the homogeneous starting model is implemented")
        s = complex(math.cos(c.pha0 / 1e3) / c.bet0, -math.sin(c.pha0 / 1e3) / c.bet0)
        return np.full(self.manz, s, np.complex128)

    def misfit(self, sigmaa):
        d = self.data
        return dmisft(d.dat, sigmaa, d.wmatd, d.wmatdr, d.wmatdp)

    def roughness(self, par, lfpi: bool = False) -> float:
        """src/brough_mod.f90 (lprior = .false.): Re(R p . conj(p)), or
        Im(R p) . Im(p) in the final phase improvement."""
        if self.cfg.ltri == 0:
            sm = self.smatm
            M, nx = self.manz, self.cfg.nx
            rp = sm[:, 0] * par
            rp[1:] += sm[:-1, 1] * par[:-1]
            rp[:-1] += sm[:-1, 1] * par[1:]
            rp[nx:] += sm[:-nx, 2] * par[:-nx]
            rp[:-nx] += sm[:-nx, 2] * par[nx:]
            _ = M
        else:
            n = self.nachbar.shape[1] - 1
            rp = np.zeros_like(par)
            for j in range(n):
                nb = self.nachbar[:, j]
                has = nb > 0
                rp[has] += self.smatm[has, j] * par[nb[has] - 1]
            rp += self.smatm[:, n] * par
        if lfpi:
            return float(np.sum(rp.imag * par.imag))
        return float(np.sum((rp * np.conj(par)).real))

    def _start(self):
        """Forward at the starting model, the set-up polarity check, misfit
        and Jacobian (src/inv.f90:426-519, :739-743).  Runs once per
        Inversion: the polarity check edits the data it keeps."""
        if getattr(self, "_started", False):
            raise RuntimeError("the starting pass of this Inversion has already run")
        self._started = True
        sig0 = self.start_model()
        ldc = self.cfg.ldc
        volt, sa0 = self.ctx.forward(sig0, ldc=ldc, mode=0)
        # set-up polarity check (inv.f90:510-519): corrected data / response,
        # swapped potential electrodes and excluded readings
        d = self.data
        dat, sa0, vnr, wdfak = chkpol(d.dat, sa0, d.vnr, lsetup=True)
        self.data = dataclasses.replace(d, dat=dat, vnr=vnr, wdfak=wdfak)
        self.ctx.set_data(dat, d.wmatd, wdfak)
        nrmsd0 = self.misfit(sa0)[0]
        # J / V is unchanged by the simultaneous swap of P1/P2 and sign of V,
        # so the Jacobian of this forward pass is used as is
        self.ctx.jacobian(mode=1 if ldc else 0, copy=False)
        if np.any(vnr != d.vnr):
            self.ctx.set_configs(d.strnr, vnr)
        return sig0, sa0, nrmsd0

    def trial_lambdas(self, lams, eps: float = 1e-4, ncgmax: Optional[int] = None, step: float = 1.0,
                      precond: int = 0):
        """The lambda trials of src/inv.f90:769-912 for the first update, side
        by side: after the starting pass, one crt_update_lambdas call gives
        every candidate's model (1 .. 8 lambdas, one read of J per CG
        iteration for all), and each model is forwarded for the misfit and
        roughness the reference's lambda logic compares."""
        sig0, sa0, nrmsd0 = self._start()
        ldc = self.cfg.ldc
        lam_ = np.asarray(lams, np.float64)
        prm = Context.params(0.0, eps=eps, ncgmax=ncgmax or self.ncgmax, ldc=ldc, step=step, precond=precond)
        par = np.log(sig0)
        up = self.ctx.update_lambdas(prm, lam_, par, sigmaa=sa0)
        trials = []
        for b, lam in enumerate(lam_):
            p = up["par"][b]
            _, sa = self.ctx.forward(np.exp(p), ldc=ldc, mode=0)
            trials.append(dict(lam=float(lam), ncg=int(up["ncg"][b]), bdpar=float(up["bdpar"][b]),
                               nrmsd=self.misfit(sa)[0], rough=self.roughness(p), par=p, sigmaa=sa))
        return dict(nrmsd0=nrmsd0, sigmaa0=sa0, trials=trials)

    def first_step(self, eps: float = 1e-4, ncgmax: Optional[int] = None, step: float = 1.0):
        """IT 0 and the first UP row of inv.ctr: forward at the starting
        model, misfit, Jacobian, lam0, update, forward at the new model."""
        if self.lam0 is None:
            raise NotImplementedError("lam0 from blam0's Jacobian estimate is not wired up yet")
        sig0, sa0, nrmsd0 = self._start()
        ldc = self.cfg.ldc
        prm = Context.params(self.lam0, eps=eps, ncgmax=ncgmax or self.ncgmax, ldc=ldc, step=step)
        par = np.log(sig0)
        up = self.ctx.update(prm, par, sigmaa=sa0)
        par1 = up["par"]
        rough = self.roughness(par1)
        sig1 = np.exp(par1)
        _, sa1 = self.ctx.forward(sig1, ldc=ldc, mode=0)
        nrmsd1 = self.misfit(sa1)[0]
        return dict(nrmsd0=nrmsd0, nrmsd1=nrmsd1, bdpar=up["bdpar"], rough=rough, ncg=up["ncg"],
                    cgres=up["cgres"], lam=self.lam0, par=par1, sigmaa0=sa0, sigmaa1=sa1)

    # -- the whole Gauss-Newton loop ----------------------------------------
    # control constants of src/rall.f90:196-220
    NRMSDM, MQRMS, STPMIN, BDMIN, NLAM, FSTART, FSTOP = 1.0, 2e-2, 1e-3, 1e-3, 30, 0.5, 0.9

    def _polarity(self, sigmaa, setup: bool):
        """chkpol (src/chkpol.f90:43-128) on the current data: corrected data,
        swapped potential electrodes and excluded readings go to the device;
        returns the corrected response."""
        d = self.data
        dat, sa, vnr, wdfak = chkpol(d.dat, sigmaa, d.vnr, lsetup=setup)
        changed_v = np.any(vnr != d.vnr)
        self.data = dataclasses.replace(d, dat=dat, vnr=vnr, wdfak=wdfak)
        self.ctx.set_data(dat, self.data.wmatd, wdfak)
        if changed_v:
            self.ctx.set_configs(d.strnr, vnr)
        return sa

    def _misfit(self, sigmaa, lfpi: bool):
        """dmisft (src/dmisft.f90:75-125): every reading, each with its local
        phase correction (chkpo2)."""
        d = self.data
        return dmisft(d.dat, sigmaa, d.wmatd, d.wmatdr, d.wmatdp, lfpi=lfpi)

    def _lam0(self, lfpi: bool, lamnull_fpi: float) -> float:
        """blam0 (src/blam0.f90:45-167): the presets, else the Jacobian
        estimate on the device."""
        c = self.cfg
        if not lfpi and self.lam0 is not None:
            return self.lam0
        if (c.llamf & 1) or lamnull_fpi > np.finfo(float).eps:
            return float(lamnull_fpi)
        return self.ctx.blam0(c.alfx, c.alfz, ldc=c.ldc, lfpi=lfpi)

    def run(self, itmax: Optional[int] = None, eps: float = 1e-4, precond: int = 0, lamnull_fpi: float = 0.0,
            ncgmax: Optional[int] = None, out_dir: Optional[str] = None):
        """The Gauss-Newton loop of src/inv.f90:332-956 around the device
        calls: forward and bvolti at every trial model, chkpol and dmisft,
        the stop tests (:562-605), the final phase improvement (:606-684),
        the Jacobian at every accepted iterate (:702-745), the lambda search
        (:769-880: blam0 at the start of a stage, the multiplicative update
        by dlam, the step halving and parfit's parabolic step length,
        :880-912) and update / bsigma / brough (:914-944).  refsig
        (:949) only matters for singularity removal, which is not built.
        Returns the inv.ctr rows (kont2, src/kont2.f90) as dicts, the model
        of every accepted iterate (wout), the final model and response, and
        the stop code (the reference's errnr2: 79 iterations, 80 optimal
        RMS, 81 no CHI improvement, 92 repeated step length, 109 minimal
        update; 82 a zero voltage, the model reset to the last iterate).
        With out_dir, the files of an inversion directory are written as the
        reference writes them: rhoNN.* / voltNN.dat at every wout, and at
        the end coverage.mag (bbsens, from the last Jacobian) and the rows of
        inv.ctr."""
        c = self.cfg
        if c.lrobust:
            raise NotImplementedError("robust data weighting (lrobust) is outside the implemented path")
        itmax = c.itmax if itmax is None else itmax
        ncgmax = ncgmax or self.ncgmax
        ldc = c.ldc
        lfphai = c.lfphai and not ldc
        lffhom = c.stabp0 < 0
        rows, models, events = [], [], {}
        espx, espy = self.mesh.midpoints()
        betrms = pharms = 0.0

        def wout(it_, sig_, sa_):
            d = self.data
            models.append(dict(it=it_, sigma=sig_.copy(), sigmaa=sa_.copy(), betrms=betrms, pharms=pharms,
                               vnr=d.vnr.copy(), wdfak=d.wdfak.copy()))
            if out_dir:
                writers.write_model(out_dir, it_, espx, espy, sig_, betrms, pharms, ldc)
                writers.write_volt_iterate(out_dir, it_, d.strnr, d.vnr, sa_, d.wdfak, ldc)

        if out_dir:
            os.makedirs(out_dir, exist_ok=True)
        it = itr = 0
        lsetup, lsetip, lfpi, llam, ldlami, lstep, lfstep = True, False, False, False, True, False, False
        step, stpalt, alam = 1.0, 1.0, 0.0
        rmsalt, lamalt, bdpar, bdalt = 0.0, 1.0, 1.0, 1.0
        if c.llamf & 1:
            lamalt = c.lamfix
        lam, dlam, dlalt, ldlamf, rmsreg = 0.0, 1.0, 1.0, False, 0.0
        ncg, ncg2, rough = 0, 0, 0.0
        sigma = self.start_model()
        sigma2, sgmaa2 = sigma.copy(), None
        dpar = np.zeros(self.manz, np.complex128)
        dpar2 = dpar.copy()
        stop = 0
        while True:
            try:
                _, sigmaa = self.ctx.forward(sigma, ldc=ldc, mode=0)
            except CRTError as exc:    # bvolti: zero voltage -> back to the last iterate
                if exc.errnr != 82 or sgmaa2 is None:
                    raise
                sigma, sigmaa, stop = sigma2, sgmaa2, 82
                break
            if lsetup or lsetip:
                sigmaa = self._polarity(sigmaa, True)
            nrmsd, betrms, pharms, npol = self._misfit(sigmaa, lfpi)
            if nrmsd < 1e-12:
                nrmsd = self.NRMSDM * (1.0 - self.MQRMS)
            if it == 0 and not rows:
                wout(0, sigma, sigmaa)
            rows.append(self._kont2_row(lsetup or lsetip, llam and not lstep, lfpi, it, itr, nrmsd, bdpar, lam,
                                        rough, ncg, betrms, pharms, npol, step))
            if llam and not lstep:
                sigmaa = self._polarity(sigmaa, lsetup or lsetip)
                errnr2 = 0
                if stpalt == 0.0:
                    errnr2 = 92
                if abs(1.0 - rmsalt / nrmsd) <= self.MQRMS:
                    errnr2 = 81
                if abs(1.0 - nrmsd / self.NRMSDM) <= self.MQRMS and ldlamf:
                    errnr2 = 80
                if it >= itmax:
                    errnr2 = 79
                if abs(1.0 - _quot(bdpar, bdalt)) < self.BDMIN:
                    errnr2 = 109
                if errnr2:
                    if lfphai and errnr2 != 79:
                        # final phase improvement: phase weights, lambda search
                        # restarted, phase-only update
                        wout(it, sigma, sigmaa)
                        events.setdefault(len(rows), []).append("FPI")
                        self.data = dataclasses.replace(self.data, wmatd=self.data.wmatdp.copy())
                        self.ctx.set_data(self.data.dat, self.data.wmatd, self.data.wdfak)
                        lfpi, lsetip, lfphai, llam, ldlami, lfstep, step = True, True, False, False, True, True, 1.0
                        if lffhom:
                            a = np.abs(sigma)
                            sigma = a * complex(math.cos(c.pha0 / 1e3), -math.sin(c.pha0 / 1e3))
                            lsetup = True
                            events.setdefault(len(rows), []).append("RESET")
                            continue
                        lsetup = False
                        nrmsd, betrms, pharms, npol = self._misfit(sigmaa, lfpi)
                        rows.append(self._kont2_row(True, False, lfpi, it, itr, nrmsd, bdpar, lam, rough, ncg,
                                                    betrms, pharms, npol, step))
                    else:
                        stop = errnr2
                        break
                else:
                    lamalt = lam
                    wout(it, sigma, sigmaa)
            if (llam and not lstep) or lsetup or lsetip:
                it += 1
                itr, rmsreg, dlam, dlalt, ldlamf, bdpar, bdalt = 0, 0.0, 1.0, 1.0, False, 1.0, 1.0
                rmsalt = nrmsd
                if it > 1:
                    lamalt = lam
                sigma2, sgmaa2 = sigma.copy(), sigmaa.copy()
                self.ctx.jacobian(mode=1 if ldc else 0, copy=False)
            else:
                sigma, sigmaa = sigma2.copy(), sgmaa2.copy()
            if itmax == 0:
                stop = 109
                break
            if c.llamf & 1:
                lam = c.lamfix
                if (c.llamf & 2) and it > 1:
                    lam = c.lamfix / (2.0 * (it - 1))
                llam = False
                lsetup = lsetip = False
            elif not lstep:
                if llam:
                    llam, step = False, 1.0
                else:
                    itr += 1
                    lr = math.log(nrmsd / self.NRMSDM)
                    search = ((((nrmsd < rmsreg and itr <= self.NLAM) or (dlam > 1.0 and itr <= self.NLAM))
                               and (not ldlamf or dlalt <= 1.0) and abs(1.0 - _quot(bdpar, bdalt)) > self.BDMIN
                               and abs(1.0 - rmsreg / self.NRMSDM) > self.MQRMS) or rmsreg == 0.0)
                    if search:
                        if lsetup or lsetip:
                            lam = self._lam0(lfpi, lamnull_fpi)
                            lamalt = lam
                        else:
                            dlalt = dlam
                            if ldlami:
                                ldlami = False
                                alam = max(abs(lr), math.log(1.0 + self.MQRMS))
                                dlam = self.FSTART
                            else:
                                alam = max(alam, abs(lr))
                                dlam = math.exp(math.log(self.FSTOP) * math.copysign(1.0, lr)
                                                + math.log(self.FSTART / self.FSTOP) * lr / alam)
                            lam *= dlam
                            if dlalt > 1.0 and dlam < 1.0:
                                ldlamf = True
                    else:
                        # no CHI decrease: back to the last lambda, shorter step
                        llam = True
                        lam /= dlam
                        if lfstep:
                            lfstep = False
                        else:
                            lstep, step = True, 0.5
                    if lsetup or lsetip:
                        lsetup = lsetip = False
                    elif not lstep:
                        rmsreg = nrmsd
            else:
                lstep = False
                step = parfit(rmsalt, nrmsd, rmsreg, self.NRMSDM, self.STPMIN)
                stpalt = 0.0 if (step == self.STPMIN and stpalt == self.STPMIN) else step
            # bpar, update, bsigma, brough
            par = np.log(sigma)
            bdalt = bdpar
            if not llam:
                dpar2, ncg2 = dpar, ncg
                prm = Context.params(lam, eps=eps, ncgmax=ncgmax, ldc=ldc, lfpi=lfpi, step=step, precond=precond)
                up = self.ctx.update(prm, par, sigmaa=sigmaa)
                par, dpar, ncg, bdpar = up["par"], up["dpar"], up["ncg"], up["bdpar"]
            else:
                dpar, ncg = dpar2, ncg2
                par = par + step * dpar
                bdpar = float(np.sum(np.abs(dpar) ** 2)) * step
            sigma = np.exp(par)
            rough = self.roughness(par, lfpi)
            if c.llamf & 1:
                llam = True
        wout(it, sigma, sigmaa)            # the final wout (inv.f90:1026)
        if out_dir:
            self._write_coverage(os.path.join(out_dir, "coverage.mag"), lfpi, espx, espy)
            writers.write_inv_ctr_rows(os.path.join(out_dir, "inv.ctr"), rows, events)
        return dict(rows=rows, models=models, sigma=sigma, sigmaa=sigmaa, stop=stop, it=it, events=events)

    def _write_coverage(self, path: str, lfpi: bool, espx, espy):
        """bbsens (src/bbsens.f90) on the device-resident Jacobian: the
        weights of the current phase (lelerr: wmatd_cri, else wmatdr, in the
        final phase improvement; wmatd otherwise), |Re J| for the FPI file."""
        c, d = self.cfg, self.data
        lelerr = (not c.lfphai and not c.ldc) or bool(c.mswitch & (1 << 5))
        w, w_fpi = writers.bbsens_weights(d.wmatd, d.wmatdr, d.wmatd_cri, d.wdfak, lfpi, lelerr)
        cs = self.ctx.coverage(0, w)
        cs_fpi = self.ctx.coverage(1, w_fpi) if w_fpi is not None else None
        return writers.write_coverage(path, espx, espy, cs, cs_fpi)

    @staticmethod
    def _kont2_row(first, accepted, lfpi, it, itr, nrmsd, bdpar, lam, rough, ncg, betrms, pharms, npol, step):
        """One control row of inv.ctr (src/kont2.f90:63-128): IT / PIT rows of
        a starting pass or an accepted iterate, UP / PUP rows of the lambda
        and step-length trials."""
        p = "P" if lfpi else ""
        if first:
            return dict(kind=p + "IT", it=it, rms=nrmsd, betrms=betrms, pharms=pharms, npol=npol)
        if accepted:
            return dict(kind=p + "IT", it=it, rms=nrmsd, step=bdpar, lam=lam, rough=rough, ncg=ncg, betrms=betrms,
                        pharms=pharms, npol=npol, steplength=step)
        return dict(kind=p + "UP", it=itr, rms=nrmsd, step=bdpar, lam=lam, rough=rough, ncg=ncg, steplength=step)

    def close(self):
        self.ctx.close()


def parfit(fa: float, fb: float, fc: float, fmin: float, smin: float) -> float:
    """src/parfit.f90:38-186: the step length where the parabola through the
    misfits (0, fa), (0.5, fb), (1, fc) has its minimum, or where the misfit
    crosses fmin by linear interpolation, clamped to [smin, 1]."""
    a, b, c = 0.0, 0.5, 1.0

    def parab():
        num = (b - a) ** 2 * (fb - fc) - (b - c) ** 2 * (fb - fa)
        den = (b - a) * (fb - fc) - (b - c) * (fb - fa)
        return b - num / (2.0 * den)

    lin_ab = lambda: a + (b - a) * (fmin - fa) / (fb - fa)  # noqa: E731
    lin_bc = lambda: b + (c - b) * (fmin - fb) / (fc - fb)  # noqa: E731
    if fa > fb:
        if fb <= fc:
            if fb <= fmin:
                step = lin_bc() if (fa < fmin and fc > fa) else lin_ab()
            else:
                step = parab()
        else:
            step = lin_ab() if fb <= fmin else (lin_bc() if fc <= fmin else c)
    elif fa < fb:
        if fb >= fc:
            if fb >= fmin:
                step = lin_bc() if (fa > fmin and fc < fa) else lin_ab()
            else:
                step = parab()
        else:
            step = lin_ab() if fb >= fmin else (lin_bc() if fc >= fmin else c)
    else:
        if fb > fc:
            step = parab() if fb < fmin else (lin_bc() if fc <= fmin else c)
        elif fb < fc:
            step = parab() if fb > fmin else (lin_bc() if fc >= fmin else c)
        else:
            step = smin
    return min(c, max(smin, step))


def load_tomodir_inversion(exe_dir: str, device: int = 0) -> Inversion:
    """Set up an Inversion from a tomodir's exe/ directory (crtomo.cfg)."""
    cfg = read_crtomo_cfg(os.path.join(exe_dir, "crtomo.cfg"))
    mesh = io.read_elem(io.resolve(exe_dir, cfg.elem))
    enr = io.read_elec(io.resolve(exe_dir, cfg.elec))
    data = error_model(io.read_volt(io.resolve(exe_dir, cfg.volt)), cfg)
    return Inversion(mesh, enr, data, cfg, device=device)


def chkpol(dat: np.ndarray, sigmaa: np.ndarray, vnr: np.ndarray, lsetup: bool, lpol: bool = False):
    """Polarity check of src/chkpol.f90:43-128.  Returns corrected copies
    (dat, sigmaa, vnr, wdfak): readings whose model response and datum sit on
    opposite sides of +-pi/2 in phase get their potential electrodes swapped
    and, unless lpol, are excluded (wdfak = 0)."""
    pi = math.acos(-1.0)
    dat = np.array(dat, np.complex128)
    sigmaa = np.array(sigmaa, np.complex128)
    vnr = np.array(vnr, np.int32)
    wdfak = np.ones(len(dat), np.int32)
    for i in range(len(dat)):
        e3 = int(vnr[i]) % 10000
        e4 = (int(vnr[i]) - e3) // 10000
        redat, imdat = dat[i].real, dat[i].imag
        resig, imsig = sigmaa[i].real, sigmaa[i].imag
        idat = -1 if imdat > pi / 2 else (1 if imdat <= -pi / 2 else 0)
        isig = -1 if imsig > pi / 2 else (1 if imsig <= -pi / 2 else 0)
        if idat == 0 and isig != 0:
            vnr[i] = e3 * 10000 + e4
            sigmaa[i] = complex(resig, imsig + isig * pi)
            if lpol:
                if not lsetup:
                    wdfak[i] = 0
            else:
                dat[i] = complex(redat, imdat - math.copysign(pi, imdat))
                wdfak[i] = 0
        elif idat != 0 and isig == 0:
            if lpol:
                dat[i] = complex(redat, imdat + idat * pi)
                if not lsetup:
                    wdfak[i] = 0
            else:
                wdfak[i] = 0
        elif idat != 0 and isig != 0:
            vnr[i] = e3 * 10000 + e4
            sigmaa[i] = complex(resig, imsig + isig * pi)
            dat[i] = complex(redat, imdat + idat * pi)
    return dat, sigmaa, vnr, wdfak


def synthetic_inversion(s, device: int = 0, itmax: int = 20, precision: int = 0, noise=(0.03, 0.1),
                        seed: int = 20261203, bet0: float = 100.0, pha0: float = 0.0, ctx=None) -> Inversion:
    """A complex inversion of a synthetic survey (crtomo_stable_b200.synth):
    the 'observed' data are the true model's response with seeded Gaussian
    noise (relative magnitude noise[0], phase noise[1] mrad), the error model
    of src/rdati.f90 with the same levels (A1 = 100 noise[0] %, A3 =
    noise[1] mrad), the regular-grid smoothness regulariser of
    src/bsmatm_mod.f90:190-362 on quadrilateral grids (nx x nz elements, row
    by row) or the triangular one otherwise, lambda_0 from blam0's Jacobian
    estimate, a homogeneous start (bet0 Ohm m, pha0 mrad) and no final phase
    improvement.  ctx: a stand-in context (as for Inversion), default a
    new device Context."""
    if ctx is None:
        ctx = Context(s.mesh, s.enr, s.strnr, s.vnr, device=device, precision=precision)
    _, sa_true = ctx.forward(s.sigma)
    rng = np.random.default_rng(seed)
    bet = np.exp(-sa_true.real) * (1.0 + noise[0] * rng.standard_normal(len(sa_true)))
    pha = -1e3 * sa_true.imag + noise[1] * rng.standard_normal(len(sa_true))
    d = io.Data(np.asarray(s.strnr, np.int32), np.asarray(s.vnr, np.int32), np.abs(bet), pha)
    quads = int(s.mesh.typ[0]) == 8 and s.nx * s.nz == s.mesh.elanz
    cfg = CRTomoConfig(mswitch=0, elem="", elec="", volt="", ramd="", ldiff=False,
                       nx=s.nx if quads else 0, nz=s.nz if quads else 0, alfx=1.0, alfz=1.0, itmax=itmax,
                       ldc=False, lrobust=False, lfphai=False, stabw0=100.0 * noise[0], stabm0=0.0, stabpA1=0.0,
                       stabpB=0.0, stabpA2=0.0, stabp0=noise[1], lrho0=True, bet0=bet0, pha0=pha0,
                       lagain=False, swrtr=1, lsink=False, nsink=0, lrandb2=False, randb="",
                       ltri=0 if quads else 1)
    return Inversion(s.mesh, s.enr, error_model(d, cfg), cfg, ctx=ctx)
