"""ctypes binding of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The shipped package never
imports this module.

``OracleProblem`` wraps one forward / inversion problem in the reference's
module-array layout and exposes the restated routines (see crt_oracle.h for
the Fortran routine each one follows).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def build(fast_math: bool = False) -> str:
    lib = os.path.join(HERE, "liboracle_fm.so" if fast_math else "liboracle.so")
    src = os.path.join(HERE, "crt_oracle.c")
    if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)
    return lib


_LIBS = {}


def lib(fast_math: bool = False):
    if fast_math not in _LIBS:
        L = C.CDLL(build(fast_math))
        _declare(L)
        _LIBS[fast_math] = L
    return _LIBS[fast_math]


i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)


class orc_problem(C.Structure):
    _fields_ = [
        ("sanz", C.c_int32), ("typanz", C.c_int32), ("mb", C.c_int32),
        ("elanz", C.c_int32), ("relanz", C.c_int32), ("maxnodes", C.c_int32),
        ("typ", i32p), ("nelanz", i32p), ("selanz", i32p),
        ("snr", i32p), ("sx", f64p), ("sy", f64p),
        ("nrel", i32p), ("rnr", i32p),
        ("eanz", C.c_int32), ("enr", i32p),
        ("nanz", C.c_int32), ("strnr", i32p), ("vnr", i32p),
        ("kwnanz", C.c_int32), ("swrtr", C.c_int32), ("kwn", f64p), ("kwnwi", f64p),
        ("elbg", f64p), ("relbg", f64p), ("kg", f64p),
        ("lbeta", C.c_int32), ("lrandb", C.c_int32), ("lrandb2", C.c_int32),
        ("lsink", C.c_int32), ("nsink", C.c_int32),
        ("rwdanz", C.c_int32), ("rwdnr", i32p), ("rwd", C.c_void_p),
    ]


class orc_cg_params(C.Structure):
    _fields_ = [
        ("manz", C.c_int32), ("nanz", C.c_int32), ("ltri", C.c_int32), ("nx", C.c_int32),
        ("nnb", C.c_int32), ("ldc", C.c_int32), ("lfpi", C.c_int32), ("ncgmax", C.c_int32),
        ("lam", C.c_double), ("eps", C.c_double),
        ("smatm", f64p), ("nachbar", i32p), ("wmatd", f64p), ("wdfak", i32p),
    ]


def _declare(L):
    P = C.POINTER(orc_problem)
    vp = C.c_void_p
    L.orc_rwaven.argtypes = [P, i32p, f64p, f64p, f64p, f64p]
    L.orc_precal.argtypes = [P, C.c_int, f64p, f64p, f64p, i32p, i32p]
    L.orc_forward.argtypes = [P, vp, C.c_int, C.c_int, vp]
    L.orc_rtrafo.argtypes = [P, vp, vp]
    L.orc_rtrafo.restype = None
    L.orc_bvolti.argtypes = [P, vp, vp, vp]
    L.orc_bvolt.argtypes = [P, vp, vp, vp, vp]
    L.orc_bvolt.restype = None
    L.orc_bkfak.argtypes = [P, f64p]
    L.orc_bsensi.argtypes = [P, vp, vp, vp, C.c_int, vp]
    L.orc_bsensi.restype = None
    L.orc_bsendc.argtypes = [P, vp, vp, vp, C.c_int, vp]
    L.orc_bsendc.restype = None
    L.orc_bsens.argtypes = [P, vp, vp, C.c_int, vp]
    L.orc_bsens.restype = None
    L.orc_refsig.argtypes = [P, vp]
    L.orc_refsig.restype = C.c_double * 2
    L.orc_bnachbar.argtypes = [P, i32p]
    L.orc_bnachbar.restype = None
    L.orc_esp.argtypes = [P, f64p, f64p]
    L.orc_esp.restype = None
    L.orc_bsmatmtri.argtypes = [P, i32p, f64p, f64p, C.c_double, C.c_double, f64p]
    L.orc_bsmatmtri.restype = None
    L.orc_bsmatmreg.argtypes = [P, C.c_int, C.c_int, C.c_double, C.c_double, f64p]
    L.orc_bsmatmreg.restype = None
    CP = C.POINTER(orc_cg_params)
    L.orc_update.argtypes = [CP, vp, vp, vp, vp, C.c_double, vp, vp, f64p, vp, f64p, i32p, f64p]
    L.orc_update.restype = None
    L.orc_cjggra.argtypes = [CP, vp, f64p, vp, vp, f64p, i32p]
    L.orc_cjggra.restype = None
    L.orc_brough.argtypes = [CP, vp]
    L.orc_brough.restype = C.c_double
    L.orc_dmisft.argtypes = [C.c_int, vp, vp, f64p, f64p, f64p, C.c_int, C.c_int, f64p, f64p, i32p]
    L.orc_dmisft.restype = C.c_double
    L.orc_blam0.argtypes = [CP, vp, vp, C.c_double, C.c_double]
    L.orc_blam0.restype = C.c_double
    L.orc_parfit.argtypes = [C.c_double] * 5
    L.orc_parfit.restype = C.c_double
    L.orc_bessk0.argtypes = [C.c_double]
    L.orc_bessk0.restype = C.c_double
    L.orc_bessk1.argtypes = [C.c_double]
    L.orc_bessk1.restype = C.c_double
    L.orc_kompab.argtypes = [P, C.c_int, C.c_int, vp, vp, vp]
    L.orc_scalab.argtypes = [P, vp, vp, f64p]
    L.orc_chol.argtypes = [P, vp]
    L.orc_vre.argtypes = [P, vp, vp, vp]
    L.orc_vre.restype = None


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _v(a):
    return C.c_void_p(a.ctypes.data)


class OracleProblem:
    """One problem in the reference's array layout.

    mesh: crtomo_stable_b200.io.Mesh (or anything with the same fields),
    enr: electrode node numbers, strnr/vnr: measurement configurations.
    """

    def __init__(self, mesh, enr, strnr, vnr, swrtr=1, lsink=False, nsink=0,
                 kwn=None, kwnwi=None, rwdnr=None, rwd=None, fast_math=False,
                 lsytop=False):
        self.L = lib(fast_math)
        self.mesh = mesh
        self.keep = []
        m = mesh
        self.typ = np.ascontiguousarray(m.typ, np.int32)
        self.nelanz = np.ascontiguousarray(m.nelanz, np.int32)
        self.selanz = np.ascontiguousarray(m.selanz, np.int32)
        self.snr = np.ascontiguousarray(m.snr, np.int32)
        self.sx = np.ascontiguousarray(m.sx, np.float64)
        self.sy = np.ascontiguousarray(m.sy, np.float64)
        self.nrel = np.asfortranarray(m.nrel, np.int32)
        self.rnr = np.ascontiguousarray(m.rnr if len(m.rnr) else np.zeros(1), np.int32)
        self.enr = np.ascontiguousarray(enr, np.int32)
        self.strnr = np.ascontiguousarray(strnr, np.int32)
        self.vnr = np.ascontiguousarray(vnr, np.int32)
        p = orc_problem()
        p.sanz, p.typanz, p.mb = m.sanz, m.typanz, m.mb
        p.elanz, p.relanz, p.maxnodes = m.elanz, m.relanz, m.maxnodes
        p.typ, p.nelanz, p.selanz = _p(self.typ, C.c_int32), _p(self.nelanz, C.c_int32), _p(self.selanz, C.c_int32)
        p.snr, p.sx, p.sy = _p(self.snr, C.c_int32), _p(self.sx, C.c_double), _p(self.sy, C.c_double)
        p.nrel, p.rnr = _p(self.nrel, C.c_int32), _p(self.rnr, C.c_int32)
        p.eanz, p.enr = len(self.enr), _p(self.enr, C.c_int32)
        p.nanz, p.strnr, p.vnr = len(self.strnr), _p(self.strnr, C.c_int32), _p(self.vnr, C.c_int32)
        p.swrtr = swrtr
        p.lsink, p.nsink = int(bool(lsink)), int(nsink)
        if rwdnr is not None and len(rwdnr):
            self.rwdnr = np.ascontiguousarray(rwdnr, np.int32)
            self.rwd = np.ascontiguousarray(rwd, np.complex128)
            p.lrandb2, p.rwdanz = 1, len(self.rwdnr)
            p.rwdnr, p.rwd = _p(self.rwdnr, C.c_int32), self.rwd.ctypes.data
        self.p = p
        # wavenumbers (src/rwaven.f90, or 2D: k = 0 in CRMod / 1e-6 in CRTomo)
        if kwn is None:
            if swrtr == 0:
                kwn, kwnwi = np.zeros(1), np.zeros(1)
            else:
                kw = np.zeros(30)
                ww = np.zeros(30)
                n = C.c_int32()
                amin, amax = C.c_double(), C.c_double()
                err = self.L.orc_rwaven(C.byref(p), C.byref(n), _p(kw, C.c_double), _p(ww, C.c_double),
                                        C.byref(amin), C.byref(amax))
                if err:
                    raise RuntimeError(f"rwaven errnr {err}")
                kwn, kwnwi = kw[: n.value].copy(), ww[: n.value].copy()
                self.amin, self.amax = amin.value, amax.value
        self.kwn = np.ascontiguousarray(kwn, np.float64)
        self.kwnwi = np.ascontiguousarray(kwnwi, np.float64)
        p.kwnanz, p.kwn, p.kwnwi = len(self.kwn), _p(self.kwn, C.c_double), _p(self.kwnwi, C.c_double)
        # precal
        nmn = m.maxnodes * (m.maxnodes + 1) // 2
        K, E, R, L_ = len(self.kwn), m.elanz, max(m.relanz, 1), len(self.enr)
        self.elbg = np.zeros(E * nmn * K)
        self.relbg = np.zeros(R * nmn)
        self.kg = np.zeros(R * L_ * K)
        lbeta, lrandb = C.c_int32(), C.c_int32()
        err = self.L.orc_precal(C.byref(p), int(lsytop), _p(self.elbg, C.c_double), _p(self.relbg, C.c_double),
                                _p(self.kg, C.c_double), C.byref(lbeta), C.byref(lrandb))
        if err:
            raise RuntimeError(f"precal errnr {err}")
        p.elbg, p.relbg, p.kg = _p(self.elbg, C.c_double), _p(self.relbg, C.c_double), _p(self.kg, C.c_double)
        p.lbeta, p.lrandb = lbeta.value, lrandb.value

    # -- forward ------------------------------------------------------------
    def forward(self, sigma, ldc=False, nthreads=1):
        """kpot(sanz, eanz, kwnanz) complex, Fortran order."""
        m = self.mesh
        sig = np.ascontiguousarray(sigma, np.complex128)
        kpot = np.zeros((m.sanz, len(self.enr), len(self.kwn)), np.complex128, order="F")
        err = self.L.orc_forward(C.byref(self.p), _v(sig), int(bool(ldc)), int(nthreads), _v(kpot))
        if err:
            raise RuntimeError(f"forward errnr {err}")
        return kpot

    def rtrafo(self, kpot):
        hpot = np.zeros((self.mesh.sanz, len(self.enr)), np.complex128, order="F")
        kp = np.asfortranarray(kpot, np.complex128)
        self.L.orc_rtrafo(C.byref(self.p), _v(kp), _v(hpot))
        return hpot

    def bvolti(self, hpot):
        n = len(self.strnr)
        volt = np.zeros(n, np.complex128)
        sa = np.zeros(n, np.complex128)
        hp = np.asfortranarray(hpot, np.complex128)
        err = self.L.orc_bvolti(C.byref(self.p), _v(hp), _v(volt), _v(sa))
        if err:
            raise RuntimeError(f"bvolti errnr {err}")
        return volt, sa

    def bvolt(self, hpot, kfak=None):
        n = len(self.strnr)
        volt = np.zeros(n, np.complex128)
        sa = np.zeros(n, np.complex128)
        hp = np.asfortranarray(hpot, np.complex128)
        kf = None if kfak is None else np.ascontiguousarray(kfak, np.float64)
        self.L.orc_bvolt(C.byref(self.p), _v(hp), None if kf is None else _v(kf), _v(volt), _v(sa))
        return volt, sa

    def bkfak(self):
        kf = np.zeros(len(self.strnr))
        err = self.L.orc_bkfak(C.byref(self.p), _p(kf, C.c_double))
        if err:
            raise RuntimeError(f"bkfak errnr {err}")
        return kf

    # -- sensitivities --------------------------------------------------------
    def bsensi(self, kpot, sigma, volt, nthreads=1):
        n, E = len(self.strnr), self.mesh.elanz
        sens = np.zeros((n, E), np.complex128, order="F")
        kp = np.asfortranarray(kpot, np.complex128)
        sg = np.ascontiguousarray(sigma, np.complex128)
        vt = np.ascontiguousarray(volt, np.complex128)
        self.L.orc_bsensi(C.byref(self.p), _v(kp), _v(sg), _v(vt), int(nthreads), _v(sens))
        return sens

    def bsendc(self, kpot, sigma, volt, nthreads=1):
        n, E = len(self.strnr), self.mesh.elanz
        sens = np.zeros((n, E), np.float64, order="F")
        kp = np.asfortranarray(kpot, np.complex128)
        sg = np.ascontiguousarray(sigma, np.complex128)
        vt = np.ascontiguousarray(volt, np.complex128)
        self.L.orc_bsendc(C.byref(self.p), _v(kp), _v(sg), _v(vt), int(nthreads), _v(sens))
        return sens

    def bsens(self, kpot, strom=None, nthreads=1):
        n, E = len(self.strnr), self.mesh.elanz
        sens = np.zeros((n, E), np.complex128, order="F")
        kp = np.asfortranarray(kpot, np.complex128)
        st = None if strom is None else np.ascontiguousarray(strom, np.float64)
        self.L.orc_bsens(C.byref(self.p), _v(kp), None if st is None else _v(st), int(nthreads), _v(sens))
        return sens

    def refsig(self, sigma):
        sg = np.ascontiguousarray(sigma, np.complex128)
        r = self.L.orc_refsig(C.byref(self.p), _v(sg))
        return complex(r[0], r[1])

    # -- regularisation -------------------------------------------------------
    def bnachbar(self):
        E, n = self.mesh.elanz, self.mesh.maxnodes
        nb = np.zeros((E, n + 1), np.int32, order="F")
        self.L.orc_bnachbar(C.byref(self.p), _p(nb, C.c_int32))
        return nb

    def esp(self):
        E = self.mesh.elanz
        ex, ey = np.zeros(E), np.zeros(E)
        self.L.orc_esp(C.byref(self.p), _p(ex, C.c_double), _p(ey, C.c_double))
        return ex, ey

    def bsmatmtri(self, nachbar, alfx, alfz):
        E, n = self.mesh.elanz, self.mesh.maxnodes
        ex, ey = self.esp()
        sm = np.zeros((E, n + 1), np.float64, order="F")
        nb = np.asfortranarray(nachbar, np.int32)
        self.L.orc_bsmatmtri(C.byref(self.p), _p(nb, C.c_int32), _p(ex, C.c_double), _p(ey, C.c_double),
                             float(alfx), float(alfz), _p(sm, C.c_double))
        return sm

    def bsmatmreg(self, nx, nz, alfx, alfz):
        sm = np.zeros((nx * nz, 3), np.float64, order="F")
        self.L.orc_bsmatmreg(C.byref(self.p), int(nx), int(nz), float(alfx), float(alfz), _p(sm, C.c_double))
        return sm


class OracleCG:
    """Inner-solve state (src/update.f90, src/cg_mod.f90)."""

    def __init__(self, manz, nanz, ltri, smatm, nachbar=None, nx=0, nnb=0, wmatd=None,
                 wdfak=None, lam=1.0, eps=1e-4, ncgmax=None, ldc=False, lfpi=False,
                 fast_math=False):
        self.L = lib(fast_math)
        self.smatm = np.asfortranarray(smatm, np.float64)
        self.nachbar = np.asfortranarray(nachbar if nachbar is not None else np.zeros((1, 1)), np.int32)
        self.wmatd = np.ascontiguousarray(wmatd, np.float64)
        self.wdfak = np.ascontiguousarray(wdfak if wdfak is not None else np.ones(nanz), np.int32)
        c = orc_cg_params()
        c.manz, c.nanz, c.ltri, c.nx, c.nnb = manz, nanz, ltri, nx, nnb
        c.ldc, c.lfpi = int(bool(ldc)), int(bool(lfpi))
        c.ncgmax = ncgmax if ncgmax is not None else (manz // 10 if ltri < 5 else manz)
        c.lam, c.eps = float(lam), float(eps)
        c.smatm, c.nachbar = _p(self.smatm, C.c_double), _p(self.nachbar, C.c_int32)
        c.wmatd, c.wdfak = _p(self.wmatd, C.c_double), _p(self.wdfak, C.c_int32)
        self.c = c

    def update(self, sens, dat, sigmaa, par, step=1.0, sensdc=None):
        manz = self.c.manz
        sens_ = np.asfortranarray(sens if sens is not None else np.zeros((1, 1)), np.complex128)
        sdc = np.asfortranarray(sensdc if sensdc is not None else np.zeros((1, 1)), np.float64)
        dat_ = np.ascontiguousarray(dat, np.complex128)
        sa = np.ascontiguousarray(sigmaa, np.complex128)
        par_ = np.array(par, np.complex128)
        dpar = np.zeros(manz, np.complex128)
        cgfac = np.zeros(manz)
        rhs = np.zeros(manz, np.complex128)
        cgres = np.zeros(self.c.ncgmax + 2)
        ncg = C.c_int32()
        bdpar = C.c_double()
        self.L.orc_update(C.byref(self.c), _v(sens_), _v(sdc), _v(dat_), _v(sa), float(step), _v(par_),
                          _v(dpar), _p(cgfac, C.c_double), _v(rhs), _p(cgres, C.c_double), C.byref(ncg),
                          C.byref(bdpar))
        return dict(par=par_, dpar=dpar, cgfac=cgfac, rhs=rhs, cgres=cgres[: ncg.value + 1],
                    ncg=ncg.value, bdpar=bdpar.value)

    def cjggra(self, sens, cgfac, rhs):
        manz = self.c.manz
        sens_ = np.asfortranarray(sens, np.complex128)
        bvec = np.array(rhs, np.complex128)
        dpar = np.zeros(manz, np.complex128)
        cgres = np.zeros(self.c.ncgmax + 2)
        ncg = C.c_int32()
        cg = np.ascontiguousarray(cgfac, np.float64)
        self.L.orc_cjggra(C.byref(self.c), _v(sens_), _p(cg, C.c_double), _v(bvec), _v(dpar),
                          _p(cgres, C.c_double), C.byref(ncg))
        return dpar, cgres[: ncg.value + 1], ncg.value

    def blam0(self, sens=None, sensdc=None, alfx=1.0, alfz=1.0):
        """lambda_0 of src/blam0.f90:131-167 from the Jacobian."""
        s_ = np.asfortranarray(sens if sens is not None else np.zeros((1, 1)), np.complex128)
        d_ = np.asfortranarray(sensdc if sensdc is not None else np.zeros((1, 1)), np.float64)
        return self.L.orc_blam0(C.byref(self.c), _v(s_), _v(d_), float(alfx), float(alfz))

    def brough(self, par):
        p = np.ascontiguousarray(par, np.complex128)
        return self.L.orc_brough(C.byref(self.c), _v(p))


def dmisft(dat, sigmaa, wmatd, wmatdr=None, wmatdp=None, lfpi=False, lpol=False):
    L = lib()
    d = np.ascontiguousarray(dat, np.complex128)
    s = np.ascontiguousarray(sigmaa, np.complex128)
    w = np.ascontiguousarray(wmatd, np.float64)
    wr = None if wmatdr is None else np.ascontiguousarray(wmatdr, np.float64)
    wp = None if wmatdp is None else np.ascontiguousarray(wmatdp, np.float64)
    br, ph = C.c_double(), C.c_double()
    npol = C.c_int32()
    r = L.orc_dmisft(len(d), _v(d), _v(s), _p(w, C.c_double),
                     None if wr is None else _p(wr, C.c_double), None if wp is None else _p(wp, C.c_double),
                     int(lfpi), int(lpol), C.byref(br), C.byref(ph), C.byref(npol))
    return r, br.value, ph.value, npol.value


def parfit(fa, fb, fc, fmin=1.0, smin=1e-3):
    """src/parfit.f90:38-186."""
    return lib().orc_parfit(float(fa), float(fb), float(fc), float(fmin), float(smin))
