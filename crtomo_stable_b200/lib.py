"""ctypes binding of libcrt_b200.so (the C ABI declared in include/crt_b200.h).

Loading fails loudly: there is no CPU fallback for any of the entry points
that compute on the device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcrt_b200.so")

i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)

ERRNR_TEXT = {
    0: "ok", 3: "inconsistent input", 18: "unknown element type", 19: "band width violated (kompab)",
    26: "element orientation (elem3/elem8)", 27: "zero diagonal (scalab)", 28: "non-positive pivot (chol)",
    29: "electrode node > sanz", 35: "degenerate boundary segment (beta)", 46: "electrode number out of range",
    73: "duplicate electrodes (rwaven)", 82: "zero voltage (bvolti)", 89: "regular grid needs nx, nz",
    93: "zero geometric factor (bkfak)", 97: "allocation problem", 101: "mixed and Dirichlet boundaries",
    111: "border to element context", 200: "CUDA runtime failure", 201: "option not implemented",
}


class CRTError(RuntimeError):
    def __init__(self, errnr: int, msg: str = ""):
        self.errnr = int(errnr)
        super().__init__(f"errnr {errnr} ({ERRNR_TEXT.get(int(errnr), '?')}): {msg}")


class crt_mesh(C.Structure):
    _fields_ = [
        ("sanz", C.c_int32), ("typanz", C.c_int32), ("mb", C.c_int32),
        ("typ", i32p), ("nelanz", i32p), ("selanz", i32p),
        ("snr", i32p), ("sx", f64p), ("sy", f64p),
        ("nrel", i32p), ("rnr", i32p),
    ]


class crt_survey(C.Structure):
    _fields_ = [
        ("eanz", C.c_int32), ("enr", i32p),
        ("nanz", C.c_int32), ("strnr", i32p), ("vnr", i32p),
        ("kwnanz", C.c_int32), ("swrtr", C.c_int32), ("kwn", f64p), ("kwnwi", f64p),
        ("elbg", f64p), ("relbg", f64p), ("kg", f64p),
        ("lsink", C.c_int32), ("nsink", C.c_int32),
        ("rwdanz", C.c_int32), ("rwdnr", i32p), ("rwd", f64p),
        ("lsytop", C.c_int32),
    ]


class crt_cg_params(C.Structure):
    _fields_ = [
        ("lam", C.c_double), ("eps", C.c_double), ("ncgmax", C.c_int32),
        ("ldc", C.c_int32), ("lfpi", C.c_int32), ("step", C.c_double),
        ("precond", C.c_int32),
    ]


EXPORTS = [
    "crt_abi_version", "crt_create", "crt_destroy", "crt_last_error", "crt_rwaven", "crt_precal",
    "crt_forward", "crt_potentials", "crt_jacobian", "crt_set_jacobian", "crt_set_regularizer",
    "crt_set_data", "crt_set_configs", "crt_update", "crt_update_lambdas", "crt_gn_step", "crt_set_model", "crt_gn_step_device",
    "crt_get_model", "crt_model_backup", "crt_last_timings", "crt_launch_count", "crt_dmisft",
    "crt_voltages_noalloc", "crt_cg_info", "crt_rcm_order", "crt_last_timings_ex",
    "crt_set_refinement", "crt_set_refinement_tol", "crt_gnn_nparam", "crt_gnn_status", "crt_gnn_init", "crt_gnn_set_weights", "crt_gnn_get_weights", "crt_gnn_collect",
    "crt_gnn_clear", "crt_gnn_train", "crt_gnn_record", "crt_gnn_record_grad", "crt_batch_create",
    "crt_batch_destroy", "crt_batch_error", "crt_batch_set_models", "crt_batch_run", "crt_batch_status",
    "crt_batch_results", "crt_set_workspace_limit", "crt_set_forward_form", "crt_forward_info", "crt_blam0",
    "crt_coverage",
]

_LIB = None


def load(path: str = LIB_PATH):
    """Load (and on first use build) the CUDA library."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        from . import build as _b
        _b.build()
    L = C.CDLL(path)
    vp = C.c_void_p
    P = C.POINTER
    L.crt_abi_version.restype = C.c_int32
    L.crt_create.argtypes = [C.c_int32, P(crt_mesh), P(crt_survey), C.c_int32, i32p]
    L.crt_create.restype = vp
    L.crt_destroy.argtypes = [vp]
    L.crt_destroy.restype = None
    L.crt_last_error.argtypes = [vp]
    L.crt_last_error.restype = C.c_char_p
    L.crt_rwaven.argtypes = [P(crt_mesh), C.c_int32, i32p, C.c_int32, i32p, i32p, i32p, f64p, f64p]
    L.crt_rwaven.restype = C.c_int32
    L.crt_precal.argtypes = [vp, f64p, f64p, f64p, i32p, i32p]
    L.crt_precal.restype = C.c_int32
    L.crt_forward.argtypes = [vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp]
    L.crt_forward.restype = C.c_int32
    L.crt_potentials.argtypes = [vp, vp]
    L.crt_potentials.restype = C.c_int32
    L.crt_jacobian.argtypes = [vp, C.c_int32, vp, vp]
    L.crt_jacobian.restype = C.c_int32
    L.crt_set_jacobian.argtypes = [vp, C.c_int32, vp]
    L.crt_set_jacobian.restype = C.c_int32
    L.crt_set_regularizer.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp]
    L.crt_set_regularizer.restype = C.c_int32
    L.crt_set_configs.argtypes = [vp, i32p, i32p]
    L.crt_set_configs.restype = C.c_int32
    L.crt_set_data.argtypes = [vp, vp, vp, vp]
    L.crt_set_data.restype = C.c_int32
    L.crt_update.argtypes = [vp, P(crt_cg_params), vp, vp, vp, vp, vp, i32p, f64p]
    L.crt_update.restype = C.c_int32
    L.crt_update_lambdas.argtypes = [vp, P(crt_cg_params), C.c_int32, f64p, vp, vp, vp, vp, i32p, f64p]
    L.crt_update_lambdas.restype = C.c_int32
    L.crt_gn_step.argtypes = [vp, P(crt_cg_params), vp, vp, vp, i32p, f64p]
    L.crt_gn_step.restype = C.c_int32
    L.crt_set_model.argtypes = [vp, vp]
    L.crt_set_model.restype = C.c_int32
    L.crt_get_model.argtypes = [vp, vp]
    L.crt_get_model.restype = C.c_int32
    L.crt_model_backup.argtypes = [vp, C.c_int32]
    L.crt_model_backup.restype = C.c_int32
    L.crt_gn_step_device.argtypes = [vp, P(crt_cg_params), i32p]
    L.crt_gn_step_device.restype = C.c_int32
    L.crt_last_timings.argtypes = [vp, f64p]
    L.crt_last_timings.restype = C.c_int32
    L.crt_set_refinement.argtypes = [vp, C.c_int32]
    L.crt_set_refinement.restype = C.c_int32
    L.crt_set_refinement_tol.argtypes = [vp, C.c_double]
    L.crt_set_refinement_tol.restype = C.c_int32
    L.crt_batch_create.argtypes = [P(vp), C.c_int32, C.c_int32, C.c_int32, i32p]
    L.crt_batch_create.restype = vp
    L.crt_batch_destroy.argtypes = [vp]
    L.crt_batch_destroy.restype = None
    L.crt_batch_error.argtypes = [vp]
    L.crt_batch_error.restype = C.c_char_p
    L.crt_batch_set_models.argtypes = [vp, P(vp)]
    L.crt_batch_set_models.restype = C.c_int32
    L.crt_batch_run.argtypes = [vp, P(C.c_double)]
    L.crt_batch_run.restype = C.c_int32
    L.crt_batch_status.argtypes = [vp, C.c_int32]
    L.crt_batch_status.restype = C.c_int32
    L.crt_batch_results.argtypes = [vp, C.c_int32, vp, vp, vp]
    L.crt_batch_results.restype = C.c_int32
    L.crt_set_workspace_limit.argtypes = [vp, C.c_int64]
    L.crt_set_workspace_limit.restype = C.c_int32
    L.crt_blam0.argtypes = [vp, C.c_int32, C.c_int32, C.c_double, C.c_double, f64p]
    L.crt_blam0.restype = C.c_int32
    L.crt_coverage.argtypes = [vp, C.c_int32, vp, vp]
    L.crt_coverage.restype = C.c_int32
    L.crt_set_forward_form.argtypes = [vp, C.c_int32]
    L.crt_set_forward_form.restype = C.c_int32
    L.crt_forward_info.argtypes = [vp, i32p, i32p, i32p, i32p]
    L.crt_forward_info.restype = C.c_int32
    L.crt_last_timings_ex.argtypes = [vp, f64p, C.c_int32]
    L.crt_last_timings_ex.restype = C.c_int32
    L.crt_cg_info.argtypes = [vp, i32p, i32p, i32p]
    L.crt_cg_info.restype = C.c_int32
    L.crt_rcm_order.argtypes = [C.c_int32, i32p, i32p, i32p, i32p]
    L.crt_rcm_order.restype = C.c_int32
    f32p = P(C.c_float)
    L.crt_gnn_nparam.restype = C.c_int32
    L.crt_gnn_status.argtypes = [vp, i32p, i32p, i32p, i32p, i32p]
    L.crt_gnn_status.restype = C.c_int32
    L.crt_gnn_init.argtypes = [vp, C.c_uint64]
    L.crt_gnn_set_weights.argtypes = [vp, f32p, C.c_int32, C.c_int32]
    L.crt_gnn_get_weights.argtypes = [vp, f32p, C.c_int32, i32p]
    L.crt_gnn_collect.argtypes = [vp, P(crt_cg_params), C.c_int32, C.c_int32, C.c_int32, i32p]
    L.crt_gnn_clear.argtypes = [vp]
    L.crt_gnn_train.argtypes = [vp, C.c_int32, C.c_int32, C.c_float, C.c_uint64, f32p]
    L.crt_gnn_record.argtypes = [vp, C.c_int32, f32p, f32p, f32p, i32p, f32p]
    L.crt_gnn_record_grad.argtypes = [vp, C.c_int32, f32p, f64p]
    for nm in ("crt_gnn_init", "crt_gnn_set_weights", "crt_gnn_get_weights", "crt_gnn_collect", "crt_gnn_clear",
               "crt_gnn_train", "crt_gnn_record", "crt_gnn_record_grad"):
        getattr(L, nm).restype = C.c_int32
    L.crt_launch_count.argtypes = [vp]
    L.crt_launch_count.restype = C.c_int64
    L.crt_dmisft.argtypes = [C.c_int32, vp, vp, vp, vp, vp, C.c_int32, C.c_int32, f64p, f64p, i32p]
    L.crt_dmisft.restype = C.c_double
    L.crt_voltages_noalloc.argtypes = [vp, vp, vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                       C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp]
    L.crt_voltages_noalloc.restype = C.c_int32
    _LIB = L
    return L


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def _vp(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def rwaven(mesh, enr, strnr, vnr):
    """Wavenumbers and weights (src/rwaven.f90) through the C ABI."""
    L = load()
    keep = []
    m = _mesh_struct(mesh, keep)
    enr = np.ascontiguousarray(enr, np.int32)
    s = np.ascontiguousarray(strnr, np.int32)
    v = np.ascontiguousarray(vnr, np.int32)
    kwn = np.zeros(30)
    kwnwi = np.zeros(30)
    n = C.c_int32()
    e = L.crt_rwaven(C.byref(m), len(enr), _ptr(enr, C.c_int32), len(s), _ptr(s, C.c_int32),
                     _ptr(v, C.c_int32), C.byref(n), _ptr(kwn, C.c_double), _ptr(kwnwi, C.c_double))
    if e:
        raise CRTError(e, "rwaven")
    return kwn[: n.value].copy(), kwnwi[: n.value].copy()


def rcm_order(xadj, adj):
    """Reverse Cuthill-McKee ordering of a CSR graph through the C ABI:
    (order, bandwidth); order[k] is the vertex at position k."""
    L = load()
    xadj = np.ascontiguousarray(xadj, np.int32)
    adj = np.ascontiguousarray(adj, np.int32)
    n = len(xadj) - 1
    order = np.zeros(n, np.int32)
    bw = C.c_int32()
    e = L.crt_rcm_order(n, _ptr(xadj, C.c_int32), _ptr(adj, C.c_int32), _ptr(order, C.c_int32), C.byref(bw))
    if e:
        raise CRTError(e, "rcm_order")
    return order, bw.value


def _mesh_struct(mesh, keep):
    arrs = dict(
        typ=np.ascontiguousarray(mesh.typ, np.int32),
        nelanz=np.ascontiguousarray(mesh.nelanz, np.int32),
        selanz=np.ascontiguousarray(mesh.selanz, np.int32),
        snr=np.ascontiguousarray(mesh.snr, np.int32),
        sx=np.ascontiguousarray(mesh.sx, np.float64),
        sy=np.ascontiguousarray(mesh.sy, np.float64),
        nrel=np.asfortranarray(mesh.nrel, np.int32),
        rnr=np.ascontiguousarray(mesh.rnr if len(mesh.rnr) else np.zeros(1), np.int32),
    )
    keep.append(arrs)
    m = crt_mesh()
    m.sanz, m.typanz, m.mb = int(mesh.sanz), int(mesh.typanz), int(mesh.mb)
    for k in ("typ", "nelanz", "selanz", "snr", "nrel", "rnr"):
        setattr(m, k, _ptr(arrs[k], C.c_int32))
    m.sx = _ptr(arrs["sx"], C.c_double)
    m.sy = _ptr(arrs["sy"], C.c_double)
    return m


PREC_FP64 = 0
PREC_MIXED = 1
PRECOND_JACOBI = 0
PRECOND_BLOCK = 1
PRECOND_GNN = 2
PRECOND_BLOCK_GNN = 3
FORWARD_AUTO = 0
FORWARD_DIRECT = 1
FORWARD_SCHUR = 2


class Context:
    """One device context: a mesh, its electrodes, measurements and
    wavenumbers (the state the Fortran modules hold across calls).
    """

    def __init__(self, mesh, enr, strnr, vnr, kwn=None, kwnwi=None, swrtr=1, lsink=False, nsink=0,
                 rwdnr=None, rwd=None, device=0, elbg=None, relbg=None, kg=None, lsytop=False, precision=0):
        self.L = load()
        self._keep = []
        self.mesh = mesh
        self.enr = np.ascontiguousarray(enr, np.int32)
        self.strnr = np.ascontiguousarray(strnr, np.int32)
        self.vnr = np.ascontiguousarray(vnr, np.int32)
        if kwn is None:
            if swrtr == 0:
                kwn, kwnwi = np.zeros(1), np.zeros(1)
            else:
                kwn, kwnwi = rwaven(mesh, self.enr, self.strnr, self.vnr)
        self.kwn = np.ascontiguousarray(kwn, np.float64)
        self.kwnwi = np.ascontiguousarray(kwnwi, np.float64)
        self.swrtr = swrtr
        m = _mesh_struct(mesh, self._keep)
        s = crt_survey()
        s.eanz, s.enr = len(self.enr), _ptr(self.enr, C.c_int32)
        s.nanz, s.strnr, s.vnr = len(self.strnr), _ptr(self.strnr, C.c_int32), _ptr(self.vnr, C.c_int32)
        s.kwnanz, s.swrtr = len(self.kwn), int(swrtr)
        s.kwn, s.kwnwi = _ptr(self.kwn, C.c_double), _ptr(self.kwnwi, C.c_double)
        if elbg is not None:
            self._pre = [np.asfortranarray(elbg, np.float64), np.asfortranarray(relbg, np.float64),
                         np.asfortranarray(kg, np.float64)]
            s.elbg, s.relbg, s.kg = (_ptr(a, C.c_double) for a in self._pre)
        s.lsink, s.nsink = int(bool(lsink)), int(nsink)
        if rwdnr is not None and len(rwdnr):
            self._rw = [np.ascontiguousarray(rwdnr, np.int32), np.ascontiguousarray(rwd, np.complex128)]
            s.rwdanz, s.rwdnr = len(self._rw[0]), _ptr(self._rw[0], C.c_int32)
            s.rwd = C.cast(C.c_void_p(self._rw[1].ctypes.data), f64p)
        s.lsytop = int(bool(lsytop))
        err = C.c_int32()
        h = self.L.crt_create(int(device), C.byref(m), C.byref(s), int(precision), C.byref(err))
        if not h:
            raise CRTError(err.value, "crt_create failed")
        self.h = C.c_void_p(h)
        self.nanz = len(self.strnr)
        self.elanz = mesh.elanz

    def close(self):
        if getattr(self, "h", None):
            self.L.crt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, e, what):
        if e:
            raise CRTError(e, f"{what}: {self.L.crt_last_error(self.h).decode(errors='replace')}")

    # -- set-up -------------------------------------------------------------
    def precal(self):
        """elbg(elanz, nmn, K), relbg(relanz, nmn), kg(relanz, eanz, K) and
        lbeta / lrandb, computed on the device."""
        m = self.mesh
        nmn = m.maxnodes * (m.maxnodes + 1) // 2
        K, E, R, Le = len(self.kwn), m.elanz, max(m.relanz, 1), len(self.enr)
        elbg = np.zeros((E, nmn, K), order="F")
        relbg = np.zeros((R, nmn), order="F")
        kg = np.zeros((R, Le, K), order="F")
        lb, lr = C.c_int32(), C.c_int32()
        self._check(self.L.crt_precal(self.h, _ptr(elbg, C.c_double), _ptr(relbg, C.c_double),
                                      _ptr(kg, C.c_double), C.byref(lb), C.byref(lr)), "crt_precal")
        return elbg, relbg, kg, lb.value, lr.value

    # -- forward ------------------------------------------------------------
    def forward(self, sigma, ldc=False, mode=0, kfak=None, want_kpot=False):
        """Returns (volt, sigmaa[, kpot]) -- bvolti (mode 0) or bvolt (mode 1)."""
        sig = np.ascontiguousarray(sigma, np.complex128)
        volt = np.zeros(self.nanz, np.complex128)
        sa = np.zeros(self.nanz, np.complex128)
        kp = None
        if want_kpot:
            kp = np.zeros((self.mesh.sanz, len(self.enr), len(self.kwn)), np.complex128, order="F")
        kf = None if kfak is None else np.ascontiguousarray(kfak, np.float64)
        self._check(self.L.crt_forward(self.h, _vp(sig), int(bool(ldc)), int(mode), _vp(kf), _vp(volt),
                                       _vp(sa), _vp(kp)), "crt_forward")
        return (volt, sa, kp) if want_kpot else (volt, sa)

    def potentials(self):
        hp = np.zeros((self.mesh.sanz, len(self.enr)), np.complex128, order="F")
        self._check(self.L.crt_potentials(self.h, _vp(hp)), "crt_potentials")
        return hp

    def jacobian(self, mode=0, strom=None, copy=True):
        st = None if strom is None else np.ascontiguousarray(strom, np.float64)
        out = None
        if copy:
            dt = np.float64 if mode == 1 else np.complex128
            out = np.zeros((self.nanz, self.elanz), dt, order="F")
        self._check(self.L.crt_jacobian(self.h, int(mode), _vp(st), _vp(out)), "crt_jacobian")
        return out

    def set_jacobian(self, sens, real=False):
        a = np.asfortranarray(sens, np.float64 if real else np.complex128)
        self._check(self.L.crt_set_jacobian(self.h, int(bool(real)), _vp(a)), "crt_set_jacobian")

    # -- inversion ----------------------------------------------------------
    def set_regularizer(self, ltri, smatm, nachbar=None, nx=0):
        sm = np.asfortranarray(smatm, np.float64)
        nb = None if nachbar is None else np.asfortranarray(nachbar, np.int32)
        nnb = 0 if nachbar is None else nb.shape[1] - 1
        self._reg = (sm, nb)
        self._check(self.L.crt_set_regularizer(self.h, int(ltri), int(nx), int(nnb), _vp(sm), _vp(nb)),
                    "crt_set_regularizer")

    def set_configs(self, strnr, vnr):
        s = np.ascontiguousarray(strnr, np.int32)
        v = np.ascontiguousarray(vnr, np.int32)
        self._check(self.L.crt_set_configs(self.h, _ptr(s, C.c_int32), _ptr(v, C.c_int32)), "crt_set_configs")
        self.strnr, self.vnr = s, v

    def set_data(self, dat, wmatd, wdfak=None):
        d = np.ascontiguousarray(dat, np.complex128)
        w = np.ascontiguousarray(wmatd, np.float64)
        wf = None if wdfak is None else np.ascontiguousarray(wdfak, np.int32)
        self._check(self.L.crt_set_data(self.h, _vp(d), _vp(w), _vp(wf)), "crt_set_data")

    @staticmethod
    def params(lam, eps=1e-4, ncgmax=100, ldc=False, lfpi=False, step=1.0, precond=0):
        p = crt_cg_params()
        p.lam, p.eps, p.ncgmax = float(lam), float(eps), int(ncgmax)
        p.ldc, p.lfpi, p.step = int(bool(ldc)), int(bool(lfpi)), float(step)
        p.precond = int(precond)
        return p

    def update(self, prm, par, sigmaa=None):
        par_ = np.array(par, np.complex128)
        M = self.elanz
        dpar = np.zeros(M, np.complex128)
        cgfac = np.zeros(M)
        cgres = np.zeros(prm.ncgmax + 2)
        ncg = C.c_int32()
        bd = C.c_double()
        sa = None if sigmaa is None else np.ascontiguousarray(sigmaa, np.complex128)
        self._check(self.L.crt_update(self.h, C.byref(prm), _vp(sa), _vp(par_), _vp(dpar), _vp(cgfac),
                                      _vp(cgres), C.byref(ncg), C.byref(bd)), "crt_update")
        return dict(par=par_, dpar=dpar, cgfac=cgfac, cgres=cgres[: ncg.value + 1], ncg=ncg.value,
                    bdpar=bd.value)

    def update_lambdas(self, prm, lams, par, sigmaa=None):
        """crt_update for every lambda in `lams` (1 .. 8 candidates, Jacobi
        form) on one Jacobian; each CG iteration reads J once for all."""
        lam_ = np.ascontiguousarray(lams, np.float64)
        nl = int(lam_.size)
        M = self.elanz
        par_ = np.ascontiguousarray(par, np.complex128)
        out = np.zeros((nl, M), np.complex128)
        dpar = np.zeros((nl, M), np.complex128)
        ncg = np.zeros(nl, np.int32)
        bd = np.zeros(nl)
        sa = None if sigmaa is None else np.ascontiguousarray(sigmaa, np.complex128)
        self._check(self.L.crt_update_lambdas(self.h, C.byref(prm), nl, _ptr(lam_, C.c_double), _vp(sa), _vp(par_),
                                              _vp(out), _vp(dpar), _ptr(ncg, C.c_int32), _ptr(bd, C.c_double)),
                    "crt_update_lambdas")
        return dict(par=out, dpar=dpar, ncg=ncg, bdpar=bd)

    def gn_step(self, prm, par):
        par_ = np.array(par, np.complex128)
        sa = np.zeros(self.nanz, np.complex128)
        cgres = np.zeros(prm.ncgmax + 2)
        ncg = C.c_int32()
        bd = C.c_double()
        self._check(self.L.crt_gn_step(self.h, C.byref(prm), _vp(par_), _vp(sa), _vp(cgres), C.byref(ncg),
                                       C.byref(bd)), "crt_gn_step")
        return dict(par=par_, sigmaa=sa, cgres=cgres[: ncg.value + 1], ncg=ncg.value, bdpar=bd.value)

    def set_model(self, par):
        p = np.ascontiguousarray(par, np.complex128)
        self._check(self.L.crt_set_model(self.h, _vp(p)), "crt_set_model")

    def get_model(self):
        p = np.zeros(self.elanz, np.complex128)
        self._check(self.L.crt_get_model(self.h, _vp(p)), "crt_get_model")
        return p

    def model_backup(self, restore=False):
        self._check(self.L.crt_model_backup(self.h, int(bool(restore))), "crt_model_backup")

    def gn_step_device(self, prm):
        ncg = C.c_int32()
        self._check(self.L.crt_gn_step_device(self.h, C.byref(prm), C.byref(ncg)), "crt_gn_step_device")
        return ncg.value

    TIMING_NAMES = ["factor", "solve", "volt", "jacobian", "cg_setup", "cg_iter", "total", "factor_prep",
                    "factor_kernel", "factor_launches", "refine_residual", "refine_solve", "panel",
                    "schur_forward", "schur_gram", "schur_chol", "schur_back", "schur_iter"]

    def timings(self):
        t = np.zeros(len(self.TIMING_NAMES))
        self._check(self.L.crt_last_timings_ex(self.h, _ptr(t, C.c_double), len(t)), "crt_last_timings_ex")
        return dict(zip(self.TIMING_NAMES, t))

    def launch_count(self):
        return int(self.L.crt_launch_count(self.h))

    def blam0(self, alfx, alfz, ldc=False, lfpi=False):
        """lambda_0 from the device-resident Jacobian (crt_blam0)."""
        v = C.c_double()
        self._check(self.L.crt_blam0(self.h, int(bool(ldc)), int(bool(lfpi)), float(alfx), float(alfz),
                                     C.byref(v)), "crt_blam0")
        return v.value

    def set_forward_form(self, form):
        """FORWARD_AUTO, FORWARD_DIRECT or FORWARD_SCHUR (crt_set_forward_form)."""
        self._check(self.L.crt_set_forward_form(self.h, int(form)), "crt_set_forward_form")

    def coverage(self, part=0, weight=None):
        """csens (bbsens.f90) from the device-resident Jacobian (crt_coverage):
        sum_i |J_ij| w_i, |Re J_ij| for part 1; weight None = sqrt(wmatd wdfak)."""
        w = None if weight is None else np.ascontiguousarray(weight, np.float64)
        out = np.zeros(self.elanz)
        self._check(self.L.crt_coverage(self.h, int(part), _vp(w), _vp(out)), "crt_coverage")
        return out

    def forward_info(self):
        """(form of the last forward, boundary nodes, interior nodes, interior band)."""
        v = [C.c_int32() for _ in range(4)]
        self._check(self.L.crt_forward_info(self.h, *(C.byref(x) for x in v)), "crt_forward_info")
        return tuple(x.value for x in v)

    def set_refinement(self, steps):
        self._check(self.L.crt_set_refinement(self.h, int(steps)), "crt_set_refinement")

    def set_refinement_tol(self, tau):
        """Normwise backward error at which a system's refinement stops."""
        self._check(self.L.crt_set_refinement_tol(self.h, float(tau)), "crt_set_refinement_tol")

    def set_workspace_limit(self, nbytes):
        """Upper bound of the band-factor workspace (0: default)."""
        self._check(self.L.crt_set_workspace_limit(self.h, int(nbytes)), "crt_set_workspace_limit")

    # -- learned correction of the preconditioner -------------------------
    def gnn_nparam(self):
        return int(self.L.crt_gnn_nparam())

    def gnn_status(self):
        v = [C.c_int32() for _ in range(5)]
        self._check(self.L.crt_gnn_status(self.h, *[C.byref(x) for x in v]), "crt_gnn_status")
        return dict(zip(["available", "trained", "form", "nrec", "guard_fired"], [x.value for x in v]))

    def gnn_init(self, seed=1):
        self._check(self.L.crt_gnn_init(self.h, int(seed)), "crt_gnn_init")

    def gnn_set_weights(self, w, form):
        w = np.ascontiguousarray(w, np.float32)
        self._check(self.L.crt_gnn_set_weights(self.h, _ptr(w, C.c_float), len(w), int(form)), "crt_gnn_set_weights")

    def gnn_get_weights(self):
        w = np.zeros(self.gnn_nparam(), np.float32)
        f = C.c_int32()
        self._check(self.L.crt_gnn_get_weights(self.h, _ptr(w, C.c_float), len(w), C.byref(f)), "crt_gnn_get_weights")
        return w, f.value

    def gnn_collect(self, prm, base_block=False, stride=8, nmax=256):
        n = C.c_int32()
        self._check(self.L.crt_gnn_collect(self.h, C.byref(prm), int(bool(base_block)), int(stride), int(nmax),
                                           C.byref(n)), "crt_gnn_collect")
        return n.value

    def gnn_clear(self):
        self._check(self.L.crt_gnn_clear(self.h), "crt_gnn_clear")

    def gnn_train(self, epochs=10, batch=8, lr=1e-3, seed=1):
        hist = np.zeros(epochs, np.float32)
        self._check(self.L.crt_gnn_train(self.h, int(epochs), int(batch), float(lr), int(seed), _ptr(hist, C.c_float)),
                    "crt_gnn_train")
        return hist

    def gnn_record(self, idx):
        M = self.elanz
        x = np.zeros((M, 4), np.float32)
        t = np.zeros((M, 2), np.float32)
        a = np.zeros((M, 4), np.float32)
        nb = np.zeros((M, 4), np.int32)
        tn = C.c_float()
        self._check(self.L.crt_gnn_record(self.h, int(idx), _ptr(x, C.c_float), _ptr(t, C.c_float),
                                          _ptr(a, C.c_float), _ptr(nb, C.c_int32), C.byref(tn)), "crt_gnn_record")
        return dict(x=x, t=t, a=a, nbr=nb, tnorm2=tn.value)

    def gnn_record_grad(self, idx):
        g = np.zeros(self.gnn_nparam(), np.float32)
        L_ = C.c_double()
        self._check(self.L.crt_gnn_record_grad(self.h, int(idx), _ptr(g, C.c_float), C.byref(L_)),
                    "crt_gnn_record_grad")
        return g, L_.value

    def cg_info(self):
        """(form of the last CG, block size of the block preconditioner or 0,
        regulariser half-bandwidth after reverse Cuthill-McKee)."""
        f, b, w = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self.L.crt_cg_info(self.h, C.byref(f), C.byref(b), C.byref(w)), "crt_cg_info")
        return f.value, b.value, w.value


def dmisft(dat, sigmaa, wmatd, wmatdr=None, wmatdp=None, lfpi=False, lpol=False):
    """src/dmisft.f90 through the C ABI (host FP64). Returns (nrmsd, betrms, pharms, npol)."""
    L = load()
    d = np.ascontiguousarray(dat, np.complex128)
    s = np.ascontiguousarray(sigmaa, np.complex128)
    w = np.ascontiguousarray(wmatd, np.float64)
    wr = None if wmatdr is None else np.ascontiguousarray(wmatdr, np.float64)
    wp = None if wmatdp is None else np.ascontiguousarray(wmatdp, np.float64)
    br, ph = C.c_double(), C.c_double()
    npol = C.c_int32()
    r = L.crt_dmisft(len(d), _vp(d), _vp(s), _vp(w), _vp(wr), _vp(wp), int(lfpi), int(lpol), C.byref(br),
                     C.byref(ph), C.byref(npol))
    return r, br.value, ph.value, npol.value


class Batch:
    """Forward (and Jacobian) of many independent contexts as one CUDA graph
    (crt_batch_*): the contexts are the graph's independent branches; the
    first run executes every instance eagerly (workspaces, panel autotuning)
    and captures the graph, later runs replay it."""

    def __init__(self, contexts, ldc=False, jacobian_mode=0):
        self.L = load()
        self.contexts = list(contexts)
        arr = (C.c_void_p * len(self.contexts))(*[c.h.value for c in self.contexts])
        self._arr = arr
        err = C.c_int32()
        h = self.L.crt_batch_create(arr, len(self.contexts), int(bool(ldc)), int(jacobian_mode), C.byref(err))
        if not h:
            raise CRTError(err.value, "crt_batch_create failed")
        self.h = C.c_void_p(h)
        self.jacobian_mode = int(jacobian_mode)
        self._sig = None

    def close(self):
        if getattr(self, "h", None):
            self.L.crt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, e, what):
        if e:
            raise CRTError(e, f"{what}: {self.L.crt_batch_error(self.h).decode(errors='replace')}")

    def set_models(self, sigmas):
        self._sig = [np.ascontiguousarray(s_, np.complex128) for s_ in sigmas]
        ptrs = (C.c_void_p * len(self._sig))(*[a.ctypes.data for a in self._sig])
        self._check(self.L.crt_batch_set_models(self.h, ptrs), "crt_batch_set_models")

    def run(self):
        """Runs (replays) the batch; returns the device time in ms."""
        ms = C.c_double()
        self._check(self.L.crt_batch_run(self.h, C.byref(ms)), "crt_batch_run")
        return ms.value

    def status(self, i):
        return int(self.L.crt_batch_status(self.h, int(i)))

    def results(self, i, sens=False):
        c = self.contexts[i]
        volt = np.zeros(c.nanz, np.complex128)
        sa = np.zeros(c.nanz, np.complex128)
        J = None
        if sens:
            dt = np.float64 if self.jacobian_mode == 1 else np.complex128
            J = np.zeros((c.nanz, c.elanz), dt, order="F")
        self._check(self.L.crt_batch_results(self.h, int(i), _vp(volt), _vp(sa), _vp(J)), "crt_batch_results")
        return (volt, sa, J) if sens else (volt, sa)
