"""The C ABI library without a GPU: it loads, exports every entry point that
include/crt_b200.h declares, and its host-only entry points agree with the
oracle."""
import ctypes as C
import os
import re

import numpy as np

from fixtures import GOLDEN

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    with open(os.path.join(ROOT, "include", "crt_b200.h")) as fh:
        txt = fh.read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(crt_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_entry_point():
    from crtomo_stable_b200 import lib
    L = lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert set(lib.EXPORTS) == set(names)
    assert L.crt_abi_version() == 2


def test_fortran_module_binds_every_entry_point():
    """include/crt_b200.f90 has one BIND(C) interface per header function,
    and INTEGRATION.md shows that file verbatim."""
    with open(os.path.join(ROOT, "include", "crt_b200.f90")) as fh:
        mod = fh.read()
    bound = re.findall(r"NAME='(crt_[a-z0-9_]+)'", mod)
    assert sorted(bound) == declared_functions()
    assert len(bound) == len(set(bound))
    # each interface's dummy-argument count matches the C prototype
    with open(os.path.join(ROOT, "include", "crt_b200.h")) as fh:
        h = re.sub(r"/\*.*?\*/", "", fh.read(), flags=re.S)
    for name in bound:
        proto = re.search(r"\b" + name + r"\s*\(([^;]*?)\)\s*;", h, flags=re.S).group(1)
        nc = 0 if proto.strip() in ("", "void") else proto.count(",") + 1
        head = re.search(r"(?:FUNCTION|SUBROUTINE)\s+" + name + r"\s*\(([^)]*)\)", mod, flags=re.S).group(1)
        head = head.replace("&", " ")
        nf = 0 if not head.strip() else head.count(",") + 1
        assert nc == nf, (name, nc, nf)
    with open(os.path.join(ROOT, "INTEGRATION.md")) as fh:
        assert mod in fh.read()


def test_rwaven_host_entry_point_matches_oracle():
    from crtomo_stable_b200 import io, lib
    from oracle.oracle import OracleProblem
    for name in ("minimal", "TestModInv", "dc_problem_complex"):
        base = os.path.join(GOLDEN, name)
        m = io.read_elem(os.path.join(base, "grid", "elem.dat"))
        e = io.read_elec(os.path.join(base, "grid", "elec.dat"))
        d = io.read_volt(os.path.join(base, "mod", "volt.dat"))
        kwn, kwnwi = lib.rwaven(m, e, d.strnr, d.vnr)
        op = OracleProblem(m, e, d.strnr, d.vnr)
        np.testing.assert_allclose(kwn, op.kwn, rtol=1e-14)
        np.testing.assert_allclose(kwnwi, op.kwnwi, rtol=1e-13)


def test_dmisft_host_entry_point_matches_oracle():
    from crtomo_stable_b200 import lib
    from oracle import oracle
    rng = np.random.default_rng(5)
    n = 300
    dat = rng.normal(size=n) + 1j * rng.uniform(-3.5, 3.5, n)
    sa = dat + rng.normal(scale=0.1, size=n) + 1j * rng.normal(scale=0.5, size=n)
    w = rng.uniform(10, 100, n)
    wr = rng.uniform(10, 100, n)
    wp = rng.uniform(10, 100, n)
    for lfpi in (False, True):
        a = lib.dmisft(dat, sa, w, wr, wp, lfpi=lfpi)
        b = oracle.dmisft(dat, sa, w, wr, wp, lfpi=lfpi)
        np.testing.assert_allclose(a[:3], b[:3], rtol=1e-13)
        assert a[3] == b[3]


def test_create_without_device_fails_loudly():
    """No silent CPU path: without a CUDA device crt_create returns NULL
    with an error number."""
    import pytest
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    from crtomo_stable_b200 import io, lib
    from crtomo_stable_b200.lib import CRTError, Context
    base = os.path.join(GOLDEN, "minimal")
    m = io.read_elem(os.path.join(base, "grid", "elem.dat"))
    e = io.read_elec(os.path.join(base, "grid", "elec.dat"))
    d = io.read_volt(os.path.join(base, "mod", "volt.dat"))
    with pytest.raises(CRTError) as ei:
        Context(m, e, d.strnr, d.vnr)
    assert ei.value.errnr == 200


def test_library_resolves_its_own_templates():
    """Every kernel launcher the library instantiates is defined in it (an
    explicit instantiation missing for one precision would only fail when the
    library is loaded on a GPU box)."""
    import shutil
    import subprocess
    from crtomo_stable_b200 import build
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm not available")
    lib = build.build()
    out = subprocess.run([nm, "-D", "--undefined-only", lib], capture_output=True, text=True).stdout
    own = [ln for ln in out.splitlines() if "launch_" in ln or "crt_" in ln or "gnn_" in ln or "spc_" in ln]
    assert not own, own


def test_null_context_is_rejected_before_any_device_work():
    """Entry points given no context return errnr 3 (inconsistent input)
    without touching a device: the refinement controls and the batched
    lambda update."""
    from crtomo_stable_b200 import lib
    L = lib.load()
    assert L.crt_set_refinement(None, 2) == 3
    assert L.crt_set_refinement_tol(None, 1e-14) == 3
    lams = np.array([1.0, 10.0])
    par = np.zeros(4, np.complex128)
    out = np.zeros(8, np.complex128)
    assert L.crt_update_lambdas(None, None, 2, lams.ctypes.data_as(C.POINTER(C.c_double)), None,
                                C.c_void_p(par.ctypes.data), C.c_void_p(out.ctypes.data), None, None, None) == 3
