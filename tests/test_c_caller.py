"""The C ABI as a C compiler sees it: tests/c_caller/crt_c_caller.c,
compiled by gcc against include/crt_b200.h and linked with libcrt_b200.so,
runs the first pass of the CRTomo loop on the `minimal` tomodir; its outputs
are compared with the FP64 oracle.  The compile-and-link check needs no GPU.
"""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from fixtures import load_forward_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_caller", "crt_c_caller.c")
LIBDIR = os.path.join(ROOT, "crtomo_stable_b200")


def _build(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    exe = str(tmp_path / "crt_c_caller")
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-O2", "-I", os.path.join(ROOT, "include"),
                           SRC, "-o", exe, "-L", LIBDIR, "-l:libcrt_b200.so", "-Wl,-rpath," + LIBDIR, "-lm"])
    return exe


def _rec(a):
    b = np.ascontiguousarray(a).tobytes(order="F") if isinstance(a, np.ndarray) else a
    return struct.pack("<q", len(b)) + b


def _read_recs(path):
    out = []
    with open(path, "rb") as fh:
        data = fh.read()
    pos = 0
    while pos < len(data):
        (n,) = struct.unpack_from("<q", data, pos)
        pos += 8
        out.append(data[pos:pos + n])
        pos += n
    return out


def test_c_caller_compiles_and_links_against_the_header(tmp_path):
    """The header compiles as strict C99 (-Wall -Werror -pedantic) and every
    entry point the program calls resolves in libcrt_b200.so."""
    from crtomo_stable_b200 import build
    build.build()
    exe = _build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_c_caller_first_gn_pass_matches_oracle(tmp_path):
    from crtomo_stable_b200 import regularization
    from oracle.oracle import OracleCG, OracleProblem
    exe = _build(tmp_path)
    case = load_forward_case("minimal")
    m, d = case["mesh"], case["volt"]
    sig = np.full(m.elanz, 0.01 * np.exp(-0.005j))
    dat = -np.log(d.bet) - 1j * d.pha / 1e3
    wmatd = 1.0 / (1e-2 + 1e-3 / d.bet) ** 2
    nb = regularization.nachbar(m)
    sm = regularization.smatm_tri(m, nb, 10.0, 1.0)
    lam, eps, ncgmax = 300.0, 1e-4, m.elanz // 10
    i32 = lambda v: struct.pack("<i", int(v))  # noqa: E731
    f64 = lambda v: struct.pack("<d", float(v))  # noqa: E731
    recs = [i32(m.sanz), i32(m.typanz), i32(m.mb), np.asarray(m.typ, np.int32), np.asarray(m.nelanz, np.int32),
            np.asarray(m.selanz, np.int32), np.asarray(m.snr, np.int32), np.asarray(m.sx, np.float64),
            np.asarray(m.sy, np.float64), np.asfortranarray(m.nrel, np.int32),
            np.asarray(m.rnr if len(m.rnr) else np.zeros(1), np.int32), i32(m.elanz),
            np.asarray(case["enr"], np.int32), np.asarray(d.strnr, np.int32), np.asarray(d.vnr, np.int32),
            np.asarray(sig, np.complex128), i32(1), i32(0), i32(nb.shape[1] - 1), np.asfortranarray(sm, np.float64),
            np.asfortranarray(nb, np.int32), np.asarray(dat, np.complex128), np.asarray(wmatd, np.float64),
            f64(lam), f64(eps), i32(ncgmax)]
    inp, outp = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as fh:
        for r in recs:
            fh.write(_rec(r) if isinstance(r, np.ndarray) else struct.pack("<q", len(r)) + r)
    res = subprocess.run([exe, str(inp), str(outp)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    o = _read_recs(outp)
    K = struct.unpack("<i", o[0])[0]
    kwn, kwnwi = np.frombuffer(o[1]), np.frombuffer(o[2])
    volt, sa = np.frombuffer(o[3], np.complex128), np.frombuffer(o[4], np.complex128)
    N, E = len(d.strnr), m.elanz
    sens = np.frombuffer(o[5], np.complex128).reshape((N, E), order="F")
    nrmsd = struct.unpack("<d", o[6])[0]
    par, dpar = np.frombuffer(o[7], np.complex128), np.frombuffer(o[8], np.complex128)
    cgfac = np.frombuffer(o[9])
    ncg = struct.unpack("<i", o[10])[0]
    form = struct.unpack("<i", o[12])[0]
    op = OracleProblem(m, case["enr"], d.strnr, d.vnr)
    assert K == len(op.kwn)
    np.testing.assert_allclose(kwn, op.kwn, rtol=1e-14)
    np.testing.assert_allclose(kwnwi, op.kwnwi, rtol=1e-14)
    kp = op.forward(sig, nthreads=4)
    volt_o, sa_o = op.bvolti(op.rtrafo(kp))
    np.testing.assert_allclose(volt, volt_o, rtol=1e-10, atol=1e-10 * np.abs(volt_o).max())
    np.testing.assert_allclose(sa, sa_o, rtol=1e-10, atol=1e-10)
    J_o = op.bsensi(kp, sig, volt_o, nthreads=4)
    colmax = np.abs(J_o).max(axis=0, keepdims=True) + 1e-300
    assert (np.abs(sens - J_o) / colmax).max() <= 1e-9
    from oracle.oracle import dmisft
    assert abs(nrmsd / dmisft(dat, sa_o, wmatd)[0] - 1) < 1e-10
    cg = OracleCG(E, N, 1, sm, nachbar=nb, nnb=m.maxnodes, wmatd=wmatd, lam=lam, eps=eps, ncgmax=ncgmax)
    ref = cg.update(J_o, dat, sa_o, np.log(sig), 1.0)
    assert form == 0 and ncg == ref["ncg"]
    np.testing.assert_allclose(cgfac, ref["cgfac"], rtol=1e-11)
    np.testing.assert_allclose(dpar, ref["dpar"], rtol=1e-7, atol=1e-7 * np.abs(ref["dpar"]).max())
    np.testing.assert_allclose(par, ref["par"], rtol=1e-9, atol=1e-9)
