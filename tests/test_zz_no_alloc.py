"""crt_voltages_noalloc: the allocation-free voltage entry point, for callers
that own all their device memory up front and cannot call cudaMalloc while
they evaluate voltages.  It must give crt_forward's voltages for the same
potentials, on consecutive calls that share its static scratch table.

This file is collected last, so a run that stops at the first failure has
run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from fixtures import load_forward_case

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-10


def _device_inputs(torch, ctx, case, kpot):
    dev = torch.device("cuda", 0)
    d = dict(
        kpot=torch.from_numpy(np.asfortranarray(kpot).ravel(order="F").copy()).to(dev),
        kwnwi=torch.from_numpy(np.ascontiguousarray(ctx.kwnwi)).to(dev),
        enr=torch.from_numpy(np.ascontiguousarray(case["enr"], np.int32)).to(dev),
        strnr=torch.from_numpy(np.ascontiguousarray(case["volt"].strnr, np.int32)).to(dev),
        vnr=torch.from_numpy(np.ascontiguousarray(case["volt"].vnr, np.int32)).to(dev),
        volt=torch.zeros(len(case["volt"].strnr), dtype=torch.complex128, device=dev),
        sigmaa=torch.zeros(len(case["volt"].strnr), dtype=torch.complex128, device=dev),
    )
    torch.cuda.synchronize()
    return d


def _call(L, case, ctx, d, mode, eanz=None, ldc=0, kfak=None):
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    return L.crt_voltages_noalloc(P(d["kpot"]), P(d["kwnwi"]), P(d["enr"]), P(d["strnr"]), P(d["vnr"]),
                                  int(case["mesh"].sanz), int(eanz or len(case["enr"])), int(len(ctx.kwnwi)),
                                  int(len(case["volt"].strnr)), int(ctx.swrtr), int(ldc), int(mode),
                                  None if kfak is None else P(kfak), P(d["volt"]), P(d["sigmaa"]), None)


def _setup(torch, name="minimal", ldc=False, mode=0, kfak=None):
    from crtomo_stable_b200 import lib
    from crtomo_stable_b200.lib import Context
    L = lib.load()
    case = load_forward_case(name)
    c = case["cfg"]
    ctx = Context(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr, swrtr=c.swrtr,
                  lsink=c.lsink, nsink=c.nsink)
    volt_ref, sa_ref, kpot = ctx.forward(case["sigma"], ldc=ldc, mode=mode, kfak=kfak, want_kpot=True)
    return L, case, ctx, volt_ref, sa_ref, _device_inputs(torch, ctx, case, kpot)


@pytest.mark.parametrize("name,mode", [("minimal", 0), ("grid_decoupling", 1)])
def test_voltages_noalloc_matches_crt_forward(name, mode):
    torch = pytest.importorskip("torch")
    from crtomo_stable_b200 import lib
    from crtomo_stable_b200.lib import Context
    L = lib.load()
    case = load_forward_case(name)
    c = case["cfg"]
    ctx = Context(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr, swrtr=c.swrtr,
                  lsink=c.lsink, nsink=c.nsink)
    volt_ref, sa_ref, kpot = ctx.forward(case["sigma"], mode=mode, want_kpot=True)
    d = _device_inputs(torch, ctx, case, kpot)
    for _ in range(2):   # two calls in a row share the static scratch
        d["volt"].zero_()
        d["sigmaa"].zero_()
        torch.cuda.synchronize()
        assert _call(L, case, ctx, d, mode) == 0
        volt = d["volt"].cpu().numpy()
        sa = d["sigmaa"].cpu().numpy()
        np.testing.assert_allclose(volt, volt_ref, rtol=RTOL_FP64, atol=RTOL_FP64 * np.abs(volt_ref).max())
        np.testing.assert_allclose(sa, sa_ref, rtol=RTOL_FP64, atol=RTOL_FP64 * np.abs(sa_ref).max())
    ctx.close()


def test_voltages_noalloc_rejects_too_many_electrodes():
    torch = pytest.importorskip("torch")
    from crtomo_stable_b200 import lib
    from crtomo_stable_b200.lib import Context
    L = lib.load()
    case = load_forward_case("minimal")
    ctx = Context(case["mesh"], case["enr"], case["volt"].strnr, case["volt"].vnr)
    _, _, kpot = ctx.forward(case["sigma"], want_kpot=True)
    d = _device_inputs(torch, ctx, case, kpot)
    assert _call(L, case, ctx, d, 0, eanz=513) == 3
    ctx.close()


def test_voltages_noalloc_geometric_factors_and_real_path():
    """bvolt with a kfak vector (mode 1) and the real (ldc) path: the same
    numbers as crt_forward with those options."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(7)
    case = load_forward_case("minimal")
    kfak = rng.uniform(0.5, 50.0, len(case["volt"].strnr))
    for ldc, mode, kf in ((0, 1, kfak), (1, 0, None), (1, 1, kfak)):
        L, case, ctx, volt_ref, sa_ref, d = _setup(torch, ldc=bool(ldc), mode=mode, kfak=kf)
        dk = None if kf is None else torch.from_numpy(np.ascontiguousarray(kf)).to("cuda:0")
        torch.cuda.synchronize()
        assert _call(L, case, ctx, d, mode, ldc=ldc, kfak=dk) == 0
        volt = d["volt"].cpu().numpy()
        sa = d["sigmaa"].cpu().numpy()
        np.testing.assert_allclose(volt, volt_ref, rtol=RTOL_FP64, atol=RTOL_FP64 * np.abs(volt_ref).max())
        np.testing.assert_allclose(sa, sa_ref, rtol=RTOL_FP64, atol=RTOL_FP64 * np.abs(sa_ref).max())
        if ldc:
            assert np.abs(volt.imag).max() == 0.0
        ctx.close()


def test_voltages_noalloc_error_codes():
    """The status codes of the reference's input checks and of bvolti, each
    from one planted fault: an electrode number above eanz in a
    configuration (46), an electrode node above sanz (29), a reading whose
    current electrodes coincide (zero voltage, 82).  A clean call after
    each returns 0 again: the status word starts at zero on every call."""
    torch = pytest.importorskip("torch")
    L, case, ctx, volt_ref, sa_ref, d = _setup(torch)
    eanz = len(case["enr"])
    strnr0, enr0 = d["strnr"].clone(), d["enr"].clone()
    bad = strnr0.clone()
    bad[3] = (eanz + 1) + 10000 * 1
    d["strnr"].copy_(bad)
    torch.cuda.synchronize()
    assert _call(L, case, ctx, d, 0) == 46
    d["strnr"].copy_(strnr0)
    torch.cuda.synchronize()
    assert _call(L, case, ctx, d, 0) == 0
    bad = enr0.clone()
    bad[1] = case["mesh"].sanz + 5
    d["enr"].copy_(bad)
    torch.cuda.synchronize()
    assert _call(L, case, ctx, d, 0) == 29
    d["enr"].copy_(enr0)
    bad = strnr0.clone()
    c1 = int(strnr0[0].item()) % 10000
    bad[0] = c1 + 10000 * c1
    d["strnr"].copy_(bad)
    torch.cuda.synchronize()
    assert _call(L, case, ctx, d, 0) == 82
    d["strnr"].copy_(strnr0)
    torch.cuda.synchronize()
    assert _call(L, case, ctx, d, 0) == 0
    np.testing.assert_allclose(d["sigmaa"].cpu().numpy(), sa_ref, rtol=RTOL_FP64,
                               atol=RTOL_FP64 * np.abs(sa_ref).max())
    ctx.close()
