"""Gauss-Newton step benchmark (forward + Jacobian + inner CG to relative
residual 1e-6) on the seeded synthetic 60k-triangle / 128-electrode
configuration, through the C ABI of libcrt_b200.so.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0.  `value` is the GN-step wall time with all
inputs resident in device memory (CUDA events on the library's stream, max
over ranks); `e2e` is the same step through crt_gn_step with host buffers
(model upload, model / response / CG-history download inside the timed
region).  Multi-GPU runs are independent replicas (the reference's hot path
has no exchange step), so the per-step time is reported as the max over
ranks with "scaling": "weak".
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GN-step wall time, learned-PCG/FP32-refined vs plain CG on B200 at rel-res 1e-6"

# CG iterations of the reference's own iteration (cgfac-preconditioned
# cjggra) to |r|^2 <= 1e-12 |r0|^2 on each synthetic workload, as counted by
# the FP64 Jacobi form on the device (whose iteration counts equal the
# oracle's in the parity tests).  The CPU baseline scales its timed CG
# sample by this count.
REF_NCG = {"C5": 1589}

# FP64 FMA pipe of a B200 SM (non-tensor): 64 FMA per clock, the roofline
# of the forward's FP64 kernels.
FP64_FMA_PER_CLK_SM = 64


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="C5")
    ap.add_argument("--eps", type=float, default=1e-12, help="|r|^2 <= eps |r0|^2 (1e-12 = rel-res 1e-6)")
    ap.add_argument("--ncgmax", type=int, default=20000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--refine", type=int, default=None,
                    help="FP64 refinement steps of the complex64 forward (default: the library's)")
    ap.add_argument("--forms", default="both", choices=["both", "mixed"],
                    help="'mixed' skips the plain FP64 comparison run (profiling)")
    ap.add_argument("--count", type=int, default=256, help="instances of the batched configuration C4")
    ap.add_argument("--lambdas", type=int, default=4,
                    help="lambda candidates of the batched Jacobi-form update measured after the step (0: skip)")
    ap.add_argument("--lambda-iters", type=int, default=100, help="CG iterations of that measurement")
    ap.add_argument("--inversion", action="store_true",
                    help="run the configuration's whole Gauss-Newton inversion (inv.f90's loop) to its stop "
                         "criterion and print one JSON line with its iterations and wall time")
    ap.add_argument("--itmax", type=int, default=20, help="iteration limit of --inversion")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(pg, local, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def make_problem(config: str):
    """Synthetic survey, its 'observed' data (the true model's response with
    3 % + 0.1 mrad seeded Gaussian noise, computed on the device once) and
    the homogeneous starting model."""
    from crtomo_stable_b200 import regularization, synth
    s = synth.CONFIGS[config]()
    return s


def setup_context(s, device: int, precision: int = 0):
    from crtomo_stable_b200 import regularization
    from crtomo_stable_b200.lib import Context
    ctx = Context(s.mesh, s.enr, s.strnr, s.vnr, device=device, precision=precision)
    # observed data: forward of the true model + seeded noise
    _, sa_true = ctx.forward(s.sigma)
    rng = np.random.default_rng(20261203)
    mag = np.exp(-sa_true.real)
    pha = -sa_true.imag
    mag = mag * (1.0 + 0.03 * rng.standard_normal(len(mag)))
    pha = pha + 1e-4 * rng.standard_normal(len(pha))
    dat = -np.log(np.abs(mag)) - 1j * pha
    stabw = 0.03 + 1e-4 / np.abs(mag)
    wmatd = 1.0 / stabw ** 2
    nb = regularization.nachbar(s.mesh)
    sm = regularization.smatm_tri(s.mesh, nb, 1.0, 1.0)
    ctx.set_regularizer(1, sm, nachbar=nb)
    ctx.set_data(dat, wmatd)
    rho0 = float(np.exp(np.mean(np.log(np.abs(1.0 / s.sigma)))))
    par0 = np.full(s.mesh.elanz, np.log(1.0 / rho0) + 0j)
    lam = float(max(s.mesh.elanz, len(s.strnr)))
    return ctx, dat, wmatd, par0, lam, nb, sm


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def schur_work(s, K: int, m_boundary: int, n_interior: int, mb_interior: int):
    """Algorithmic complex multiply-adds of the Schur-form kernels (8 flops
    each) on survey s with K wavenumbers: the boundary set G is every node of
    a type-11 segment, a column's first non-zero interior row is its
    source's row (source columns) or that of the first interior neighbour
    of its boundary node (coupling columns); the forward sweep runs each
    column from that row, the Gram products over the rows where both columns
    can be non-zero, the rebuild over V^'s non-zero rows, the back sweep and
    the interior factorisation over the whole band."""
    m = s.mesh
    n = m.sanz
    typ = np.repeat(m.typ, m.nelanz)
    rows = np.nonzero(typ == 11)[0]
    isg = np.zeros(n, bool)
    isg[np.unique(m.nrel[rows, :2].ravel()) - 1] = True
    posI = -np.ones(n, np.int64)
    posI[~isg] = np.arange(int((~isg).sum()))
    gpos = -np.ones(n, np.int64)
    gpos[isg] = np.arange(int(isg.sum()))
    nI, M, L, mb = n_interior, m_boundary, len(s.enr), mb_interior
    assert nI == int((~isg).sum()) and M == int(isg.sum())
    nk = int(m.selanz[0])
    area = m.nrel[: m.elanz, :nk] - 1
    first_g = np.full(M, nI)
    ga, gb = [], []
    for a in range(nk):
        for b in range(nk):
            ga.append(area[:, a])
            gb.append(area[:, b])
    ga, gb = np.concatenate(ga), np.concatenate(gb)
    sel = isg[ga] & ~isg[gb]
    np.minimum.at(first_g, gpos[ga[sel]], posI[gb[sel]])
    first_s = posI[s.enr - 1]
    first_s = np.where(first_s < 0, nI, first_s)
    fg = np.sort(first_g)
    vtv = sum(float(np.sum(nI - np.maximum(f, fg[: i + 1]))) for i, f in enumerate(fg))
    vtu = float(sum(np.sum(nI - np.maximum(f, first_s)) for f in first_g))
    return {
        "factor": K * nI * mb * mb / 2.0,
        "forward": K * float(np.sum(nI - first_g) + np.sum(nI - first_s)) * mb,
        "gram": K * (vtv + vtu),
        "chol": K * L * (M ** 3 / 6.0 + M * M),
        # iterative form: one reference factor per 16 electrodes, then per
        # system and iteration the residual (S0 x) and the two triangular
        # solves, m^2 each (times the mean iteration count, supplied later)
        "chol_ref": K * ((L + 15) // 16) * (M ** 3 / 6.0 + M * M),
        "chol_it": K * L * 2.0 * M * M,
        "back": K * (float(np.sum(nI - first_g)) * L + L * nI * mb),
    }


# ---------------------------------------------------------------------------
def workload_name(s, K: int) -> str:
    """The workload string both arms print (identical for the same survey)."""
    m = s.mesh
    kind = "triangles" if int(m.typ[0]) == 3 else "quadrilaterals"
    L, N = len(s.enr), len(s.strnr)
    return (f"{s.name}: {m.elanz} {kind}, n={m.sanz}, mb={m.mb}, {L} electrodes, {N} readings, K={K}; one GN step "
            f"from a homogeneous model (forward {K * L} band systems + Jacobian + CG to rel-res 1e-6)")


def _cpu_problem(s):
    """Oracle problem of the survey (wavenumbers from the oracle's own rwaven,
    precal of all electrodes), the homogeneous starting model, a data
    vector and weights for the CG timing (the starting model's response
    stands in for the data: a CG iteration's cost does not depend on the
    values) and the regulariser (ltri = 1, as the GPU arm)."""
    from crtomo_stable_b200 import regularization
    from oracle.oracle import OracleProblem
    m = s.mesh
    op = OracleProblem(m, s.enr, s.strnr, s.vnr)
    rho0 = float(np.exp(np.mean(np.log(np.abs(1.0 / s.sigma)))))
    sig0 = np.full(m.elanz, 1.0 / rho0 + 0j)
    nb = regularization.nachbar(m)
    sm = regularization.smatm_tri(m, nb, 1.0, 1.0)
    return op, sig0, nb, sm


def guided_makespan(n: int, threads: int, min_chunk: int) -> int:
    """Readings of the busiest thread when OpenMP's SCHEDULE(GUIDED, c)
    hands out n equal-cost iterations to `threads` threads (chunk =
    max(c, ceil(remaining / threads)), each to the thread that frees first)."""
    import heapq
    load = [0] * max(threads, 1)
    heapq.heapify(load)
    rem = n
    while rem > 0:
        ch = min(rem, max(min_chunk, -(-rem // max(threads, 1))))
        heapq.heappush(load, heapq.heappop(load) + ch)
        rem -= ch
    return max(load)


def _cg_iteration_s(J, E, N, nb, sm, lam, iters=2):
    """Seconds per serial cjggra iteration (src/cg_mod.f90:426-518, no
    OpenMP in the reference) on the given Jacobian: `iters` iterations at
    eps = 0 on a unit right-hand side."""
    from oracle.oracle import OracleCG
    cg = OracleCG(E, N, 1, sm, nachbar=nb, nnb=sm.shape[1] - 1, wmatd=np.ones(N), lam=lam, eps=0.0, ncgmax=iters)
    t = time.perf_counter()
    _, _, ncg = cg.cjggra(J, np.ones(E), np.ones(E, np.complex128))
    return (time.perf_counter() - t) / max(ncg, 1)


def oracle_full_step(s, nthreads: int, ncg_ref: int):
    """The reference's CPU path (the oracle: the FP64 C restatement of the
    Fortran, OpenMP where the reference has it) on the whole workload,
    measured once: the complete forward (every wavenumber x source electrode
    system; OpenMP over wavenumbers with min(K, cores) threads as
    src/inv.f90:426-484) with rtrafo and bvolti, and the complete bsensi
    (every reading; OpenMP over readings on all cores as
    src/bsensi.f90:90-96).  The CG is not run to its end (at rel-res 1e-6 the
    reference's serial cjggra needs ncg_ref iterations, hours on this
    survey): two iterations on the real Jacobian give its per-iteration time
    and the projection ncg_ref x that, reported apart from the measured
    value."""
    op, sig0, nb, sm = _cpu_problem(s)
    m = s.mesh
    E, N, K = m.elanz, len(s.strnr), len(op.kwn)
    tf = min(K, nthreads)
    # warm-up: one source electrode's systems (threads spun up, pages in)
    from oracle.oracle import OracleProblem
    one, zero = np.array([1], np.int32), np.array([0], np.int32)
    OracleProblem(m, s.enr[:1], one, zero, kwn=op.kwn, kwnwi=op.kwnwi).forward(sig0, nthreads=tf)
    t0 = time.perf_counter()
    kp = op.forward(sig0, nthreads=tf)
    volt, sa = op.bvolti(op.rtrafo(kp))
    t1 = time.perf_counter()
    J = op.bsensi(kp, sig0, volt, nthreads=nthreads)
    t2 = time.perf_counter()
    del kp
    lam = float(max(E, N))
    t_it = _cg_iteration_s(J, E, N, nb, sm, lam)
    return dict(forward_s=t1 - t0, jacobian_s=t2 - t1, cg_iteration_s=t_it, projected_cg_s=t_it * ncg_ref,
                ncg_ref=ncg_ref, forward_threads=tf, jacobian_threads=nthreads, K=K)


def cpu_sample(s, nthreads: int, ncg_ref: int, le: int = 16, ni_frac: float = 0.125, ni_max: int = 96):
    """A bounded sample of the same step on the oracle, extrapolated (and
    labelled so): the forward of all wavenumbers for `le` of the L source
    electrodes (min(K, cores) threads), scaled by L / le -- the systems of
    one electrode cost the same as any other's; bsensi for a sample of the
    readings on one thread, scaled to all readings and divided by the
    parallel width of the reference's schedule; the serial CG iteration timed
    twice on a Jacobian of the full size, projected to ncg_ref iterations.
    The scaling method is checked end to end on the 60 x 20 survey (C1),
    where the whole step runs in seconds (validate_scaling)."""
    from oracle.oracle import OracleProblem
    op, sig0, nb, sm = _cpu_problem(s)
    m = s.mesh
    L, N, E, K = len(s.enr), len(s.strnr), m.elanz, len(op.kwn)
    tf = min(K, nthreads)
    le = min(le, L)
    one, zero = np.array([1], np.int32), np.array([0], np.int32)
    opf = OracleProblem(m, s.enr[:le], one, zero, kwn=op.kwn, kwnwi=op.kwnwi)
    opf.forward(sig0, nthreads=tf)   # warm-up
    t = time.perf_counter()
    opf.forward(sig0, nthreads=tf)
    t_fwd = (time.perf_counter() - t) * L / le
    # bsensi: `ni` readings on one thread, scaled to the readings of the
    # busiest thread under the reference's SCHEDULE(GUIDED, 256) (a
    # reading's cost does not depend on which reading it is)
    ni = max(1, min(ni_max, int(N * ni_frac)))
    span = guided_makespan(N, nthreads, 256)
    width = N / span
    opj = OracleProblem(m, s.enr, s.strnr[:ni], s.vnr[:ni], kwn=op.kwn, kwnwi=op.kwnwi)
    kp = np.zeros((m.sanz, L, K), np.complex128, order="F")
    t = time.perf_counter()
    opj.bsensi(kp, sig0, np.ones(ni, np.complex128), nthreads=1)
    t_jac = (time.perf_counter() - t) / ni * span
    del kp
    J = np.full((N, E), 1e-3 + 1e-4j, order="F")
    t_it = _cg_iteration_s(J, E, N, nb, sm, float(max(E, N)))
    del J
    sample = (f"oracle (FP64 C restatement, OpenMP as the reference), extrapolated: forward of all {K} "
              f"wavenumbers x {le} of {L} source electrodes on {tf} threads (x{L / le:g}); bsensi on {ni} of {N} "
              f"readings on 1 thread, scaled to the {span} readings of the busiest of {nthreads} threads under GUIDED(256); CG projected: 2 serial cjggra iterations on the "
              f"full-size {N} x {E} Jacobian x {ncg_ref} iterations")
    return dict(forward_s=t_fwd, jacobian_s=t_jac, cg_iteration_s=t_it, projected_cg_s=t_it * ncg_ref,
                sample=sample, cores=nthreads)


def validate_scaling(nthreads: int):
    """The sampling of cpu_sample checked end to end on C1 (60 x 20 quads,
    40 electrodes, 268 readings), where the oracle's whole step -- forward,
    bsensi and the CG run to rel-res 1e-6 -- is measured in seconds: the
    measured phases beside the same extrapolations (forward from 4 of 40
    electrodes, bsensi from 1/8 of the readings, the CG from two iterations
    times the iteration count the measured run needed)."""
    from crtomo_stable_b200 import synth
    from oracle.oracle import OracleCG, OracleProblem
    s = synth.config1()
    op, sig0, nb, sm = _cpu_problem(s)
    m = s.mesh
    L, N, E, K = len(s.enr), len(s.strnr), m.elanz, len(op.kwn)
    tf = min(K, nthreads)
    op.forward(sig0, nthreads=tf)   # warm-up
    t0 = time.perf_counter()
    kp = op.forward(sig0, nthreads=tf)
    volt, sa = op.bvolti(op.rtrafo(kp))
    t1 = time.perf_counter()
    J = op.bsensi(kp, sig0, volt, nthreads=nthreads)
    t2 = time.perf_counter()
    lam = float(max(E, N))
    cg = OracleCG(E, N, 1, sm, nachbar=nb, nnb=sm.shape[1] - 1, wmatd=np.ones(N), lam=lam, eps=1e-12, ncgmax=50000)
    t3 = time.perf_counter()
    _, _, ncg = cg.cjggra(J, np.ones(E), np.ones(E, np.complex128))
    t4 = time.perf_counter()
    est = cpu_sample(s, nthreads, ncg, le=4)
    measured = {"forward_s": t1 - t0, "jacobian_s": t2 - t1, "cg_s": t4 - t3, "cg_iterations": int(ncg)}
    extrap = {"forward_s": est["forward_s"], "jacobian_s": est["jacobian_s"], "cg_s": est["projected_cg_s"]}
    return {"workload": "C1 (60 x 20 quadrilaterals, 40 electrodes, 268 readings, K=%d)" % K,
            "measured": measured, "extrapolated": extrap,
            "ratio_extrapolated_to_measured": {k: extrap[k] / measured[k] for k in extrap if measured[k] > 0}}


def run_reference(args, ws, rank, pg):
    """--impl reference: the reference's CPU path on the host cores -- the
    oracle, because the Fortran reference cannot be built here -- on the
    same survey and model as the GPU arm.  It loads no library of this
    repository's product (the oracle computes its own wavenumbers).  One
    complete forward + Jacobian is measured: at ~1-2 minutes per step the
    requested --steps cannot all run within a few minutes, so the line
    reports the repeats it ran in "steps" (and the requested ones beside)."""
    if rank != 0:
        return
    s = make_problem(args.config)
    nthreads = os.cpu_count() or 1
    ncg_ref = int(os.environ.get("CRT_REF_NCG", str(REF_NCG.get(args.config, 200))))
    r = oracle_full_step(s, nthreads, ncg_ref)
    v = r["forward_s"] + r["jacobian_s"]
    line = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": 1,
            "warmup": 1, "steps_requested": args.steps, "warmup_requested": args.warmup,
            "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded)",
            "config": {"workload": workload_name(s, r["K"]), "parallelism": "host cores"},
            "impl": "reference",
            "value_covers": ("forward + Jacobian of the GN step, measured in full (all systems, all readings); "
                             "the step's CG is excluded from value and projected in projected_cg_s"),
            "phases_s": {"forward": r["forward_s"], "jacobian": r["jacobian_s"]},
            "projected_cg_s": r["projected_cg_s"],
            "projected_cg": (f"{r['ncg_ref']} serial cjggra iterations (the count of the reference's "
                             f"Jacobi-preconditioned CG to rel-res 1e-6 on this survey) x "
                             f"{r['cg_iteration_s']:.3f} s per iteration measured on the real Jacobian"),
            "cpu_baseline": {"value": v, "unit": "s", "cores": nthreads, "kind": "port",
                             "sample": (f"oracle (FP64 C restatement of the Fortran path, OpenMP as the reference): "
                                        f"one complete forward ({r['forward_threads']} threads, one per wavenumber) "
                                        f"and one complete bsensi ({r['jacobian_threads']} threads), measured")},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_batch(args, ws, rank, local, pg):
    """C4: uneven synthetic instances (complex64 factorisation with FP64
    refinement, forward + Jacobian) run as one captured CUDA graph; a step is
    one replay of the whole batch (device time of the replay).  The first
    run (eager pass, panel autotuning, capture) is reported as build_s."""
    from crtomo_stable_b200 import synth
    from crtomo_stable_b200.lib import PREC_MIXED, Batch, Context
    S = synth.config4(count=args.count)
    ctxs = [Context(s.mesh, s.enr, s.strnr, s.vnr, device=local, precision=PREC_MIXED) for s in S]
    budget = int(min(512 << 20, (64 << 30) // len(ctxs)))
    for c in ctxs:
        c.set_workspace_limit(budget)
    b = Batch(ctxs, jacobian_mode=0)
    b.set_models([s.sigma for s in S])
    t0 = time.perf_counter()
    b.run()
    build_s = time.perf_counter() - t0
    for _ in range(max(0, args.warmup - 1)):
        b.run()
    barrier(pg)
    ms = [b.run() for _ in range(args.steps)]
    barrier(pg)
    t = max_over_ranks(pg, local, float(np.mean(ms)) / 1e3)
    # the same work one instance at a time through the per-context calls
    # (crt_forward + crt_jacobian, host round trip per instance)
    t0 = time.perf_counter()
    for c, s in zip(ctxs, S):
        c.forward(s.sigma)
        c.jacobian(0, copy=False)
    seq_s = time.perf_counter() - t0
    systems = sum(len(c.kwn) * len(s.enr) for c, s in zip(ctxs, S))
    E = [s.mesh.elanz for s in S]
    line = {"metric": "batched forward + Jacobian time of the uneven instances (one graph replay)", "value": t,
            "unit": "s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64/c128", "data": "synthetic (seeded)",
            "config": {"workload": f"C4: {len(S)} instances, E {min(E)}-{max(E)} (sum {sum(E)}), "
                                   f"{sum(len(s.strnr) for s in S)} readings, {systems} band systems",
                       "form": "complex64 band factorisation, adaptive FP64 refinement (at most 8 steps, to normwise "
                               "backward error 1e-14), FP64 Jacobian stored complex64",
                       "workspace_bytes_per_instance": budget, "parallelism": f"replicas x{args.gpus}"},
            "build_s": build_s, "sequential_calls_s": seq_s,
            "panels": sorted({int(c.timings()["panel"]) for c in ctxs})}
    b.close()
    for c in ctxs:
        c.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def lambda_batch(ctx, Context, lam, par0, nlam, iters, E, N, eps, ncgmax, precond_block):
    """Lambda trials side by side: `nlam` updates for lambdas spread over
    two decades around `lam`, on the step's complex64 Jacobian, through
    crt_update_lambdas against the same updates one crt_update at a time:
    in the Jacobi form (the reference's cjggra) for exactly `iters` CG
    iterations (eps = 0), and in the block-preconditioned form to the
    step's stop rule.  Times are the library's CUDA-event phases (cg set-up,
    preconditioner factors and iterations), host copies excluded."""
    lams = lam * np.logspace(-1.0, 1.0, nlam)
    prm = Context.params(lam, eps=0.0, ncgmax=iters)
    ctx.update_lambdas(prm, lams, par0)                      # warm-up
    got = ctx.update_lambdas(prm, lams, par0)
    t = ctx.timings()
    t_batch, t_iter = t["cg_setup"] + t["cg_iter"], t["cg_iter"]
    t_seq = 0.0
    for lm in lams:
        ctx.update(Context.params(lm, eps=0.0, ncgmax=iters), par0)
        t = ctx.timings()
        t_seq += t["cg_setup"] + t["cg_iter"]
    bytes_it = 2.0 * N * E * 8 + nlam * (6.0 * E * 16 + 3.0 * N * 16)   # J (complex64) twice + vectors
    ach = bytes_it * iters / (t_iter / 1e3) / 1e9
    # the block-preconditioned form at the step's stop rule (rel-res 1e-6):
    # one S factor per candidate, factors and sweeps side by side
    pb = Context.params(lam, eps=eps, ncgmax=ncgmax, precond=precond_block)
    ctx.update_lambdas(pb, lams, par0)                       # warm-up
    gb = ctx.update_lambdas(pb, lams, par0)
    t = ctx.timings()
    tb_batch = t["cg_setup"] + t["cg_iter"]
    form_b = ctx.cg_info()[0]
    tb_seq, ncg_seq = 0.0, []
    for lm in lams:
        r = ctx.update(Context.params(lm, eps=eps, ncgmax=ncgmax, precond=precond_block), par0)
        t = ctx.timings()
        tb_seq += t["cg_setup"] + t["cg_iter"]
        ncg_seq.append(int(r["ncg"]))
    return {"candidates": nlam, "lams": [float(x) for x in lams],
            "jacobi": {"iterations": iters, "ncg": [int(x) for x in got["ncg"]],
                       "batched_ms": t_batch, "sequential_ms": t_seq,
                       "speedup": t_seq / t_batch if t_batch > 0 else None,
                       "batched_iteration_ms": t_iter / iters, "achieved_gbs": ach,
                       "form": "Jacobi (cgfac) CG per candidate (the reference's cjggra), exactly `iterations` "
                               "iterations, complex64 J read once per iteration for all candidates"},
            "block": {"ncg": [int(x) for x in gb["ncg"]], "ncg_sequential": ncg_seq,
                      "batched_ms": tb_batch, "sequential_ms": tb_seq,
                      "speedup": tb_seq / tb_batch if tb_batch > 0 else None, "cg_form": int(form_b),
                      "form": "block-preconditioned CG per candidate to rel-res 1e-6 (the GN step's solve): "
                              "one S factor per candidate, factors and sweeps on parallel streams, batched "
                              "matvecs"}}


def run_inversion(args, local):
    """The complete inversion of a synthetic survey through Inversion.run:
    forward at every trial model, Jacobian at every iterate, lambda search,
    step-length control, stop tests; wall time on the host around the whole
    loop (every device call in it is synchronous)."""
    from crtomo_stable_b200 import inversion
    s = make_problem(args.config)
    inv = inversion.synthetic_inversion(s, device=local, itmax=args.itmax)
    calls = {"forward": 0, "jacobian": 0, "update": 0}
    ctx = inv.ctx
    for name in calls:
        fn = getattr(ctx, name)

        def counted(*a, _fn=fn, _n=name, **k):
            calls[_n] += 1
            return _fn(*a, **k)
        setattr(ctx, name, counted)
    t0 = time.perf_counter()
    res = inv.run()
    wall = time.perf_counter() - t0
    rows = res["rows"]
    its = [r for r in rows if r["kind"] == "IT"]
    m = s.mesh
    print(json.dumps({
        "metric": "full GN inversion wall time", "value": round(wall, 3), "unit": "s", "impl": "ours",
        "higher_is_better": False, "n_gpus": 1, "data": "synthetic",
        "config": {"workload": f"{s.name}: {m.elanz} elements, {len(s.enr)} electrodes, {len(s.strnr)} readings, "
                               f"3 % + 0.1 mrad noise, homogeneous start, itmax {args.itmax}"},
        "stop_errnr": res["stop"], "iterations": res["it"], "rms_start": round(its[0]["rms"], 4),
        "rms_final": round(its[-1]["rms"], 4), "lambda_final": its[-1].get("lam"),
        "forwards": calls["forward"], "jacobians": calls["jacobian"], "updates": calls["update"],
        "cg_steps": int(sum(r.get("ncg", 0) for r in rows if r["kind"] in ("UP", "PUP"))),
        "rows": [{k: (round(v, 5) if isinstance(v, float) else v) for k, v in r.items()} for r in rows],
    }))
    inv.close()


def main():
    args = parse()
    ws, rank, local, pg = dist_init(args)
    if args.inversion:
        if rank == 0:
            run_inversion(args, local)
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()
        return
    if args.config == "C4" and args.impl == "ours":
        run_batch(args, ws, rank, local, pg)
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, ws, rank, pg)
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()
        return
    from crtomo_stable_b200.lib import (FORWARD_AUTO, FORWARD_DIRECT, PREC_FP64, PREC_MIXED, PRECOND_BLOCK,
                                        PRECOND_JACOBI, Context)
    s = make_problem(args.config)
    E, N = s.mesh.elanz, len(s.strnr)
    n, mb, L = s.mesh.sanz, s.mesh.mb, len(s.enr)
    names = ["factor", "solve", "volt", "jacobian", "cg_setup", "cg_iter"]
    tnames = Context.TIMING_NAMES

    def run_form(precision, steps, warmup, e2e_steps, sample_clocks, fwd_form=FORWARD_AUTO):
        ctx, dat, wmatd, par0, lam, nb, sm = setup_context(s, local, precision)
        ctx.set_forward_form(fwd_form)
        if args.refine is not None:
            ctx.set_refinement(args.refine)
        pc = PRECOND_BLOCK if precision == PREC_MIXED else PRECOND_JACOBI
        prm = Context.params(lam, eps=args.eps, ncgmax=args.ncgmax, precond=pc)
        ctx.set_model(par0)
        ctx.model_backup(restore=False)
        ncg = 0
        for _ in range(warmup):     # identical steps from the same starting model
            ctx.model_backup(restore=True)
            ncg = ctx.gn_step_device(prm)
        barrier(pg)
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
        launches0 = ctx.launch_count()
        phase = np.zeros(len(tnames))
        step_ms = []
        for _ in range(steps):
            ctx.model_backup(restore=True)
            ncg = ctx.gn_step_device(prm)
            t = ctx.timings()
            step_ms.append(t["total"])
            phase += np.array([t[k] for k in tnames])
        launches = (ctx.launch_count() - launches0) // max(steps, 1)
        barrier(pg)
        clocks = sampler.stop() if sampler else None
        t_step = max_over_ranks(pg, local, float(np.mean(step_ms)) / 1e3)
        phase /= max(steps, 1)
        e2e_ms = []
        for _ in range(e2e_steps):   # through crt_gn_step with host buffers
            p = par0.copy()
            t0 = time.perf_counter()
            ctx.gn_step(prm, p)
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
        t_e2e = max_over_ranks(pg, local, float(np.mean(e2e_ms)) / 1e3) if e2e_ms else None
        K = ctx.kwn.size
        form, blk, bw = ctx.cg_info()
        lam_batch = None
        if precision == PREC_MIXED and args.lambdas > 0:
            lam_batch = lambda_batch(ctx, Context, lam, par0, args.lambdas, args.lambda_iters, E, N, args.eps,
                                     args.ncgmax, PRECOND_BLOCK)
        finfo = ctx.forward_info()
        ctx.close()
        return dict(t=t_step, phase=phase, ncg=ncg, launches=int(launches), clocks=clocks, e2e=t_e2e, lam=lam, K=K,
                    finfo=finfo,
                    cg_form=form, cg_block=blk, cg_bw=bw, c64=precision == PREC_MIXED, lam_batch=lam_batch)

    mixed = run_form(PREC_MIXED, args.steps, args.warmup, args.steps, True)
    plain = None
    if args.forms == "both":
        # the reference's algorithm on the GPU: one FP64 band system per
        # wavenumber and electrode, the Jacobi-preconditioned CG
        plain = run_form(PREC_FP64, max(1, args.steps // 3), max(1, args.warmup // 3), 0, False, FORWARD_DIRECT)
    t_step, phase, ncg, K = mixed["t"], mixed["phase"], mixed["ncg"], mixed["K"]
    ph = dict(zip(tnames, [float(x) for x in phase]))
    h2d = E * 16
    d2h = E * 16 + N * 16 + (ncg + 1) * 8 + 8
    peak_gbs, peak_kind = load_peaks()
    sm_mhz = (mixed["clocks"] or {}).get("sm_max_mhz") or 1965.0
    # Rooflines of the forward's kernels.  In the Schur form (mixed
    # boundaries) every kernel computes in FP64 on the CUDA cores: the FP64
    # FMA pipe (64 FMA / clk / SM x 148 SMs at the max SM clock) is the peak
    # of each; achieved = algorithmic flops (schur_work: 8 per complex
    # multiply-add) / the kernel's CUDA-event time in the step.  The
    # dominant one (the longest) is the line's `roofline`.
    fp64_peak = FP64_FMA_PER_CLK_SM * 2 * 148 * sm_mhz * 1e6 / 1e12
    form_used, m_b, n_i, mb_i = mixed["finfo"]
    kernels = []
    if form_used == 2:
        w = schur_work(s, K, m_b, n_i, mb_i)
        it_mean = ph.get("schur_iter", 0.0)
        chol_label = ("k_schur_chol (dense Cholesky of every S_l, fused forward solve, back solve)" if it_mean == 0 else
                      "k_schur_s0 + k_schur_chol<REF> (a reference factor per 16 electrodes) + k_schur_iter "
                      "(preconditioned iteration per electrode, %.1f iterations)" % it_mean)
        if it_mean > 0:
            w["chol"] = w["chol_ref"] + it_mean * w["chol_it"]
        # the forward sweep runs beside the factor (second stream) unless
        # CRT_B200_SCHUR_OVERLAP=0: its span is the factor's time plus the
        # part after the factor (the `schur_forward` phase)
        overlap = os.environ.get("CRT_B200_SCHUR_OVERLAP", "1") != "0"
        fwd_label = ("k_schur_sweep (forward sweep of [F r_I | F A_IG], beside the factor: span from the factor's "
                     "start) + factor transpose" if overlap else
                     "k_schur_sweep (forward sweep of [F r_I | F A_IG]) + factor transpose")
        for name, key, label in (("factor", "factor_kernel", "k_band_factor_blk<cd> (interior band Cholesky, one system per wavenumber)"),
                                 ("forward", "schur_forward", fwd_label),
                                 ("gram", "schur_gram", "k_schur_gram (V^T [u^ | V^])"),
                                 ("chol", "schur_chol", chol_label),
                                 ("back", "schur_back", "k_schur_zrebuild + k_schur_sweep back + k_schur_out_gam")):
            t_ms = ph.get(key, 0.0)
            if name == "forward" and overlap:
                t_ms += ph.get("factor_kernel", 0.0)
            fl = 8.0 * w[name]
            ach = fl / (t_ms / 1e3) / 1e12 if t_ms > 0 else 0.0
            ent = {"kernel": label, "ms": t_ms, "flops": fl, "achieved": ach, "peak": fp64_peak,
                   "unit": "TFLOP/s", "frac": ach / fp64_peak}
            if name == "factor":
                # one CTA of 512 threads per wavenumber: K of the 148 SMs
                ent["sms_used"] = K
                ent["frac_of_used_sms"] = ach / (fp64_peak * K / 148.0)
                ent["note"] = ("a system per CTA: every row's pivot (complex square root and reciprocal, then the "
                               "update of the next diagonal entry) is a chain of dependent FP64 operations, about "
                               "1 us per row; the forward sweep runs beside it on the other SMs")
            kernels.append(ent)
    # the dominant kernel: the longest phase whose time is its own (the
    # overlapped sweep's span contains the factor)
    dom = max((k_ for k_ in kernels if "span" not in k_["kernel"]), key=lambda k_: k_["ms"]) if kernels else None
    roof = None
    if dom is not None:
        roof = {"kernel": dom["kernel"], "bound": "fp64", "achieved": dom["achieved"], "peak": fp64_peak,
                "unit": "TFLOP/s", "frac": dom["frac"], "traffic": None,
                "traffic_unit": "bytes per launch (ncu dram read + write)",
                "peak_source": ("FP64 FMA pipe, 64 FMA/clk/SM x 148 SMs at the max SM clock (the Schur kernels run "
                                "in FP64 on the CUDA cores; MEASURED_PEAKS.json holds HBM and bf16 tensor figures only)"),
                "algorithmic_flops_per_launch": dom["flops"], "launch_ms": dom["ms"], "launches": 1.0}
        for key in ("sms_used", "frac_of_used_sms", "note"):
            if key in dom:
                roof[key] = dom[key]
    roof_cg = None
    if ncg > 0:
        bytes_it = 2.0 * N * E * 8 + 6.0 * E * 16 + 3.0 * N * 16   # J (complex64) read twice + vectors
        ach_cg = bytes_it * ncg / (ph["cg_iter"] / 1e3) / 1e9
        roof_cg = {"kernel": "CG iteration (k_cg_jv + k_cg_jhv on the complex64 J, preconditioner apply)",
                   "bound": "hbm", "achieved": ach_cg, "peak": peak_gbs, "unit": "GB/s", "frac": ach_cg / peak_gbs,
                   "peak_source": peak_kind, "algorithmic_bytes_per_iteration": bytes_it}
    ref_ncg = plain["ncg"] if plain is not None else REF_NCG.get(args.config, ncg)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            nth = os.cpu_count() or 1
            info = cpu_sample(s, nth, ref_ncg)
            v = info["forward_s"] + info["jacobian_s"]
            cpu = {"value": v, "unit": "s", "cores": info["cores"], "kind": "port", "sample": info["sample"],
                   "extrapolated": True,
                   "value_covers": "forward + Jacobian of the GN step (the CG is projected apart)",
                   "phases_s": {"forward": info["forward_s"], "jacobian": info["jacobian_s"]},
                   "projected_cg_s": info["projected_cg_s"], "cg_iteration_s": info["cg_iteration_s"],
                   "scaling_check": validate_scaling(nth)}
        except Exception as exc:  # the baseline must not hide the GPU number
            cpu = {"value": None, "unit": "s", "cores": 0, "kind": "port", "sample": f"failed: {exc}"}
    if rank == 0:
        line = {"metric": METRIC, "value": t_step, "unit": "s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "c128/c64", "data": "synthetic (seeded)",
                "config": {"workload": workload_name(s, K),
                           "form": (("forward by elimination of the mixed-boundary nodes in FP64 (one interior band "
                                     "factorisation per wavenumber, dense Schur complement per electrode)"
                                     if mixed["finfo"][0] == 2 else
                                     "forward per band system: complex64 factorisation with adaptive FP64 refinement")
                                    + "; Jacobian formed in FP64, stored complex64; CG with FP64 accumulation and dots, "
                                    + ("preconditioned by cgfac and the block-tridiagonal S^-1 (FP32) of the sparse part"
                                       if mixed["cg_form"] == 1 else "diagonal-PCG (block preconditioner unavailable)")),
                           "plain_form": ("FP64 per band system (the reference's loop) and the reference's "
                                          "Jacobi-preconditioned CG, on the GPU"),
                           "cg_block": mixed["cg_block"], "cg_bandwidth": mixed["cg_bw"],
                           "cg_iterations": ncg, "lam": mixed["lam"],
                           "l2": "inputs larger than L2 (J alone is %.1f GB in complex64)" % (N * E * 8 / 1e9),
                           "parallelism": f"replicas x{ws}"},
                "phases_ms": ph,
                "plain_fp64": None if plain is None else
                {"value": plain["t"], "unit": "s", "cg_iterations": plain["ncg"],
                 "phases_ms": dict(zip(tnames, [float(x) for x in plain["phase"]]))},
                "e2e": {"value": mixed["e2e"], "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "roofline": roof, "kernels_forward": kernels, "roofline_cg": roof_cg, "lambda_batch": mixed["lam_batch"],
                "cpu_baseline": cpu, "clocks": mixed["clocks"],
                "gpu_launches": mixed["launches"]}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
