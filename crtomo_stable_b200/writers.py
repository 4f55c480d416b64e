"""Output files of the CRTomo / CRMod drivers, in the reference's layouts.

* wout (src/wout.f90:30-165): per written iterate rhoNN.mag (log10 |rho|),
  rhoNN.modl (1/Re(sigma), phase), rhoNN.pha and rhoNN.sig (complex runs)
  and voltNN.dat (|R|, phase, wdfak);
* bbsens (src/bbsens.f90:52-110): coverage.mag (log10 of the normalised
  column sums of |J| w) and coverage.mag_fpi in the final phase improvement;
* kont2 (src/kont2.f90:35-128): the IT / UP / PIT / PUP rows of inv.ctr;
* wsens (src/wsens.f90:30-80) and wpot / bpot (src/wpot.f90, src/bpot.f90):
  CRMod's per-reading sensitivity and potential files.

Numbers are written the way the reference's Fortran writes them: list-
directed REAL(4) with 9 and REAL(8) with 17 significant digits, explicit
G / F / I edit descriptors where the reference gives them.  Readers of these
files split on blanks, so the spacing between fields is not reproduced
byte for byte.
"""
from __future__ import annotations

import math
import os
from typing import Iterable, Optional, Sequence

import numpy as np


# -- Fortran edit descriptors --------------------------------------------------
def _neg(v: float) -> bool:
    return math.copysign(1.0, v) < 0.0


def _fixed(a: float, dec: int) -> str:
    """Fd editing of a magnitude (Fortran keeps the point at d = 0)."""
    return f"{a:.{dec}f}" + ("." if dec == 0 else "")


def fortran_g(v: float, w: int, d: int) -> str:
    """Gw.d output editing: F(w-4).(d-k) and four blanks where the rounded
    magnitude is within [0.1, 10**d), else Ew.d (0.ddddE+ee)."""
    v = float(v)
    if not math.isfinite(v):
        return ("NaN" if math.isnan(v) else ("-Infinity" if v < 0 else "Infinity")).rjust(w)
    a = abs(v)
    sign = "-" if _neg(v) else ""
    if a == 0.0:
        return (sign + f"{0.0:.{d - 1}f}").rjust(w - 4) + "    "
    k = int(f"{a:.{d - 1}e}".split("e")[1]) + 1          # 10**(k-1) <= rounded a < 10**k
    if 0 <= k <= d:
        return (sign + _fixed(a, d - k)).rjust(w - 4) + "    "
    m = f"{a:.{d - 1}e}"                                    # d.ddd e+xx, same rounding
    digits = m.split("e")[0].replace(".", "")
    return (sign + "0." + digits + f"E{k:+03d}").rjust(w)


def fortran_f(v: float, w: int, d: int) -> str:
    return f"{float(v):{w}.{d}f}"


def _ld_real(v: float, sig: int) -> str:
    """A list-directed REAL item: F form with `sig` significant digits in
    [0.1, 10**sig), E form otherwise."""
    v = float(v)
    if not math.isfinite(v):
        return " " + ("NaN" if math.isnan(v) else ("-Infinity" if v < 0 else "Infinity"))
    a = abs(v)
    sign = "-" if _neg(v) else " "
    if a == 0.0:
        return "  " + sign.strip() + f"{0.0:.{sig - 1}f}" + "    "
    m = f"{a:.{sig - 1}e}"
    k = int(m.split("e")[1]) + 1
    if 0 <= k <= sig:
        return " " + sign + _fixed(a, sig - k) + "    "
    mant, ex = m.split("e")
    return " " + sign + mant + f"E{int(ex):+03d}"


def ld_r4(v) -> str:
    return _ld_real(float(np.float32(v)), 9)


def ld_r8(v) -> str:
    return _ld_real(float(v), 17)


def ld_i(v) -> str:
    return f"{int(v):12d}"


# -- wout ---------------------------------------------------------------------
def write_model(inv_dir: str, it: int, espx, espy, sigma, betrms: float, pharms: float, ldc: bool) -> list:
    """rhoNN.mag / .modl (and .pha / .sig for complex runs) of src/wout.f90:
    log10 |1/sigma|, 1/Re(sigma) with the phase of 1/sigma in mrad (G12.4),
    the phase, and Re / Im of sigma."""
    sig = np.asarray(sigma, np.complex128)
    rho = 1.0 / sig
    base = os.path.join(inv_dir, f"rho{it:02d}")
    paths = []
    with open(base + ".mag", "w") as fh:
        fh.write(f"{ld_i(len(sig))} \t{ld_r8(betrms)}\n")
        for x, y, r in zip(espx, espy, rho):
            fh.write(f"{ld_r4(x)}{ld_r4(y)}{ld_r4(math.log10(abs(r)))}\n")
    paths.append(base + ".mag")
    with open(base + ".modl", "w") as fh:
        fh.write(f"{len(sig):7d}\n")
        for s_, r in zip(sig, rho):
            ph = float(np.float32(1e3 * math.atan2(r.imag, r.real)))
            fh.write(" " + fortran_g(float(np.float32(1.0) / np.float32(s_.real)), 12, 4) + " "
                     + fortran_g(ph, 12, 4) + "\n")
    paths.append(base + ".modl")
    if not ldc:
        with open(base + ".pha", "w") as fh:
            fh.write(f"{ld_i(len(sig))} \t{ld_r8(pharms)}\n")
            for x, y, r in zip(espx, espy, rho):
                fh.write(f"{ld_r4(x)}{ld_r4(y)}{ld_r4(1e3 * math.atan2(r.imag, r.real))}\n")
        paths.append(base + ".pha")
        with open(base + ".sig", "w") as fh:
            fh.write(f"{ld_i(len(sig))}{ld_r8(betrms)}{ld_r8(pharms)}\n")
            for s_ in sig:
                fh.write(f"{ld_r4(s_.real)}{ld_r4(s_.imag)}\n")
        paths.append(base + ".sig")
    return paths


def write_volt_iterate(inv_dir: str, it: int, strnr, vnr, sigmaa, wdfak, ldc: bool) -> str:
    """voltNN.dat of src/wout.f90:140-160: |R| = exp(-Re sigmaa) and the
    phase -1000 Im sigmaa (REAL(4)), and wdfak."""
    path = os.path.join(inv_dir, f"volt{it:02d}.dat")
    sa = np.asarray(sigmaa, np.complex128)
    with open(path, "w") as fh:
        fh.write(ld_i(len(sa)) + "\n")
        for s, v, z, w in zip(strnr, vnr, sa, wdfak):
            row = f"{ld_i(s)}{ld_i(v)}{ld_r4(1.0 / math.exp(z.real))}"
            if not ldc:
                row += ld_r4(-1e3 * z.imag)
            fh.write(row + ld_i(w) + "\n")
    return path


# -- bbsens -------------------------------------------------------------------
def write_coverage(path: str, espx, espy, csens, csens_fpi=None) -> list:
    """coverage.mag (src/bbsens.f90:80-95): manz and max(csens), then
    log10(csens / max) per cell; with csens_fpi also coverage.mag_fpi."""
    out = []
    cmax = float(np.max(csens))
    with open(path, "w") as fh:
        fh.write(f"{ld_i(len(csens))}{ld_r8(cmax)}\n")
        for x, y, c in zip(espx, espy, csens):
            fh.write(f"{ld_r8(x)}{ld_r8(y)}{ld_r8(math.log10(c / cmax) if c > 0 else -math.inf)}\n")
    out.append(path)
    if csens_fpi is not None:
        fmax = float(np.max(csens_fpi))
        with open(path + "_fpi", "w") as fh:
            fh.write(ld_i(len(csens_fpi)) + "\n")
            for x, y, c in zip(espx, espy, csens_fpi):
                fh.write(f"{ld_r8(x)}{ld_r8(y)}{ld_r8(math.log10(c / fmax) if c > 0 else -math.inf)}\n")
            fh.write(f" Max:{ld_r8(fmax)}\n")
        out.append(path + "_fpi")
    return out


def bbsens_weights(wmatd, wmatdr, wmatd_cri, wdfak, lfpi: bool, lelerr: bool):
    """The per-reading weights of src/bbsens.f90:52-70: (w, w_fpi), w_fpi
    None outside the final phase improvement."""
    wdfak = np.asarray(wdfak, np.float64)
    if not lfpi:
        return np.sqrt(np.asarray(wmatd)) * wdfak, None
    w = np.sqrt(np.asarray(wmatd_cri if lelerr else wmatdr)) * wdfak
    return w, np.sqrt(np.asarray(wmatd)) * wdfak


# -- kont2 --------------------------------------------------------------------
STARS = "*" * 109 + " "


def _tab_line(fields: Sequence) -> str:
    """Fields (1-based column, text) placed as Fortran's Tn descriptors do."""
    line = ""
    for col, text in fields:
        if len(line) < col - 1:
            line += " " * (col - 1 - len(line))
        line = line[: col - 1] + text
    return line


def kont2_line(r: dict) -> str:
    """One row of inv.ctr in formats 101 / 111 / 105 of src/kont2.f90."""
    kind = f"{r['kind']:>3s}"
    if "step" not in r:      # starting row (format 101)
        return _tab_line([(1, kind), (5, f"{r['it']:3d}"), (11, fortran_g(r["rms"], 10, 4)),
                          (69, fortran_g(r["betrms"], 10, 4)), (81, fortran_g(r["pharms"], 10, 4)),
                          (93, f"{r['npol']:4d}")])
    if "betrms" in r:        # accepted iterate (format 111)
        return _tab_line([(1, kind), (5, f"{r['it']:3d}"), (11, fortran_g(r["rms"], 10, 4)),
                          (23, fortran_g(r["step"], 10, 4)), (34, fortran_g(r["lam"], 10, 4)),
                          (46, fortran_g(r["rough"], 10, 4)), (58, f"{r['ncg']:6d}"),
                          (69, fortran_g(r["betrms"], 10, 4)), (81, fortran_g(r["pharms"], 10, 4)),
                          (93, f"{r['npol']:4d}"), (105, fortran_f(r["steplength"], 5, 3))])
    return _tab_line([(1, kind), (5, f"{r['it']:3d}"), (11, fortran_g(r["rms"], 10, 4)),
                      (23, fortran_g(r["step"], 9, 3)), (34, fortran_g(r["lam"], 10, 4)),
                      (46, fortran_g(r["rough"], 10, 4)), (58, f"{r['ncg']:6d}"),
                      (105, fortran_f(r["steplength"], 5, 3))])


def write_inv_ctr_rows(path: str, rows: Iterable[dict], events: Optional[dict] = None) -> str:
    """The trajectory part of inv.ctr: starting and accepted rows between
    star lines, trial rows plain, the final phase improvement's separator
    and phase-model reset notes before the row index they precede."""
    events = events or {}
    with open(path, "a") as fh:
        for i, r in enumerate(rows):
            for ev in events.get(i, ()):
                if ev == "FPI":
                    fh.write("\n" + "-" * 113 + "\n\n")
                elif ev == "RESET":
                    fh.write("  ******* Resetting phase model ********\n")
            boxed = "step" not in r or "betrms" in r
            if boxed:
                fh.write(STARS + "\n")
            fh.write(kont2_line(r) + "\n")
            if boxed:
                fh.write(STARS + "\n")
        fh.write("***finished***\n")
    return path


# -- CRMod outputs ----------------------------------------------------------------
def numbered_path(pattern: str, i: int, ndig: int) -> str:
    """src/wsens.f90 / src/wpot.f90 file names: the pattern's stem with the
    reading number, zero-padded to ndig = int(log10(nanz)) + 1 digits."""
    d, f = os.path.split(pattern)
    stem, ext = os.path.splitext(f)
    return os.path.join(d, f"{stem}{i:0{ndig}d}{ext}")


def write_sensitivities(pattern: str, sens: np.ndarray, espx, espy) -> list:
    """wsens: per reading i, |sum_j J_ij| and its phase in mrad, then
    (espx, espy, Re J_ij, Im J_ij) per cell."""
    nanz = sens.shape[0]
    ndig = int(math.log10(float(np.float32(nanz)))) + 1
    paths = []
    for i in range(nanz):
        p = numbered_path(pattern, i + 1, ndig)
        row = np.asarray(sens[i])
        summe = complex(np.sum(row))
        with open(p, "w") as fh:
            if abs(summe) > 0.0:
                fh.write(f"{ld_r4(abs(summe))}{ld_r4(1e3 * math.atan2(summe.imag, summe.real))}\n")
            else:
                fh.write(f"{ld_r4(0.0)}{ld_r4(0.0)}\n")
            for x, y, z in zip(espx, espy, row):
                fh.write(f"{ld_r4(x)}{ld_r4(y)}{ld_r4(z.real)}{ld_r4(z.imag)}\n")
        paths.append(p)
    return paths


def write_potentials(pattern: str, hpot: np.ndarray, strnr, node_x, node_y, strom=None) -> list:
    """bpot + wpot: per reading i the potential of its current dipole,
    (hpot[:, e2] - hpot[:, e1]) * strom_i, as (x, y, Re, Im) per node."""
    nanz = len(strnr)
    ndig = int(math.log10(float(np.float32(nanz)))) + 1
    strom = np.ones(nanz) if strom is None else np.asarray(strom, np.float64)
    paths = []
    for i, s in enumerate(strnr):
        e1, e2 = int(s) % 10000, int(s) // 10000
        pot = np.zeros(hpot.shape[0], np.complex128)
        if e2 > 0:
            pot += hpot[:, e2 - 1]
        if e1 > 0:
            pot -= hpot[:, e1 - 1]
        pot *= strom[i]
        p = numbered_path(pattern, i + 1, ndig)
        with open(p, "w") as fh:
            for x, y, z in zip(node_x, node_y, pot):
                fh.write(f"{ld_r4(x)}{ld_r4(y)}{ld_r4(z.real)}{ld_r4(z.imag)}\n")
        paths.append(p)
    return paths
