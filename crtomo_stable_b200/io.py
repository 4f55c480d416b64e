"""Readers and writers for the CRMod / CRTomo tomodir file formats.

The formats are kept exactly as the reference reads and writes them, so a
tomodir prepared for the Fortran programs works unchanged:

* ``elem.dat``   -- src/relem.f90:62-151 (+ the border-element fix-up of
  src/relem.f90:163-252, "check 2", which rewrites ``rnr`` in memory)
* ``elec.dat``   -- src/relectr.f90:46-68
* ``rho.dat``    -- src/rsigma.f90:74-115 (magnitude in Ohm m, phase in mrad)
* ``config.dat`` -- src/rdatm.f90:45-84 (``C1*10000+C2 P1*10000+P2`` or four
  electrode columns)
* ``volt.dat``   -- written by src/wdatm.f90:55-79, read by src/rdati.f90
* ``crmod.cfg``  -- src/fem.f90:163-184
* ``crtomo.cfg`` -- src/rall.f90:234-472

Arrays follow the Fortran layout that the C ABI receives: ``nrel`` is
``(elanz+relanz, maxnodes)`` column-major with 1-based node numbers.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional

import numpy as np


def _tokens(line: str) -> List[str]:
    return line.replace(",", " ").split()


def _fortran_bool(tok: str) -> bool:
    t = tok.strip().lstrip(".").upper()
    if t.startswith("T"):
        return True
    if t.startswith("F"):
        return False
    raise ValueError(f"not a Fortran logical: {tok!r}")


def _ffloat(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "e"))


@dataclasses.dataclass
class Mesh:
    """elemmod state (src/elemmod.f90)."""

    sanz: int
    typanz: int
    mb: int
    typ: np.ndarray        # int32 [typanz]
    nelanz: np.ndarray     # int32 [typanz]
    selanz: np.ndarray     # int32 [typanz]
    snr: np.ndarray        # int32 [sanz]
    sx: np.ndarray         # f64 [sanz]
    sy: np.ndarray         # f64 [sanz]
    nrel: np.ndarray       # int32 Fortran-ordered (elanz+relanz, maxnodes)
    rnr: np.ndarray        # int32 [relanz]

    @property
    def elanz(self) -> int:
        return int(sum(int(n) for t, n in zip(self.typ, self.nelanz) if t <= 10))

    @property
    def relanz(self) -> int:
        return int(sum(int(n) for t, n in zip(self.typ, self.nelanz) if t > 10))

    @property
    def maxnodes(self) -> int:
        return int(max(self.selanz))

    def node_xy(self, node: np.ndarray):
        """Coordinates of 1-based node numbers (sx(snr(node)))."""
        idx = self.snr[np.asarray(node) - 1] - 1
        return self.sx[idx], self.sy[idx]

    def area_nodes(self) -> np.ndarray:
        """(elanz, maxnodes) 1-based node numbers of the area elements."""
        return np.asarray(self.nrel[: self.elanz, :])

    def element_types(self) -> np.ndarray:
        """Type of every element (area and boundary), in file order."""
        return np.repeat(self.typ, self.nelanz).astype(np.int32)

    def midpoints(self):
        """espx/espy as src/relem.f90 computes them (area elements)."""
        out_x = np.zeros(self.elanz)
        out_y = np.zeros(self.elanz)
        start = 0
        for t, n, s in zip(self.typ, self.nelanz, self.selanz):
            if t < 10:
                nodes = self.nrel[start:start + n, :s]
                x, y = self.node_xy(nodes)
                # same summation order as the reference (k = 1..selanz)
                sxs = np.zeros(n)
                sys_ = np.zeros(n)
                for k in range(s):
                    sxs = sxs + x[:, k]
                    sys_ = sys_ + y[:, k]
                out_x[start:start + n] = sxs / s
                out_y[start:start + n] = sys_ / s
            start += n
        return out_x, out_y


def read_elem(path: str, fix_borders: bool = True) -> Mesh:
    """Read ``elem.dat`` (src/relem.f90:62-151)."""
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines()]
    pos = 0

    def next_line():
        nonlocal pos
        while pos < len(lines) and not lines[pos].strip():
            pos += 1
        if pos >= len(lines):
            raise EOFError(f"{path}: unexpected end of file")
        ln = lines[pos]
        pos += 1
        return _tokens(ln)

    h = next_line()
    sanz, typanz, mb = int(h[0]), int(h[1]), int(h[2])
    typ, nel, sel = [], [], []
    for _ in range(typanz):
        t = next_line()
        typ.append(int(t[0]))
        nel.append(int(t[1]))
        sel.append(int(t[2]))
    # one READ for all node triples: values may span lines arbitrarily
    vals: List[str] = []
    while len(vals) < 3 * sanz:
        vals.extend(next_line())
    arr = np.array([_ffloat(v) for v in vals[: 3 * sanz]]).reshape(sanz, 3)
    snr = arr[:, 0].astype(np.int32)
    sx = arr[:, 1].copy()
    sy = arr[:, 2].copy()
    maxnodes = max(sel)
    ntot = sum(nel)
    nrel = np.zeros((ntot, maxnodes), dtype=np.int32, order="F")
    row = 0
    for t, n, s in zip(typ, nel, sel):
        for _ in range(n):
            toks = next_line()
            while len(toks) < s:
                toks = toks + next_line()
            nrel[row, :s] = [int(v) for v in toks[:s]]
            row += 1
    relanz = sum(n for t, n in zip(typ, nel) if t > 10)
    rvals: List[str] = []
    while len(rvals) < relanz:
        rvals.extend(next_line())
    rnr = np.array([int(v) for v in rvals[:relanz]], dtype=np.int32)
    mesh = Mesh(sanz, typanz, mb, np.array(typ, np.int32), np.array(nel, np.int32),
                np.array(sel, np.int32), snr, sx, sy, nrel, rnr)
    if fix_borders and relanz > 0:
        _fix_border_elements(mesh)
    return mesh


def _fix_border_elements(mesh: Mesh) -> None:
    """"check 2" of src/relem.f90:190-216: every border segment is attached
    to the area element that contains both of its nodes."""
    elanz = mesh.elanz
    s1 = int(mesh.selanz[0])
    area = np.asarray(mesh.nrel[:elanz, :s1])
    # node -> elements map
    node_elems = {}
    for e in range(elanz):
        for nd in area[e]:
            node_elems.setdefault(int(nd), set()).add(e + 1)
    for i in range(mesh.relanz):
        ik1 = int(mesh.nrel[elanz + i, 0])
        ik2 = int(mesh.nrel[elanz + i, 1])
        both = node_elems.get(ik1, set()) & node_elems.get(ik2, set())
        # the reference scans k = 1..elanz and keeps the last matching k
        for k in sorted(both):
            if mesh.rnr[i] != k:
                mesh.rnr[i] = k
    bad = np.count_nonzero((mesh.rnr < 1) | (mesh.rnr > elanz))
    if bad:
        raise ValueError("border to element context is wrong (errnr 111)")


def write_elem(path: str, mesh: Mesh) -> None:
    """Write ``elem.dat`` in the layout relem reads."""
    with open(path, "w") as fh:
        fh.write(f"{mesh.sanz:12d}{mesh.typanz:12d}{mesh.mb:12d}\n")
        for t, n, s in zip(mesh.typ, mesh.nelanz, mesh.selanz):
            fh.write(f"{int(t):12d}{int(n):12d}{int(s):12d}\n")
        for i in range(mesh.sanz):
            fh.write(f"{int(mesh.snr[i]):9d} {mesh.sx[i]:.10g} {mesh.sy[i]:.10g}\n")
        row = 0
        for t, n, s in zip(mesh.typ, mesh.nelanz, mesh.selanz):
            for _ in range(n):
                fh.write(" ".join(f"{int(v):9d}" for v in mesh.nrel[row, :s]) + "\n")
                row += 1
        for v in mesh.rnr:
            fh.write(f"{int(v):9d}\n")


def read_elec(path: str) -> np.ndarray:
    """``elec.dat`` (src/relectr.f90:46-68): eanz, then one node per line."""
    with open(path) as fh:
        toks = fh.read().split()
    eanz = int(toks[0])
    return np.array([int(t) for t in toks[1:1 + eanz]], dtype=np.int32)


def write_elec(path: str, enr: np.ndarray) -> None:
    with open(path, "w") as fh:
        fh.write(f"{len(enr):12d}\n")
        for v in enr:
            fh.write(f"{int(v):12d}\n")


def read_rho(path: str, elanz: Optional[int] = None) -> np.ndarray:
    """``rho.dat`` -> complex conductivities sigma (src/rsigma.f90:80-115):
    sigma = (cos(phi)/|rho|, -sin(phi)/|rho|), phi in mrad."""
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines() if ln.strip()]
    n = int(_tokens(lines[0])[0])
    if elanz is not None and n != elanz:
        raise ValueError(f"{path}: {n} values for {elanz} elements")
    sig = np.zeros(n, dtype=np.complex128)
    for i in range(n):
        t = _tokens(lines[1 + i])
        bet = _ffloat(t[0])
        pha = 1e-3 * _ffloat(t[1]) if len(t) > 1 else 0.0
        if bet < 1e-12:
            raise ValueError(f"{path}: resistivity {bet} too small (errnr 11)")
        sig[i] = complex(math.cos(pha) / bet, -math.sin(pha) / bet)
    return sig


def write_rho(path: str, sigma: np.ndarray) -> None:
    rho = 1.0 / np.asarray(sigma)
    with open(path, "w") as fh:
        fh.write(f"{len(rho):12d}\n")
        for r in rho:
            fh.write(f"{abs(r):.10g} {1e3 * math.atan2(r.imag, r.real):.10g}\n")


def _decode_configs(rows):
    """rows of ints -> (strnr, vnr); crtf rule of src/rdatm.f90:51-53."""
    first = rows[0][0]
    crtf = (first - 10000) >= 0
    strnr, vnr = [], []
    for r in rows:
        if crtf:
            strnr.append(int(r[0]))
            vnr.append(int(r[1]))
        else:
            strnr.append(int(r[0]) * 10000 + int(r[1]))
            vnr.append(int(r[2]) * 10000 + int(r[3]))
    return np.array(strnr, np.int32), np.array(vnr, np.int32), crtf


def check_configs(strnr, vnr, eanz: int) -> None:
    """Electrode-number checks of src/rdatm.f90:67-84 (errnr 46 / 73)."""
    for i, (s, v) in enumerate(zip(strnr, vnr)):
        e1, e2 = int(s) % 10000, int(s) // 10000
        e3, e4 = int(v) % 10000, int(v) // 10000
        if min(e1, e2, e3, e4) < 0 or max(e1, e2, e3, e4) > eanz:
            raise ValueError(f"Electrode pair {i + 1} not correct (errnr 46)")
        if (e1 == e2 or e3 == e4 or (((e1 == e3) or (e1 == e4)) and e1 != 0)
                or (((e2 == e3) or (e2 == e4)) and e2 != 0)):
            raise ValueError(f"duplicate electrodes for reading {i + 1} (errnr 73)")


def read_config(path: str):
    """``config.dat`` -> (strnr, vnr)."""
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines() if ln.strip()]
    n = int(_tokens(lines[0])[0])
    rows = [[int(float(x)) for x in _tokens(lines[1 + i])] for i in range(n)]
    s, v, _ = _decode_configs(rows)
    return s, v


def write_config(path: str, strnr, vnr) -> None:
    with open(path, "w") as fh:
        fh.write(f"{len(strnr):12d}\n")
        for s, v in zip(strnr, vnr):
            fh.write(f"{int(s):12d}{int(v):12d}\n")


@dataclasses.dataclass
class Data:
    strnr: np.ndarray
    vnr: np.ndarray
    bet: np.ndarray            # |R| (Ohm)
    pha: np.ndarray            # phase (mrad)
    stabw: Optional[np.ndarray] = None   # individual errors (lindiv)
    stabwp: Optional[np.ndarray] = None


def read_volt(path: str) -> Data:
    """``volt.dat`` as rdati reads it (src/rdati.f90:71-245)."""
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines() if ln.strip()]
    head = _tokens(lines[0])
    n = int(head[0])
    lindiv = len(head) > 1 and _fortran_bool(head[1])
    rows = [_tokens(lines[1 + i]) for i in range(n)]
    ints = [[int(float(x)) for x in r[:4]] for r in rows]
    first = ints[0][0]
    crtf = (first - 10000) >= 0
    ncfg = 2 if crtf else 4
    s, v, _ = _decode_configs(ints)
    bet = np.array([_ffloat(r[ncfg]) for r in rows])
    pha = np.array([_ffloat(r[ncfg + 1]) if len(r) > ncfg + 1 else 0.0 for r in rows])
    d = Data(s, v, bet, pha)
    if lindiv:
        d.stabw = np.array([_ffloat(r[ncfg + 2]) for r in rows])
        d.stabwp = np.array([_ffloat(r[ncfg + 3]) if len(r) > ncfg + 3 else 0.0 for r in rows])
    return d


def write_volt(path: str, strnr, vnr, sigmaa: np.ndarray) -> np.ndarray:
    """wdatm (src/wdatm.f90:55-79): ``|sigmaa|`` and phase in mrad as
    float32, flipping the voltage-electrode order when the phase is near
    +-pi.  Returns the (possibly flipped) vnr."""
    vnr_out = np.array(vnr, dtype=np.int64).copy()
    pi = math.acos(-1.0)
    with open(path, "w") as fh:
        fh.write(f"{len(strnr):12d}\n")
        for i, z in enumerate(np.asarray(sigmaa)):
            bet = abs(z)
            pha = math.atan2(z.imag, z.real)
            q = pha / pi   # dnint: round half away from zero
            npi = math.copysign(math.floor(abs(q) + 0.5), q) * pi
            if abs(npi) > 1e-12:
                pha = pha - npi
                ie1 = int(vnr_out[i]) % 10000
                ie2 = (int(vnr_out[i]) - ie1) // 10000
                vnr_out[i] = ie1 * 10000 + ie2
            fh.write(f"{int(strnr[i]):12d}{int(vnr_out[i]):12d}"
                     f"{float(np.float32(bet)):16.8E}{float(np.float32(1e3 * pha)):16.8E}\n")
    return vnr_out


@dataclasses.dataclass
class CRModConfig:
    """crmod.cfg (src/fem.f90:163-184)."""

    elem: str
    elec: str
    rho: str
    config: str
    lpot: bool
    pot: str
    lvolt: bool
    volt: str
    lsens: bool
    sens: str
    lagain: bool
    swrtr: int
    lsink: bool
    nsink: int
    lrandb2: bool
    randb: str
    mswitch: int = 0


def read_crmod_cfg(path: str) -> CRModConfig:
    with open(path) as fh:
        lines = fh.read().splitlines()
    it = iter(lines)
    next(it)  # ***FILES***

    def s():
        return next(it).split("!")[0].strip()

    elem, elec, rho, cfg = s(), s(), s(), s()
    lpot = _fortran_bool(s())
    pot = s()
    lvolt = _fortran_bool(s())
    volt = s()
    lsens = _fortran_bool(s())
    sens = s()
    lagain = _fortran_bool(s())
    swrtr = int(s().split()[0])
    lsink = _fortran_bool(s())
    nsink = int(s().split()[0])
    lrandb2 = _fortran_bool(s())
    randb = s()
    mswitch = 0
    try:
        mswitch = int(s().split()[0])
    except (StopIteration, ValueError, IndexError):
        pass
    return CRModConfig(elem, elec, rho, cfg, lpot, pot, lvolt, volt, lsens, sens,
                       lagain, swrtr, lsink, nsink, lrandb2, randb, mswitch)


def resolve(base_dir: str, rel: str) -> str:
    return rel if os.path.isabs(rel) else os.path.normpath(os.path.join(base_dir, rel))
