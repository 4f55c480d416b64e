"""Regularisation operator set-up (host, FP64, once per inversion).

* ``nachbar``   -- edge neighbours of every area element (src/bnachbar.f90:
  52-90: element j is neighbour k of element i when it shares the edge
  (node k, node k+1 mod n) in either orientation).  The reference scans all
  element pairs; here edges are matched through a sort, which gives the same
  table for any conforming mesh.
* ``smatm_tri`` -- src/bsmatm_mod.f90:364-460 (ltri = 1/2).
* ``smatm_reg`` -- src/bsmatm_mod.f90:190-362 (ltri = 0, regular nx x nz grid).
"""
from __future__ import annotations

import numpy as np


def nachbar(mesh) -> np.ndarray:
    E, n = mesh.elanz, mesh.maxnodes
    nodes = np.asarray(mesh.nrel[:E, :n], dtype=np.int64)
    nxt = np.roll(nodes, -1, axis=1)
    a = np.minimum(nodes, nxt).ravel()
    b = np.maximum(nodes, nxt).ravel()
    elem = np.repeat(np.arange(E), n)
    slot = np.tile(np.arange(n), E)
    key = a * (int(mesh.sanz) + 1) + b
    order = np.lexsort((elem, key))
    ks = key[order]
    nb = np.zeros((E, n + 1), dtype=np.int32, order="F")
    same = np.nonzero(ks[1:] == ks[:-1])[0]
    for pos in same:
        i0, i1 = order[pos], order[pos + 1]
        e0, e1 = elem[i0], elem[i1]
        if e0 == e1:
            continue
        nb[e0, slot[i0]] = e1 + 1
        nb[e1, slot[i1]] = e0 + 1
    nb[:, n] = np.count_nonzero(nb[:, :n], axis=1)
    return nb


def smatm_tri(mesh, nb: np.ndarray, alfx: float, alfz: float) -> np.ndarray:
    E, n = mesh.elanz, mesh.maxnodes
    espx, espy = mesh.midpoints()
    nodes = np.asarray(mesh.nrel[:E, :n])
    x, y = mesh.node_xy(nodes)
    xn, yn = np.roll(x, -1, axis=1), np.roll(y, -1, axis=1)
    edglen = np.sqrt((x - xn) * (x - xn) + (y - yn) * (y - yn))
    sm = np.zeros((E, n + 1), dtype=np.float64, order="F")
    for k in range(n):
        j = nb[:, k]
        has = j > 0
        jj = np.where(has, j - 1, 0)
        dx = espx - espx[jj]
        dy = espy - espy[jj]
        dist = np.sqrt(dx * dx + dy * dy)
        ang = np.arctan2(dy, dx)
        cx = alfx * np.cos(ang)
        sz = alfz * np.sin(ang)
        alfgeo = np.sqrt(cx * cx + sz * sz)
        with np.errstate(divide="ignore", invalid="ignore"):
            rs = edglen[:, k] / dist * alfgeo
        sm[:, k] = np.where(has, -rs, 0.0)
        sm[:, n] = sm[:, n] + np.where(has, rs, 0.0)
    return sm


def smatm_reg(mesh, nx: int, nz: int, alfx: float, alfz: float) -> np.ndarray:
    manz = nx * nz
    nodes = np.asarray(mesh.nrel[:manz, :4])
    x, y = mesh.node_xy(nodes)
    xm = (((x[:, 0] + x[:, 1]) + x[:, 2]) + x[:, 3]) / 4.0
    zm = (((y[:, 0] + y[:, 1]) + y[:, 2]) + y[:, 3]) / 4.0
    sm = np.zeros((manz, 3), dtype=np.float64, order="F")
    idx = np.arange(manz)
    i = idx // nx   # row (z)
    j = idx % nx    # column (x)
    dzleft = np.abs(y[:, 3] - y[:, 0])
    dzright = np.abs(y[:, 2] - y[:, 1])
    dxup = np.abs(x[:, 2] - x[:, 3])
    dxdown = np.abs(x[:, 1] - x[:, 0])
    left = j > 0
    d = np.where(left, alfx * dzleft / np.abs(xm - np.where(left, xm[idx - 1], 1.0 + xm)), 0.0)
    sm[:, 0] = d
    right = j < nx - 1
    jr = np.where(right, idx + 1, idx)
    dum = np.where(right, alfx * dzright / np.abs(np.where(right, xm[jr], xm + 1.0) - xm), 0.0)
    sm[:, 0] = sm[:, 0] + dum
    sm[:, 1] = np.where(right, -dum, 0.0)
    up = i > 0
    iu = np.where(up, idx - nx, idx)
    dum = np.where(up, alfz * dxup / np.abs(np.where(up, zm[iu], zm + 1.0) - zm), 0.0)
    sm[:, 0] = sm[:, 0] + dum
    down = i < nz - 1
    idn = np.where(down, idx + nx, idx)
    dum = np.where(down, alfz * dxdown / np.abs(zm - np.where(down, zm[idn], zm + 1.0)), 0.0)
    sm[:, 0] = sm[:, 0] + dum
    sm[:, 2] = np.where(down, -dum, 0.0)
    return sm
