"""Seeded synthetic tomodirs for the benchmark configurations.

The reference ships no benchmark inputs; these generators build structured
meshes in the reference's conventions (src/relem.f90, src/elem3.f90,
src/elem8.f90):

* area elements counter-clockwise, listed row by row from the surface
  (x fastest), so the regular-grid regulariser (src/bsmatm_mod.f90:190-362,
  element k(i, j) = (i-1) nx + j) applies to quadrilateral grids;
* nodes numbered column by column, depth fastest, which gives the band
  width (nz + 1 for quadrilaterals and split quadrilaterals) a Cuthill-McKee
  ordering of such a grid reaches;
* boundary segments traversed clockwise around the domain, the orientation
  whose normal src/beta.f90 treats as outward: the surface as no-flow
  (type 12), sides and bottom as mixed boundaries (type 11), each with the
  area element it borders (rnr).

Seeds follow 20261203 + configuration number.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Tuple

import numpy as np

from .io import Mesh

SEED0 = 20261203


@dataclasses.dataclass
class Survey:
    mesh: Mesh
    enr: np.ndarray            # electrode nodes (1-based)
    strnr: np.ndarray
    vnr: np.ndarray
    sigma: np.ndarray          # complex conductivity per area element
    name: str = ""
    nx: int = 0
    nz: int = 0


def graded_depths(nz: int, dz0: float, growth: float) -> np.ndarray:
    d = [0.0]
    dz = dz0
    for _ in range(nz):
        d.append(d[-1] + dz)
        dz *= growth
    return np.array(d)


def structured_mesh(xs: np.ndarray, depths: np.ndarray, triangles: bool,
                    topo=None, side_type: int = 11) -> Mesh:
    """Quadrilateral (type 8) or split-quadrilateral triangle (type 3) grid.
    The sides and the bottom are mixed boundaries (side_type 11) or
    homogeneous Dirichlet boundaries (side_type 13, src/randb.f90)."""
    nx, nz = len(xs) - 1, len(depths) - 1
    ncol = nz + 1

    def node(ix, iz):
        return ix * ncol + iz + 1

    sanz = (nx + 1) * ncol
    X = np.repeat(xs, ncol)
    surf = np.zeros_like(xs) if topo is None else topo(xs)
    Y = (np.repeat(surf, ncol) - np.tile(depths, nx + 1))
    snr = np.arange(1, sanz + 1, dtype=np.int32)
    area = []
    for iz in range(nz):
        for ix in range(nx):
            a, b = node(ix, iz), node(ix + 1, iz)
            c, d = node(ix + 1, iz + 1), node(ix, iz + 1)
            if triangles:
                area.append((d, b, a))
                area.append((d, c, b))
            else:
                area.append((d, c, b, a))
    area_elems_per_cell = 2 if triangles else 1

    def elem_of(iz, ix, which):
        base = (iz * nx + ix) * area_elems_per_cell
        return base + (which if triangles else 0) + 1

    top, mixed = [], []
    rnr_top, rnr_mixed = [], []
    for ix in range(nx):
        top.append((node(ix, 0), node(ix + 1, 0)))
        rnr_top.append(elem_of(0, ix, 0))
    for iz in range(nz):
        mixed.append((node(nx, iz), node(nx, iz + 1)))
        rnr_mixed.append(elem_of(iz, nx - 1, 1))
    for ix in range(nx - 1, -1, -1):
        mixed.append((node(ix + 1, nz), node(ix, nz)))
        rnr_mixed.append(elem_of(nz - 1, ix, 1))
    for iz in range(nz - 1, -1, -1):
        mixed.append((node(0, iz + 1), node(0, iz)))
        rnr_mixed.append(elem_of(iz, 0, 0))
    nk = 3 if triangles else 4
    E, R12, R11 = len(area), len(top), len(mixed)
    nrel = np.zeros((E + R12 + R11, nk), dtype=np.int32, order="F")
    nrel[:E, :nk] = np.array(area, dtype=np.int32)
    nrel[E:E + R12, :2] = np.array(top, dtype=np.int32)
    nrel[E + R12:, :2] = np.array(mixed, dtype=np.int32)
    mb = int(max(np.max(np.array(area), axis=1) - np.min(np.array(area), axis=1)))
    typ = np.array([3 if triangles else 8, 12, side_type], np.int32)
    nel = np.array([E, R12, R11], np.int32)
    sel = np.array([nk, 2, 2], np.int32)
    rnr = np.array(rnr_top + rnr_mixed, np.int32)
    return Mesh(sanz, 3, mb, typ, nel, sel, snr, X.astype(np.float64), Y.astype(np.float64), nrel, rnr)


def centroids(mesh: Mesh):
    E = mesh.elanz
    nodes = mesh.nrel[:E, : int(mesh.selanz[0])]
    x, y = mesh.node_xy(nodes)
    return x.mean(axis=1), y.mean(axis=1)


def sigma_from(rho: np.ndarray, pha_mrad: np.ndarray) -> np.ndarray:
    p = pha_mrad / 1e3
    return np.cos(p) / rho - 1j * np.sin(p) / rho


# -- measurement configurations (1-based electrode numbers) --------------
def dipole_dipole(nel: int, spacings=(1,), nmax=8) -> List[Tuple[int, int, int, int]]:
    out = []
    for a in spacings:
        for n in range(1, nmax + 1):
            for A in range(1, nel + 1):
                B = A + a
                M = B + n * a
                N = M + a
                if N <= nel:
                    out.append((A, B, M, N))
    return out


def wenner(nel: int, amax: int) -> List[Tuple[int, int, int, int]]:
    out = []
    for a in range(1, amax + 1):
        for A in range(1, nel + 1):
            M, N, B = A + a, A + 2 * a, A + 3 * a
            if B <= nel:
                out.append((A, B, M, N))
    return out


def gradient(nel: int, span: int, step: int) -> List[Tuple[int, int, int, int]]:
    out = []
    for A in range(1, nel - span + 1, step):
        B = A + span
        for M in range(A + 1, B - 1):
            out.append((A, B, M, M + 1))
    return out


def encode(configs):
    c = np.array(configs, dtype=np.int64)
    strnr = (c[:, 0] + 10000 * c[:, 1]).astype(np.int32)
    vnr = (c[:, 2] + 10000 * c[:, 3]).astype(np.int32)
    return strnr, vnr


def surface_electrodes(mesh: Mesh, xs: np.ndarray, x_el: np.ndarray, nz: int) -> np.ndarray:
    ncol = nz + 1
    ix = np.array([int(np.argmin(np.abs(xs - x))) for x in x_el])
    return (ix * ncol + 1).astype(np.int32)


# -- the configurations ---------------------------------------------------
def config1(seed: int = SEED0 + 1) -> Survey:
    """60 x 20 quads (1 m x 0.5 m), 40 electrodes from x = 10 m at 1 m,
    100 Ohm m with a 10 Ohm m block of 5 x 3 cells, DD a = 1, n = 1..8."""
    rng = np.random.default_rng(seed)
    xs = np.arange(61, dtype=np.float64)
    depths = np.arange(21, dtype=np.float64) * 0.5
    mesh = structured_mesh(xs, depths, triangles=False)
    rho = np.full(mesh.elanz, 100.0)
    bx = int(rng.integers(15, 40))
    bz = int(rng.integers(1, 12))
    for iz in range(bz, bz + 3):
        for ix in range(bx, bx + 5):
            rho[iz * 60 + ix] = 10.0
    enr = surface_electrodes(mesh, xs, 10.0 + np.arange(40), 20)
    strnr, vnr = encode(dipole_dipole(40, (1,), 8))
    return Survey(mesh, enr, strnr, vnr, sigma_from(rho, np.zeros_like(rho)), "C1", 60, 20)


def _ellipse_mask(cx, cy, x0, y0, a, b):
    return ((cx - x0) / a) ** 2 + ((cy - y0) / b) ** 2 <= 1.0


def config2(seed: int = SEED0 + 2) -> Survey:
    """~8000 triangles with sinusoidal topography (1 m, 20 m), 48 electrodes
    at 1 m, 100 Ohm m / -5 mrad with two seeded ellipses, DD n = 1..10 plus
    Wenner."""
    rng = np.random.default_rng(seed)
    nx, nz = 100, 40
    xs = np.linspace(-26.0, 74.0, nx + 1)
    depths = graded_depths(nz, 0.25, 1.06)
    topo = lambda x: 1.0 * np.sin(2 * np.pi * x / 20.0)  # noqa: E731
    mesh = structured_mesh(xs, depths, triangles=True, topo=topo)
    cx, cy = centroids(mesh)
    rho = np.full(mesh.elanz, 100.0)
    pha = np.full(mesh.elanz, -5.0)
    for r_, p_ in ((20.0, -20.0), (500.0, -1.0)):
        x0 = rng.uniform(8, 40)
        y0 = topo(np.array([x0]))[0] - rng.uniform(2, 8)
        m = _ellipse_mask(cx, cy, x0, y0, rng.uniform(2, 5), rng.uniform(1, 3))
        rho[m], pha[m] = r_, p_
    enr = surface_electrodes(mesh, xs, np.arange(48, dtype=np.float64), nz)
    cfg = dipole_dipole(48, (1,), 10) + wenner(48, 15)
    strnr, vnr = encode(cfg)
    return Survey(mesh, enr, strnr, vnr, sigma_from(rho, pha), "C2", nx, nz)


def config3(seed: int = SEED0 + 3) -> Survey:
    """200 x 100 quads (20k elements), 96 electrodes, ~4000 DD readings of a
    seeded 3-anomaly model."""
    rng = np.random.default_rng(seed)
    nx, nz = 200, 100
    xs = np.linspace(-52.0, 148.0, nx + 1)
    depths = graded_depths(nz, 0.25, 1.035)
    mesh = structured_mesh(xs, depths, triangles=False)
    cx, cy = centroids(mesh)
    rho = np.full(mesh.elanz, 100.0)
    pha = np.full(mesh.elanz, -5.0)
    for r_, p_ in ((10.0, -25.0), (1000.0, -2.0), (30.0, -15.0)):
        x0 = rng.uniform(10, 85)
        y0 = -rng.uniform(2, 15)
        m = _ellipse_mask(cx, cy, x0, y0, rng.uniform(3, 8), rng.uniform(1.5, 4))
        rho[m], pha[m] = r_, p_
    enr = surface_electrodes(mesh, xs, np.arange(96, dtype=np.float64), nz)
    strnr, vnr = encode(dipole_dipole(96, (1, 2, 3, 4), 12))
    return Survey(mesh, enr, strnr, vnr, sigma_from(rho, pha), "C3", nx, nz)


def config5(seed: int = SEED0 + 5, nx: int = 235, nz: int = 128) -> Survey:
    """~60k triangles (235 x 128 split cells, n = 30,444 nodes, mb = 129),
    128 surface electrodes at 1 m, ~12,000 dipole-dipole + gradient
    readings, seeded layered-plus-block complex model."""
    rng = np.random.default_rng(seed)
    x0 = -53.5
    xs = x0 + np.arange(nx + 1, dtype=np.float64)
    depths = graded_depths(nz, 0.25, 1.03)
    mesh = structured_mesh(xs, depths, triangles=True)
    cx, cy = centroids(mesh)
    # layers
    n_layers = 3
    bounds = np.sort(rng.uniform(2.0, 30.0, n_layers - 1))
    lrho = np.exp(rng.uniform(np.log(20), np.log(500), n_layers))
    lpha = -rng.uniform(1, 30, n_layers)
    depth = -cy
    rho = np.full(mesh.elanz, lrho[0])
    pha = np.full(mesh.elanz, lpha[0])
    for k, b in enumerate(bounds):
        rho[depth > b] = lrho[k + 1]
        pha[depth > b] = lpha[k + 1]
    for _ in range(3):
        bx0 = rng.uniform(10, 115)
        bz0 = rng.uniform(1, 20)
        w, h = rng.uniform(4, 15), rng.uniform(2, 8)
        m = (np.abs(cx - bx0) <= w / 2) & (np.abs(depth - bz0) <= h / 2)
        rho[m] = np.exp(rng.uniform(np.log(10), np.log(1000)))
        pha[m] = -rng.uniform(1, 30)
    enr = surface_electrodes(mesh, xs, np.arange(128, dtype=np.float64), nz)
    cfg = dipole_dipole(128, tuple(range(1, 11)), 10)
    cfg += gradient(128, 32, 2) + gradient(128, 64, 4) + gradient(128, 48, 4)
    strnr, vnr = encode(cfg)
    return Survey(mesh, enr, strnr, vnr, sigma_from(rho, pha), "C5", nx, nz)


def config4(seed: int = SEED0 + 4, count: int = 256, emin: int = 2000, emax: int = 30000) -> List[Survey]:
    """`count` independent instances of uneven size for the batched forward
    and Jacobian: split-quadrilateral triangle meshes of E log-uniform in
    [emin, emax] elements (depth 6-64 cells, so mb = nz + 1 <= 65), L uniform
    in 24..96 surface electrodes, dipole-dipole readings with a random set of
    dipole lengths and n up to 4..12 (which puts the wavenumber count of the
    reference's rwaven rule between 8 and 15), and per-element resistivities
    log-uniform in 10..1000 Ohm m with phases uniform in -30..-1 mrad."""
    out = []
    spacing_sets = [(1,), (1, 2), (1, 2, 3), (1, 2, 4), (1, 3, 6)]
    for i in range(count):
        rng = np.random.default_rng([seed, i])
        E = float(np.exp(rng.uniform(np.log(emin), np.log(emax))))
        L = int(rng.integers(24, 97))
        pad = 4
        nx_min = L + 2 * pad + 2
        nz = int(min(rng.integers(16, 65), max(6, E // (2 * nx_min))))
        nx = max(nx_min, int(round(E / (2 * nz))))
        core = nx - 2 * pad
        w = 1.5 ** np.arange(1, pad + 1)
        xs = np.concatenate([-np.cumsum(w)[::-1], np.arange(core + 1, dtype=np.float64), core + np.cumsum(w)])
        depths = graded_depths(nz, 0.25, 1.04)
        mesh = structured_mesh(xs, depths, triangles=True)
        rho = np.exp(rng.uniform(np.log(10.0), np.log(1000.0), mesh.elanz))
        pha = -rng.uniform(1.0, 30.0, mesh.elanz)
        step = max(1, core // (L - 1))
        x_el = (core - step * (L - 1)) // 2 + step * np.arange(L, dtype=np.float64)
        enr = surface_electrodes(mesh, xs, x_el, nz)
        spacings = spacing_sets[int(rng.integers(0, len(spacing_sets)))]
        cfg = dipole_dipole(L, spacings, int(rng.integers(4, 13)))
        strnr, vnr = encode(cfg)
        out.append(Survey(mesh, enr, strnr, vnr, sigma_from(rho, pha), f"C4.{i}", nx, nz))
    return out


def small_triangles(seed: int = SEED0 + 100, nx: int = 24, nz: int = 10, nel: int = 12) -> Survey:
    """A small triangle mesh for quick parity tests."""
    rng = np.random.default_rng(seed)
    xs = np.arange(nx + 1, dtype=np.float64) - 6.0
    depths = graded_depths(nz, 0.5, 1.1)
    mesh = structured_mesh(xs, depths, triangles=True, topo=lambda x: 0.3 * np.sin(x / 3.0))
    rho = np.exp(rng.uniform(np.log(10), np.log(1000), mesh.elanz))
    pha = -rng.uniform(1, 30, mesh.elanz)
    enr = surface_electrodes(mesh, xs, np.arange(nel, dtype=np.float64), nz)
    strnr, vnr = encode(dipole_dipole(nel, (1, 2), 4))
    return Survey(mesh, enr, strnr, vnr, sigma_from(rho, pha), "small", nx, nz)


CONFIGS = {"C1": config1, "C2": config2, "C3": config3, "C5": config5}
