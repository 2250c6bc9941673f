"""Small parity cases shared by the golden-fixture generator and the tests.

Models are closed-form (no random numbers), so any machine rebuilds the same
float32 inputs.  Each case is small enough for the reference CPU path to run
in about a second.
"""
from __future__ import annotations

import numpy as np

CASES = {
    # two-layer, square cells, split spread around a mid-surface source
    "twolayer_split_nb32": dict(
        nb=32, nx=160, nz=120, dx=10.0, dz=10.0, T=0.4, dt=0.001, ddt=0.001, f=12.0,
        model="twolayer", geom=("shot", [(800.0, 20.0, 121, 0, 10.0, 1)])),
    # vertical gradient + circular anomaly + variable density, rectangular
    # cells, decimated recording (dt_factor 2), end-on-left spread, nb=40
    "gradient_endonleft_nb40": dict(
        nb=40, nx=150, nz=100, dx=12.0, dz=8.0, T=0.5, dt=0.0008, ddt=0.0016, f=10.0,
        model="gradient_anomaly", geom=("shot", [(1500.0, 16.0, 100, 0, 12.0, 2)])),
    # end-on-right spread with a near offset, nb=32
    "layers_endonright_near_nb32": dict(
        nb=32, nx=141, nz=97, dx=10.0, dz=10.0, T=0.35, dt=0.001, ddt=0.001, f=12.0,
        model="layers", geom=("shot", [(300.0, 10.0, 90, 20.0, 10.0, 3)])),
    # explicit geometry: source and receivers on the grid edges and at depth
    # (edge rows of the derivative operators), odd sizes
    "edges_explicit_nb32": dict(
        nb=32, nx=137, nz=93, dx=10.0, dz=10.0, T=0.3, dt=0.001, ddt=0.002, f=12.0,
        model="layers", geom=("explicit", "edges")),
    # source in the first column and row, nb=40
    "corner_source_nb40": dict(
        nb=40, nx=120, nz=90, dx=10.0, dz=10.0, T=0.3, dt=0.001, ddt=0.001, f=12.0,
        model="gradient_anomaly", geom=("explicit", "corner")),
    # the 7.62 m grid spacing and 0.6 ms step of the salt configuration, its
    # 50-cell sponge, a split spread at a non-integer receiver spacing, dt_factor 2
    "salt_grid_nb50": dict(
        nb=50, nx=200, nz=120, dx=7.62, dz=7.62, T=0.24, dt=0.0006, ddt=0.0012, f=15.0,
        model="gradient_anomaly", geom=("shot", [(762.0, 15.24, 81, 0, 15.24, 1)])),
    # the 5 m spacing, 0.5 ms step, 20 Hz and 60-cell sponge of the large
    # two-layer configuration
    "twolayer_5m_nb60": dict(
        nb=60, nx=180, nz=140, dx=5.0, dz=5.0, T=0.2, dt=0.0005, ddt=0.0005, f=20.0,
        model="twolayer", geom=("shot", [(450.0, 10.0, 161, 0, 5.0, 1)])),
}


def model(name: str, nx: int, nz: int, dx: float, dz: float):
    """Return ``(vp, rho)`` as float32 ``[nx][nz]``."""
    x = (np.arange(nx, dtype=np.float64)[:, None]) * dx
    z = (np.arange(nz, dtype=np.float64)[None, :]) * dz
    if name == "twolayer":
        vp = np.where(np.broadcast_to(z, (nx, nz)) < (nz // 2) * dz, 1500.0, 3000.0)
        rho = np.where(np.broadcast_to(z, (nx, nz)) < (nz // 2) * dz, 1000.0, 2000.0)
    elif name == "gradient_anomaly":
        zmax = (nz - 1) * dz
        vp = 1500.0 + 1000.0 * (z / zmax) + 0.0 * x
        cx, cz, r = 0.55 * (nx - 1) * dx, 0.6 * zmax, 0.15 * zmax
        inside = (x - cx) ** 2 + (z - cz) ** 2 < r * r
        vp = np.where(inside, vp + 400.0, vp)
        rho = 310.0 * vp ** 0.25
    elif name == "layers":
        zz = np.broadcast_to(z, (nx, nz))
        xx = np.broadcast_to(x, (nx, nz))
        b1 = 0.3 * (nz - 1) * dz + 0.05 * xx
        b2 = 0.7 * (nz - 1) * dz - 0.03 * xx
        vp = np.where(zz < b1, 1600.0, np.where(zz < b2, 2200.0, 2900.0))
        rho = np.where(zz < b1, 1100.0, np.where(zz < b2, 1800.0, 2300.0))
    else:
        raise KeyError(name)
    return vp.astype(np.float32), rho.astype(np.float32)


def explicit_geometry(kind: str, nx: int, nz: int, dx: float, dz: float):
    """``[((sx, sz), [(gx, gz), ...])]`` in metres, on grid nodes."""
    xmax, zmax = (nx - 1) * dx, (nz - 1) * dz
    if kind == "edges":
        src = (40 * dx, 0.0)
        recs = [(i * dx, 0.0) for i in range(0, nx, 4)]
        recs += [(xmax, j * dz) for j in range(0, nz, 6)]
        recs += [(0.0, zmax), (xmax, zmax), (20 * dx, zmax), (70 * dx, 45 * dz)]
        return [(src, recs)]
    if kind == "corner":
        src = (0.0, 0.0)
        recs = [(i * dx, 2 * dz) for i in range(0, nx, 3)] + [(5 * dx, j * dz) for j in range(0, nz, 5)]
        return [(src, recs)]
    raise KeyError(kind)
