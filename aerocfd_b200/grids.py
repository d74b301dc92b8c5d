"""Seeded, analytic generators of the synthetic cases the solver is measured on.

The reference ships no grids, bcinfo or Control.in files, so every case is
generated here with the shapes, sizes and boundary layouts of the workloads
the path is quoted on:

* ``bump_channel``  - single-block channel of length 3, height 1, with a
  circular-arc bump of height h on x in [1, 2]; uniform in x, geometric in y;
  inflow / outflow / wall / symmetry (k faces symmetry).
* ``naca_ogrid``    - NACA 4-digit O-grid split into ``nblk`` blocks around the
  airfoil, block interfaces on the i faces, wall at j=1, farfield at j=max.
* ``bump_batch``    - many bump channels of uneven size (a Mach/geometry sweep).
* ``bump_channel_2d`` - the bump channel in 2-D mode (iflag_dimension = 2) as
  two blocks, the second turned by 180 degrees in the plane, so their shared
  face runs in opposite directions (2-D orientation code 3).

``naca_ogrid`` builds its 2-D form (one plane, no k faces, orientation code 2)
when the configuration asks for iflag_dimension = 2.
"""
from __future__ import annotations

import math
from typing import List, Optional

import numpy as np

from .case import (BC_FARFIELD, BC_INFLOW, BC_OUTFLOW, BC_SYMM, BC_WALL, IFLAG_2D, IFLAG_EULERSOLVER,
                   IFLAG_NSSOLVER, Block, Case, Config, Subface)


def _set_coords(blk: Block, X: np.ndarray, Y: np.ndarray, Z: np.ndarray) -> None:
    """Stores physical-node coordinates (shape (nk, nj, ni)) into the block's
    x, y, z arrays; ghost coordinates come from the coordinate halo."""
    s = blk.sl(blk.box0)
    blk.fields["x"][s] = X
    blk.fields["y"][s] = Y
    blk.fields["z"][s] = Z


def bump_channel(ni: int = 97, nj: int = 49, nk: int = 5, h: float = 0.10, length: float = 3.0,
                 ratio: float = 1.05, dz: float = 0.05, cfg: Optional[Config] = None,
                 name: str = "bump") -> Case:
    """Circular-arc bump channel, Euler.  The arc of chord 1 on x in [1,2] has
    radius R = (1/4 + h^2)/(2h) and centre (1.5, h - R)."""
    cfg = cfg or Config(solver=IFLAG_EULERSOLVER, ma=0.5, re=1.0e6, cfl=5.0)
    subs = [
        Subface(1, 1, 1, 1, 1, nj, 1, nk, BC_INFLOW),
        Subface(2, 2, ni, ni, 1, nj, 1, nk, BC_OUTFLOW),
        Subface(3, 3, 1, ni, 1, 1, 1, nk, BC_WALL),
        Subface(4, 4, 1, ni, nj, nj, 1, nk, BC_SYMM),
        Subface(5, 5, 1, ni, 1, nj, 1, 1, BC_SYMM),
        Subface(6, 6, 1, ni, 1, nj, nk, nk, BC_SYMM),
    ]
    blk = Block(1, ni, nj, nk, subs, cfg.buffer_length, cfg.dimension)
    x = np.linspace(0.0, length, ni)
    R = (0.25 + h * h) / (2.0 * h)
    ywall = np.where((x >= 1.0) & (x <= 2.0),
                     np.sqrt(np.maximum(R * R - (x - 1.5) ** 2, 0.0)) - (R - h), 0.0)
    n = nj - 1
    eta = (ratio ** np.arange(nj) - 1.0) / (ratio ** n - 1.0)
    Y2 = ywall[None, :] + (1.0 - ywall[None, :]) * eta[:, None]          # (nj, ni)
    X2 = np.broadcast_to(x[None, :], (nj, ni))
    zs = dz * np.arange(nk)
    X = np.broadcast_to(X2[None], (nk, nj, ni)).copy()
    Y = np.broadcast_to(Y2[None], (nk, nj, ni)).copy()
    Z = np.broadcast_to(zs[:, None, None], (nk, nj, ni)).copy()
    _set_coords(blk, X, Y, Z)
    return Case(name, cfg, [blk])


def naca4_surface(x: np.ndarray, t: float, m: float = 0.0, p: float = 0.4):
    """Upper and lower surface of a NACA 4-digit section (standard thickness
    law, open trailing edge of thickness 0.0021*t/0.01... at x = 1), chord 1."""
    yt = 5.0 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1015 * x ** 4)
    if m > 0.0:
        yc = np.where(x < p, m / p ** 2 * (2 * p * x - x ** 2), m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * x - x ** 2))
        dyc = np.where(x < p, 2 * m / p ** 2 * (p - x), 2 * m / (1 - p) ** 2 * (p - x))
        th = np.arctan(dyc)
        xu, yu = x - yt * np.sin(th), yc + yt * np.cos(th)
        xl, yl = x + yt * np.sin(th), yc - yt * np.cos(th)
    else:
        xu, yu, xl, yl = x, yt, x, -yt
    return xu, yu, xl, yl


def naca4_loop(n: int, t: float, m: float = 0.0, p: float = 0.4, n_cap: int = 8):
    """Closed surface loop of n intervals, clockwise from the trailing-edge tip:
    a semicircular cap of n_cap intervals closes the blunt trailing edge (its
    lower half first), then the lower surface to the leading edge and the upper
    surface back.  x is clustered toward the leading edge and mildly toward the
    trailing edge."""
    half = (n - n_cap) // 2
    tt = np.linspace(0.0, 1.0, half + 1)
    xs = 0.5 * (0.5 * (1.0 - np.cos(np.pi * tt))) + 0.5 * (1.0 - np.cos(0.5 * np.pi * tt))  # 0 -> 1
    xu, yu, xl, yl = naca4_surface(xs, t, m, p)
    # trailing-edge cap: centre midway between the TE corners, radius half the gap
    cx, cy = 0.5 * (xu[-1] + xl[-1]), 0.5 * (yu[-1] + yl[-1])
    r = 0.5 * np.hypot(xu[-1] - xl[-1], yu[-1] - yl[-1])
    ang0 = np.arctan2(yl[-1] - cy, xl[-1] - cx)     # lower corner (about -pi/2)
    k = n_cap // 2
    a_low = np.linspace(0.0, ang0, k + 1)           # tip (0) -> lower corner
    a_up = np.linspace(-ang0, 0.0, n_cap - k + 1)    # upper corner -> tip
    cap_lo_x, cap_lo_y = cx + r * np.cos(a_low), cy + r * np.sin(a_low)
    cap_up_x, cap_up_y = cx + r * np.cos(a_up), cy + r * np.sin(a_up)
    lx, ly = xl[::-1], yl[::-1]                     # TE -> LE along the lower surface
    X = np.concatenate([cap_lo_x, lx[1:], xu[1:], cap_up_x[1:]])
    Y = np.concatenate([cap_lo_y, ly[1:], yu[1:], cap_up_y[1:]])
    assert len(X) == n + 1, (len(X), n)
    return X, Y


def radial_distribution(nj: int, first: float, ratio: float, outer: float = 1.0,
                        n_inner: Optional[int] = None) -> np.ndarray:
    """Wall-normal node positions 0..outer over nj nodes in two geometric
    segments: ``n_inner`` intervals growing at ``ratio`` from spacing ``first``,
    then a second ratio solved so the last node lands on ``outer`` (a single
    ratio of 1.08 over 64 intervals would reach only ~0.17 chord)."""
    n = nj - 1
    n1 = n // 2 if n_inner is None else n_inner
    inner = first * (ratio ** np.arange(n1 + 1) - 1.0) / (ratio - 1.0)
    d = first * ratio ** (n1 - 1) if n1 > 0 else first
    n2 = n - n1
    left = outer - inner[-1]
    lo, hi = 1.0 + 1e-12, 10.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        val = d * mid * (mid ** n2 - 1.0) / (mid - 1.0)
        lo, hi = (mid, hi) if val < left else (lo, mid)
    r2 = 0.5 * (lo + hi)
    outer_part = inner[-1] + d * r2 * (r2 ** np.arange(1, n2 + 1) - 1.0) / (r2 - 1.0)
    out = np.concatenate([inner, outer_part])
    out[-1] = outer
    return out


def naca_ogrid(nblk: int = 4, ni: int = 129, nj: int = 65, nk: int = 3, t: float = 0.12,
               m: float = 0.0, p: float = 0.4, first: float = 1.0e-4, ratio: float = 1.08,
               outer: float = 20.0, dz: float = 0.1, cfg: Optional[Config] = None,
               name: str = "naca_ogrid") -> Case:
    """O-grid around a NACA 4-digit section (blunt trailing edge closed by a
    small semicircular cap).  i runs clockwise around the airfoil starting at
    the trailing-edge tip (lower surface first), j outward, k
    spanwise.  Block b covers i-intervals [b*(ni-1), (b+1)*(ni-1)] of the loop;
    neighbouring blocks share their i interface plane (overlap nodes) and are
    connected face 2 -> face 1 with orientation code 2 (the reference's
    transposed (l,m) convention between an i+ and an i- face)."""
    cfg = cfg or Config(solver=IFLAG_NSSOLVER, ma=0.5, re=5000.0, aoa_deg=2.0, cfl=2.0)
    two = cfg.dimension == IFLAG_2D
    if two:
        nk = 1                           # one plane, z = 0 (sub_init_allocatememory.f90:389-401)
    ntot = nblk * (ni - 1)               # intervals around the loop
    sx, sy = naca4_loop(ntot, t, m, p)
    # outer circle, clockwise from angle 0, at the same loop fraction
    theta = 2.0 * math.pi * np.arange(ntot + 1) / ntot
    cx, cy = 0.5, 0.0
    ox = cx + outer * np.cos(-theta)
    oy = cy + outer * np.sin(-theta)
    # wall-normal distribution reaching the outer circle; blend surface -> circle
    dist = radial_distribution(nj, first / outer, ratio, 1.0)
    blocks: List[Block] = []
    zs = dz * np.arange(nk)
    for b in range(nblk):
        lo = b * (ni - 1)
        idx = np.arange(lo, lo + ni) % ntot
        bx = sx[idx]; by = sy[idx]; ex = ox[idx]; ey = oy[idx]
        # initial direction: surface normal blended toward the straight line
        X2 = bx[None, :] + (ex - bx)[None, :] * dist[:, None]
        Y2 = by[None, :] + (ey - by)[None, :] * dist[:, None]
        left = nblk if b == 0 else b          # neighbour on face 1 (i-)
        right = 1 if b == nblk - 1 else b + 2  # neighbour on face 2 (i+)
        # in 2-D the shared i faces run the same way in j: orientation code 2
        # (same order); in 3-D code 2 is the transposed (l,m) convention
        subs = [
            Subface(1, 1, 1, 1, 1, nj, 1, nk, left, 2, 2),
            Subface(2, 2, ni, ni, 1, nj, 1, nk, right, 1, 2),
            Subface(3, 3, 1, ni, 1, 1, 1, nk, BC_WALL),
            Subface(4, 4, 1, ni, nj, nj, 1, nk, BC_FARFIELD),
        ]
        if not two:
            subs += [Subface(5, 5, 1, ni, 1, nj, 1, 1, BC_SYMM),
                     Subface(6, 6, 1, ni, 1, nj, nk, nk, BC_SYMM)]
        blk = Block(b + 1, ni, nj, nk, subs, cfg.buffer_length, cfg.dimension)
        X = np.broadcast_to(X2[None], (nk, nj, ni)).copy()
        Y = np.broadcast_to(Y2[None], (nk, nj, ni)).copy()
        Z = np.zeros((nk, nj, ni)) if two else np.broadcast_to(zs[:, None, None], (nk, nj, ni)).copy()
        _set_coords(blk, X, Y, Z)
        blocks.append(blk)
    return Case(name, cfg, blocks)


def bump_channel_2d(ni: int = 97, nj: int = 49, h: float = 0.10, length: float = 3.0,
                    ratio: float = 1.05, cfg: Optional[Config] = None, name: str = "bump2d") -> Case:
    """The bump channel of ``bump_channel`` in 2-D mode, as two blocks that
    share the node line x = x_mid (ni points in total along x, the split at
    node ni // 2 + 1).  Block 1 is the left part in (x, y) index order; block 2
    is the right part turned by 180 degrees in the plane (its i runs from the
    outlet back to the split, its j from the top down), so the grid stays
    right-handed, its wall is face 4, its outflow face 1, and the shared
    faces (face 2 of both blocks) run in opposite directions: orientation
    code 3 (sub_bc_updatebuffer2d.f90:284-293)."""
    cfg = cfg or Config(solver=IFLAG_EULERSOLVER, ma=0.5, re=1.0e6, cfl=5.0, dimension=IFLAG_2D)
    if cfg.dimension != IFLAG_2D:
        raise ValueError("bump_channel_2d needs a 2-D configuration")
    x = np.linspace(0.0, length, ni)
    R = (0.25 + h * h) / (2.0 * h)
    ywall = np.where((x >= 1.0) & (x <= 2.0),
                     np.sqrt(np.maximum(R * R - (x - 1.5) ** 2, 0.0)) - (R - h), 0.0)
    n = nj - 1
    eta = (ratio ** np.arange(nj) - 1.0) / (ratio ** n - 1.0)
    Y2 = ywall[None, :] + (1.0 - ywall[None, :]) * eta[:, None]          # (nj, ni)
    X2 = np.broadcast_to(x[None, :], (nj, ni))
    mid = ni // 2                                                        # 0-based split node
    n1, n2 = mid + 1, ni - mid
    s1 = [
        Subface(1, 1, 1, 1, 1, nj, 1, 1, BC_INFLOW),
        Subface(2, 2, n1, n1, 1, nj, 1, 1, 2, 2, 3),
        Subface(3, 3, 1, n1, 1, 1, 1, 1, BC_WALL),
        Subface(4, 4, 1, n1, nj, nj, 1, 1, BC_SYMM),
    ]
    s2 = [
        Subface(1, 1, 1, 1, 1, nj, 1, 1, BC_OUTFLOW),
        Subface(2, 2, n2, n2, 1, nj, 1, 1, 1, 2, 3),
        Subface(3, 3, 1, n2, 1, 1, 1, 1, BC_SYMM),
        Subface(4, 4, 1, n2, nj, nj, 1, 1, BC_WALL),
    ]
    b1 = Block(1, n1, nj, 1, s1, cfg.buffer_length, cfg.dimension)
    b2 = Block(2, n2, nj, 1, s2, cfg.buffer_length, cfg.dimension)
    _set_coords(b1, X2[None, :, :n1].copy(), Y2[None, :, :n1].copy(), np.zeros((1, nj, n1)))
    # block 2 node (i', j') = global node (ni - i', nj + 1 - j') (1-based)
    X2r = X2[::-1, ::-1][:, :n2]
    Y2r = Y2[::-1, ::-1][:, :n2]
    _set_coords(b2, X2r[None].copy(), Y2r[None].copy(), np.zeros((1, nj, n2)))
    return Case(name, cfg, [b1, b2])


def bump_batch(ncase: int = 64, seed: int = 0, nk: int = 5):
    """Uneven bump-channel sweep: ni ~ U{65..257}, nj ~ U{33..97}, nk = 5,
    h ~ U[0.05, 0.12], M ~ U[0.3, 0.7]."""
    rng = np.random.default_rng(seed)
    cases = []
    for c in range(ncase):
        ni = int(rng.integers(65, 258))
        nj = int(rng.integers(33, 98))
        h = float(rng.uniform(0.05, 0.12))
        ma = float(rng.uniform(0.3, 0.7))
        cfg = Config(solver=IFLAG_EULERSOLVER, ma=ma, re=1.0e6, cfl=5.0)
        cases.append(bump_channel(ni, nj, nk, h=h, cfg=cfg, name=f"bump{c:02d}"))
    return cases


def batch_case(cases, name: str = "batch"):
    """Independent cases as the blocks of one registered set (a batch):
    returns the Case (blocks renumbered 1..n in case order, each keeping its
    own arrays; the interface partners of a multi-block case shifted with
    them) and {m: Config} with every block's own Control.in values, for
    GpuCase(..., block_params=...).  The flags (solver, time advance, ...) of
    the first case apply to all."""
    import dataclasses
    from .case import Block as _Block
    blocks, params = [], {}
    off = 0
    for c in cases:
        for b in c.blocks:
            subs = [dataclasses.replace(sf, blk_t=sf.blk_t + off if sf.blk_t > 0 else sf.blk_t)
                    for sf in b.subfaces]
            nb = _Block(off + b.m, b.ni, b.nj, b.nk, subs, c.cfg.buffer_length, c.cfg.dimension)
            for k, v in b.fields.items():
                nb.fields[k][...] = v
            blocks.append(nb)
            params[nb.m] = c.cfg
        off += len(c.blocks)
    blocks.sort(key=lambda b: b.m)
    return Case(name, cases[0].cfg, blocks), params


def batch_members(cases):
    """The 0-based block range [first, last) of every case in the batch that
    batch_case builds from `cases`."""
    out, off = [], 0
    for c in cases:
        out.append((off, off + len(c.blocks)))
        off += len(c.blocks)
    return out


def unbatch(batch: Case, cases, i: int) -> Case:
    """Case i of a batch as a stand-alone case with its own numbering (arrays
    copied from the batch's host arrays)."""
    import dataclasses
    from .case import Block as _Block
    first, last = batch_members(cases)[i]
    c = cases[i]
    blocks = []
    for b, src in zip(c.blocks, batch.blocks[first:last]):
        nb = _Block(b.m, b.ni, b.nj, b.nk, [dataclasses.replace(sf) for sf in b.subfaces], c.cfg.buffer_length,
                    c.cfg.dimension)
        for k, v in src.fields.items():
            nb.fields[k][...] = v
        blocks.append(nb)
    return Case(f"{c.name}_member{i}", c.cfg, blocks)


def geometric_nodes(n: int, first: float, length: float) -> np.ndarray:
    """n intervals from 0 to `length` growing geometrically from `first`."""
    if abs(first * n - length) < 1e-15 * length:
        return np.linspace(0.0, length, n + 1)
    lo, hi = (1.0 + 1e-12, 10.0) if first * n < length else (1e-6, 1.0 - 1e-12)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        val = first * (mid ** n - 1.0) / (mid - 1.0)
        lo, hi = (mid, hi) if val < length else (lo, mid)
    r = 0.5 * (lo + hi)
    s = first * (r ** np.arange(n + 1) - 1.0) / (r - 1.0)
    s[-1] = length
    return s


def flat_plate(nbi: int = 2, nbj: int = 2, nbk: int = 2, ni: int = 193, nj: int = 129, nk: int = 33,
               x_up: float = 0.5, dx_le: float = 2.0e-3, dy_wall: float = 5.0e-6, ratio_y: float = 1.1,
               span: float = 0.32, cfg: Optional[Config] = None, name: str = "flat_plate") -> Case:
    """Turbulent flat plate of length 1 split into nbi x nbj x nbk blocks that
    share their interface planes (ni = nbi*(bi-1)+1 etc.).  The leading edge
    sits on the first i-interface, so the j=1 faces of the upstream blocks are
    symmetry planes and those of the downstream blocks no-slip walls.  x is
    clustered geometrically at the leading edge from both sides, y grows from
    the wall spacing dy_wall at ratio_y, z is uniform.  Inflow at i=1, outflow
    at i=max, farfield at j=max, symmetry on both k faces."""
    cfg = cfg or Config(solver=IFLAG_NSSOLVER, turbulence=2, ma=0.2, re=5.0e6, cfl=2.0, nutinf=3.0)
    bi, bj, bk = (ni - 1) // nbi + 1, (nj - 1) // nbj + 1, (nk - 1) // nbk + 1
    assert nbi * (bi - 1) + 1 == ni and nbj * (bj - 1) + 1 == nj and nbk * (bk - 1) + 1 == nk
    i_le = bi  # global index of the leading edge
    up = geometric_nodes(i_le - 1, dx_le, x_up)[::-1] * -1.0
    down = geometric_nodes(ni - i_le, dx_le, 1.0)
    X = np.concatenate([up, down[1:]])
    Y = dy_wall * (ratio_y ** np.arange(nj) - 1.0) / (ratio_y - 1.0)
    Z = np.linspace(0.0, span, nk)
    blocks: List[Block] = []

    def bid(a, b, c):
        return 1 + a + nbi * (b + nbj * c)

    for c in range(nbk):
        for b in range(nbj):
            for a in range(nbi):
                m = bid(a, b, c)
                subs = []
                fno = 0

                def add(face, box, kind, partner=0):
                    nonlocal fno
                    fno += 1
                    subs.append(Subface(fno, face, *box, kind, partner, 2 if kind > 0 else 0))
                full = {1: (1, 1, 1, bj, 1, bk), 2: (bi, bi, 1, bj, 1, bk), 3: (1, bi, 1, 1, 1, bk),
                        4: (1, bi, bj, bj, 1, bk), 5: (1, bi, 1, bj, 1, 1), 6: (1, bi, 1, bj, bk, bk)}
                # face 1, 2 (i)
                add(1, full[1], bid(a - 1, b, c) if a > 0 else BC_INFLOW)
                add(2, full[2], bid(a + 1, b, c) if a < nbi - 1 else BC_OUTFLOW)
                # face 3, 4 (j)
                wall = BC_WALL if a * (bi - 1) + 1 >= i_le else BC_SYMM
                add(3, full[3], bid(a, b - 1, c) if b > 0 else wall)
                add(4, full[4], bid(a, b + 1, c) if b < nbj - 1 else BC_FARFIELD)
                # face 5, 6 (k)
                add(5, full[5], bid(a, b, c - 1) if c > 0 else BC_SYMM)
                add(6, full[6], bid(a, b, c + 1) if c < nbk - 1 else BC_SYMM)
                blk = Block(m, bi, bj, bk, subs, cfg.buffer_length, cfg.dimension)
                xs = X[a * (bi - 1):a * (bi - 1) + bi]
                ys = Y[b * (bj - 1):b * (bj - 1) + bj]
                zs = Z[c * (bk - 1):c * (bk - 1) + bk]
                ZZ, YY, XX = np.meshgrid(zs, ys, xs, indexing="ij")
                _set_coords(blk, XX, YY, ZZ)
                blocks.append(blk)
    # interface partners: face 1 <-> face 2 (subface 1 <-> 2), 3 <-> 4, 5 <-> 6
    pair = {1: 2, 2: 1, 3: 4, 4: 3, 5: 6, 6: 5}
    for blk in blocks:
        for s in blk.subfaces:
            if s.blk_t > 0:
                s.subface_t = pair[s.face]
    return Case(name, cfg, blocks)
