"""Learned warm start for families of cases (no counterpart in the reference).

A small MLP (aero_mlp_*: BF16 weights, FP32 accumulation, tcgen05 GEMMs) is
trained on converged fields the solver generates for seeded members of a case
family, and predicts the primitive variables of a new member from its
parameters and node coordinates; the solver then starts from that field instead
of the freestream.  The freestream start stays the fallback and the yardstick
for the result: a warm-started run is iterated to the same residual level as
the cold one and their wall forces are compared.

The family here is the bump channel (a fixed grid of ni x nj x nk, bump height
h ~ U[0.05, 0.12], Mach ~ U[0.3, 0.7]) with farfield (Riemann-invariant)
boundaries on the inflow, outflow and top faces: its steady state is unique
and the scheme converges to machine zero from any start, which the warm start
is compared against.  (With the fixed inflow and extrapolated outflow of the
reference's own channel set-up the converged pressure level depends on the
start, so converged forces cannot tell two starts apart.)  Node inputs are
(x, y, wall distance, h, M), outputs the freestream-normalised perturbations of
(rho, u, v, p).
"""
from __future__ import annotations

import ctypes
import time
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import _lib, grids
from .case import BC_FARFIELD, Case, Config, IFLAG_EULERSOLVER

GAMMA = 1.4


def family(n: int, seed: int, ni: int = 97, nj: int = 49, nk: int = 5) -> List[Tuple[Case, float, float]]:
    """n bump channels with seeded (h, M): (case, h, M)."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(n):
        h = float(rng.uniform(0.05, 0.12))
        ma = float(rng.uniform(0.3, 0.7))
        cfg = Config(solver=IFLAG_EULERSOLVER, ma=ma, re=1.0e6, cfl=5.0)
        case = grids.bump_channel(ni, nj, nk, h=h, cfg=cfg, name=f"bump_h{h:.3f}_m{ma:.3f}")
        for sf in case.blocks[0].subfaces:
            if sf.face in (1, 2, 4):
                sf.blk_t = BC_FARFIELD
        out.append((case, h, ma))
    return out


def features(case: Case, h: float, ma: float) -> np.ndarray:
    """Per physical node of the first k-plane: x/3, y, y - y_wall(x), h/0.12,
    (M - 0.5)/0.2 (float32, nj*ni rows, i fastest)."""
    b = case.blocks[0]
    s = b.sl(b.box0)
    x = b.fields["x"][s][0]
    y = b.fields["y"][s][0]
    dist = y - y[0:1, :]
    nj, ni = x.shape
    f = np.stack([x / 3.0, y, dist, np.full_like(x, h / 0.12), np.full_like(x, (ma - 0.5) / 0.2)], -1)
    return f.reshape(nj * ni, 5).astype(np.float32)


def targets(case: Case) -> np.ndarray:
    """(rho - 1, u - 1, v, p/p0 - 1) on the first k-plane of the physical
    nodes (the freestream is rho = u = 1, v = 0, p = p0 = 1/(gamma M^2))."""
    b = case.blocks[0]
    s = b.sl(b.box0)
    pri = b.fields["pri_v"][s][0]
    p0 = 1.0 / GAMMA / case.cfg.ma ** 2
    t = np.stack([pri[..., 0] - 1.0, pri[..., 1] - 1.0, pri[..., 2], pri[..., 4] / p0 - 1.0], -1)
    return t.reshape(-1, 4).astype(np.float32)


def set_state(case: Case, pred: np.ndarray) -> None:
    """Conservative variables of every node of the case from predicted
    perturbations on the first k-plane (copied along k; ghost nodes take the
    nearest physical node's value before the start-up BCs overwrite them)."""
    b = case.blocks[0]
    ma = case.cfg.ma
    p0 = 1.0 / GAMMA / ma ** 2
    nk, nj, ni = b.nk, b.nj, b.ni
    pr = pred.reshape(nj, ni, 4).astype(np.float64)
    rho = 1.0 + pr[..., 0]
    u = 1.0 + pr[..., 1]
    v = pr[..., 2]
    p = p0 * (1.0 + pr[..., 3])
    q = np.stack([rho, rho * u, rho * v, np.zeros_like(rho), p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v)], -1)
    full = b.fields["q"]
    is_, ie, js, je, ks, ke = b.box
    ii = np.clip(np.arange(is_, ie + 1), 1, ni) - 1
    jj = np.clip(np.arange(js, je + 1), 1, nj) - 1
    full[...] = q[jj][:, ii][None, :, :, :]


class Network:
    """aero_mlp_* through the C-ABI."""

    def __init__(self, n_in=5, n_out=4, width=256, depth=8, batch=8192, seed=1):
        self.L = _lib.load()
        _lib.check(self.L.aero_mlp_create(n_in, n_out, width, depth, batch, ctypes.c_ulonglong(seed)), "aero_mlp_create")
        self.shape = (n_in, n_out, width, depth, batch)

    def train(self, x: np.ndarray, t: np.ndarray, steps: int, lr: float = 1e-3, seed: int = 2) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        hist = np.zeros(steps, dtype=np.float32)
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        _lib.check(self.L.aero_mlp_train(p(x), p(t), ctypes.c_longlong(len(x)), steps, ctypes.c_float(lr),
                                         ctypes.c_ulonglong(seed), p(hist)), "aero_mlp_train")
        return hist

    def predict(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((len(x), self.shape[1]), dtype=np.float32)
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        _lib.check(self.L.aero_mlp_predict(p(x), ctypes.c_longlong(len(x)), p(y)), "aero_mlp_predict")
        return y

    def close(self) -> None:
        self.L.aero_mlp_destroy()


def run_batch(solver, members: Sequence[Tuple[Case, float, float]], iters: int, chunk: int = 50,
              warm: Dict[int, np.ndarray] = None, mixed: bool = False):
    """Runs the members as one batch for `iters` iterations; warm maps member
    index -> predicted field (else a freestream start).  Returns the per-member
    density residual after iteration 1 and after every further chunk (row r is
    iteration 1 + r*chunk), the wall time and the batch case (host arrays
    synchronised)."""
    cases = [m[0] for m in members]
    batch, params = grids.batch_case(cases)
    gc = solver.GpuCase(batch, block_params=params)
    try:
        gc.compute_geometry()
        gc.init_flowfield()
        if warm:
            gc.sync_to_host(solver.ALL)
            for i, pred in warm.items():
                set_state(Case("member", cases[i].cfg, [batch.blocks[i]]), pred)
            gc.sync_to_device(solver.mask("q"))
        gc.start()
        gc.set_precision(mixed)
        gc.use_graphs(True)
        t0 = time.perf_counter()
        gc.step(1, history=False)
        res = [gc.residual_blocks()[:, 0]]  # iteration 1
        for _ in range(iters // chunk):
            gc.step(chunk, history=False)
            res.append(gc.residual_blocks()[:, 0])
        wall = time.perf_counter() - t0
        gc.sync_to_host(solver.ALL)
        return np.array(res), wall, batch
    finally:
        gc.close()


def member(batch: Case, i: int, cfg: Config) -> Case:
    """Block i of a batch as a stand-alone single-block case (arrays copied)."""
    from .case import Block
    b = batch.blocks[i]
    nb = Block(1, b.ni, b.nj, b.nk, b.subfaces, cfg.buffer_length, cfg.dimension)
    for k, v in b.fields.items():
        nb.fields[k][...] = v
    return Case(f"member{i}", cfg, [nb])


def first_below(hist: np.ndarray, level: np.ndarray, chunk: int) -> np.ndarray:
    """Iteration (chunk resolution) at which each member's residual first falls
    below its level (rows as run_batch returns them); -1 if never."""
    out = np.full(hist.shape[1], -1)
    for m in range(hist.shape[1]):
        hit = np.nonzero(hist[:, m] <= level[m])[0]
        if len(hit):
            out[m] = 1 + hit[0] * chunk
    return out


def wall_force(solver, case: Case) -> np.ndarray:
    """Pressure + viscous force on the walls (clcd_output) of a solved case."""
    gc = solver.GpuCase(case)
    try:
        gc.sync_to_device(solver.ALL)
        return gc.clcd_output(1.0)
    finally:
        gc.close()


# ---------------------------------------------------------------------------
# NACA 4-digit family with the SA model on the 4-block O-grid
#
# Family parameters (seeded): thickness t ~ U[0.08, 0.15], camber m ~
# U[0, 0.04] at p ~ U[0.2, 0.6], angle of attack ~ U[-2, 6] deg, M ~
# U[0.3, 0.7], Re ~ U[1e6, 1e7]; SA with nu_t,inf = 3 nu_inf.  Every member
# has its own grid (the section shape changes it), so a batch of members is a
# set of 4-block cases (grids.batch_case).  Node inputs: x, y, the distance to
# the wall, and the six member parameters, scaled to O(1); outputs: the
# perturbations of rho, u, v, p from the freestream and log(nu_t / nu_t,inf).

NACA_IN, NACA_OUT = 9, 5


def naca_family(n: int, seed: int, ni: int = 129, nj: int = 65, nk: int = 3, first: float = 5.0e-6,
                cfl: float = 3.0):
    """n members of the NACA family: [(case, params)], params a dict of the
    member's t, m, p, aoa_deg, ma, re."""
    from .case import IFLAG_NSSOLVER
    rng = np.random.default_rng(seed)
    out = []
    for c in range(n):
        prm = {"t": float(rng.uniform(0.08, 0.15)), "m": float(rng.uniform(0.0, 0.04)),
               "p": float(rng.uniform(0.2, 0.6)), "aoa_deg": float(rng.uniform(-2.0, 6.0)),
               "ma": float(rng.uniform(0.3, 0.7)), "re": float(rng.uniform(1.0e6, 1.0e7))}
        cfg = Config(solver=IFLAG_NSSOLVER, turbulence=2, ma=prm["ma"], re=prm["re"], aoa_deg=prm["aoa_deg"],
                     cfl=cfl, nutinf=3.0)
        case = grids.naca_ogrid(ni=ni, nj=nj, nk=nk, t=prm["t"], m=prm["m"], p=prm["p"], first=first, cfg=cfg,
                                name=f"naca_{c:03d}")
        out.append((case, prm))
    return out


def _plane(b, name):
    s = b.sl(b.box0)
    return b.fields[name][s][0]


def naca_features(case: Case, prm) -> np.ndarray:
    """Per physical node of the first k-plane of every block (block order,
    i fastest): x, y (chord units, y scaled by 1/2), log10 of the distance to
    the nearest wall node, and the member parameters scaled to O(1)."""
    wall = np.concatenate([np.stack([_plane(b, "x")[0], _plane(b, "y")[0]], -1) for b in case.blocks])
    rows = []
    for b in case.blocks:
        x, y = _plane(b, "x"), _plane(b, "y")
        pts = np.stack([x.ravel(), y.ravel()], -1)
        d = np.full(len(pts), np.inf)
        for c0 in range(0, len(wall), 256):
            w = wall[c0:c0 + 256]
            d = np.minimum(d, np.min(np.hypot(pts[:, None, 0] - w[None, :, 0], pts[:, None, 1] - w[None, :, 1]), 1))
        n = len(pts)
        par = [(prm["t"] - 0.115) / 0.035, prm["m"] / 0.02 - 1.0, (prm["p"] - 0.4) / 0.2,
               (prm["aoa_deg"] - 2.0) / 4.0, (prm["ma"] - 0.5) / 0.2, (np.log10(prm["re"]) - 6.5) / 0.5]
        f = np.stack([np.tanh(pts[:, 0] - 0.5), np.tanh(pts[:, 1]), np.log10(np.maximum(d, 1e-7)) / 3.0 + 1.0]
                     + [np.full(n, v) for v in par], -1)
        rows.append(f)
    return np.concatenate(rows).astype(np.float32)


def naca_targets(case: Case) -> np.ndarray:
    """(rho - 1, u - cos aoa, v - sin aoa, p/p0 - 1, log(nu_t / nu_t,inf)) on
    the first k-plane of the physical nodes of every block."""
    cfg = case.cfg
    a = np.deg2rad(cfg.aoa_deg)
    p0 = 1.0 / GAMMA / cfg.ma ** 2
    rows = []
    for b in case.blocks:
        pri = _plane(b, "pri_v")
        nut = _plane(b, "nut")
        t = np.stack([pri[..., 0] - 1.0, pri[..., 1] - np.cos(a), pri[..., 2] - np.sin(a), pri[..., 4] / p0 - 1.0,
                      np.log(np.maximum(nut, 1e-12) / cfg.nutinf)], -1)
        rows.append(t.reshape(-1, NACA_OUT))
    return np.concatenate(rows).astype(np.float32)


def naca_set_state(cfg: Config, blocks, pred: np.ndarray) -> None:
    """q and nu_t of every node of the member's blocks from the predicted
    first-plane values (copied along k; ghost nodes take the nearest physical
    node's value before the start-up BCs and halos overwrite them)."""
    a = np.deg2rad(cfg.aoa_deg)
    p0 = 1.0 / GAMMA / cfg.ma ** 2
    off = 0
    for b in blocks:
        nj, ni = b.nj, b.ni
        pr = pred[off:off + nj * ni].reshape(nj, ni, NACA_OUT).astype(np.float64)
        off += nj * ni
        rho = np.maximum(1.0 + pr[..., 0], 0.05)
        u = np.cos(a) + pr[..., 1]
        v = np.sin(a) + pr[..., 2]
        p = p0 * np.maximum(1.0 + pr[..., 3], 0.05)
        nut = cfg.nutinf * np.exp(np.clip(pr[..., 4], -20.0, 20.0))
        q = np.stack([rho, rho * u, rho * v, np.zeros_like(rho), p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v)], -1)
        is_, ie, js, je, ks, ke = b.box
        ii = np.clip(np.arange(is_, ie + 1), 1, ni) - 1
        jj = np.clip(np.arange(js, je + 1), 1, nj) - 1
        b.fields["q"][...] = q[jj][:, ii][None, :, :, :]
        b.fields["nut"][...] = nut[jj][:, ii][None, :, :]


def case_residuals(batch: Case, cases, r_blocks: np.ndarray) -> np.ndarray:
    """Each member's density residual norm from its blocks' norms (the norm
    over the member's nodes: block sums weighted by their node counts)."""
    out = []
    for first, last in grids.batch_members(cases):
        nodes = np.array([b.nodes for b in batch.blocks[first:last]], dtype=float)
        out.append(np.sqrt(np.sum(r_blocks[first:last, 0] ** 2 * nodes) / np.sum(nodes)))
    return np.array(out)


def run_family_batch(solver, members, iters: int, chunk: int = 100, warm: Dict[int, np.ndarray] = None,
                     mixed: bool = False):
    """The members (multi-block cases) as one batch for `iters` iterations
    from the freestream or, for the members in `warm`, from the predicted
    field.  Returns each member's density residual after iteration 1 and after
    every further chunk (rows), the wall time and the batch case (host arrays
    synchronised)."""
    cases = [m[0] for m in members]
    batch, params = grids.batch_case(cases)
    gc = solver.GpuCase(batch, block_params=params)
    try:
        gc.compute_geometry()
        gc.init_flowfield()
        if warm:
            gc.sync_to_host(solver.ALL)
            spans = grids.batch_members(cases)
            for i, pred in warm.items():
                first, last = spans[i]
                naca_set_state(cases[i].cfg, batch.blocks[first:last], pred)
            gc.sync_to_device(solver.mask("q", "nut"))
        gc.start()
        gc.set_precision(mixed)
        gc.set_retirement(True)
        gc.use_graphs(True)
        t0 = time.perf_counter()
        gc.step(1, history=False)
        res = [case_residuals(batch, cases, gc.residual_blocks())]
        for _ in range(iters // chunk):
            gc.step(chunk, history=False)
            res.append(case_residuals(batch, cases, gc.residual_blocks()))
        wall = time.perf_counter() - t0
        gc.sync_to_host(solver.ALL)
        # each member's status: the OR of its blocks' words (a retired member
        # is frozen where it failed)
        bst = gc.block_status()
        status = np.array([np.bitwise_or.reduce(bst[a:e]) for a, e in grids.batch_members(cases)])
        return np.array(res), wall, batch, status
    finally:
        gc.close()
