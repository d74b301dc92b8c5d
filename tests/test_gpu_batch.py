"""Batches of independent cases (aero_set_block_params): each block of the
batch follows the oracle's run of its case alone (Mach number, size and bump
height differ per case), step by step; CUDA-graph replay gives bit-identical
results; aero_autotune restores the state it started from and changes no
result."""
import numpy as np
import pytest

from aerocfd_b200 import grids
from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def gpu():
    from aerocfd_b200 import build, solver
    build.build()
    return solver


def small_batch():
    rng = np.random.default_rng(7)
    cases = []
    for c in range(5):
        cfg = grids.Config(solver=grids.IFLAG_EULERSOLVER, ma=float(rng.uniform(0.3, 0.7)), re=1.0e6, cfl=5.0)
        cases.append(grids.bump_channel(int(rng.integers(17, 40)), int(rng.integers(9, 20)), 5,
                                        h=float(rng.uniform(0.05, 0.12)), cfg=cfg, name=f"b{c}"))
    return cases


def run_oracle(oracle_mod, case, nsteps):
    oc = oracle_mod.OracleCase(case)
    oc.geometry()
    oc.init_flowfield()
    oc.start()
    return oc.iterate(nsteps)


def started_batch(gpu, cases):
    batch, params = grids.batch_case(cases)
    gc = gpu.GpuCase(batch, block_params=params)
    gc.compute_geometry()
    gc.init_flowfield()
    gc.start()
    return batch, gc


def test_batch_blocks_follow_their_own_cases(gpu, oracle_mod):
    cases = small_batch()
    nsteps = 4
    hist = [run_oracle(oracle_mod, c, nsteps) for c in cases]
    batch, gc = started_batch(gpu, small_batch())
    try:
        for s in range(nsteps):
            gc.step(1, history=False)
            r = gc.residual_blocks()
            for m, h in enumerate(hist):
                scale = np.maximum(np.abs(h[s, :5]), 1e-6 * np.abs(h[s, :5]).max())
                assert np.max(np.abs(r[m, :5] - h[s, :5]) / scale) <= 1e-10, (s, m)
        gc.sync_to_host(gpu.mask("q"))
        for m, c in enumerate(cases):
            assert relerr(batch.blocks[m].fields["q"], c.blocks[0].fields["q"]) <= TOL
    finally:
        gc.close()


def test_graphs_and_autotune_change_no_result(gpu):
    qs = []
    for mode in ("plain", "graphs", "autotuned"):
        batch, gc = started_batch(gpu, small_batch())
        try:
            if mode == "autotuned":
                gc.sync_to_host(gpu.mask("q"))
                q_before = [b.fields["q"].copy() for b in batch.blocks]
                desc = gc.autotune(2)
                assert "inviscid_tile=" in desc
                gc.sync_to_host(gpu.mask("q"))
                for b, q in zip(batch.blocks, q_before):
                    assert np.array_equal(b.fields["q"], q)   # state restored
            if mode != "plain":
                gc.use_graphs(True)
            h = gc.step(6)
            gc.sync_to_host(gpu.mask("q"))
            qs.append((h, [b.fields["q"].copy() for b in batch.blocks]))
            assert gc.status() == 0
        finally:
            gc.close()
    for h, q in qs[1:]:
        assert np.array_equal(h, qs[0][0])
        for a, b in zip(q, qs[0][1]):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("make", [lambda: grids.naca_ogrid(nblk=4, ni=33, nj=17, nk=3),
                                  lambda: grids.flat_plate(ni=17, nj=13, nk=7, dy_wall=1e-3),
                                  lambda: naca_2d_sa()])
def test_every_launch_shape_gives_the_same_bits(gpu, make):
    """All launch shapes the autotuner can pick, including the face-based
    inviscid kernels (tile 0, -6 / -8 under register bounds, -10 with its
    stencils staged in shared memory), in FP64 and mixed precision: identical
    histories and states (the default shape is the one checked against the
    oracle)."""
    shapes = [(64, 256, 128, 128, 4), (0, 128, 64, 64, 2), (32, 512, 256, 256, 3), (128, 256, 128, 128, 4),
              (-6, 256, 128, 128, 4), (-8, 128, 256, 64, 3), (-10, 256, 128, 128, 4)]
    for mixed in (False, True):
        ref = None
        for x, shape in enumerate(shapes):
            case = make()
            gc = gpu.GpuCase(case)
            try:
                gc.set_tuning(*shape)
                gc.set_register_bound(x % 2 == 1)  # the register-bounded viscous kernel too
                gc.set_precision(mixed)
                gc.compute_geometry()
                gc.init_flowfield()
                gc.start()
                h = gc.step(4)
                gc.sync_to_host(gpu.mask("q", "rhsi"))
                out = (h, [b.fields["q"].copy() for b in case.blocks], [b.fields["rhsi"].copy() for b in case.blocks])
            finally:
                gc.close()
            if ref is None:
                ref = out
                continue
            assert np.array_equal(out[0], ref[0]), (mixed, shape)
            for a, b in zip(out[1] + out[2], ref[1] + ref[2]):
                assert np.array_equal(a, b), (mixed, shape)


def naca_2d_sa():
    from aerocfd_b200.case import IFLAG_2D, IFLAG_NSSOLVER, IFLAG_SA, Config
    cfg = Config(solver=IFLAG_NSSOLVER, ma=0.5, re=5000.0, aoa_deg=2.0, cfl=2.0, dimension=IFLAG_2D,
                 turbulence=IFLAG_SA)
    return grids.naca_ogrid(nblk=4, ni=33, nj=17, first=1e-3, cfg=cfg)


@pytest.mark.parametrize("make", [lambda: grids.naca_ogrid(nblk=4, ni=33, nj=17, nk=3),
                                  lambda: grids.flat_plate(ni=17, nj=13, nk=7, dy_wall=1e-3),
                                  lambda: grids.bump_channel(129, 65, 9), naca_2d_sa])
def test_sweep_cluster_gives_the_same_bits(gpu, make):
    """The LU-SGS sweep on one CTA per block (staged in shared memory, or from
    global memory when the planes are too large: the 129 x 65 x 9 bump) and
    on clusters of 2, 4 and 8 CTAs per block passing plane values through L2,
    by bulk copies between shared memories, or pipelined by k-slabs, and on
    clusters of 16 CTAs (bulk copies or slabs; a non-portable cluster size,
    taken where the device holds one); the SA sweep (the plate) on one CTA or
    on clusters of k-slabs: identical histories and states, in FP64 and mixed
    precision.  Slab clusters larger than a block's k-extent leave CTAs idle
    (the aerofoil: one k-offset; the 2-D aerofoil: a single plane, so one
    active CTA per slab cluster), and slabs too wide for one CTA fall back to
    the bulk or the L2 exchange (the bump on 2 and 4 CTAs)."""
    from aerocfd_b200 import _lib
    for mixed in (False, True):
        ref = None
        for ctas, exch, sa_ctas in ((1, "l2", 1), (2, "l2", 1), (4, "l2", 1), (8, "l2", 1), (2, "shared", 1),
                                    (4, "shared", 1), (8, "shared", 1), (16, "shared", 1), (2, "slab", 2),
                                    (4, "slab", 4), (8, "slab", 8), (16, "slab", 16), (8, "slab", 1),
                                    (1, "l2", 4), (4, "shared2", 1), (8, "shared2", 2), (8, "shared", 0)):
            case = make()
            gc = gpu.GpuCase(case)
            try:
                try:
                    gc.set_sweep_cluster(ctas)
                    if sa_ctas == 0:  # the bulk sweep prefetching four planes ahead
                        gc.set_sweep_prefetch(4)
                        sa_ctas = 1
                    gc.set_sa_sweep_cluster(sa_ctas)
                except _lib.AeroError:
                    assert 16 in (ctas, sa_ctas)  # the device holds no 16-CTA cluster
                    continue
                gc.set_sweep_exchange(exch)
                gc.set_precision(mixed)
                gc.compute_geometry()
                gc.init_flowfield()
                gc.start()
                h = gc.step(4)
                assert gc.status() == 0, (ctas, exch, sa_ctas)
                gc.sync_to_host(gpu.mask("q", "nut"))
                out = (h, [b.fields["q"].copy() for b in case.blocks], [b.fields["nut"].copy() for b in case.blocks])
            finally:
                gc.close()
            if ref is None:
                ref = out
                continue
            assert np.array_equal(out[0], ref[0]), (mixed, ctas, exch, sa_ctas)
            for a, b in zip(out[1] + out[2], ref[1] + ref[2]):
                assert np.array_equal(a, b), (mixed, ctas, exch, sa_ctas)



def test_failed_case_is_retired_and_the_others_follow_their_own_cases(gpu, oracle_mod):
    """A NaN planted on the host in one case of a running batch (between two
    steps, at an interior node): the next step raises that block's own
    non-finite-residual bit and no other block's; with retirement on, the
    failed case is frozen from then on (its q keeps the bits it had after the
    failing step, its residual counts as 0), and every other case still
    follows the oracle's run of that case alone, to the end."""
    ST_NONFINITE = 2
    cases = small_batch()
    nsteps = 7
    hist = [run_oracle(oracle_mod, c, nsteps) for c in cases]
    batch, gc = started_batch(gpu, small_batch())
    bad = 2
    try:
        gc.set_retirement(True)
        gc.step(2, history=False)
        assert not gc.block_status().any()
        gc.sync_to_host(gpu.mask("q"))
        b = batch.blocks[bad]
        i, j, k = b.box1[0] + 3, b.box1[2] + 2, b.box1[4] + 1
        b.fields["q"][k - b.box[4], j - b.box[2], i - b.box[0], 0] = np.nan
        gc.sync_to_device(gpu.mask("q"))
        gc.step(1, history=False)
        st = gc.block_status()
        assert st[bad] & ST_NONFINITE, st
        assert not np.delete(st, bad).any(), st
        gc.sync_to_host(gpu.mask("q"))
        frozen = b.fields["q"].copy()
        assert np.isnan(frozen).any()
        gc.step(nsteps - 3, history=False)
        r = gc.residual_blocks()
        assert np.array_equal(gc.block_status(), st)
        gc.sync_to_host(gpu.mask("q"))
        assert np.array_equal(b.fields["q"], frozen, equal_nan=True)
        assert np.all(r[bad] == 0.0)
        for m, c in enumerate(cases):
            if m == bad:
                continue
            h = hist[m][-1, :5]
            scale = np.maximum(np.abs(h), 1e-6 * np.abs(h).max())
            assert np.max(np.abs(r[m, :5] - h) / scale) <= 1e-10, m
            assert relerr(batch.blocks[m].fields["q"], c.blocks[0].fields["q"]) <= TOL, m
        gc.clear_block_status()
        assert not gc.block_status().any()
    finally:
        gc.close()


def test_batch_of_multiblock_sa_members_matches_each_member_alone(gpu):
    """Three NACA/SA members (4-block O-grids around different sections,
    all at the same place in space) run as one batch: every member's wall
    distance is to its own aerofoil, and after 5 iterations every member's
    q and nut equal, bit for bit, the same member run alone (the batch shares
    no value between cases)."""
    from aerocfd_b200 import warmstart

    def family():
        return [c for c, _ in warmstart.naca_family(3, seed=7, ni=33, nj=17)]

    alone = []
    for case in family():
        gc = gpu.GpuCase(case)
        try:
            gc.compute_geometry()
            gc.init_flowfield()
            gc.start()
            gc.step(5, history=False)
            assert gc.status() == 0
            gc.sync_to_host(gpu.mask("q", "nut", "dist"))
            alone.append([{f: b.fields[f].copy() for f in ("q", "nut", "dist")} for b in case.blocks])
        finally:
            gc.close()
    cases = family()
    batch, params = grids.batch_case(cases)
    gc = gpu.GpuCase(batch, block_params=params)
    try:
        gc.compute_geometry()
        gc.init_flowfield()
        gc.start()
        gc.step(5, history=False)
        assert gc.status() == 0
        gc.sync_to_host(gpu.mask("q", "nut", "dist"))
    finally:
        gc.close()
    for i, (first, last) in enumerate(grids.batch_members(cases)):
        for ref, b in zip(alone[i], batch.blocks[first:last]):
            for f in ("dist", "q", "nut"):
                assert np.array_equal(b.fields[f], ref[f]), (i, b.m, f)
