"""Reference input formats (aerocfd_b200.io): Control.in, grid and bcinfo
readers follow the reference's list-directed reads
(sub_init_readcontrolfile.f90:30-47, sub_init_allocatememory.f90:36-71 and
:380-410, sub_init_readbcinfo.f90:45-104); the writers' output reads back
exactly."""
import numpy as np

from aerocfd_b200 import grids, io


def test_case_round_trip(tmp_path):
    for make in (lambda: grids.naca_ogrid(nblk=4, ni=33, nj=17, nk=3), lambda: grids.flat_plate(ni=17, nj=13, nk=5)):
        case = make()
        path = io.save_case(case, str(tmp_path / case.name))
        back, ctl = io.load_case(path)
        assert back.cfg.iflags().tolist() == case.cfg.iflags().tolist()
        assert np.array_equal(back.cfg.params()[:6], case.cfg.params()[:6])
        for a, b in zip(case.blocks, back.blocks):
            assert (a.ni, a.nj, a.nk) == (b.ni, b.nj, b.nk)
            assert a.box == b.box and a.box0 == b.box0 and a.box1 == b.box1
            assert [vars(s) for s in a.subfaces] == [vars(s) for s in b.subfaces]
            s = a.sl(a.box0)
            for n in ("x", "y", "z"):
                assert np.array_equal(a.fields[n][s], b.fields[n][s])


CONTROL = """! comment
! comment
3, 0, 0, 2.5d0, 1.0D-3
!
!
0.5 5000.0 288.15 2.0
!
!
2.0 2.0 1.0 4.0 1.5 0.0
!
!
3 4 0 2 2 0
!
!
100 3000 'naca.grd' "naca.inp" 0 'restart.dat' 0 0
!
!
0 0.0 0.0 0 0 0 0 0 0 0
"""


def test_control_list_directed(tmp_path):
    p = tmp_path / "Control.in"
    p.write_text(CONTROL)
    c = io.read_control(str(p))
    assert (c.iflag_dimension, c.iflag_solver, c.iflag_time) == (3, 0, 0)
    assert c.cfl == 2.5 and c.dt == 1e-3
    assert (c.ma, c.re, c.tinf, c.aoa) == (0.5, 5000.0, 288.15, 2.0)
    assert (c.scale_x, c.scale_y, c.lref, c.sref) == (2.0, 2.0, 4.0, 1.5)
    assert (c.iflag_inviscid, c.iflag_timeadvance, c.iflag_turbulence) == (4, 2, 2)
    assert (c.grid, c.bcinfo, c.ntstep) == ("naca.grd", "naca.inp", 3000)
    cfg = c.config()
    assert cfg.buffer_length == 2 and cfg.turbulence == 2 and cfg.aoa_deg == 2.0


def test_grid_records_scaling_and_2d(tmp_path):
    # values spread over records of any length, repeat counts, d exponents
    p = tmp_path / "g.dat"
    p.write_text("1\n3 2\n0.0 1.0d0 2*2.0\n  3.0, 4.0\n5*7.0 8.0\n")
    (ni, nj, nk, X, Y, Z), = io.read_grid(str(p), dimension=2, scale=(2.0, 1.0, 1.0), lref=0.5)
    assert (ni, nj, nk) == (3, 2, 1)
    assert np.array_equal(X.ravel(), np.array([0.0, 1.0, 2.0, 2.0, 3.0, 4.0]) * 4.0)
    assert np.array_equal(Y.ravel(), np.array([7.0] * 5 + [8.0]) * 2.0)
    assert not Z.any()


def test_bcinfo_2d_rows(tmp_path):
    p = tmp_path / "bc.dat"
    p.write_text("h\nh\nh\nb\nb\n2\nh\n1 1 1 1 1 9 -50 0 0 0\n2 3 1 5 1 1 2 3 1 0\nend\n")
    (subs,) = io.read_bcinfo(str(p), 1, dimension=2)
    assert [(s.face, s.is_, s.ie, s.js, s.je, s.ks, s.ke, s.blk_t, s.subface_t, s.ori) for s in subs] == [
        (1, 1, 1, 1, 9, 1, 1, -50, 0, 0), (3, 1, 5, 1, 1, 1, 1, 2, 3, 1)]


def test_flowfield_restart_round_trip(tmp_path, oracle_mod):
    """A flow field written by write_flowfield restarts the same state: q
    within a few ulps (q is rebuilt from d, u, v, w, p), nut exactly, and the
    primitive variables the reference's restart derives, with its quirks
    (q2 = d**2 + u**2 + v**2 in t, hence p; c = sqrt(p)/ma); those feed the first physical_bc
    of the start-up, so a restarted run does not continue the original one bit
    for bit in the reference either."""
    make = lambda: grids.flat_plate(ni=17, nj=13, nk=5)
    ca = make()
    oa = oracle_mod.OracleCase(ca)
    oa.geometry()
    oa.init_flowfield()
    oa.start()
    oa.iterate(5)
    path = str(tmp_path / "flowfield.dat")
    io.write_flowfield(path, ca)
    cb = make()
    io.read_restart(path, cb)
    ma, gamma = cb.cfg.ma, 1.4
    cv = 1.0 / gamma / (gamma - 1.0) / ma / ma
    for a, b in zip(ca.blocks, cb.blocks):
        s = a.sl(a.box0)
        qa, qb = a.fields["q"][s], b.fields["q"][s]
        assert np.max(np.abs(qa - qb) / np.maximum(np.abs(qa), 1e-300)) < 1e-14
        assert np.array_equal(a.fields["nut"][s], b.fields["nut"][s])
        pa, pb = a.fields["pri_v"][s], b.fields["pri_v"][s]
        assert np.allclose(pb[..., :4], pa[..., :4], rtol=1e-14, atol=1e-15)
        d, u, v = pb[..., 0], pb[..., 1], pb[..., 2]
        assert np.array_equal(pb[..., 5], (qb[..., 4] / d - 0.5 * (d ** 2 + u ** 2 + v ** 2)) / cv)
        assert np.array_equal(pb[..., 4], d * pb[..., 5] / gamma / ma / ma)
        assert np.array_equal(pb[..., 6], np.sqrt(pb[..., 4]) / ma)
        assert np.all(b.fields["dt"][s] == cb.cfg.dt) and np.all(b.fields["amu"][s][..., 0] == 1.0)
        assert not b.fields["rhs"][s].any()


def test_surface_file_round_trip(tmp_path):
    """write_surface / read_surface: headers and values survive exactly,
    including a zone without nodes."""
    rng = np.random.default_rng(0)
    zones = np.array([[1, 3, 5, 1, 3], [2, 4, 0, 1, 3], [2, 5, 2, 4, 1]])
    rows = rng.standard_normal((15 + 8, 4)) * 10.0 ** rng.integers(-8, 8, (23, 4))
    path = tmp_path / "surfcp.dat"
    io.write_surface(str(path), zones, rows)
    back = io.read_surface(str(path))
    assert [z for z, _ in back] == [(5, 1, 3), (0, 1, 3), (2, 4, 1)]
    assert np.array_equal(np.concatenate([r for _, r in back]), rows)
    assert io.surface_path(12, 3) == "result/surfcp_000012_0003.dat"


def test_flowfield_and_restart_2d(tmp_path):
    """2-D mode: flowfield_output writes x, y, d, u, v, w, p, nut and a zone
    without a k extent (sub_output_flowfield.f90:36-57); the 2-D restart
    (sub_init_flowfield.f90:163-210) reads seven values per record, x, y, d,
    u, v, p, nut, with w = 0."""
    from aerocfd_b200.case import IFLAG_2D
    case = grids.bump_channel_2d(ni=9, nj=5)
    rng = np.random.default_rng(0)
    for b in case.blocks:
        s = b.sl(b.box0)
        b.fields["pri_v"][s] = 1.0 + rng.random(b.fields["pri_v"][s].shape)
        b.fields["nut"][s] = rng.random(b.fields["nut"][s].shape)
    path = tmp_path / "ff2d.dat"
    io.write_flowfield(str(path), case)
    lines = path.read_text().splitlines()
    assert lines[0].split() == ["variables", "=", "x,y,d,u,v,w,p,nut"]
    assert lines[1].split() == ["zone", "i=", str(case.blocks[0].ni), "j=", str(case.blocks[0].nj),
                                "datapacking=point"]
    assert len(lines[2].split()) == 8
    # a restart file in the 2-D record layout (seven values per line)
    rst = tmp_path / "restart2d.dat"
    want = {}
    with open(rst, "w") as f:
        for b in case.blocks:
            n = b.ni * b.nj
            vals = 0.5 + rng.random((n, 7))
            want[b.m] = vals
            f.write(" variables = x,y,d,u,v,p,nut\n zone\n")
            for row in vals:
                f.write(" ".join(f"{v:.17e}" for v in row) + "\n")
    cb = grids.bump_channel_2d(ni=9, nj=5)
    cb.cfg.turbulence = 2
    io.read_restart(str(rst), cb)
    for b in cb.blocks:
        s = b.sl(b.box0)
        v = want[b.m]
        col = lambda c: v[:, c].reshape(1, b.nj, b.ni)
        d, u, vv, p = col(2), col(3), col(4), col(5)
        q = b.fields["q"][s]
        assert np.array_equal(q[..., 0], d)
        assert np.array_equal(q[..., 1], d * u) and np.array_equal(q[..., 2], d * vv)
        assert np.all(q[..., 3] == 0.0)
        assert np.array_equal(b.fields["nut"][s], col(6))
        gamma, ma = 1.4, cb.cfg.ma
        cv = 1.0 / gamma / (gamma - 1.0) / ma / ma
        t = p / d * gamma * ma * ma
        assert np.array_equal(q[..., 4], d * t * cv + 0.5 * d * (u * u + vv * vv + 0.0 * 0.0))
    assert cb.cfg.dimension == IFLAG_2D
