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
