"""Known-answer tests that pin the CPU oracle (the reference ships no golden
vectors and cannot be compiled here, so the restatement is pinned by
identities the discretisation must satisfy)."""
import ctypes

import numpy as np
import pytest

from aerocfd_b200 import grids
from aerocfd_b200.case import Block, Case, Config, Subface, BC_SYMM, IFLAG_NSSOLVER
from conftest import perturb


def _d(x):
    return ctypes.byref(ctypes.c_double(x))


def _i(x):
    return ctypes.byref(ctypes.c_int(x))


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def small_bump(**kw):
    return grids.bump_channel(ni=25, nj=13, nk=5, **kw)


def test_freestream_preserved_on_curvilinear_grid(oracle_mod):
    """Uniform flow on the bump grid: the conservative metrics make the WENO3 +
    Roe residual vanish to round-off, the viscous residual is exactly zero and
    an implicit step leaves q unchanged."""
    case = small_bump(cfg=Config(solver=IFLAG_NSSOLVER, ma=0.5, re=1e4, cfl=5.0))
    oc = oracle_mod.OracleCase(case)
    oc.geometry()
    oc.init_flowfield()
    b = case.blocks[0]
    f = b.fields
    L = oc.L
    L.oracle_inviscid_flux_1(_p(f["rhsi"]), _p(f["q"]), _p(f["dxidx"]), _p(f["inv_j"]),
                             *oracle_mod.box_args(b.box), *oracle_mod.box_args(b.box0),
                             *oracle_mod.box_args(b.box1), _d(1.4))
    flux_scale = 1.0 / 0.5 ** 2 * np.max(np.abs(f["dxidx"][b.sl(b.box0)])) * np.max(f["inv_j"])
    assert np.max(np.abs(f["rhsi"])) < 1e-12 * flux_scale
    q0 = f["q"].copy()
    consts = oc.consts()
    L.oracle_viscous_flux(_p(f["rhsv"]), _p(f["pri_v"]), _p(f["amu"]), _p(f["vor"]), _p(f["dudx"]),
                          _p(f["tao"]), _p(f["dxidx"]), _p(f["inv_j"]), _d(288.15), _d(0.72), _d(0.9),
                          _d(1.4), _d(consts[5]), _d(1e4), *oracle_mod.box_args(b.box),
                          *oracle_mod.box_args(b.box0), *oracle_mod.box_args(b.box1), _i(1))
    assert np.all(f["rhsv"] == 0.0)
    f["rhsi"][...] = 0.0
    L.oracle_implicit1st(_p(f["q"]), _p(f["dt"]), _p(f["pri_v"]), _p(f["rhs"]), _p(f["rhsi"]),
                         _p(f["rhsv"]), _p(f["dxidx"]), _p(f["inv_j"]), *oracle_mod.box_args(b.box),
                         *oracle_mod.box_args(b.box0), *oracle_mod.box_args(b.box1), _d(1.4), _d(5.0),
                         _p(f["x"]), _p(f["y"]), _p(f["z"]))
    assert np.array_equal(f["q"], q0)


def test_weno3_reproduces_linear_data(oracle_mod):
    """Both one-sided WENO3 states of linear data equal the face value."""
    nx = 12
    b = [1, nx, 1, 1, 1, 1]
    f = np.zeros((1, 1, nx, 5))
    i = np.arange(1, nx + 1)
    for c in range(5):
        f[0, 0, :, c] = 0.7 + 0.13 * (c + 1) * i
    r0 = [2, nx - 3, 1, 1, 1, 1]
    for direction in (1, -1):
        df = np.zeros_like(f)
        oracle_mod.lib().oracle_thirdorder_weno(_p(df), _p(f), *oracle_mod.box_args(b),
                                                *oracle_mod.box_args(r0), _i(1), _i(direction))
        for face in range(r0[0] - 1, r0[1] + 1):
            if direction == -1 and face == b[0]:
                # left state at i == is is the one-sided copy f(is) (:50-51)
                want = 0.7 + 0.13 * np.arange(1, 6) * face
            else:
                want = 0.7 + 0.13 * np.arange(1, 6) * (face + 0.5)
            np.testing.assert_allclose(df[0, 0, face - 1], want, rtol=1e-14, atol=1e-14)


def test_roe_consistency(oracle_mod):
    """Equal left and right states: the Roe flux is the physical contravariant
    flux F = (rho U, rho u U + kx p, rho v U + ky p, rho w U + kz p, rho H U)
    with k the face-averaged metric/J."""
    rng = np.random.default_rng(3)
    b = [1, 2, 1, 1, 1, 1]
    for trial in range(20):
        d, u, v, w = 1 + 0.2 * rng.random(), rng.normal(), rng.normal(), rng.normal()
        p = 2.0 + rng.random()
        state = np.array([d, u, v, w, p])
        ql = np.zeros((1, 1, 2, 5)); ql[0, 0, 0] = state
        qr = ql.copy()
        dxidx = rng.normal(size=(1, 1, 2, 9))
        inv_j = 0.5 + rng.random((1, 1, 2))
        flux = np.zeros((1, 1, 2, 5))
        r0 = [2, 1, 1, 1, 1, 1]  # one face, i = 1 (between nodes 1 and 2)
        oracle_mod.lib().oracle_roe_3d(_p(ql), _p(qr), _p(flux), _p(dxidx), _p(inv_j), _d(1.4),
                                       *oracle_mod.box_args(b), *oracle_mod.box_args(r0), _i(1))
        k = 0.5 * (dxidx[0, 0, 0, :3] * inv_j[0, 0, 0] + dxidx[0, 0, 1, :3] * inv_j[0, 0, 1])
        U = u * k[0] + v * k[1] + w * k[2]
        H = 1.4 * p / (0.4 * d) + 0.5 * (u * u + v * v + w * w)
        want = np.array([d * U, d * u * U + k[0] * p, d * v * U + k[1] * p, d * w * U + k[2] * p, d * H * U])
        np.testing.assert_allclose(flux[0, 0, 0], want, rtol=1e-13, atol=1e-13)


def test_calc_jm_is_flux_jacobian(oracle_mod):
    """calc_jm equals the central-difference Jacobian of the contravariant flux."""
    g = 1.4
    rng = np.random.default_rng(5)

    def F(q, k):
        d, mu, mv, mw, e = q
        U = (k[0] * mu + k[1] * mv + k[2] * mw) / d
        p = (g - 1) * (e - 0.5 * (mu * mu + mv * mv + mw * mw) / d)
        return np.array([d * U, mu * U + k[0] * p, mv * U + k[1] * p, mw * U + k[2] * p, (e + p) * U])

    for _ in range(10):
        q = np.array([1 + 0.3 * rng.random(), rng.normal(), rng.normal(), rng.normal(), 0.0])
        q[4] = 3.0 + 0.5 * (q[1] ** 2 + q[2] ** 2 + q[3] ** 2) / q[0]
        k = rng.normal(size=3)
        a = np.zeros(25)
        oracle_mod.lib().oracle_calc_jm(_p(a), *[_d(x) for x in q], *[_d(x) for x in k], _d(g))
        A = a.reshape(5, 5, order="F")
        J = np.zeros((5, 5))
        h = 1e-6
        for c in range(5):
            dq = np.zeros(5); dq[c] = h
            J[:, c] = (F(q + dq, k) - F(q - dq, k)) / (2 * h)
        np.testing.assert_allclose(A, J, rtol=1e-6, atol=1e-7)


def test_lusgs_single_node_and_zero_rhs(oracle_mod):
    """With one updated node the LU-SGS update is rhs/diag/inv_j; zero rhs
    gives dq = 0."""
    case = grids.bump_channel(ni=3, nj=3, nk=3)
    oc = oracle_mod.OracleCase(case)
    oc.geometry()
    oc.init_flowfield()
    b = case.blocks[0]
    f = b.fields
    rng = np.random.default_rng(1)
    f["rhsi"][...] = rng.normal(size=f["rhsi"].shape)
    q0 = f["q"].copy()
    oc.L.oracle_implicit1st(_p(f["q"]), _p(f["dt"]), _p(f["pri_v"]), _p(f["rhs"]), _p(f["rhsi"]),
                            _p(f["rhsv"]), _p(f["dxidx"]), _p(f["inv_j"]), *oracle_mod.box_args(b.box),
                            *oracle_mod.box_args(b.box0), *oracle_mod.box_args(b.box1), _d(1.4), _d(5.0),
                            _p(f["x"]), _p(f["y"]), _p(f["z"]))
    # node (2,2,2) is the only updated node
    n = (1, 1, 1)
    pri = f["pri_v"][n]
    m = f["dxidx"][n]
    diag = 1.0 / f["dt"][n]
    for d in range(3):
        k = m[3 * d:3 * d + 3]
        diag += abs(k @ pri[1:4]) + abs(pri[6] * np.sqrt(k @ k))
    want = q0[n] + f["rhsi"][n] / diag / f["inv_j"][n]
    np.testing.assert_allclose(f["q"][n], want, rtol=1e-14)
    outside = np.ones(f["q"].shape[:3], bool); outside[n] = False
    assert np.array_equal(f["q"][outside], q0[outside])


def ogrid_case(nblk=4, ni=17, nj=9, nk=3):
    return grids.naca_ogrid(nblk=nblk, ni=ni, nj=nj, nk=nk)


def test_halo_coordinates_continuous_across_ogrid_interfaces(oracle_mod):
    """After the coordinate halo, the two ghost layers of every block equal
    the neighbour's first two interior layers (orientation code 2 between an
    i+ and an i- face)."""
    case = ogrid_case()
    oc = oracle_mod.OracleCase(case)
    oc.L.oracle_updatebuffercoordinate()
    nb = len(case.blocks)
    for m, b in enumerate(case.blocks):
        left = case.blocks[(m - 1) % nb]
        right = case.blocks[(m + 1) % nb]
        for name in ("x", "y", "z"):
            a = b.fields[name]
            # ghost i = 0, -1 (array index 1, 0) <- left block's i = ni-1, ni-2
            la = left.fields[name]
            ni = b.ni
            np.testing.assert_array_equal(a[:, :, 1], la[:, :, (ni - 1) - left.box[0]])
            np.testing.assert_array_equal(a[:, :, 0], la[:, :, (ni - 2) - left.box[0]])
            ra = right.fields[name]
            np.testing.assert_array_equal(a[:, :, ni + 1 - b.box[0]], ra[:, :, 2 - right.box[0]])
            np.testing.assert_array_equal(a[:, :, ni + 2 - b.box[0]], ra[:, :, 3 - right.box[0]])


@pytest.mark.parametrize("ori", [1, 2, 3, 4])
def test_halo_orientation_round_trip(oracle_mod, ori):
    """Two single-block-wide cubes joined i+ -> i- with each orientation code:
    the ghost layers receive a permutation of the neighbour's interior layers
    that the matching code maps back (every donor value arrives exactly once)."""
    n = 5
    cfg = Config()
    subs_a = [Subface(1, 2, n, n, 1, n, 1, n, 2, 1, ori)] + [
        Subface(2 + f, f, *(1, 1, 1, n, 1, n) if f == 1 else (1, n, 1, 1, 1, n) if f == 3 else
                (1, n, n, n, 1, n) if f == 4 else (1, n, 1, n, 1, 1) if f == 5 else (1, n, 1, n, n, n),
                BC_SYMM) for f in (1, 3, 4, 5, 6)]
    partner = {1: 1, 2: 2, 3: 3, 4: 4}[ori]
    subs_b = [Subface(1, 1, 1, 1, 1, n, 1, n, 1, 1, partner)] + [
        Subface(2 + f, f, *(n, n, 1, n, 1, n) if f == 2 else (1, n, 1, 1, 1, n) if f == 3 else
                (1, n, n, n, 1, n) if f == 4 else (1, n, 1, n, 1, 1) if f == 5 else (1, n, 1, n, n, n),
                BC_SYMM) for f in (2, 3, 4, 5, 6)]
    A = Block(1, n, n, n, subs_a)
    B = Block(2, n, n, n, subs_b)
    case = Case("pair", cfg, [A, B])
    rng = np.random.default_rng(ori)
    for blk in (A, B):
        blk.fields["q"][...] = rng.random(blk.fields["q"].shape)
    oc = oracle_mod.OracleCase(case)
    oc.updatebuffer()
    # every ghost value of A is one of B's layer-1/2 interior values, bijectively
    ga = A.fields["q"][:, :, n - A.box[0] + 1:, 0].ravel()
    src = B.fields["q"][:, :, 1 - B.box[0] + 1:1 - B.box[0] + 3, 0].ravel()
    assert sorted(ga) == sorted(src)
    gb = B.fields["q"][:, :, :2, 0].ravel()
    srcb = A.fields["q"][:, :, n - A.box[0] - 2:n - A.box[0], 0].ravel()
    assert sorted(gb) == sorted(srcb)


def test_average_is_symmetric(oracle_mod):
    """average1 + average2 leave both copies of every shared interface node
    equal to (a+b)/2."""
    case = ogrid_case()
    for b in case.blocks:
        b.fields["q"][...] = np.random.default_rng(b.m).random(b.fields["q"].shape)
    before = [b.fields["q"].copy() for b in case.blocks]
    oc = oracle_mod.OracleCase(case)
    oc.average1()
    oc.average2()
    nb = len(case.blocks)
    for m, b in enumerate(case.blocks):
        right = case.blocks[(m + 1) % nb]
        mine = b.fields["q"][:, :, b.ni - b.box[0]]
        theirs = right.fields["q"][:, :, 1 - right.box[0]]
        np.testing.assert_array_equal(mine, theirs)
        want = (before[m][:, :, b.ni - b.box[0]] + before[(m + 1) % nb][:, :, 1 - right.box[0]]) * 0.5
        np.testing.assert_array_equal(mine, want)


def test_residual_of_known_field(oracle_mod):
    case = small_bump()
    oc = oracle_mod.OracleCase(case)
    b = case.blocks[0]
    s1 = b.sl(b.box1)
    b.fields["rhs"][s1] = 2.0
    b.fields["dt"][...] = 0.5
    b.fields["inv_j"][...] = 1.0
    r = oc.residual()
    n1 = (b.box1[1] - b.box1[0] + 1) * (b.box1[3] - b.box1[2] + 1) * (b.box1[5] - b.box1[4] + 1)
    np.testing.assert_allclose(r[:5], np.sqrt(n1 / b.nodes), rtol=1e-15)
    assert r[5] == 0.0


def test_sa_source_vanishes_at_zero_eddy_viscosity(oracle_mod):
    """nut = 0 everywhere: advection, diffusion, production and destruction of
    the SA equation are zero, so sa_rhs = 0.  (The implicit diagonal is NaN
    there: the source linearisation evaluates 0 * g**(-7) with g = 0,
    sub_tur_sa.f90:615-616, so nut itself is not checked.)"""
    cfg = Config(solver=IFLAG_NSSOLVER, turbulence=2, ma=0.3, re=1e5)
    case = small_bump(cfg=cfg)
    oc = oracle_mod.OracleCase(case)
    oc.geometry(walldist=False)
    oc.init_flowfield()
    b = case.blocks[0]
    f = b.fields
    f["nut"][...] = 0.0
    f["dist"][...] = 0.1
    oc.L.oracle_sa_model(_p(f["nut"]), _p(f["sa_rhs"]), _p(f["dt"]), _p(f["pri_v"]), _p(f["amu"]),
                         _p(f["dudx"]), _p(f["vor"]), _p(f["dxidx"]), _p(f["inv_j"]), _p(f["alpha"]),
                         _p(f["beta"]), _p(f["ggamma"]), _p(f["length"]), _p(f["dist"]),
                         _p(f["spacing"]), _d(1e5), _d(5.0), *oracle_mod.box_args(b.box),
                         *oracle_mod.box_args(b.box0), *oracle_mod.box_args(b.box1))
    assert np.all(f["sa_rhs"] == 0.0)


def test_iteration_reduces_residual_on_bump(oracle_mod):
    """The assembled iteration (main.f90:343-447) converges on the bump."""
    case = small_bump()
    oc = oracle_mod.OracleCase(case)
    oc.geometry()
    oc.init_flowfield()
    oc.start()
    h = oc.iterate(40)
    assert np.all(np.isfinite(h))
    assert h[-1, 0] < 0.5 * h[0, 0]


# ------------------------------------------- extension inviscid schemes
def _cartesian_line(oracle_mod, n, inviscid, ny=9, nz=9, amp=0.2):
    """A Cartesian n x ny x nz box of spacing h with physical faces only, the
    flow varying along x alone: rho = 1 + 0.2 sin(pi x / 2), u = 0.5, v = w = 0,
    p = 1/1.4.  Returns the oracle's rhsi / inv_j on the centre line and the
    exact -dF/dx there (the metric gives the face flux h^2 F, so
    rhsi / inv_j approximates -dF/dx)."""
    cfg = Config(ma=0.5, inviscid=inviscid)
    subs = [Subface(f, f, *box, BC_SYMM) for f, box in enumerate(
        [(1, 1, 1, ny, 1, nz), (n, n, 1, ny, 1, nz), (1, n, 1, 1, 1, nz), (1, n, ny, ny, 1, nz),
         (1, n, 1, ny, 1, 1), (1, n, 1, ny, nz, nz)], start=1)]
    blk = Block(1, n, ny, nz, subs, cfg.buffer_length, cfg.dimension)
    case = Case("line", cfg, [blk])
    oc = oracle_mod.OracleCase(case)  # configures the oracle's flags
    h = 1.0 / (n - 1)
    x = (np.arange(n) * h)[None, None, :] * np.ones((nz, ny, 1))
    f = blk.fields
    rho = 1.0 + amp * np.sin(np.pi * x / 2.0)
    u, p, gam = 0.5, 1.0 / 1.4, 1.4
    f["q"][..., 0] = rho
    f["q"][..., 1] = rho * u
    f["q"][..., 2] = 0.0
    f["q"][..., 3] = 0.0
    f["q"][..., 4] = p / (gam - 1.0) + 0.5 * rho * u * u
    f["dxidx"][...] = 0.0
    for c in (0, 4, 8):
        f["dxidx"][..., c] = 1.0 / h
    f["inv_j"][...] = h ** 3
    name = {5: "weno5", 8: "wcns5"}[inviscid]
    getattr(oc.L, f"oracle_inviscid_flux_{name}")(_p(f["rhsi"]), _p(f["q"]), _p(f["dxidx"]), _p(f["inv_j"]),
                                                  *oracle_mod.box_args(blk.box), *oracle_mod.box_args(blk.box0),
                                                  *oracle_mod.box_args(blk.box1), _d(1.4))
    jc, kc = ny // 2, nz // 2
    got = f["rhsi"][kc, jc, :, :] / h ** 3
    xs = x[0, 0, :]
    drho = amp * np.pi / 2.0 * np.cos(np.pi * xs / 2.0)
    exact = -np.stack([drho * u, drho * u * u, 0 * xs, 0 * xs, 0.5 * drho * u ** 3], axis=1)
    return got, exact, f["rhsi"]


@pytest.mark.parametrize("inviscid,order", [(5, 4.0), (8, 3.6)])
def test_extension_scheme_order_of_accuracy(oracle_mod, inviscid, order):
    """Steger-Warming + WENO5 (5th order) and WCNS5 with the hybrid 4th-order
    difference, on smooth monotone data away from the boundary closures: the
    error of -dF/dx falls at least at the stated rate when h halves."""
    errs = []
    for n in (33, 65):
        got, exact, _ = _cartesian_line(oracle_mod, n, inviscid)
        sl = slice(5, n - 5)
        errs.append(np.max(np.abs(got[sl] - exact[sl])))
    rate = np.log2(errs[0] / errs[1])
    print("errors", errs, "observed order", rate)
    assert rate >= order


@pytest.mark.parametrize("inviscid", [5, 8])
def test_extension_schemes_keep_uniform_flow_on_cartesian_grid(oracle_mod, inviscid):
    """Uniform flow on a Cartesian box: the interior faces see identical
    stencils, so the residual is zero there to the last bit."""
    got, exact, rhsi = _cartesian_line(oracle_mod, 21, inviscid, amp=0.0)
    assert np.all(np.isfinite(rhsi))
    assert np.all(got[5:-5] == 0.0)


def test_buffer_length_follows_the_scheme():
    """bufferLength is derived from iflag_inviscid (main.f90:81): 2 for the
    3rd-order WENO, 3 for the 5th-order extension schemes, an error otherwise."""
    assert Config(inviscid=4).buffer_length == 2
    assert Config(inviscid=5).buffer_length == 3
    assert Config(inviscid=8).buffer_length == 3
    with pytest.raises(ValueError):
        Config(inviscid=6).buffer_length
