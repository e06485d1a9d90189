"""The oracle's Lagrangian-particle routines (orc_bspline3 ... orc_particle_stats).

The reference's particle tracker (weno/src/ParticleTrack.cpp,
update.cpp:1082-1303) interpolates with einspline, an external library that
is absent here and never pinned by the reference; its Evolve loop never calls
the tracker, so no reference run produces particle output.  The oracle
restates einspline's natural cubic B-spline from the mathematics, and these
tests pin that restatement independently: against scipy's natural cubic spline
(a tensor-product spline evaluated by successive 1-D interpolation), against
the interpolation and end conditions it must satisfy, and the tracker and
statistics against direct numpy statements of ParticleTrack.cpp:43-65 and
update.cpp:1134-1181.
"""

import numpy as np
import pytest
from scipy.interpolate import CubicSpline

import gks_ic


def successive_natural(grids, data, p):
    """Value and gradient of the tensor-product natural cubic spline at p (3,)
    by natural 1-D splines along z, then x, then y."""
    y, x, z = p
    A = CubicSpline(grids[2], data, axis=2, bc_type="natural")
    vz, dz = A(z), A(z, 1)
    B = CubicSpline(grids[1], vz, axis=1, bc_type="natural")
    vx, dx = B(x), B(x, 1)
    dzx = CubicSpline(grids[1], dz, axis=1, bc_type="natural")(x)
    C = CubicSpline(grids[0], vx, bc_type="natural")
    g = [C(y, 1), CubicSpline(grids[0], dx, bc_type="natural")(y), CubicSpline(grids[0], dzx, bc_type="natural")(y)]
    return C(y), np.array(g)


@pytest.mark.parametrize("shape", [(9, 11, 10), (4, 6, 5), (14, 14, 14)])
def test_bspline_equals_scipy_natural_spline(oracle, shape):
    rng = np.random.default_rng(sum(shape))
    data = rng.standard_normal(shape)
    h = np.array([0.3, 0.5, 0.7])
    st = np.array([-0.2, 0.1, 1.0])
    grids = [st[a] + h[a] * np.arange(shape[a]) for a in range(3)]
    coef = oracle.bspline3(data)
    n = 40
    pos = np.stack([st[a] + h[a] * (shape[a] - 1) * rng.random(n) for a in range(3)])
    val, grad = oracle.spline_eval(coef, st, 1.0 / h, pos)
    for m in range(n):
        v, g = successive_natural(grids, data, pos[:, m])
        assert abs(val[m] - v) <= 1e-12 * np.abs(data).max()
        assert np.all(np.abs(grad[:, m] - g) <= 1e-12 * np.abs(data).max() / h.min())


def test_bspline_interpolates_and_has_natural_ends(oracle):
    rng = np.random.default_rng(7)
    data = rng.standard_normal((8, 9, 10))
    coef = oracle.bspline3(data)
    # the interpolant equals the data at every node
    idx = np.stack(np.meshgrid(*[np.arange(s) for s in data.shape], indexing="ij")).reshape(3, -1).astype(float)
    val, _ = oracle.spline_eval(coef, [0.0, 0.0, 0.0], [1.0, 1.0, 1.0], idx)
    assert np.abs(val - data.reshape(-1)).max() < 1e-13
    # natural ends: c_0 - 2 c_1 + c_2 = 0 and c_{N-1} - 2 c_N + c_{N+1} = 0 along every axis
    for ax in range(3):
        c = np.moveaxis(coef, ax, 0)
        assert np.abs(c[0] - 2 * c[1] + c[2]).max() < 1e-12
        assert np.abs(c[-3] - 2 * c[-2] + c[-1]).max() < 1e-12


def dhit_block(nc, seed):
    case = gks_ic.make_dhit(nc, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=seed)
    return case, gks_ic.to_conservative_padded(case)


def test_particle_props_of_the_field(oracle):
    """Properties at particles on nodes equal generateSplines' primitives there;
    between nodes they follow the spline of those primitives."""
    nc = 12
    case, W = dhit_block(nc, 3)
    prm = oracle.params(nc, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    dx = prm.dx
    nt = nc + 6
    # particles at the cell centres (j, i, k) = (2, 5, 7) and (0, 0, 11)
    cells = np.array([[2, 5, 7], [0, 0, 11]])
    n = len(cells)
    rec = np.zeros((oracle.PREC_FIELDS, n))
    rec[0:3] = ((cells + 0.5) * dx).T
    oracle.particle_props(W, prm, rec)
    for a, (j, i, k) in enumerate(cells):
        w = W[:, j + 3, i + 3, k + 3]
        den, u, v, ww = w[0], w[1] / w[0], w[2] / w[0], w[3] / w[0]
        p = (den * (case.gam - 1)) * (w[4] / den - 0.5 * (u * u + v * v + ww * ww))
        np.testing.assert_allclose(rec[3:8, a], [den, u, v, ww, p], rtol=1e-12, atol=1e-14)
    # off-node: the same spline, evaluated directly from its coefficients
    rng = np.random.default_rng(5)
    m = 16
    rec = np.zeros((oracle.PREC_FIELDS, m))
    rec[0:3] = rng.random((3, m)) * 2 * np.pi
    oracle.particle_props(W, prm, rec)
    u_nodes = W[1] / W[0]
    start = -3 * dx + 0.5 * dx
    hinv = 1.0 / (((start + (nt - 1) * dx) - start) / (nt - 1))
    val, grad = oracle.spline_eval(oracle.bspline3(u_nodes), [start] * 3, [hinv] * 3, np.ascontiguousarray(rec[0:3]))
    np.testing.assert_array_equal(rec[4], val)
    np.testing.assert_array_equal(rec[11:14], grad)


def test_track_moves_and_wraps_like_update_position(oracle):
    twopi = 2 * np.arctan(1.0) * 4.0
    n = 6
    rec = np.zeros((oracle.PREC_FIELDS, n))
    rec[0] = [0.1, 6.2, 3.0, 0.0, twopi, 1.0]      # y
    rec[1] = [6.25, 0.01, 3.0, 0.0, twopi, 2.0]    # x
    rec[2] = [3.0, 3.0, 0.001, 0.0, twopi, 3.0]    # z
    rec[4] = [1.0, -1.0, 0.5, 0.0, 0.3, 0.0]       # u moves x
    rec[5] = [-2.0, 1.5, 0.0, 0.0, 0.3, 0.0]       # v moves y
    rec[6] = [0.0, 0.0, -0.2, 0.0, 0.3, 0.0]       # w moves z
    dt = 0.05
    want = rec.copy()
    for q, vel in ((0, 5), (1, 4), (2, 6)):
        x = want[q] + want[vel] * dt
        x = np.where(x > twopi, x - twopi, x)
        x = np.where(x < 0, twopi + x, x)
        want[q] = x
    oracle.particle_track(rec, dt)
    np.testing.assert_array_equal(rec, want)
    assert np.all((rec[0:3] >= 0) & (rec[0:3] <= twopi))


def test_particle_stats_formulas(oracle):
    rng = np.random.default_rng(11)
    n = 500
    rec = rng.standard_normal((oracle.PREC_FIELDS, n))
    out = oracle.particle_stats(np.ascontiguousarray(rec))
    U = rec[4:7]
    gu, gv, gw = rec[11:14], rec[14:17], rec[17:20]  # (d/dy, d/dx, d/dz)
    dudx, dudy, dudz = gu[1], gu[0], gu[2]
    dvdx, dvdy, dvdz = gv[1], gv[0], gv[2]
    dwdx, dwdy, dwdz = gw[1], gw[0], gw[2]
    sij = dudx**2 + 0.5 * (dudy + dvdx) ** 2 + 0.5 * (dudz + dwdx) ** 2 + 0.5 * (dwdy + dvdz) ** 2 + dvdy**2 + dwdz**2
    want = [np.mean((U**2).sum(0)), sij.mean(), np.mean(dudx**2), np.mean(dudx**3), np.mean(dwdz**2),
            np.mean(dwdz**3)]
    want += [want[3] / want[2] ** 1.5, want[5] / want[4] ** 1.5, n]
    np.testing.assert_allclose(out, want, rtol=1e-12)


def test_bench_particle_cpu_baseline_runs(oracle):
    """bench.py's particle CPU leg times the oracle on the bench's field: a
    small case finishes and reports a port on one core."""
    import os
    import sys

    from conftest import ROOT

    sys.path.insert(0, ROOT)
    import bench

    case = gks_ic.make_dhit(8, k0=4.0, Mt=0.3, seed=1)
    W = gks_ic.to_conservative_padded(case)
    out = bench.particle_cpu_baseline(W, case, 64)
    assert out["kind"] == "port" and out["cores"] == 1 and out["props_ms"] > 0
    assert os.path.basename(bench.__file__) == "bench.py"


def test_particle_positions_are_seeded_and_in_the_box():
    a = gks_ic.particle_positions(100, 3)
    b = gks_ic.particle_positions(100, 3)
    assert np.array_equal(a, b) and a.shape == (3, 100)
    assert np.all((a >= 0) & (a < 2 * np.pi))
