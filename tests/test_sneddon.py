"""Known-answer checks against Sneddon's pressurised penny crack, the analytical
solution the reference's static_solver_1 / postprocessing_1 tests use
(src/Solvers/_test/solver_test.cpp:16-57, test_radial_crack_static.cpp:27-305),
here with seeded points instead of std::random_device."""
import numpy as np

from conftest import golden

G, NU = 1.0, 0.35


def test_sneddon_opening_121(ora):
    # tip_type 0 mesh, sigma_zz = 1 -> pressure 1; the reference test excludes
    # nodes within r_tol of the tip and allows 0.1 absolute
    g = golden('ref_c1')
    nods, conn = g['nods'], g['conn']
    ne = conn.shape[1]
    dd = ora.dd_from_solution(g['x'], g['dof'], ne)
    r_tol = 0.2 * np.sqrt(np.pi / ne / np.sqrt(3.0))
    worst = 0.0
    for e in range(ne):
        v = nods[:3, conn[:3, e]]
        nodes = list(v.T) + [0.5 * (v[:, (a + 1) % 3] + v[:, (a + 2) % 3]) for a in range(3)]
        for k, x in enumerate(nodes):
            if 1.0 - np.hypot(x[0], x[1]) < r_tol:
                continue
            ref = ora.sneddon_dd(G, NU, 1.0, 1.0, x)
            worst = max(worst, abs(dd[6 * e + k, 2] - ref[2]))
    assert worst < 0.1


def test_sneddon_stress_121(ora):
    g = golden('ref_c1')
    nods, conn = g['nods'], g['conn']
    dd = ora.dd_from_solution(g['x'], g['dof'], conn.shape[1])
    rng = np.random.default_rng(3)
    pts = []
    while len(pts) < 5:
        p = rng.uniform(-2, 2, 3)
        if abs(p[2]) > 0.3:
            pts.append(p)
    pts = np.array(pts).T
    st = ora.stress(nods, conn, dd, pts, [0, 0, 1.0, 0, 0, 0])
    for i in range(pts.shape[1]):
        ref = ora.sneddon_stress(G, NU, 1.0, 1.0, pts[:, i])
        # oracle stress adds sigma_inf; Sneddon's field already includes the far field
        assert np.abs(st[i] - ref).max() < 0.1
