"""The FP64 adjoint of the oracle step against FP64 central differences.

orc_adjoint_step (oracle/pbf_adjoint.c) is the CPU reference gradient the GPU
adjoint is checked against; here it is checked itself.  Loss = mean squared
distance of the final positions to a seeded target; directional derivatives
along seeded random unit directions in initial-velocity, initial-position
and SDF-translation space are compared with central differences.

The step is piecewise smooth: the trilinear SDF has kinks on cell faces and
the neighbour sets, contacts and clamps switch discretely.  A difference
quotient straddling a kink carries an O(eps) error, so eps is chosen per
case small enough that none is straddled (in FP64 that still leaves
roundoff far below the tolerance).  With s_corr on (k = 0.1 at unit mass)
the Jacobi iterations amplify perturbations by orders of magnitude per
substep; those cases use one substep.
"""
import numpy as np
import pytest

import oracle as O
from adjoint_cases import loss, mk_sdf, setup


CASES = [
    # (setup kwargs, eps, rel tol)
    (dict(subs=2, iters=2, sdf=False, scorr=False, visc=True, vort=True), 1e-4, 1e-6),
    (dict(subs=2, iters=2, sdf=True, scorr=False, visc=True, vort=True), 1e-7, 1e-5),
    (dict(subs=1, iters=4, sdf=False, scorr=True, visc=True, vort=True), 1e-7, 1e-5),
    (dict(subs=2, iters=1, sdf=False, scorr=True, visc=False, vort=False), 1e-7, 1e-5),
    (dict(subs=1, iters=2, sdf=True, scorr=True, visc=True, vort=True), 1e-7, 1e-5),
]


@pytest.mark.parametrize("kw,eps,tol", CASES)
def test_adjoint_matches_central_differences(kw, eps, tol):
    _, P, pos, vel, grid, target = setup(**kw)
    n = len(pos)
    t0 = np.zeros(3)
    L0, pT, vT = loss(P, pos, vel, grid, t0, target)
    gp0, gv0, gt, pT2, vT2 = O.adjoint_step(P, pos, vel, gpos=2 * (pT - target) / n, sdf=mk_sdf(grid, t0))
    assert np.array_equal(pT2, pT) and np.array_equal(vT2, vT)  # the recorded forward is orc_step
    rng = np.random.default_rng(5)
    for _ in range(2):
        u = rng.normal(size=vel.shape)
        u /= np.linalg.norm(u)
        up = rng.normal(size=pos.shape)
        up /= np.linalg.norm(up)
        fd_v = (loss(P, pos, vel + eps * u, grid, t0, target)[0] -
                loss(P, pos, vel - eps * u, grid, t0, target)[0]) / (2 * eps)
        fd_p = (loss(P, pos + eps * up, vel, grid, t0, target)[0] -
                loss(P, pos - eps * up, vel, grid, t0, target)[0]) / (2 * eps)
        assert abs(fd_v - (gv0 * u).sum()) <= tol * abs(fd_v), (fd_v, (gv0 * u).sum())
        assert abs(fd_p - (gp0 * up).sum()) <= tol * abs(fd_p), (fd_p, (gp0 * up).sum())
        if grid is not None:
            ut = rng.normal(size=3)
            ut /= np.linalg.norm(ut)
            fd_t = (loss(P, pos, vel, grid, t0 + eps * ut, target)[0] -
                    loss(P, pos, vel, grid, t0 - eps * ut, target)[0]) / (2 * eps)
            assert abs(fd_t - gt @ ut) <= tol * abs(fd_t), (fd_t, gt @ ut)


def test_velocity_loss_adjoint():
    """Adjoint of a loss on the final velocities (exercises the velocity
    chain of integrate and the vorticity pass)."""
    _, P, pos, vel, grid, target = setup(subs=2, iters=2, sdf=True, scorr=False)
    n = len(pos)
    t0 = np.zeros(3)
    wv = np.random.default_rng(9).normal(size=vel.shape)

    def lv(v0):
        return (loss(P, pos, v0, grid, t0, target)[2] * wv).sum()

    gp0, gv0, gt, _, _ = O.adjoint_step(P, pos, vel, gvel=wv, sdf=mk_sdf(grid, t0))
    u = np.random.default_rng(3).normal(size=vel.shape)
    u /= np.linalg.norm(u)
    eps = 1e-7
    fd = (lv(vel + eps * u) - lv(vel - eps * u)) / (2 * eps)
    assert abs(fd - (gv0 * u).sum()) <= 1e-6 * abs(fd)
