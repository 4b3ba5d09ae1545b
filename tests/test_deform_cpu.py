"""Host deformation solver (pbf_deform_*) against dense FP64 restatements.

The reference's LaplacianDeformation needs Eigen, CHOLMOD and OpenMesh, none of
which exists here, so it cannot be run; these tests restate its math with numpy
(cotangent Laplacian of src/deformation/LaplacianDeformation.cpp:69-183, the
soft least-squares solve :497-616, the hard-constraint system of the
incremental path :25-66/:620-675, the k-ring patch solve :215-417) and the
application's handle driver (src/main.cpp:870-944), and compare.
"""
import numpy as np
import pytest

from pbf_b200 import scenes
from pbf_b200.deform import Deformer, default_params


def cot_laplacian(V, F):
    n = len(V)
    W = np.zeros((n, n))
    opp = {}
    for f in F:
        for e in range(3):
            a, b, c = f[e], f[(e + 1) % 3], f[(e + 2) % 3]
            opp.setdefault((min(a, b), max(a, b)), []).append(c)
    for (a, b), cs in opp.items():
        cot = 0.0
        for c in cs:
            s, e = V[a] - V[c], V[b] - V[c]
            sn = np.linalg.norm(np.cross(s, e))
            if sn > 1e-6:
                cot += s @ e / sn
        W[a, b] = W[b, a] = max(0.5 * cot, 1e-4)
    L = np.eye(n) - W / W.sum(1, keepdims=True)
    return L, W > 0


@pytest.fixture(scope="module")
def sphere():
    V, F = scenes.icosphere(2, 0.2, (0.0, 0.0, 0.0))  # 162 vertices
    return V, F


def test_soft_global_matches_least_squares(sphere):
    V, F = sphere
    L, _ = cot_laplacian(V, F)
    n = len(V)
    d = Deformer(V, F)
    d.set_mode(use_local=False, use_incremental=False)
    anchors = list(np.argsort(V[:, 1])[:5])
    for a in anchors:
        d.add_anchor(a)
    hidx = [int(np.argmax(V[:, 1])), int(np.argmax(V[:, 0]))]
    tgt = V[hidx] + np.array([[0.0, -0.05, 0.0], [0.03, 0.0, 0.01]])
    d.set_control_points(hidx, tgt)
    d.precompute()
    d.solve()
    got = d.vertices()
    A = np.vstack([L] + [np.eye(n)[[a]] for a in anchors] + [np.eye(n)[[h]] for h in hidx])
    b = np.vstack([L @ V] + [V[[a]] for a in anchors] + [tgt])
    ref = np.linalg.solve(A.T @ A, A.T @ b)
    assert np.abs(got - ref).max() < 1e-9


def _hard_solution(L, V, cons, tgt):
    n = len(V)
    A = L.T @ L + 1e-8 * np.eye(n)
    b = L.T @ (L @ V)
    free = np.setdiff1d(np.arange(n), cons)
    x = np.zeros_like(V)
    x[cons] = tgt
    x[free] = np.linalg.solve(A[np.ix_(free, free)], b[free] - A[np.ix_(free, cons)] @ tgt)
    return x


def test_incremental_hard_constraints_and_updates(sphere):
    V, F = sphere
    L, _ = cot_laplacian(V, F)
    d = Deformer(V, F)
    d.set_mode(use_local=False, use_incremental=True)
    anchors = [int(i) for i in np.argsort(V[:, 1])[:6]]
    for a in anchors:
        d.add_anchor(a)
    rng = np.random.default_rng(3)
    sets = [[10, 20, 30], [10, 20, 31, 40, 41], [5], [5, 6, 7, 8, 100, 120]]
    for hs in sets:  # each change goes through the tree-path column update
        tgt = V[hs] + rng.normal(0, 0.02, (len(hs), 3))
        d.set_control_points(hs, tgt)
        d.precompute()
        d.solve()
        cons = sorted(set(anchors) | set(hs))
        targets = np.array([V[c] if c in anchors else tgt[hs.index(c)] for c in cons])
        ref = _hard_solution(L, V, np.array(cons), targets)
        got = d.vertices()
        assert np.abs(got - ref).max() < 1e-8, hs
        assert np.abs(got[hs] - tgt).max() < 1e-12  # hard: handles sit on their targets
        assert 0 <= d.verify_incremental() < 1e-9


def test_local_patch_matches_dense_patch_solve(sphere):
    V, F = sphere
    L, adj = cot_laplacian(V, F)
    n = len(V)
    d = Deformer(V, F)
    d.set_mode(use_local=True, kring=2)
    anchors = [int(i) for i in np.argsort(V[:, 1])[:4]]
    for a in anchors:
        d.add_anchor(a)
    hs = [int(np.argmax(V[:, 1]))]
    tgt = V[hs] + np.array([[0.01, -0.04, 0.0]])
    d.set_control_points(hs, tgt)
    d.precompute()
    d.solve()
    got = d.vertices()
    # k-ring interior (anchors excluded), neighbours of it held fixed
    ring = set(hs)
    frontier = set(hs)
    for _ in range(2):
        frontier = {j for v in frontier for j in np.nonzero(adj[v])[0]} - ring
        ring |= frontier
    interior = sorted(ring - set(anchors))
    outer = sorted(set(range(n)) - set(interior))
    Lii, Lio = L[np.ix_(interior, interior)], L[np.ix_(interior, outer)]
    rhs = Lii.T @ ((L @ V)[interior] - Lio @ V[outer])
    M = Lii.T @ Lii
    hl = [interior.index(h) for h in hs]
    M[hl, hl] += 1.0
    rhs[hl] += tgt
    xi = np.linalg.solve(M, rhs)
    ref = V.copy()
    ref[interior] = xi
    assert d.patch_size() == len(interior)
    assert np.abs(got - ref).max() < 1e-9


def test_deform_step_handle_policy(sphere):
    """The per-frame driver against a restatement of src/main.cpp:870-944:
    hysteresis of the handle set, per-frame and total clamps, elastic restore,
    refactor only when the set changes."""
    V, F = sphere
    n = len(V)
    prm = default_params(stiffness=1.0, max_displacement=0.01, max_total_disp=0.03, restore_enabled=1,
                         restore_strength=0.05, control_threshold=1.0, control_threshold_low=0.5)
    d = Deformer(V, F)
    d.set_mode(use_local=False, use_incremental=True)
    anchors = [int(i) for i in np.argsort(V[:, 1])[:6]]
    for a in anchors:
        d.add_anchor(a)
    rng = np.random.default_rng(4)
    last = []
    cur = V.copy()
    for frame in range(6):
        f = np.zeros((n, 3), np.float32)
        hit = rng.choice(n, 12, replace=False)
        f[hit] = rng.normal(0, 1.2, (12, 3)).astype(np.float32)
        dt = np.float32(1 / 60)
        # restatement
        handles, targets = [], []
        for i in range(n):
            if i in anchors:
                continue
            fmag = np.float32(np.sqrt(np.float32(f[i] @ f[i])))
            wasH = i in last
            pushed = fmag >= np.float32(prm.control_threshold) or (wasH and fmag >= np.float32(prm.control_threshold_low))
            relaxing = bool(prm.restore_enabled) and wasH and np.linalg.norm(cur[i] - V[i]) > 1e-3
            if not (pushed or relaxing):
                continue
            t = cur[i].copy()
            if pushed:
                disp = f[i] * np.float32(prm.stiffness * dt)
                dm = np.float32(np.sqrt(np.float32(disp @ disp)))
                if dm > np.float32(prm.max_displacement) and dm > 1e-12:
                    disp = disp * np.float32(np.float32(prm.max_displacement) / dm)
                t = t + disp.astype(np.float64)
            t = t + np.float64(np.float32(prm.restore_strength)) * (V[i] - t)
            off = np.linalg.norm(t - V[i])
            if off > np.float32(prm.max_total_disp):
                t = V[i] + (t - V[i]) * (np.float64(np.float32(prm.max_total_disp)) / off)
            handles.append(i)
            targets.append(t)
        hc, refactored, moved = d.step(f, dt, prm)
        assert hc == len(handles)
        assert refactored == (handles != last)
        if handles or refactored:
            L, _ = cot_laplacian(V, F)
            cons = sorted(set(anchors) | set(handles))
            tg = np.array([V[c] if c in anchors else targets[handles.index(c)] for c in cons])
            cur = _hard_solution(L, V, np.array(cons), tg)
        assert moved == bool(handles or refactored)
        assert np.abs(d.vertices() - cur).max() < 1e-8, frame
        last = handles
