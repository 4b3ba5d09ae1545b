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


def _script(n, A, rng, steps=8):
    """Constraint masks (a growing and shrinking contact patch), full or
    column-update factorizations with the changed columns (entering/leaving
    vertices and their neighbours), random right-hand sides."""
    import scipy.sparse as sp
    Ac = sp.csc_matrix(A)
    Ac.sort_indices()
    masks = np.zeros((steps, n), np.int8)
    full = np.zeros(steps, np.int32)
    changed, cptr = [], [0]
    prev = np.zeros(n, bool)
    for s in range(steps):
        cur = prev.copy()
        if s == 0:
            cur[rng.choice(n, 12, replace=False)] = True
            full[s] = 1
        else:
            cur[rng.choice(n, 5, replace=False)] = True
            cur[rng.choice(np.flatnonzero(cur), 3, replace=False)] = False
            full[s] = 1 if s == steps - 1 else 0
        diff = np.flatnonzero(cur != prev)
        ch = set(diff.tolist())
        for k in diff:
            ch.update(Ac.indices[Ac.indptr[k]:Ac.indptr[k + 1]].tolist())
        changed += sorted(ch)
        cptr.append(len(changed))
        masks[s] = cur
        prev = cur
    rhs = rng.normal(size=(steps, n))
    return (Ac.indptr.astype(np.int32), Ac.indices.astype(np.int32), Ac.data.astype(np.float64), masks, full,
            np.array(cptr, np.int32), np.array(changed, np.int32), rhs)


def _run(fn, n, script):
    import ctypes as C
    p, i, x, masks, full, cptr, ch, rhs = script
    out = np.zeros_like(rhs)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = fn(n, ptr(p), ptr(i), ptr(x), len(full), ptr(masks), ptr(full), ptr(cptr), ptr(ch), ptr(rhs), ptr(out))
    assert rc == 0
    return out


def test_incremental_cholesky_matches_reference_build(tmp_path, sphere):
    """The library's IncrementalCholesky against the reference's own
    src/deformation/IncrementalCholesky.cpp (oracle/_ref/libpbfref_chol.so),
    replaying the same analyze / setConstrained / factorizeFull / updateColumns
    / solveInPlace script on the C1-style normal matrix of a cotangent
    Laplacian (2-ring pattern).  Both follow the up-looking LDL^T recurrence
    in the same order, so the solutions are bit-identical."""
    import ctypes as C
    import os
    import subprocess
    import oracle as O
    ref_so = os.path.join(os.path.dirname(O.__file__), "_ref", "libpbfref_chol.so")
    if not os.path.exists(ref_so):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    so = str(tmp_path / "libchol_harness.so")
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I" + os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "chol_harness.cpp"),
                    os.path.join(root, "realtime-fsi-engine_b200", "host", "IncrementalCholesky.cpp"), "-o", so],
                   check=True, capture_output=True, text=True)
    mine = C.CDLL(so).chol_run
    ref = C.CDLL(ref_so).cholref_run
    for fn in (mine, ref):
        fn.restype = C.c_int
    V, F = sphere
    L, _ = cot_laplacian(V, F)
    n = len(V)
    A = L.T @ L + 1e-3 * np.eye(n)
    A[np.abs(A) < 1e-15] = 0.0
    script = _script(n, A, np.random.default_rng(4))
    got, want = _run(mine, n, script), _run(ref, n, script)
    assert np.array_equal(got, want)
    # and both solve A^B x = b
    masks, rhs = script[3], script[7]
    for s in range(len(rhs)):
        B = masks[s].astype(bool)
        AB = A.copy()
        AB[B, :] = 0.0
        AB[:, B] = 0.0
        AB[B, B] = 1.0
        assert np.abs(AB @ want[s] - rhs[s]).max() < 1e-8 * np.abs(rhs[s]).max()
