"""CPU tests of the oracle itself (no GPU): it must reproduce the exact FP32
AABB-overlap pair set on every frame of the schedule, its FP32 SAT must agree
bit for bit with the reference's own predicate compiled from the reference
header (oracle/_ref), and its trees must satisfy the reference's integrity
checks."""
import numpy as np
import pytest

from treecheck import check_tree, pick_roots


def _run_pipeline(po, faces, frames, cull, restr=True, marks=()):
    p = po.Pipeline(restructure=restr, cull_adjacent=cull, narrow=True)
    out = []
    for f, pos in enumerate(frames):
        b, fr = po.schedule(f)
        p.frame(faces, pos, b, fr)
        out.append((p.info(), po.canon_pairs(p.pairs()), po.canon_pairs(p.pairs(narrow=True)), p.tree()))
        if f in marks:
            p.mark_restructure(marks[f](p.tree()))
    return out


@pytest.mark.parametrize("cull", [0, 1])
def test_pipeline_pairs_equal_brute_force(oracle, cloth_c1, cull):
    faces, frames = cloth_c1
    res = _run_pipeline(oracle, faces, frames[:14], cull)
    for f, (info, pairs, hits, tree) in enumerate(res):
        ref = oracle.brute_pairs(faces, frames[f], cull)
        assert pairs.shape == ref.shape and np.array_equal(pairs, ref), f"frame {f}"
        # each unordered pair once
        assert len(np.unique(pairs, axis=0)) == len(pairs)
        assert not check_tree(tree, faces.shape[0]), f"frame {f}"
        # the narrow phase keeps exactly the pairs whose triangles intersect
        keep = oracle.narrow(pairs, faces, frames[f]).astype(bool)
        assert np.array_equal(hits, pairs[keep])


# front operations in orders the reference's schedules never produce: two
# balances in a row, keeps between balances, a balance right after generation
ANY_ORDER = [(0, 1), (1, 3), (1, 3), (1, 4), (1, 3), (1, 2), (1, 3), (1, 4), (1, 4), (1, 3), (1, 3), (1, 2)]


def test_pipeline_any_operation_order(oracle, cloth_c1):
    faces, frames = cloth_c1
    p = oracle.Pipeline(False, True, True)
    for f, (b, fr) in enumerate(ANY_ORDER):
        p.frame(faces, frames[f], b, fr)
        assert np.array_equal(oracle.canon_pairs(p.pairs()), oracle.brute_pairs(faces, frames[f], 1)), f
        for which in (0, 1):
            fr_ = p.front(which)
            assert len(np.unique(fr_, axis=0)) == len(fr_), (f, which)


def test_schedule_table(oracle):
    # STATIC_MANDATORY with divergent marks, BenchmarkLogic.hpp:102-117
    got = [oracle.schedule(f) for f in range(26)]
    B, R = 0, 1
    GEN, UPD, REO, KEEP = 1, 2, 3, 4
    exp = [(B, GEN), (R, KEEP), (R, KEEP), (R, KEEP), (R, KEEP), (R, REO), (R, UPD), (R, KEEP),
           (R, KEEP), (R, KEEP), (R, KEEP), (R, KEEP), (B, GEN), (R, KEEP), (R, KEEP), (R, KEEP),
           (R, KEEP), (R, REO), (R, UPD), (R, KEEP), (R, KEEP), (R, KEEP), (R, KEEP), (R, KEEP),
           (B, GEN), (R, KEEP)]
    assert got == exp


def test_restructure_keeps_pairs_and_tree(oracle, cloth_c1):
    faces, frames = cloth_c1
    res = _run_pipeline(oracle, faces, frames[:6], 1, marks={2: pick_roots})
    info, pairs, _, tree = res[3]
    assert info["opt_tag"] == 1, "the marked subtrees must be restructured"
    assert info["num_rt_int"] * 8 >= faces.shape[0] - 1
    for f in range(6):
        ref = oracle.brute_pairs(faces, frames[f], 1)
        assert np.array_equal(res[f][1], ref)
        assert not check_tree(res[f][3], faces.shape[0])
    # restructured subtrees are Morton-ordered inside
    codes = tree["codes"]
    leaf_root = np.zeros(faces.shape[0], np.int64)
    inode = tree["inode"]
    for r in pick_roots(res[2][3]):
        lo, hi = inode[r, 4], inode[r, 5]
        assert np.all(np.diff(codes[lo:hi + 1].astype(np.int64)) >= 0)


def test_restructure_decision_thresholds(oracle, cloth_c1):
    faces, frames = cloth_c1
    # a handful of marked nodes: fewer than 1/8 of the internal nodes -> refit
    res = _run_pipeline(oracle, faces, frames[:5], 1, marks={2: lambda t: pick_roots(t, frac=0.01)})
    assert res[3][0]["opt_tag"] == 0
    # more than half -> rebuild
    res = _run_pipeline(oracle, faces, frames[:5], 1, marks={2: lambda t: np.array([0], np.int32)})
    assert res[3][0]["opt_tag"] == 2
    ref = oracle.brute_pairs(faces, frames[3], 1)
    assert np.array_equal(res[3][1], ref)


def _tri_cases(rng, n):
    P = rng.uniform(0, 1, (n, 3, 3)).astype(np.float32)
    Q = (P[:, :1, :] + rng.normal(0, 0.3, (n, 3, 3))).astype(np.float32)
    # coplanar
    P2, Q2 = P.copy(), Q.copy()
    P2[..., 2] = 0.25
    Q2[..., 2] = 0.25
    # shared vertex / shared edge (touching)
    P3, Q3 = P.copy(), Q.copy()
    Q3[:, 0] = P3[:, 1]
    P4, Q4 = P.copy(), Q.copy()
    Q4[:, 0] = P4[:, 0]
    Q4[:, 1] = P4[:, 2]
    # near-touching: Q offset by tiny amounts along the normal of P
    n_ = np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
    n_ /= np.linalg.norm(n_, axis=1, keepdims=True) + 1e-30
    Q5 = (P[:, [0, 1, 2]] + n_[:, None, :] * rng.choice([-1e-7, 0.0, 1e-7], (n, 1, 1))).astype(np.float32)
    Q5 = Q5[:, [1, 2, 0]]
    return [(P, Q), (P2, Q2), (P3, Q3), (P4, Q4), (P, Q5)]


def _narrow_batch(fn, P, Q):
    n = P.shape[0]
    faces = np.arange(6 * n, dtype=np.int32).reshape(2 * n, 3)
    verts = np.concatenate([P.reshape(-1, 3), Q.reshape(-1, 3)]).astype(np.float32)
    pairs = np.stack([np.arange(n), np.arange(n) + n], 1).astype(np.int32)
    return fn(pairs, faces, verts)


def test_sat32_matches_reference_predicate(oracle):
    if oracle.ref_lib() is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    rng = np.random.default_rng(7)
    for P, Q in _tri_cases(rng, 4000):
        a = _narrow_batch(oracle.narrow, P, Q)
        b = _narrow_batch(oracle.ref_narrow, P, Q)
        assert np.array_equal(a, b)


def test_exact_predicate_agrees_off_degenerate_cases(oracle):
    rng = np.random.default_rng(11)
    P, Q = _tri_cases(rng, 3000)[0]
    a = _narrow_batch(oracle.narrow, P, Q)
    c = _narrow_batch(lambda p, f, v: oracle.narrow(p, f, v, exact=True), P, Q)
    assert (a != c).sum() == 0
    # touching triangles intersect under both (closed triangles)
    P3, Q3 = _tri_cases(rng, 500)[2]
    assert _narrow_batch(lambda p, f, v: oracle.narrow(p, f, v, exact=True), P3, Q3).all()
    assert _narrow_batch(oracle.narrow, P3, Q3).all()


def test_morton_codes_known_values(oracle):
    # one triangle per corner of the unit cube: codes of normalised centres
    faces = np.arange(6, dtype=np.int32).reshape(2, 3)
    verts = np.array([[0, 0, 0], [0, 0, 0], [0, 0, 0], [1, 1, 1], [1, 1, 1], [1, 1, 1]], np.float32)
    box = np.zeros(6, np.float32)
    oracle.lib().orc_scene_box(2, faces, verts, box)
    codes = np.zeros(2, np.uint32)
    oracle.lib().orc_morton_codes(2, faces, verts, box, codes)
    assert codes[0] == 0 and codes[1] == (1 << 30) - 1


def _boxes(faces, verts):
    t = np.asarray(verts, np.float32)[np.asarray(faces)]
    return t.min(axis=1), t.max(axis=1)


def test_inter_pairs_equal_all_pairs_enumeration(oracle):
    """The inter oracle (sweep and prune over two joined meshes) against every
    pair of boxes tested, on meshes whose vertex ids overlap numerically."""
    rng = np.random.default_rng(21)
    va = rng.uniform(0, 1, (300, 3)).astype(np.float32)
    vb = rng.uniform(0.3, 1.3, (200, 3)).astype(np.float32)
    fa = rng.integers(0, 300, (400, 3)).astype(np.int32)
    fb = rng.integers(0, 200, (250, 3)).astype(np.int32)
    va[:, 2] *= 0.05  # thin slabs: a sparse set of pairs
    vb[:, 2] *= 0.05
    lo_a, hi_a = _boxes(fa, va)
    lo_b, hi_b = _boxes(fb, vb)
    ov = np.all((lo_a[:, None, :] <= hi_b[None, :, :]) & (lo_b[None, :, :] <= hi_a[:, None, :]), axis=2)
    exp = np.argwhere(ov).astype(np.int64)
    got = oracle.brute_inter_pairs(fa, va, fb, vb)
    assert 0 < exp.shape[0] < ov.size
    assert np.array_equal(got, exp)
    # the SAT takes the obstacle's triangle first
    hit = oracle.inter_narrow(got, fa, va, fb, vb)
    n = got.shape[0]
    P = vb[fb[got[:, 1]]].reshape(n, 9)
    Q = va[fa[got[:, 0]]].reshape(n, 9)
    assert np.array_equal(hit, _narrow_batch(oracle.narrow, P, Q))
    # either mesh empty: no pairs
    empty = np.zeros((0, 3), np.int32)
    assert oracle.brute_inter_pairs(empty, va, fb, vb).shape == (0, 2)
    assert oracle.brute_inter_pairs(fa, va, empty, vb).shape == (0, 2)
