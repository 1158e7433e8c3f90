"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Integer and index results (tree topology, DFS ids, escape links, Morton
codes, fronts as multisets, pair sets) must be bit-exact; so must the FP32
boxes, which are exact min/max of FP32 inputs.  The narrow phase is an FP32
predicate evaluated in the same operation order without contraction on both
sides, so its hit set must match exactly too.
"""
import numpy as np
import pytest

from treecheck import check_tree, pick_roots

pytestmark = pytest.mark.gpu

CAPS = dict(int_front_capacity=4_000_000, ext_front_capacity=4_000_000, pair_capacity=2_000_000)


def canon(p):
    import pyoracle
    return pyoracle.canon_pairs(p)


def sorted_rows(a):
    a = np.asarray(a).reshape(-1, 2)
    if a.size == 0:
        return a
    return a[np.lexsort((a[:, 1], a[:, 0]))]


def _new(bvhcd, T, V, restr=True, cull=True, narrow=True, auto_grow=False, caps=None):
    bvh = bvhcd.LBvh(max(T, 1), max(V, 1), enable_restr=restr)
    front = bvhcd.BvttFront(bvh, cull_adjacent=cull, narrow_phase=narrow, auto_grow=auto_grow,
                            **(caps or CAPS))
    return bvh, front


def _tree_equal(a, b):
    for k in ("inode", "ibox", "leaf", "lbox", "lca", "codes", "primmap"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


def test_build_and_refit_bit_exact(cuda, lib_built, oracle, cloth_c1):
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    bvh, front = _new(lib_built, T, V)
    p = oracle.Pipeline(True, True, True)
    bvh.maintain(lib_built.BVH_BUILD, frames[0], faces)
    p.frame(faces, frames[0], 0, 1)
    g, o = bvh.export(), p.tree()
    _tree_equal(g, o)
    assert not check_tree(g, T)
    front.maintain(lib_built.FRONT_GENERATE)
    bvh.maintain(lib_built.BVH_REFIT, frames[1], faces)
    p.frame(faces, frames[1], 1, 4)
    _tree_equal(bvh.export(), p.tree())


@pytest.mark.parametrize("cull", [1, 0])
def test_pipeline_parity_over_schedule(cuda, lib_built, oracle, cloth_c1, cull):
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    bvh, front = _new(lib_built, T, V, cull=bool(cull))
    p = oracle.Pipeline(True, bool(cull), True)
    for f, pos in enumerate(frames):
        b, fr = lib_built.schedule(f)
        bvh.maintain(b, pos, faces, faces_static=f > 0)  # unchanged faces: keeps may skip entries
        front.maintain(fr)
        p.frame(faces, pos, b, fr)
        st, info = front.stats(), p.info()
        assert st["overflow"] == 0
        assert st["front_op_run"] == info["front_op"], f
        assert st["bvh_opt_tag"] == info["opt_tag"], f
        assert (st["int_front"], st["ext_front"]) == (info["F_int"], info["F_ext"]), f
        assert (st["broad_pairs"], st["narrow_hits"]) == (info["P"], info["H"]), f
        assert np.array_equal(canon(front.pairs()), canon(p.pairs())), f
        assert np.array_equal(canon(front.pairs(narrow=True)), canon(p.pairs(narrow=True))), f
        if f in (0, 6, 7, 12, 18):
            assert np.array_equal(canon(front.pairs()), oracle.brute_pairs(faces, pos, cull)), f
            for which in (0, 1):
                assert np.array_equal(sorted_rows(front.export(which)), sorted_rows(p.front(which))), (f, which)


def test_front_is_node_ordered(cuda, lib_built, cloth_c1):
    faces, frames = cloth_c1
    bvh, front = _new(lib_built, faces.shape[0], frames[0].shape[0])
    bvh.maintain(lib_built.BVH_BUILD, frames[0], faces)
    front.maintain(lib_built.FRONT_GENERATE)
    for which in (0, 1):
        nodes = front.export(which)[:, 1]
        # the counting sort orders entries by groups of 16 consecutive node ids
        assert np.all(np.diff(nodes >> 4) >= 0), "counting sort must order entries by node group"


def test_any_operation_order(cuda, lib_built, oracle, cloth_c1):
    """Front operations in orders the reference's schedules never produce: two
    balances in a row, keeps between balances, a balance right after
    generation.  Fronts (as multisets) and pairs equal the oracle's; pairs
    equal the brute-force set."""
    faces, frames = cloth_c1
    order = [(0, 1), (1, 3), (1, 3), (1, 4), (1, 3), (1, 2), (1, 3), (1, 4), (1, 4), (1, 3), (1, 3), (1, 2)]
    bvh, front = _new(lib_built, faces.shape[0], frames[0].shape[0], restr=False)
    p = oracle.Pipeline(False, True, True)
    for f, (b, fr) in enumerate(order):
        bvh.maintain(b, frames[f], faces)
        front.maintain(fr)
        p.frame(faces, frames[f], b, fr)
        for which in (0, 1):
            assert np.array_equal(sorted_rows(front.export(which)), sorted_rows(p.front(which))), (f, which)
        assert np.array_equal(canon(front.pairs()), oracle.brute_pairs(faces, frames[f], 1)), f
        assert np.array_equal(canon(front.pairs(narrow=True)), canon(p.pairs(narrow=True))), f


@pytest.mark.parametrize("step", [1, 4])
def test_long_keep_runs(cuda, lib_built, oracle, step):
    """A generation followed by keeps only, with the motion per frame scaled by
    `step` (frames skipped): the keep's expiries must never hold back an entry
    whose boxes have come to overlap.  Fronts and pairs equal the oracle's
    every frame."""
    import scenes
    faces, frames = scenes.cloth_over_sphere_frames(64, frames=1 + 12 * step, sphere_freq=8)
    frames = frames[::step]
    bvh, front = _new(lib_built, faces.shape[0], frames[0].shape[0], restr=False)
    p = oracle.Pipeline(False, True, True)
    for f, pos in enumerate(frames):
        op = (0, 1) if f == 0 else (1, 4)
        bvh.maintain(op[0], pos, faces, faces_static=f > 0)
        front.maintain(op[1])
        p.frame(faces, pos, *op)
        for which in (0, 1):
            assert np.array_equal(sorted_rows(front.export(which)), sorted_rows(p.front(which))), (f, which)
        assert np.array_equal(canon(front.pairs()), canon(p.pairs())), f
        assert np.array_equal(canon(front.pairs(narrow=True)), canon(p.pairs(narrow=True))), f
        st = front.stats()
        if f >= 2:
            # the keeps after the first one select by expiry: fewer entries tested than the front holds
            assert st["keep_tested"] < st["int_front"] + st["ext_front"], (f, st)
        elif f == 1:
            assert st["keep_tested"] == st["int_front"] + st["ext_front"], (f, st)


def _flat_grid(n):
    xs = np.linspace(0.0, 1.0, n, dtype=np.float32)
    gx, gy = np.meshgrid(xs, xs, indexing="ij")
    verts = np.stack([gx.ravel(), gy.ravel(), np.zeros(n * n, np.float32)], axis=1).astype(np.float32)
    faces = []
    for i in range(n - 1):
        for j in range(n - 1):
            a, b, c, d = i * n + j, i * n + j + 1, (i + 1) * n + j, (i + 1) * n + j + 1
            faces += [(a, b, d), (a, d, c)]
    return np.asarray(faces, np.int32), verts


def test_keep_expiry_catches_a_closing_gap(cuda, lib_built, oracle):
    """A triangle falls onto a flat, still cloth by a small step per frame,
    under keeps only (one generation on frame 0): its entries wait on their
    expiries while the gap closes, and the pairs must equal the brute-force
    set on every frame -- none may appear late, on the frame the boxes first
    touch included."""
    faces, verts = _flat_grid(24)
    nv = verts.shape[0]
    tri = np.array([[0.41, 0.43, 0.0], [0.55, 0.47, 0.0], [0.47, 0.58, 0.0]], np.float32)
    faces = np.concatenate([faces, np.array([[nv, nv + 1, nv + 2]], np.int32)])
    bvh, front = _new(lib_built, faces.shape[0], nv + 3, restr=False)
    first = None
    for f in range(40):
        pos = np.concatenate([verts, tri + np.float32([0.0, 0.0, 0.2 - 0.0125 * f])]).astype(np.float32)
        op = (0, 1) if f == 0 else (1, 4)
        bvh.maintain(op[0], pos, faces, faces_static=f > 0)
        front.maintain(op[1])
        got = canon(front.pairs())
        assert np.array_equal(got, oracle.brute_pairs(faces, pos, 1)), f
        falling = faces.shape[0] - 1
        if first is None and np.any(got == falling):
            first = f
        if f >= 2:
            st = front.stats()
            assert st["keep_tested"] < st["int_front"] + st["ext_front"], (f, st)
    assert first == 16, first  # z = 0.2 - 0.0125 * 16 = 0 touches the cloth


def test_restructure_parity(cuda, lib_built, oracle, cloth_c1):
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    bvh, front = _new(lib_built, T, V)
    p = oracle.Pipeline(True, True, True)
    for f in range(8):
        pos = frames[f]
        b, fr = lib_built.schedule(f)
        bvh.maintain(b, pos, faces)
        front.maintain(fr)
        p.frame(faces, pos, b, fr)
        assert bvh.opt_tag() == p.info()["opt_tag"], f
        _tree_equal(bvh.export(), p.tree())
        assert not check_tree(bvh.export(), T)
        assert np.array_equal(canon(front.pairs()), canon(p.pairs())), f
        if f == 2:
            roots = pick_roots(p.tree())
            bvh.request_restructure(roots)
            p.mark_restructure(roots)
        if f == 3:
            assert bvh.opt_tag() == 1
            st = front.stats()
            assert st["num_rt_int_nodes"] == p.info()["num_rt_int"]


def test_pure_bvh_cd(cuda, lib_built, oracle, cloth_c1):
    faces, frames = cloth_c1
    bvh, front = _new(lib_built, faces.shape[0], frames[0].shape[0])
    for f in (0, 5, 11):
        bvh.maintain(lib_built.BVH_BUILD if f == 0 else lib_built.BVH_REFIT, frames[f], faces)
        front.maintain(lib_built.FRONT_PURE_BVH_CD)
        assert np.array_equal(canon(front.pairs()), oracle.brute_pairs(faces, frames[f], 1))


def _edge_scene(kind):
    if kind == "empty":
        return np.zeros((0, 3), np.int32), np.zeros((0, 3), np.float32)
    if kind == "one":
        return np.array([[0, 1, 2]], np.int32), np.eye(3, dtype=np.float32)
    if kind == "two":
        return np.array([[0, 1, 2], [3, 4, 5]], np.int32), np.concatenate([np.eye(3), np.eye(3) + 0.5]).astype(np.float32)
    if kind == "three":
        v = np.random.default_rng(3).uniform(0, 1, (9, 3)).astype(np.float32)
        return np.arange(9, dtype=np.int32).reshape(3, 3), v
    if kind == "identical":  # all Morton codes equal
        v = np.tile(np.eye(3, dtype=np.float32), (200, 1))
        return np.arange(600, dtype=np.int32).reshape(200, 3), v
    if kind == "degenerate":  # zero-area triangles and a flat scene (zero z extent)
        rng = np.random.default_rng(9)
        v = rng.uniform(0, 1, (300, 3)).astype(np.float32)
        v[:, 2] = 0.0
        f = rng.integers(0, 300, (500, 3)).astype(np.int32)
        f[:50, 1] = f[:50, 0]
        return f, v
    raise KeyError(kind)


@pytest.mark.parametrize("kind", ["empty", "one", "two", "three", "identical", "degenerate"])
def test_edge_cases(cuda, lib_built, oracle, kind):
    faces, verts = _edge_scene(kind)
    T = faces.shape[0]
    bvh, front = _new(lib_built, T, verts.shape[0], cull=False)
    p = oracle.Pipeline(True, False, True)
    for f, op in enumerate([(0, 1), (1, 4), (1, 2), (1, 3), (0, 1)]):
        bvh.maintain(op[0], verts, faces)
        front.maintain(op[1])
        p.frame(faces, verts, *op)
        assert np.array_equal(canon(front.pairs()), canon(p.pairs())), (kind, f)
        assert np.array_equal(canon(front.pairs(narrow=True)), canon(p.pairs(narrow=True))), (kind, f)
        if T >= 1:
            _tree_equal(bvh.export(), p.tree())
    assert np.array_equal(canon(front.pairs()), oracle.brute_pairs(faces, verts, 0))


def test_overflow_is_reported_and_auto_grow_recovers(cuda, lib_built, oracle, cloth_c1):
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    small = dict(int_front_capacity=1000, ext_front_capacity=1000, pair_capacity=1000)
    bvh, front = _new(lib_built, T, V, caps=small)
    bvh.maintain(0, frames[0], faces)
    front.maintain(1)
    st = front.stats()
    assert st["overflow"] & 1 and st["overflow"] & 2 and st["overflow"] & 4
    with pytest.raises(lib_built.BvhcdError):
        front.pairs()
    bvh2, front2 = _new(lib_built, T, V, caps=small, auto_grow=True)
    for f in range(8):
        b, fr = lib_built.schedule(f)
        bvh2.maintain(b, frames[f], faces)
        front2.maintain(fr)
        assert front2.stats()["overflow"] == 0
        assert np.array_equal(canon(front2.pairs()), oracle.brute_pairs(faces, frames[f], 1)), f


def test_device_resident_input(cuda, lib_built, cloth_c1):
    torch = cuda
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    b1, f1 = _new(lib_built, T, V)
    b2, f2 = _new(lib_built, T, V)
    df = torch.from_numpy(faces).cuda()
    for f in range(7):
        b, fr = lib_built.schedule(f)
        b1.maintain(b, frames[f], faces)
        f1.maintain(fr)
        b2.maintain(b, torch.from_numpy(frames[f]).cuda(), df)
        f2.maintain(fr)
        assert np.array_equal(canon(f1.pairs(True)), canon(f2.pairs(True)))
        assert np.array_equal(canon(f1.pairs()), canon(f2.pairs()))
    hits, counts = f2.device_results()
    assert hits and counts


def test_cloth_over_sphere_full_size(cuda, lib_built, oracle):
    """The bench workload (512x512 cloth over a frequency-45 icosphere,
    562,742 triangles) through a whole cycle of the reference's schedule --
    build + generate (0), keeps, balance (5), prune/sprout (6), a restructure
    forced through the public marks (8), the mandatory rebuild (12) -- with
    the CPU oracle pipeline alongside.  Every frame: the broad set equals the
    brute-force set of overlapping boxes, the hits equal the FP32 SAT over it,
    sizes / op tags / front operation equal the oracle's; on the frames that
    change the front, both fronts equal the oracle's as multisets; after the
    builds, a refit and the restructure the tree equals the oracle's bit for
    bit."""
    import scenes
    faces, frames = scenes.cloth_over_sphere_frames(512, 14)
    T, V = faces.shape[0], frames[0].shape[0]
    assert T == 522242 + 40500
    caps = dict(int_front_capacity=40_000_000, ext_front_capacity=40_000_000, pair_capacity=8_000_000)
    bvh, front = _new(lib_built, T, V, caps=caps)
    p = oracle.Pipeline(True, True, True)
    ops = []
    for f in range(14):
        b, fr = lib_built.schedule(f)
        bvh.maintain(b, frames[f], faces, faces_static=f > 0)
        front.maintain(fr)
        p.frame(faces, frames[f], b, fr)
        st, info = front.stats(), p.info()
        assert st["overflow"] == 0, f
        assert st["bvh_opt_tag"] == info["opt_tag"] and st["front_op_run"] == info["front_op"], (f, st, info)
        assert (st["int_front"], st["ext_front"]) == (info["F_int"], info["F_ext"]), (f, st, info)
        assert (st["broad_pairs"], st["narrow_hits"]) == (info["P"], info["H"]), (f, st, info)
        pairs = canon(front.pairs())
        assert np.array_equal(pairs, oracle.brute_pairs(faces, frames[f], 1)), f
        hits = canon(front.pairs(narrow=True))
        keep = oracle.narrow(pairs, faces, frames[f]).astype(bool)
        assert np.array_equal(hits, pairs[keep]), f
        assert len(hits) > 0, "the cloth must cut the sphere"
        ops.append((st["bvh_opt_tag"], st["front_op_run"]))
        if f in (0, 5, 6, 8, 12):
            for which in (0, 1):
                assert np.array_equal(sorted_rows(front.export(which)), sorted_rows(p.front(which))), (f, which)
        if f in (0, 1, 8, 12):
            # builds, a refit and the restructure at full size: the single-launch
            # sort and scans and the one-exchange climb give the reference's tree
            _tree_equal(bvh.export(), p.tree())
        if f == 7:
            roots = pick_roots(p.tree())
            bvh.request_restructure(roots)
            p.mark_restructure(roots)
    assert ops[8] == (1, lib_built.FRONT_GENERATE), ops      # the forced restructure, then a regeneration
    assert ops[12][1] == lib_built.FRONT_GENERATE, ops       # the mandatory rebuild (its tag stays 0, as the reference's)
    assert ops[5][1] == lib_built.FRONT_REORDER and ops[6][1] == lib_built.FRONT_UPDATE, ops
    assert not check_tree(bvh.export(), T)
