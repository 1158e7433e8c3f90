"""Scenes given as primitive boxes (the reference's ARCSimSceneData path) on
the GPU.

A box scene whose boxes are exactly its triangles' FP32 boxes must give the
triangle scene's tree, fronts and pairs bit for bit, through builds, refits and
a restructure.  Arbitrary boxes (swept over two frames, FP64 input rounded
outward) must give the brute-force set of overlapping boxes, with adjacency
culling on the given faces.
"""
import numpy as np
import pytest

from treecheck import check_tree, pick_roots

pytestmark = pytest.mark.gpu

CAPS = dict(int_front_capacity=2_000_000, ext_front_capacity=2_000_000, pair_capacity=1_000_000)


def _rows(p):
    p = np.asarray(p, dtype=np.int64).reshape(-1, 2)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def tri_boxes(faces, pos):
    t = np.asarray(pos, np.float32)[np.asarray(faces)]
    return np.concatenate([t.min(axis=1), t.max(axis=1)], axis=1).astype(np.float32)


def round_outward(b64):
    lo, hi = b64[:, :3], b64[:, 3:]
    lo32, hi32 = lo.astype(np.float32), hi.astype(np.float32)
    m = lo32.astype(np.float64) > lo
    lo32[m] = np.nextafter(lo32[m], np.float32(-np.inf))
    m = hi32.astype(np.float64) < hi
    hi32[m] = np.nextafter(hi32[m], np.float32(np.inf))
    return np.concatenate([lo32, hi32], axis=1)


def brute_box_pairs(oracle, boxes, faces, cull):
    """Overlapping box pairs (touching counts), as canonical rows; with cull,
    without the pairs whose faces share a vertex id."""
    T = boxes.shape[0]
    # one degenerate triangle per box (its corners min, max, min): its FP32
    # box is the box itself
    verts = np.stack([boxes[:, :3], boxes[:, 3:], boxes[:, :3]], axis=1).reshape(-1, 3).astype(np.float32)
    tf = np.arange(3 * T, dtype=np.int32).reshape(T, 3)
    p = oracle.brute_pairs(tf, verts, 0)
    if cull and p.size:
        fa, fb = faces[p[:, 0]], faces[p[:, 1]]
        share = (fa[:, :, None] == fb[:, None, :]).any(axis=(1, 2))
        p = p[~share]
    return p


def _tree_equal(a, b):
    for k in ("inode", "ibox", "leaf", "lbox", "lca", "codes", "primmap"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


def test_box_scene_equals_triangle_scene(cuda, lib_built):
    bvhcd = lib_built
    import scenes
    faces, frames = scenes.cloth_over_sphere_frames(48, frames=14, sphere_freq=8)
    T, V = faces.shape[0], frames[0].shape[0]
    tb = bvhcd.LBvh(T, V, enable_restr=True)
    bb = bvhcd.LBvh(T, V, enable_restr=True)
    tf = bvhcd.BvttFront(tb, cull_adjacent=True, narrow_phase=False, **CAPS)
    bf = bvhcd.BvttFront(bb, cull_adjacent=True, narrow_phase=False, **CAPS)
    for f, pos in enumerate(frames):
        b, fr = bvhcd.schedule(f)
        tb.maintain(b, pos, faces, faces_static=f > 0)
        tf.maintain(fr)
        bb.maintain_boxes(b, tri_boxes(faces, pos), faces, faces_static=f > 0)
        bf.maintain(fr)
        if f == 4:
            assert tb.opt_tag() == 1 and bb.opt_tag() == 1
        et, eb = tb.export(), bb.export()
        _tree_equal(et, eb)
        assert not check_tree(eb, T)
        for which in (0, 1):
            assert np.array_equal(_rows(tf.export(which)), _rows(bf.export(which))), (f, which)
        assert np.array_equal(_rows(tf.pairs()), _rows(bf.pairs())), f
        assert bf.stats()["overflow"] == 0
        if f == 3:
            roots = pick_roots(et)
            tb.request_restructure(roots)
            bb.request_restructure(roots)


def test_swept_boxes_match_brute_force(cuda, lib_built, oracle):
    """Boxes swept over two frames and grown by a thickness, host FP32 input,
    every front operation; pairs against the brute-force set, culled on the
    given faces."""
    bvhcd = lib_built
    import scenes
    faces, frames = scenes.cloth_fold_frames(64, 9)
    T = faces.shape[0]
    bvh = bvhcd.LBvh(T, 0, enable_restr=False)
    front = bvhcd.BvttFront(bvh, cull_adjacent=True, narrow_phase=False, **CAPS)
    ops = [(0, 1), (1, 4), (1, 2), (1, 3), (1, 4), (1, 2), (0, 1), (1, 3)]
    for f, (b, fr) in enumerate(ops):
        a0, a1 = tri_boxes(faces, frames[f]), tri_boxes(faces, frames[f + 1])
        boxes = np.concatenate([np.minimum(a0[:, :3], a1[:, :3]) - 1e-3,
                                np.maximum(a0[:, 3:], a1[:, 3:]) + 1e-3], axis=1).astype(np.float32)
        bvh.maintain_boxes(b, boxes, faces)
        front.maintain(fr)
        assert front.stats()["overflow"] == 0
        got = front.pairs()
        import pyoracle
        assert np.array_equal(pyoracle.canon_pairs(got), brute_box_pairs(oracle, boxes, faces, True)), f


def test_f64_boxes_round_outward(cuda, lib_built, oracle):
    """FP64 boxes, from host memory and read in place from the device: the
    tree's leaf boxes are the outward-rounded FP32 boxes, which contain the
    given ones, and the pairs are theirs."""
    bvhcd = lib_built
    torch = cuda
    rng = np.random.default_rng(17)
    T = 20000
    c = rng.uniform(0.0, 1.0, (T, 3))
    h = rng.uniform(1e-4, 1.2e-2, (T, 3))
    b64 = np.concatenate([c - h, c + h], axis=1) + rng.uniform(-1e-9, 1e-9, (T, 6))
    faces = rng.integers(0, 3 * T, (T, 3)).astype(np.int32)
    b32 = round_outward(b64)
    assert np.all(b32[:, :3].astype(np.float64) <= b64[:, :3]) and np.all(b32[:, 3:].astype(np.float64) >= b64[:, 3:])
    assert (b32[:, :3].astype(np.float64) < b64[:, :3]).any()
    ref = brute_box_pairs(oracle, b32, faces, True)
    import pyoracle
    for src in ("host", "device"):
        bvh = bvhcd.LBvh(T, 0, enable_restr=False)
        front = bvhcd.BvttFront(bvh, cull_adjacent=True, narrow_phase=False, **CAPS)
        if src == "host":
            bvh.maintain_boxes(bvhcd.BVH_BUILD, b64, faces)
        else:
            bvh.maintain_boxes(bvhcd.BVH_BUILD, torch.from_numpy(b64).cuda(), torch.from_numpy(faces).cuda())
        front.maintain(bvhcd.FRONT_GENERATE)
        e = bvh.export()
        orig = e["leaf"][:, 0]
        assert np.array_equal(e["lbox"], b32[orig]), src
        assert np.array_equal(pyoracle.canon_pairs(front.pairs()), ref), src


def test_switching_scene_kinds_rebuilds(cuda, lib_built):
    """Triangles, then boxes, then triangles again on one handle (the op is
    REFIT each time after the first): each kind change rebuilds, so the tree
    equals a fresh handle's."""
    bvhcd = lib_built
    import scenes
    faces, frames = scenes.cloth_fold_frames(32, 3)
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = bvhcd.LBvh(T, V, enable_restr=False)
    bvh.maintain(bvhcd.BVH_BUILD, frames[0], faces)
    boxes = tri_boxes(faces, frames[1])
    boxes[:, 3:] += np.float32(0.01)
    bvh.maintain_boxes(bvhcd.BVH_REFIT, boxes, faces)
    fresh = bvhcd.LBvh(T, V, enable_restr=False)
    fresh.maintain_boxes(bvhcd.BVH_BUILD, boxes, faces)
    _tree_equal(bvh.export(), fresh.export())
    bvh.maintain(bvhcd.BVH_REFIT, frames[2], faces)
    fresh2 = bvhcd.LBvh(T, V, enable_restr=False)
    fresh2.maintain(bvhcd.BVH_BUILD, frames[2], faces)
    _tree_equal(bvh.export(), fresh2.export())


def test_box_scene_rejects_the_narrow_phase(cuda, lib_built):
    bvhcd = lib_built
    import scenes
    faces, frames = scenes.cloth_fold_frames(16, 1)
    T = faces.shape[0]
    bvh = bvhcd.LBvh(T, 0, enable_restr=False)
    bvh.maintain_boxes(bvhcd.BVH_BUILD, tri_boxes(faces, frames[0]), faces)
    front = bvhcd.BvttFront(bvh, narrow_phase=True, **CAPS)
    with pytest.raises(bvhcd.BvhcdError):
        front.maintain(bvhcd.FRONT_GENERATE)
    broad = bvhcd.BvttFront(bvh, narrow_phase=False, **CAPS)
    broad.maintain(bvhcd.FRONT_GENERATE)
    with pytest.raises(bvhcd.BvhcdError):
        broad.contacts(1)
