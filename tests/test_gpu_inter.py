"""Inter-object fronts on the GPU: a rigid obstacle's triangles traversing a
deformable BVH (BvttFrontLooseInter over LBvhFixedDeformable and LBvhRigid).

Whatever shape its front has, an inter front reports every (deformable
triangle, obstacle triangle) pair whose FP32 boxes overlap, each once, so
every frame's broad pairs must equal the oracle's brute-force enumeration
exactly and the hits the FP32 SAT over those pairs.  The schedule runs every
front operation, a restructure of the deformable BVH, rebuilds of both BVHs
and an intra front over the same deformable BVH, which must not disturb the
inter front (nor the inter front it).
"""
import math

import numpy as np
import pytest

from treecheck import pick_roots

pytestmark = pytest.mark.gpu

CAPS = dict(int_front_capacity=2_000_000, ext_front_capacity=2_000_000, pair_capacity=1_000_000)


def _rows(p):
    p = np.asarray(p, dtype=np.int64).reshape(-1, 2)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def _cloth(n, frames):
    """The cloth of the cloth-over-sphere scene alone: n x n vertices folded by
    a damped radial wave about z = 0.2."""
    import scenes
    faces, pos = scenes.cloth_over_sphere_frames(n, frames=frames, sphere_freq=2)
    tc, vc = 2 * (n - 1) ** 2, n * n
    assert faces[:tc].max() < vc
    return faces[:tc].copy(), [p[:vc].copy() for p in pos]


def _obstacle(freq, f, radius=0.25):
    """An icosphere moved rigidly: turned about z and carried along x."""
    import scenes
    v, faces = scenes.icosphere(freq, radius, (0.0, 0.0, 0.0))
    a = 0.05 * f
    c, s = math.cos(a), math.sin(a)
    rot = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    v = v @ rot.T + np.array([0.4 + 0.015 * f, 0.5, 0.02 * math.sin(f)])
    return faces, v.astype(np.float32)


def _check_frame(oracle, front, cf, cp, of, op, tag):
    st = front.stats()
    assert st["overflow"] == 0, (tag, st)
    exp = oracle.brute_inter_pairs(cf, cp, of, op)
    got = _rows(front.pairs())
    assert np.array_equal(got, exp), tag
    assert st["broad_pairs"] == exp.shape[0], tag
    mask = oracle.inter_narrow(exp, cf, cp, of, op).astype(bool)
    assert np.array_equal(_rows(front.pairs(narrow=True)), exp[mask]), tag
    assert st["narrow_hits"] == int(mask.sum()), tag
    return exp.shape[0], int(mask.sum())


def test_inter_schedule_matches_brute_force(cuda, lib_built, oracle):
    bvhcd = lib_built
    cf, frames = _cloth(48, 14)
    of, _ = _obstacle(8, 0)
    dbvh = bvhcd.LBvh(cf.shape[0], frames[0].shape[0], enable_restr=True)
    rbvh = bvhcd.LBvh(of.shape[0], 2000, enable_restr=False)
    intra = bvhcd.BvttFront(dbvh, cull_adjacent=True, narrow_phase=True, **CAPS)
    # cull_adjacent does not apply across two meshes: vertex ids of the
    # cloth and of the obstacle coincide without naming the same vertex
    inter = bvhcd.BvttFront(dbvh, rigid=rbvh, cull_adjacent=True, narrow_phase=True, **CAPS)
    seen = {}
    total = 0
    for f, cp in enumerate(frames):
        b, fr = bvhcd.schedule(f)
        dbvh.maintain(b, cp, cf, faces_static=f > 0)
        if f == 4:
            assert dbvh.opt_tag() == 1, "the marks of frame 3 restructure the deformable BVH"
        intra.maintain(fr)
        of, op = _obstacle(8, f)
        rbvh.maintain(bvhcd.BVH_BUILD if f in (0, 9) else bvhcd.BVH_REFIT, op, of, faces_static=f > 0)
        inter.maintain(fr)
        if f == 4:  # the restructured subtrees are re-sprouted, not the whole front regenerated
            assert inter.stats()["front_op_run"] == bvhcd.FRONT_RESTRUCTURE
        seen[fr] = seen.get(fr, 0) + 1
        p, h = _check_frame(oracle, inter, cf, cp, of, op, f)
        total += p
        assert h > 0, f
        assert np.array_equal(oracle.canon_pairs(intra.pairs()), oracle.brute_pairs(cf, cp, 1)), f
        if f == 3:
            dbvh.request_restructure(pick_roots(dbvh.export()))
    assert total > 0
    for op in (bvhcd.FRONT_GENERATE, bvhcd.FRONT_UPDATE, bvhcd.FRONT_REORDER, bvhcd.FRONT_KEEP):
        assert seen.get(op, 0) > 0, op


def test_inter_front_restructure(cuda, lib_built, oracle):
    """BvttFrontLooseInter::restructure (BvttFrontLooseInter.cu:252-318): the
    deformable BVH restructures subtrees on several frames while the inter
    front keeps or updates in between.  The frame after each restructure runs
    the front restructure (valid entries kept, the restructured subtrees
    re-sprouted) and every frame equals the brute-force pairs.  Two topology
    changes between two maintains of the front, or a rebuild, fall back to a
    regeneration."""
    bvhcd = lib_built
    cf, frames = _cloth(56, 16)
    of, _ = _obstacle(8, 0)
    dbvh = bvhcd.LBvh(cf.shape[0], frames[0].shape[0], enable_restr=True)
    rbvh = bvhcd.LBvh(of.shape[0], 2000, enable_restr=False)
    inter = bvhcd.BvttFront(dbvh, rigid=rbvh, narrow_phase=True, **CAPS)
    # the intra front over the same BVH consumes the restructure marks each
    # frame, as in the reference app (keeps only: no quality check adds marks)
    intra = bvhcd.BvttFront(dbvh, cull_adjacent=True, narrow_phase=False, **CAPS)
    ops = [bvhcd.FRONT_GENERATE, 4, 4, 4, 4, 2, 4, 4, 2, 4, 4, 4, 4, 3, 4, 4]
    restr_on = {2, 5, 8, 12}           # frames whose BVH maintain restructures (marks set the frame before)
    skip_inter = {12}                  # the front is not maintained on frame 12 ...
    restr_on_13 = True                 # ... and frame 13 restructures again: two changes -> regenerate
    runs = {}
    for f, cp in enumerate(frames):
        dbvh.maintain(bvhcd.BVH_BUILD if f == 0 else bvhcd.BVH_REFIT, cp, cf, faces_static=f > 0)
        if f in restr_on or (f == 13 and restr_on_13):
            assert dbvh.opt_tag() == 1, f
        intra.maintain(bvhcd.FRONT_GENERATE if f == 0 else bvhcd.FRONT_KEEP)
        of, op = _obstacle(8, f)
        rbvh.maintain(bvhcd.BVH_BUILD if f == 0 else bvhcd.BVH_REFIT, op, of, faces_static=f > 0)
        if f not in skip_inter:
            inter.maintain(ops[f])
            run = inter.stats()["front_op_run"]
            runs[f] = run
            if f in restr_on:
                assert run == bvhcd.FRONT_RESTRUCTURE, (f, run)
            _check_frame(oracle, inter, cf, cp, of, op, f)
        if f + 1 in restr_on or f + 1 == 13:
            dbvh.request_restructure(pick_roots(dbvh.export(), frac=0.2))
    assert runs[13] == bvhcd.FRONT_GENERATE, runs
    assert sum(1 for r in runs.values() if r == bvhcd.FRONT_RESTRUCTURE) == 3, runs


def test_inter_every_operation_every_frame(cuda, lib_built, oracle):
    """Each front operation run on every frame after the first, the obstacle
    moving through the cloth."""
    bvhcd = lib_built
    cf, frames = _cloth(40, 8)
    for fop in (bvhcd.FRONT_UPDATE, bvhcd.FRONT_REORDER, bvhcd.FRONT_KEEP, bvhcd.FRONT_PURE_BVH_CD,
                bvhcd.FRONT_RESTRUCTURE):
        of, _ = _obstacle(6, 0)
        dbvh = bvhcd.LBvh(cf.shape[0], frames[0].shape[0], enable_restr=False)
        rbvh = bvhcd.LBvh(of.shape[0], 1000, enable_restr=False)
        inter = bvhcd.BvttFront(dbvh, rigid=rbvh, narrow_phase=True, **CAPS)
        for f, cp in enumerate(frames):
            dbvh.maintain(bvhcd.BVH_BUILD if f == 0 else bvhcd.BVH_REFIT, cp, cf, faces_static=f > 0)
            of, op = _obstacle(6, 2 * f)
            rbvh.maintain(bvhcd.BVH_BUILD if f == 0 else bvhcd.BVH_REFIT, op, of, faces_static=f > 0)
            inter.maintain(bvhcd.FRONT_GENERATE if f == 0 else fop)
            _check_frame(oracle, inter, cf, cp, of, op, (fop, f))


def _tiny(kind):
    if kind == "empty":
        return np.zeros((0, 3), np.int32), np.zeros((0, 3), np.float32)
    if kind == "one":
        return np.array([[0, 1, 2]], np.int32), np.array([[0.2, 0.2, 0.0], [0.8, 0.3, 0.1],
                                                          [0.4, 0.9, 0.3]], np.float32)
    if kind == "far":
        v = np.random.default_rng(5).uniform(0, 1, (30, 3)).astype(np.float32) + 10.0
        return np.arange(30, dtype=np.int32).reshape(10, 3), v
    raise KeyError(kind)


@pytest.mark.parametrize("side,kind", [("rigid", "one"), ("rigid", "empty"), ("rigid", "far"),
                                       ("deformable", "one"), ("deformable", "empty")])
def test_inter_edge_cases(cuda, lib_built, oracle, side, kind):
    bvhcd = lib_built
    cf, frames = _cloth(24, 5)
    tf, tv = _tiny(kind)
    if side == "rigid":
        dfaces, dpos = cf, frames
        ofaces, opos = tf, [tv] * len(frames)
    else:
        of, ov = _obstacle(4, 0, radius=0.4)
        dfaces, dpos = tf, [tv] * len(frames)
        ofaces, opos = of, [ov + np.float32(0.01 * f) for f in range(len(frames))]
    dbvh = bvhcd.LBvh(max(dfaces.shape[0], 1), max(dpos[0].shape[0], 1), enable_restr=False)
    rbvh = bvhcd.LBvh(max(ofaces.shape[0], 1), max(opos[0].shape[0], 1), enable_restr=False)
    inter = bvhcd.BvttFront(dbvh, rigid=rbvh, narrow_phase=True, **CAPS)
    ops = [bvhcd.FRONT_GENERATE, bvhcd.FRONT_KEEP, bvhcd.FRONT_UPDATE, bvhcd.FRONT_REORDER, bvhcd.FRONT_KEEP]
    for f in range(len(frames)):
        dbvh.maintain(bvhcd.BVH_BUILD if f == 0 else bvhcd.BVH_REFIT, dpos[f], dfaces)
        rbvh.maintain(bvhcd.BVH_BUILD if f == 0 else bvhcd.BVH_REFIT, opos[f], ofaces)
        inter.maintain(ops[f])
        _check_frame(oracle, inter, dfaces, dpos[f], ofaces, opos[f], (side, kind, f))


def test_inter_rejections(cuda, lib_built):
    bvhcd = lib_built
    a = bvhcd.LBvh(1000, 1000)
    b = bvhcd.LBvh(1000, 1000)
    with pytest.raises(bvhcd.BvhcdError):
        bvhcd.BvttFront(a, rigid=a, **CAPS)
    with pytest.raises(bvhcd.BvhcdError):
        bvhcd.BvttFront(a, rigid=b, precision=1, **CAPS)
    inter = bvhcd.BvttFront(a, rigid=b, **CAPS)
    with pytest.raises(bvhcd.BvhcdError):
        inter.maintain(bvhcd.FRONT_GENERATE)  # neither BVH built yet
    cf, frames = _cloth(16, 1)
    a.maintain(bvhcd.BVH_BUILD, frames[0], cf)
    b.maintain(bvhcd.BVH_BUILD, frames[0], cf)
    inter.maintain(bvhcd.FRONT_GENERATE)
    with pytest.raises(bvhcd.BvhcdError):
        inter.contacts(0)
