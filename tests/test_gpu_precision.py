"""The precision mode on the GPU (front config precision = 1): hits equal to
an FP64 evaluation of every broad-phase pair (the FP64 brute-force oracle),
contact points and distances within 1e-5 of the FP64 oracle, relative to the
pair's size.  Workload: stacked cloth layers 1e-3 apart with in-plane shear
and a grazing vertical jitter, so near-coplanar pairs are frequent."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stack():
    import scenes
    return scenes.stacked_layers_frames(64, 4, 4, z_noise=0.8)


def _scale(faces, verts, pairs):
    """largest coordinate extent of the pair's six vertices, per pair"""
    a = verts[faces[pairs[:, 0]]]
    b = verts[faces[pairs[:, 1]]]
    pts = np.concatenate([a, b], axis=1)
    return (pts.max(axis=1) - pts.min(axis=1)).max(axis=1).astype(np.float64)


def _run(lib, faces, frames, precision, nframes=4):
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = lib.LBvh(T, V, enable_restr=False)
    front = lib.BvttFront(bvh, 4_000_000, 4_000_000, 2_000_000, cull_adjacent=True, narrow_phase=True,
                          precision=precision)
    for f in range(nframes):
        b, fr = lib.schedule(f)
        bvh.maintain(b, frames[f], faces)
        front.maintain(fr)
        yield f, bvh, front


def test_precision_hits_equal_fp64_bruteforce(cuda, lib_built, oracle):
    faces, frames = _stack()
    flagged = 0
    fp32_differs = 0
    for f, bvh, front in _run(lib_built, faces, frames, 1):
        broad = oracle.canon_pairs(front.pairs())
        exp_broad = oracle.brute_pairs(faces, frames[f], 1)
        assert np.array_equal(broad, exp_broad), f
        hit64, _, _ = oracle.precision_pairs(exp_broad, faces, frames[f])
        got = oracle.canon_pairs(front.pairs(narrow=True))
        assert np.array_equal(got, oracle.canon_pairs(exp_broad[hit64])), f
        st = front.stats()
        flagged += st["flagged"]
        fp32 = np.asarray(oracle.narrow(exp_broad, faces, frames[f]), bool)
        fp32_differs += int(np.sum(fp32 != hit64))
    assert flagged > 0          # the grazing layers do reach the FP64 path
    print(f"flagged pairs {flagged}, FP32-vs-FP64 decisions that differ {fp32_differs}")


@pytest.mark.parametrize("precision", [1, 0])
def test_contact_points_and_distances_against_fp64(cuda, lib_built, oracle, precision):
    faces, frames = _stack()
    worst_c = worst_d = 0.0
    for f, bvh, front in _run(lib_built, faces, frames, precision, nframes=3):
        hits = front.pairs(narrow=True)
        c, _ = front.contacts(0)
        assert c.shape[0] == hits.shape[0]
        _, con, _ = oracle.precision_pairs(hits, faces, frames[f])
        seg = ~np.isnan(con[:, 0])
        sc = _scale(faces, frames[f], hits)
        if precision:
            assert np.array_equal(np.isnan(c[:, 0]), ~seg), f        # same coplanar pairs
        both = seg & ~np.isnan(c[:, 0])
        if both.any():
            e = np.abs(c[both, :3].astype(np.float64) - con[both, :3]).max(axis=1) / sc[both]
            worst_c = max(worst_c, float(e.max()))
        broad = front.pairs()
        d, _ = front.contacts(1)
        assert d.shape[0] == broad.shape[0]
        hit64, _, dist = oracle.precision_pairs(broad, faces, frames[f])
        if precision:
            assert np.array_equal(d[:, 3] == 0, hit64), f
        sc = _scale(faces, frames[f], broad)
        dd = ~hit64
        e = np.abs(d[dd, 3].astype(np.float64) - dist[dd]) / sc[dd]
        worst_d = max(worst_d, float(e.max()))
    print(f"precision {precision}: worst relative contact-point error {worst_c:.3e}, distance {worst_d:.3e}")
    if precision:
        assert worst_c <= 1e-5 and worst_d <= 1e-5


@pytest.mark.parametrize("restr", [True, False])
def test_fp16_node_boxes_keep_exact_pairs(cuda, lib_built, oracle, cloth_c1, restr):
    """Outward-rounded FP16 node boxes in the traversals: fronts may differ,
    the broad and narrow pair sets may not."""
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = lib_built.LBvh(T, V, enable_restr=restr, node_box_fp16=True)
    front = lib_built.BvttFront(bvh, 4_000_000, 4_000_000, 2_000_000, cull_adjacent=True, narrow_phase=True)
    ref = oracle.Pipeline(restructure=restr, cull_adjacent=True, narrow=True)
    for f in range(len(frames)):
        b, fr = lib_built.schedule(f)
        bvh.maintain(b, frames[f], faces)
        front.maintain(fr)
        ref.frame(faces, frames[f], b, fr)
        assert front.stats()["overflow"] == 0
        assert np.array_equal(oracle.canon_pairs(front.pairs()), oracle.canon_pairs(ref.pairs())), f
        assert np.array_equal(oracle.canon_pairs(front.pairs(narrow=True)),
                              oracle.canon_pairs(ref.pairs(narrow=True))), f
    if restr:
        # the same frame through FP32 node boxes: a looser FP16 box can only add front entries
        # below the entries it replaces, never lose a pair; report the front growth
        st = front.stats()
        print(f"fp16 node boxes, last frame fronts {st['int_front']} / {st['ext_front']}")


def test_fp16_node_boxes_c2_brute(cuda, lib_built, oracle):
    """The 562,742-triangle cloth-over-sphere workload with FP16 node boxes,
    one regenerated and two maintained frames, against the sweep-and-prune
    enumeration of all FP32 AABB overlaps."""
    import scenes
    faces, frames = scenes.cloth_over_sphere_frames(512, 3)
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = lib_built.LBvh(T, V, enable_restr=True, node_box_fp16=True)
    front = lib_built.BvttFront(bvh, 20_000_000, 20_000_000, 4_000_000, cull_adjacent=True, narrow_phase=True)
    for f, op in enumerate([lib_built.FRONT_GENERATE, lib_built.FRONT_KEEP, lib_built.FRONT_UPDATE]):
        bvh.maintain(lib_built.BVH_BUILD if f == 0 else lib_built.BVH_REFIT, frames[f], faces)
        front.maintain(op)
        assert front.stats()["overflow"] == 0
        assert np.array_equal(oracle.canon_pairs(front.pairs()), oracle.brute_pairs(faces, frames[f], 1)), f


@pytest.mark.parametrize("z_noise", [0.0, 0.8])
def test_stacked_layers_full_size_against_exact_predicate(cuda, lib_built, oracle, z_noise):
    """The precision configuration at its stated size: four stacked 512x512
    cloths (2,088,968 triangles) 1e-3 apart with in-plane shear -- as stated
    (z_noise 0: flat layers, every broad pair coplanar inside a layer) and
    with a grazing vertical jitter of up to 0.8 gaps (layers cut each other).
    FP16 outward-rounded node records, precision = 1.  Every frame: the broad
    set equals the sweep-and-prune set of overlapping FP32 boxes and the hits
    equal the exact (expansion-arithmetic) tri-tri predicate over it; on the
    last frame the contact points and distances are within 1e-5 of the FP64
    oracle, relative to the pair's size."""
    import scenes
    faces, frames = scenes.stacked_layers_frames(512, 4, 3, z_noise=z_noise)
    T, V = faces.shape[0], frames[0].shape[0]
    assert T == 2_088_968
    bvh = lib_built.LBvh(T, V, enable_restr=False, node_box_fp16=True)
    # the grazing layers with FP16 node boxes (rounded outward by up to a quarter of the layer gap)
    # hold more than 60 internal front entries per triangle: their buffers grow as needed
    caps = (130_000_000, 90_000_000, 16_000_000) if z_noise else (60_000_000, 40_000_000, 8_000_000)
    front = lib_built.BvttFront(bvh, *caps, cull_adjacent=True, narrow_phase=True, precision=1,
                                auto_grow=1 if z_noise else 0)
    for f in range(3):
        b, fr = lib_built.schedule(f)
        bvh.maintain(b, frames[f], faces, faces_static=f > 0)
        front.maintain(fr)
        st = front.stats()
        assert st["overflow"] == 0, (f, st)
        broad = oracle.canon_pairs(front.pairs())
        exp = oracle.brute_pairs(faces, frames[f], 1)
        assert np.array_equal(broad, exp), f
        exact = oracle.narrow(exp, faces, frames[f], exact=True).astype(bool)
        hits = oracle.canon_pairs(front.pairs(narrow=True))
        assert np.array_equal(hits, exp[exact]), f
    print(f"z_noise {z_noise}: {len(broad)} broad pairs, {len(hits)} hits, {st['flagged']} flagged")
    if z_noise:
        # FP64 results (bvhcd_front_contacts64): FP32 results would carry the FP32 rounding of
        # coordinates near 1, about 1.5e-5 of these 2e-3 triangles, whatever the arithmetic
        h = front.pairs(narrow=True)
        c = front.contacts64(0)
        _, con, _ = oracle.precision_pairs(h, faces, frames[2])
        assert np.array_equal(np.isnan(c[:, 0]), np.isnan(con[:, 0]))
        both = ~np.isnan(con[:, 0])
        assert both.sum() > 0.9 * len(h)
        e = np.abs(c[both, :3] - con[both, :3]).max(axis=1) / _scale(faces, frames[2], h)[both]
        assert float(e.max()) <= 1e-5, float(e.max())
        bp = front.pairs()
        d = front.contacts64(1)
        hit64, _, dist = oracle.precision_pairs(bp, faces, frames[2])
        assert np.array_equal(d[:, 3] == 0, hit64)
        dd = ~hit64
        ed = np.abs(d[dd, 3] - dist[dd]) / _scale(faces, frames[2], bp)[dd]
        assert float(ed.max()) <= 1e-5, float(ed.max())
        print(f"contact points / distances against FP64: {float(e.max()):.2e} / {float(ed.max()):.2e} of the extent")
