"""Proximities of the broad pairs (bvhcd_front_proximity) on the GPU against
the oracle's FP64 restatement, field by field and bit for bit: intra fronts
with and without adjacency culling, positions passed in or the BVH's own, a
box scene with positions, and an inter front over two meshes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CAPS = dict(int_front_capacity=2_000_000, ext_front_capacity=2_000_000, pair_capacity=1_000_000)


def _same(a, b):
    assert a.shape == b.shape, (a.shape, b.shape)
    for k in ("pair", "kind", "fa", "fb", "dist", "n", "w"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("cull", [True, False])
def test_proximity_matches_oracle(cuda, lib_built, oracle, cull):
    bvhcd = lib_built
    import scenes
    faces, frames = scenes.stacked_layers_frames(40, layers=3, frames=3, gap=1e-3, z_noise=0.8)
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = bvhcd.LBvh(T, V, enable_restr=False)
    front = bvhcd.BvttFront(bvh, cull_adjacent=cull, narrow_phase=True, **CAPS)
    h = 2e-3
    for f, pos in enumerate(frames):
        bvh.maintain(bvhcd.BVH_BUILD if f == 0 else bvhcd.BVH_REFIT, pos, faces)
        front.maintain(bvhcd.FRONT_GENERATE if f == 0 else bvhcd.FRONT_KEEP)
        got = front.proximity(h)
        pairs = front.pairs()
        ref = oracle.proximity(pairs, faces, pos, h=h)
        assert len(ref) > 100
        _same(got, ref)
        if f == 2:
            _same(front.proximity(h, pos=cuda.from_numpy(pos).cuda()), ref)
            assert len(front.proximity(0.0)) < len(ref)


def test_proximity_of_a_box_scene(cuda, lib_built, oracle):
    """A box scene (boxes grown by the thickness, so every pair within it is a
    candidate) with its positions passed in."""
    bvhcd = lib_built
    import scenes
    faces, frames = scenes.stacked_layers_frames(32, layers=2, frames=1, gap=1e-3, z_noise=0.8)
    pos = frames[0]
    h = 3e-3
    t = pos[faces]
    boxes = np.concatenate([t.min(axis=1) - h, t.max(axis=1) + h], axis=1).astype(np.float32)
    bvh = bvhcd.LBvh(faces.shape[0], 0, enable_restr=False)
    bvh.maintain_boxes(bvhcd.BVH_BUILD, boxes, faces)
    front = bvhcd.BvttFront(bvh, cull_adjacent=True, narrow_phase=False, **CAPS)
    front.maintain(bvhcd.FRONT_GENERATE)
    with pytest.raises(bvhcd.BvhcdError):
        front.proximity(h)  # no positions of its own
    got = front.proximity(h, pos=cuda.from_numpy(pos).cuda())
    ref = oracle.proximity(front.pairs(), faces, pos, h=h)
    assert len(ref) > 100
    _same(got, ref)


def test_proximity_of_an_inter_front(cuda, lib_built, oracle):
    bvhcd = lib_built
    import scenes
    x, y, cf = scenes.cloth_grid(40)
    cpos = np.stack([x, y, np.full_like(x, 0.25)], axis=1).astype(np.float32)
    sv, sf = scenes.icosphere(6, 0.25, (0.5, 0.5, 0.0))
    sv = sv.astype(np.float32)
    dbvh = bvhcd.LBvh(cf.shape[0], cpos.shape[0], enable_restr=False)
    rbvh = bvhcd.LBvh(sf.shape[0], sv.shape[0], enable_restr=False)
    dbvh.maintain(bvhcd.BVH_BUILD, cpos, cf)
    rbvh.maintain(bvhcd.BVH_BUILD, sv, sf)
    inter = bvhcd.BvttFront(dbvh, rigid=rbvh, narrow_phase=True, **CAPS)
    inter.maintain(bvhcd.FRONT_GENERATE)
    h = 5e-3
    got = inter.proximity(h)
    ref = oracle.proximity(inter.pairs(), cf, cpos, sf, sv, h=h)
    assert len(ref) > 10
    _same(got, ref)
