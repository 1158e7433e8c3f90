"""Host-side fault handling through the C ABI, with no GPU fault: device
allocation failures injected by the library's host hook
(bvhcd_debug_fail_alloc) and non-finite vertex input.

The reference ends the process on a failed CUDA call (checkCudaErrors, and
Mine/utility/CudaThrustUtils.hpp:9-11 for Thrust) and never looks at its
input; here a failed allocation returns BVHCD_OUT_OF_MEMORY and leaves the
handle usable, and a NaN or infinite coordinate is reported through the
stats and refused by the pair export, with the next finite frame exact
again."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OOM, INVALID = 2, 1
CAPS = dict(int_front_capacity=4_000_000, ext_front_capacity=4_000_000, pair_capacity=2_000_000)


@pytest.fixture
def fail_alloc(lib_built):
    L = lib_built.lib()
    yield lambda n: L.bvhcd_debug_fail_alloc(n)
    L.bvhcd_debug_fail_alloc(0)


def test_allocation_failure_on_create_and_recovery(cuda, lib_built, oracle, cloth_c1, fail_alloc):
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    for n in (1, 3, 20):
        assert fail_alloc(n) == 0
        with pytest.raises(lib_built.BvhcdError) as ei:
            lib_built.LBvh(T, V, enable_restr=True)
        assert ei.value.status == OOM, n
    fail_alloc(0)
    bvh = lib_built.LBvh(T, V, enable_restr=True)
    for n in (1, 2, 5):
        fail_alloc(n)
        with pytest.raises(lib_built.BvhcdError) as ei:
            lib_built.BvttFront(bvh, cull_adjacent=True, narrow_phase=True, **CAPS)
        assert ei.value.status == OOM, n
    fail_alloc(0)
    front = lib_built.BvttFront(bvh, cull_adjacent=True, narrow_phase=True, **CAPS)
    for f in range(4):
        b, fr = lib_built.schedule(f)
        bvh.maintain(b, frames[f], faces)
        front.maintain(fr)
        assert np.array_equal(oracle.canon_pairs(front.pairs()), oracle.brute_pairs(faces, frames[f], 1)), f


def test_allocation_failure_while_growing(cuda, lib_built, oracle, cloth_c1, fail_alloc):
    """A BVH sized for a small scene must grow at its first maintain, and a
    front with small buffers (auto_grow = 1) must grow at its first
    generation; each growth is made to fail once, returns OUT_OF_MEMORY, and
    the same handles then give the exact pair sets."""
    faces, frames = cloth_c1
    bvh = lib_built.LBvh(100, 100, enable_restr=True)
    small = dict(int_front_capacity=1000, ext_front_capacity=1000, pair_capacity=1000)
    front = lib_built.BvttFront(bvh, cull_adjacent=True, narrow_phase=True, auto_grow=1, **small)
    fail_alloc(4)
    with pytest.raises(lib_built.BvhcdError) as ei:
        bvh.maintain(lib_built.BVH_BUILD, frames[0], faces)
    assert ei.value.status == OOM
    fail_alloc(0)
    bvh.maintain(lib_built.BVH_BUILD, frames[0], faces)
    fail_alloc(3)  # the front's first growth (its fifth new buffer) fails
    with pytest.raises(lib_built.BvhcdError) as ei:
        front.maintain(lib_built.FRONT_GENERATE)
    assert ei.value.status == OOM
    fail_alloc(0)
    for f in range(1, 9):
        b, fr = lib_built.schedule(f)
        bvh.maintain(b, frames[f], faces)
        front.maintain(fr)
        st = front.stats()
        assert st["overflow"] == 0, (f, st)
        pairs = oracle.brute_pairs(faces, frames[f], 1)
        assert np.array_equal(oracle.canon_pairs(front.pairs()), pairs), f
        hit = oracle.narrow(pairs, faces, frames[f]).astype(bool)
        assert np.array_equal(oracle.canon_pairs(front.pairs(narrow=True)), pairs[hit]), f


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_nonfinite_input_is_reported(cuda, lib_built, oracle, cloth_c1, bad):
    """A NaN / infinite coordinate on a refit frame and on a build frame: the
    stats say so and the pair export refuses the frame; the finite frames
    around them give the exact pair sets (keeps included)."""
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = lib_built.LBvh(T, V, enable_restr=False)
    front = lib_built.BvttFront(bvh, cull_adjacent=True, narrow_phase=True, **CAPS)
    plan = [(0, 1, False), (1, 4, False), (1, 4, True), (1, 4, False), (1, 4, False), (0, 1, True),
            (0, 1, False), (1, 4, False)]
    for f, (b, fr, poison) in enumerate(plan):
        pos = frames[f].copy()
        if poison:
            pos[777, 1] = bad
        bvh.maintain(b, pos, faces, faces_static=f > 0)
        front.maintain(fr)
        st = front.stats()
        assert st["nonfinite_input"] == (1 if poison else 0), (f, st)
        if poison:
            with pytest.raises(lib_built.BvhcdError) as ei:
                front.pairs()
            assert ei.value.status == INVALID
            continue
        pairs = oracle.brute_pairs(faces, pos, 1)
        assert np.array_equal(oracle.canon_pairs(front.pairs()), pairs), f
        hit = oracle.narrow(pairs, faces, pos).astype(bool)
        assert np.array_equal(oracle.canon_pairs(front.pairs(narrow=True)), pairs[hit]), f


def test_nonfinite_box_scene_is_reported(cuda, lib_built, oracle, cloth_c1):
    torch = cuda
    faces, frames = cloth_c1
    pos = frames[0]
    tri = pos[faces]
    boxes = np.concatenate([tri.min(axis=1), tri.max(axis=1)], axis=1).astype(np.float32)
    bvh = lib_built.LBvh(faces.shape[0], 0, enable_restr=False)
    front = lib_built.BvttFront(bvh, cull_adjacent=True, narrow_phase=False, **CAPS)
    dfaces = torch.from_numpy(faces).cuda()
    for f, poison in enumerate([False, True, False]):
        bx = boxes.copy()
        if poison:
            bx[123, 4] = np.nan
        bvh.maintain_boxes(0 if f == 0 else 1, torch.from_numpy(bx).cuda(), dfaces, faces_static=f > 0)
        front.maintain(1 if f == 0 else 4)
        assert front.stats()["nonfinite_input"] == int(poison), f
        if not poison:
            assert np.array_equal(oracle.canon_pairs(front.pairs()), oracle.brute_pairs(faces, pos, 1)), f
