"""Capacity overflow through the C ABI: what each auto_grow mode reports and
how the results recover.

The reference never checks its buffers (an emission past a capacity writes out
of bounds); here every emission checks, raises bits in a device word, and the
three auto_grow modes decide what follows.  A frame whose input front lost
entries keeps reporting it (bit 6) until a GENERATE, and the sticky record
(overflow_any) keeps every bit seen since the front was created."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SMALL = dict(int_front_capacity=1000, ext_front_capacity=1000, pair_capacity=1000)


def _new(bvhcd, T, V, auto_grow, caps=SMALL):
    bvh = bvhcd.LBvh(T, V, enable_restr=True)
    front = bvhcd.BvttFront(bvh, cull_adjacent=True, narrow_phase=True, auto_grow=auto_grow, **caps)
    return bvh, front


def test_overflow_carries_over_until_generate(cuda, lib_built, oracle, cloth_c1):
    """auto_grow = 0: the generation overflows; the keep that works from the
    truncated front reports bit 6 and its pairs read as CAPACITY_EXCEEDED."""
    faces, frames = cloth_c1
    bvh, front = _new(lib_built, faces.shape[0], frames[0].shape[0], 0)
    bvh.maintain(lib_built.BVH_BUILD, frames[0], faces)
    front.maintain(lib_built.FRONT_GENERATE)
    st0 = front.stats()
    assert st0["overflow"] & 1 and st0["overflow"] & 2
    bvh.maintain(lib_built.BVH_REFIT, frames[1], faces)
    front.maintain(lib_built.FRONT_KEEP)
    st1 = front.stats()
    assert st1["overflow"] & 64, st1
    assert st1["overflow"] & 3
    with pytest.raises(lib_built.BvhcdError):
        front.pairs()
    assert st1["overflow_any"] & 1 and st1["overflow_any"] & 4


def test_sync_grow_leaves_no_sticky_record(cuda, lib_built, oracle, cloth_c1):
    """auto_grow = 1 replays inside the call: every frame is complete, so
    nothing reaches the sticky record."""
    faces, frames = cloth_c1
    bvh, front = _new(lib_built, faces.shape[0], frames[0].shape[0], 1)
    for f in range(4):
        b, fr = lib_built.schedule(f)
        bvh.maintain(b, frames[f], faces)
        front.maintain(fr)
        st = front.stats()
        assert st["overflow"] == 0 and st["overflow_any"] == 0, (f, st)
        assert np.array_equal(oracle.canon_pairs(front.pairs()), oracle.brute_pairs(faces, frames[f], 1)), f


def test_deferred_grow_recovers_without_sync(cuda, lib_built, oracle, cloth_c1):
    """auto_grow = 2: the overflowed frame is reported (and its pairs refused);
    a later maintain that sees the completed counter copy grows the buffers
    and regenerates, after which every frame equals the brute-force set.  The
    sticky record keeps the overflow."""
    faces, frames = cloth_c1
    bvh, front = _new(lib_built, faces.shape[0], frames[0].shape[0], 2)
    bad, good = [], []
    for f in range(12):
        b, fr = lib_built.schedule(f)
        bvh.maintain(b, frames[f], faces)
        front.maintain(fr)
        st = front.stats()  # synchronises: the copy of this frame's counters has landed
        if st["overflow"]:
            bad.append(f)
            with pytest.raises(lib_built.BvhcdError):
                front.pairs()
        else:
            good.append(f)
            pairs = oracle.brute_pairs(faces, frames[f], 1)
            assert np.array_equal(oracle.canon_pairs(front.pairs()), pairs), f
            hit = oracle.narrow(pairs, faces, frames[f]).astype(bool)
            assert np.array_equal(oracle.canon_pairs(front.pairs(narrow=True)), pairs[hit]), f
    assert bad and bad[0] == 0, bad
    # the frame after an overflow sees the copy (the stats call waited for it) and regenerates
    assert bad == list(range(len(bad))) and len(bad) <= 2, bad
    assert good and good[-1] == 11
    assert front.stats()["overflow_any"] & 1


def test_deferred_mode_matches_plain_when_nothing_overflows(cuda, lib_built, oracle, cloth_c1):
    """With capacity to spare the deferred mode runs the same operations as
    auto_grow = 0 and gives the same pairs on every frame."""
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    caps = dict(int_front_capacity=4_000_000, ext_front_capacity=4_000_000, pair_capacity=2_000_000)
    b0, f0 = _new(lib_built, T, V, 0, caps)
    b2, f2 = _new(lib_built, T, V, 2, caps)
    for f in range(14):
        b, fr = lib_built.schedule(f)
        for bvh, front in ((b0, f0), (b2, f2)):
            bvh.maintain(b, frames[f], faces, faces_static=f > 0)
            front.maintain(fr)
        s0, s2 = f0.stats(), f2.stats()
        assert s2["overflow_any"] == 0 and s0["front_op_run"] == s2["front_op_run"], f
        assert np.array_equal(oracle.canon_pairs(f0.pairs(narrow=True)), oracle.canon_pairs(f2.pairs(narrow=True))), f
        assert np.array_equal(oracle.canon_pairs(f0.pairs()), oracle.canon_pairs(f2.pairs())), f


def test_auto_grow_mode_out_of_range_is_rejected(cuda, lib_built):
    bvh = lib_built.LBvh(16, 16, enable_restr=False)
    with pytest.raises(lib_built.BvhcdError):
        lib_built.BvttFront(bvh, auto_grow=3, **SMALL)
