"""Double-buffered position uploads (bvhcd_bvh_stage_positions) on the GPU.

Frames whose positions were staged on a copy stream while the previous frame
computed must give the same trees and pair sets as frames uploaded the
ordinary way; a second staging before the first was used is refused; graph
frames refuse staged positions.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _frames(n=48, frames=14):
    import scenes
    return scenes.cloth_over_sphere_frames(n, frames=frames, sphere_freq=8)


def test_staged_frames_equal_plain_frames(cuda, lib_built):
    import torch
    import bvhcd
    import pyoracle
    faces, frames = _frames()
    T, V = faces.shape[0], frames[0].shape[0]
    dfaces = torch.from_numpy(faces).cuda()
    host = torch.from_numpy(np.stack(frames).astype(np.float32)).pin_memory()
    stream = torch.cuda.current_stream()
    copy = torch.cuda.Stream()

    def make():
        bvh = bvhcd.LBvh(T, V, enable_restr=True)
        front = bvhcd.BvttFront(bvh, int_front_capacity=64 * T, ext_front_capacity=64 * T, pair_capacity=16 * T,
                                cull_adjacent=True, narrow_phase=True)
        return bvh, front

    a_bvh, a_front = make()
    b_bvh, b_front = make()
    staged = b_bvh.stage_positions(host[0], copy)
    for f in range(len(frames)):
        bvhcd.frame(a_bvh, a_front, f, 0, host[f].numpy(), faces, stream=stream, faces_static=f > 0)
        bvhcd.frame(b_bvh, b_front, f, 0, staged, dfaces, stream=stream, faces_static=f > 0)
        if f + 1 < len(frames):
            staged = b_bvh.stage_positions(host[f + 1], copy)
        assert a_front.stats(stream)["overflow"] == 0 and b_front.stats(stream)["overflow"] == 0, f
        for narrow in (False, True):
            pa, pb = a_front.pairs(narrow=narrow, stream=stream), b_front.pairs(narrow=narrow, stream=stream)
            assert np.array_equal(pyoracle.canon_pairs(pa), pyoracle.canon_pairs(pb)), (f, narrow)
        ta, tb = a_bvh.export(stream), b_bvh.export(stream)
        for k in ("inode", "ibox", "leaf", "lbox"):
            assert np.array_equal(ta[k], tb[k]), (f, k)


def test_second_stage_before_use_is_refused(cuda, lib_built):
    import torch
    import bvhcd
    faces, frames = _frames(n=16, frames=2)
    bvh = bvhcd.LBvh(faces.shape[0], frames[0].shape[0])
    copy = torch.cuda.Stream()
    bvh.stage_positions(frames[0], copy)
    with pytest.raises(bvhcd.BvhcdError) as err:
        bvh.stage_positions(frames[1], copy)
    assert err.value.status == 6  # BVHCD_NOT_READY


def test_graph_frames_refuse_staged_positions(cuda, lib_built):
    import torch
    import bvhcd
    faces, frames = _frames(n=16, frames=2)
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = bvhcd.LBvh(T, V, enable_restr=False)
    front = bvhcd.BvttFront(bvh, int_front_capacity=64 * T, ext_front_capacity=64 * T, pair_capacity=16 * T,
                            auto_grow=False)
    s = torch.cuda.Stream()
    staged = bvh.stage_positions(frames[0], s)
    with pytest.raises(bvhcd.BvhcdError) as err:
        bvhcd.frame_graph(bvh, front, staged, torch.from_numpy(faces).cuda(), bvhcd.BVH_BUILD,
                          bvhcd.FRONT_GENERATE, stream=s)
    assert err.value.status == 1  # BVHCD_INVALID_ARG


def test_pairs_async_equal_synchronous_read(cuda, lib_built):
    """bvhcd_front_pairs_async writes the same pairs, in the same order, as
    bvhcd_front_pairs, into mapped host memory with no synchronisation;
    capacity and unmapped memory behave as documented."""
    import ctypes
    bvhcd = lib_built
    import scenes
    faces, frames = scenes.cloth_over_sphere_frames(48, frames=4, sphere_freq=8)
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = bvhcd.LBvh(T, V, enable_restr=True)
    front = bvhcd.BvttFront(bvh, int_front_capacity=2_000_000, ext_front_capacity=2_000_000, pair_capacity=500_000)
    bufs = [bvhcd.HostPairs(500_000) for _ in range(2)]
    small = bvhcd.HostPairs(10)
    stream = cuda.cuda.Stream()
    for f, pos in enumerate(frames):
        bvhcd.frame(bvh, front, f, 0, pos, faces, stream=stream)
        front.pairs_async(bufs[0], narrow=False, stream=stream)
        front.pairs_async(bufs[1], narrow=True, stream=stream)
        front.pairs_async(small, narrow=False, stream=stream)
        stream.synchronize()
        broad, hits = front.pairs(narrow=False, stream=stream), front.pairs(narrow=True, stream=stream)
        assert np.array_equal(bufs[0].read(), broad) and np.array_equal(bufs[1].read(), hits), f
        assert small.count == broad.shape[0] and np.array_equal(small.read(), broad[:10])
    pageable = np.zeros(4, np.int64)
    st = bvhcd.lib().bvhcd_front_pairs_async(front.handle, 0, ctypes.c_void_p(pageable.ctypes.data + 16), 1,
                                             ctypes.c_void_p(pageable.ctypes.data), None)
    assert st == 1  # INVALID_ARG: not mapped host memory
    for b in bufs + [small]:
        b.close()
