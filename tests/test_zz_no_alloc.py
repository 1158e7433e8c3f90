"""The allocation-free Morton-order entry point (bvhcd_morton_order_noalloc)
against the ordinary build path.

That entry point serves callers that may not allocate device memory while
they run (a simulator that gives all device memory to its own pool, or a
real-time loop that cannot take cudaMalloc's implicit synchronisation): its
temporaries live in a fixed device array inside the library.  Its output must
equal what bvhcd_bvh_maintain(BUILD) computes -- the sorted Morton codes and
the original triangle id of every Morton slot -- bit for bit, on consecutive
calls that reuse that array.  This file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _build_order(lib, faces, pos):
    bvh = lib.LBvh(faces.shape[0], pos.shape[0], enable_restr=False)
    bvh.maintain(lib.BVH_BUILD, pos, faces)
    t = bvh.export()
    order = np.empty(faces.shape[0], np.int32)
    order[t["primmap"]] = np.arange(faces.shape[0], dtype=np.int32)
    bvh.close()
    return t["codes"], order


def _noalloc(lib, torch, dpos, dfaces, T):
    codes = torch.full((max(T, 1),), -1, dtype=torch.int32, device="cuda")
    order = torch.full((max(T, 1),), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    st = lib.lib().bvhcd_morton_order_noalloc(
        ctypes.c_void_p(dpos.data_ptr()), ctypes.c_void_p(dfaces.data_ptr()), T,
        ctypes.c_void_p(codes.data_ptr()), ctypes.c_void_p(order.data_ptr()),
        ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return st, codes.cpu().numpy().view(np.uint32)[:T], order.cpu().numpy()[:T]


def test_noalloc_morton_order_matches_build(cuda, lib_built, cloth_c1):
    torch = cuda
    faces, frames = cloth_c1
    T = faces.shape[0]
    dfaces = torch.from_numpy(faces).cuda()
    # two calls in a row on one frame, then one on another frame: the shared
    # array keeps the previous call's contents and must not leak into the next
    for f in (0, 0, 7):
        exp_codes, exp_order = _build_order(lib_built, faces, frames[f])
        st, codes, order = _noalloc(lib_built, torch, torch.from_numpy(frames[f]).cuda(), dfaces, T)
        assert st == 0
        assert np.array_equal(codes, exp_codes)
        assert np.array_equal(order, exp_order)


def test_noalloc_calls_allocate_nothing(cuda, lib_built, cloth_c1):
    """After the first call on the device (which may load the library's
    device code and with it the fixed array), further calls leave the device's
    free memory unchanged: no allocation, by the library or anything it
    calls."""
    torch = cuda
    faces, frames = cloth_c1
    T = faces.shape[0]
    dpos = torch.from_numpy(frames[3]).cuda()
    dfaces = torch.from_numpy(faces).cuda()
    codes = torch.empty(T, dtype=torch.int32, device="cuda")
    order = torch.empty(T, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    args = [ctypes.c_void_p(dpos.data_ptr()), ctypes.c_void_p(dfaces.data_ptr()), T,
            ctypes.c_void_p(codes.data_ptr()), ctypes.c_void_p(order.data_ptr()),
            ctypes.c_void_p(stream.cuda_stream)]
    assert lib_built.lib().bvhcd_morton_order_noalloc(*args) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert lib_built.lib().bvhcd_morton_order_noalloc(*args) == 0
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_sizes_beyond_its_array(cuda, lib_built):
    torch = cuda
    dummy = torch.zeros(1, dtype=torch.int32, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    # the size check comes first: the buffers are never touched
    too_many = lib_built.lib().bvhcd_morton_order_noalloc(p, p, 1048577, p, p, None)
    assert too_many == 3  # BVHCD_CAPACITY_EXCEEDED
    st, _, _ = _noalloc(lib_built, torch, dummy, dummy, 0)
    assert st == 0
