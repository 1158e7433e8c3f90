"""Python mirror of the reference's collision module interface over the C ABI
(include/bvhcd.h, libbvhcd.so built in this directory).

``LBvh`` stands in for ``LBvhFixedDeformable`` and ``BvttFront`` for
``BvttFrontLooseIntra`` (Mine/collision/lbvh/LBvhFixedDeformable.h:27-50,
Mine/collision/bvtt_front/BvttFrontLooseIntra.h:27-36): same maintenance
options, same meaning of the per-frame calls.  Inputs are numpy arrays (host,
copied each call like the reference's SceneData upload) or CUDA tensors (read
in place).  There is no fallback: the compiled library is required, and every
error status raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbvhcd.so")

BVH_BUILD, BVH_REFIT, BVH_UPDATE = 0, 1, 2
FRONT_PURE_BVH_CD, FRONT_GENERATE, FRONT_UPDATE, FRONT_REORDER, FRONT_KEEP, FRONT_RESTRUCTURE = range(6)

STATUS = {0: "ok", 1: "invalid argument", 2: "out of device memory", 3: "capacity exceeded",
          4: "CUDA error", 5: "timeout", 6: "not ready"}

EXPORTED = [
    "bvhcd_status_string", "bvhcd_device_check", "bvhcd_bvh_create", "bvhcd_bvh_destroy",
    "bvhcd_bvh_maintain", "bvhcd_bvh_sizes", "bvhcd_bvh_opt_tag", "bvhcd_bvh_export",
    "bvhcd_bvh_request_restructure", "bvhcd_bvh_stage_positions", "bvhcd_bvh_maintain_boxes", "bvhcd_obj_read",
    "bvhcd_front_create", "bvhcd_front_create_inter", "bvhcd_front_destroy", "bvhcd_front_maintain", "bvhcd_front_stats_get",
    "bvhcd_front_pairs", "bvhcd_front_device_results", "bvhcd_front_export", "bvhcd_front_proximity",
    "bvhcd_front_pairs_async", "bvhcd_host_alloc", "bvhcd_host_free",
    "bvhcd_schedule_heuristic", "bvhcd_frame", "bvhcd_profile_enable", "bvhcd_profile_read",
    "bvhcd_launch_count", "bvhcd_morton_order_noalloc", "bvhcd_bvh_set_scenes", "bvhcd_frame_graph",
    "bvhcd_front_get_shapes", "bvhcd_front_set_shapes", "bvhcd_front_autotune",
    "bvhcd_bvh_copy_state", "bvhcd_front_copy_state",
    "bvhcd_learner_create", "bvhcd_learner_destroy", "bvhcd_learner_set_params", "bvhcd_learner_get_params",
    "bvhcd_learner_frame", "bvhcd_learner_observe", "bvhcd_learner_cut", "bvhcd_learner_features",
    "bvhcd_learner_work", "bvhcd_mlp_gradient", "bvhcd_mlp_train", "bvhcd_mlp_predict",
    "bvhcd_learner_set_decide_every", "bvhcd_front_contacts", "bvhcd_debug_fail_alloc", "bvhcd_front_contacts64",
    "bvhcd_learner_set_front_cycle",
]

MLP_PARAMS = 5443

SHAPE_STAGES = ["keep", "prune_int", "prune_ext", "balance", "sprout", "narrow"]

STAGES = ["bvh_build", "bvh_refit", "bvh_restructure", "front_generate", "front_update",
          "front_keep", "front_balance", "front_reorder", "narrow", "quality", "pure_bvh_cd",
          "front_restructure"]


class BvhcdError(RuntimeError):
    def __init__(self, status, what):
        super().__init__(f"{what}: {STATUS.get(status, status)}")
        self.status = status


class BvhConfig(ctypes.Structure):
    _fields_ = [("prim_capacity", ctypes.c_int32), ("vert_capacity", ctypes.c_int32),
                ("enable_restr", ctypes.c_int32), ("node_box_fp16", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 4)]


class FrontConfig(ctypes.Structure):
    _fields_ = [("int_front_capacity", ctypes.c_int64), ("ext_front_capacity", ctypes.c_int64),
                ("pair_capacity", ctypes.c_int64), ("cull_adjacent", ctypes.c_int32),
                ("narrow_phase", ctypes.c_int32), ("auto_grow", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("reserved", ctypes.c_int32 * 4)]


class Scene(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_void_p), ("faces", ctypes.c_void_p),
                ("num_vertices", ctypes.c_int32), ("num_faces", ctypes.c_int32),
                ("on_device", ctypes.c_int32), ("faces_static", ctypes.c_int32)]


# bvhcd_proximity
PROX_DTYPE = np.dtype([("pair", np.int32), ("kind", np.int32), ("fa", np.int32), ("fb", np.int32),
                       ("dist", np.float64), ("n", np.float64, 3), ("w", np.float64, 4)], align=True)
assert PROX_DTYPE.itemsize == 80


class BoxScene(ctypes.Structure):
    _fields_ = [("boxes", ctypes.c_void_p), ("faces", ctypes.c_void_p), ("num_faces", ctypes.c_int32),
                ("boxes_f64", ctypes.c_int32), ("on_device", ctypes.c_int32), ("faces_static", ctypes.c_int32)]


class LaunchShapes(ctypes.Structure):
    _fields_ = [("unroll", ctypes.c_int32 * 6), ("block", ctypes.c_int32 * 6)]

    def as_dict(self):
        return {k: (int(self.unroll[i]), int(self.block[i])) for i, k in enumerate(SHAPE_STAGES)}


class FrontStats(ctypes.Structure):
    _fields_ = [("int_front", ctypes.c_int64), ("ext_front", ctypes.c_int64),
                ("broad_pairs", ctypes.c_int64), ("narrow_hits", ctypes.c_int64),
                ("overflow", ctypes.c_int32), ("bvh_opt_tag", ctypes.c_int32),
                ("front_op_run", ctypes.c_int32), ("restr_pending", ctypes.c_int32),
                ("num_rt_subtrees", ctypes.c_int32), ("num_rt_int_nodes", ctypes.c_int32),
                ("flagged", ctypes.c_int32), ("keep_tested", ctypes.c_int32), ("overflow_any", ctypes.c_int32),
                ("nonfinite_input", ctypes.c_int32), ("reserved", ctypes.c_int32 * 2)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


_LIB = None


def build(force: bool = False):
    """Compile libbvhcd.so in-tree (nvcc, sm_100a)."""
    if force:
        subprocess.run(["make", "-s", "-C", HERE, "clean"], check=True)
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    """The loaded C library.  Raises when it is missing: no fallback path."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; run make in {HERE}")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        sig = {
            "bvhcd_status_string": (ctypes.c_char_p, [ctypes.c_int]),
            "bvhcd_device_check": (ctypes.c_int, [i32, ctypes.POINTER(i32)]),
            "bvhcd_bvh_create": (ctypes.c_int, [ctypes.POINTER(BvhConfig), ctypes.POINTER(vp)]),
            "bvhcd_bvh_destroy": (ctypes.c_int, [vp]),
            "bvhcd_bvh_maintain": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(Scene), vp]),
            "bvhcd_bvh_sizes": (ctypes.c_int, [vp, ctypes.POINTER(i32), ctypes.POINTER(i32),
                                               ctypes.POINTER(i32)]),
            "bvhcd_bvh_opt_tag": (ctypes.c_int, [vp, ctypes.POINTER(i32)]),
            "bvhcd_bvh_export": (ctypes.c_int, [vp] + [vp] * 7 + [vp]),
            "bvhcd_bvh_request_restructure": (ctypes.c_int, [vp, vp, i32, vp]),
            "bvhcd_bvh_stage_positions": (ctypes.c_int, [vp, vp, i32, vp, ctypes.POINTER(vp)]),
            "bvhcd_bvh_maintain_boxes": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(BoxScene), vp]),
            "bvhcd_obj_read": (ctypes.c_int, [ctypes.c_char_p, vp, i32, vp, i32, ctypes.POINTER(i32),
                                              ctypes.POINTER(i32)]),
            "bvhcd_front_create": (ctypes.c_int, [vp, ctypes.POINTER(FrontConfig), ctypes.POINTER(vp)]),
            "bvhcd_front_create_inter": (ctypes.c_int, [vp, vp, ctypes.POINTER(FrontConfig), ctypes.POINTER(vp)]),
            "bvhcd_front_destroy": (ctypes.c_int, [vp]),
            "bvhcd_front_pairs_async": (ctypes.c_int, [vp, i32, vp, ctypes.c_int64, vp, vp]),
            "bvhcd_host_alloc": (ctypes.c_int, [ctypes.c_int64, ctypes.POINTER(vp)]),
            "bvhcd_host_free": (ctypes.c_int, [vp]),
            "bvhcd_front_proximity": (ctypes.c_int, [vp, vp, ctypes.c_double, vp, ctypes.c_int64,
                                                     ctypes.POINTER(ctypes.c_int64), i32, vp]),
            "bvhcd_front_maintain": (ctypes.c_int, [vp, ctypes.c_int, vp]),
            "bvhcd_front_stats_get": (ctypes.c_int, [vp, ctypes.POINTER(FrontStats), vp]),
            "bvhcd_front_pairs": (ctypes.c_int, [vp, i32, vp, i64, ctypes.POINTER(i64), i32, vp]),
            "bvhcd_front_device_results": (ctypes.c_int, [vp, ctypes.POINTER(vp), ctypes.POINTER(vp)]),
            "bvhcd_front_export": (ctypes.c_int, [vp, i32, vp, i64, ctypes.POINTER(i64), vp]),
            "bvhcd_schedule_heuristic": (ctypes.c_int, [i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]),
            "bvhcd_frame": (ctypes.c_int, [vp, vp, i32, i32, ctypes.POINTER(Scene), vp]),
            "bvhcd_profile_enable": (ctypes.c_int, [vp, i32]),
            "bvhcd_profile_read": (ctypes.c_int, [vp, vp, vp, i32]),
            "bvhcd_launch_count": (ctypes.c_int, [ctypes.POINTER(i64)]),
            "bvhcd_debug_fail_alloc": (ctypes.c_int, [i64]),
            "bvhcd_morton_order_noalloc": (ctypes.c_int, [vp, vp, i32, vp, vp, vp]),
            "bvhcd_bvh_set_scenes": (ctypes.c_int, [vp, i32, vp]),
            "bvhcd_frame_graph": (ctypes.c_int, [vp, vp, ctypes.POINTER(Scene), i32, i32, vp]),
            "bvhcd_front_get_shapes": (ctypes.c_int, [vp, ctypes.POINTER(LaunchShapes)]),
            "bvhcd_front_set_shapes": (ctypes.c_int, [vp, ctypes.POINTER(LaunchShapes)]),
            "bvhcd_front_autotune": (ctypes.c_int, [vp, i32, ctypes.POINTER(LaunchShapes), vp, vp]),
            "bvhcd_bvh_copy_state": (ctypes.c_int, [vp, vp, vp]),
            "bvhcd_front_copy_state": (ctypes.c_int, [vp, vp, vp]),
            "bvhcd_front_contacts": (ctypes.c_int, [vp, i32, vp, i64, ctypes.POINTER(i64), ctypes.POINTER(i64),
                                                    i32, vp]),
            "bvhcd_front_contacts64": (ctypes.c_int, [vp, i32, vp, i64, ctypes.POINTER(i64), i32, vp]),
            "bvhcd_learner_create": (ctypes.c_int, [vp, vp, i32, ctypes.POINTER(vp)]),
            "bvhcd_learner_destroy": (ctypes.c_int, [vp]),
            "bvhcd_learner_set_params": (ctypes.c_int, [vp, vp]),
            "bvhcd_learner_get_params": (ctypes.c_int, [vp, vp]),
            "bvhcd_learner_frame": (ctypes.c_int, [vp, ctypes.POINTER(Scene), i32, ctypes.POINTER(i32),
                                                   ctypes.POINTER(i32), vp]),
            "bvhcd_learner_observe": (ctypes.c_int, [vp, i32, i32, vp]),
            "bvhcd_learner_set_decide_every": (ctypes.c_int, [vp, i32]),
            "bvhcd_learner_set_front_cycle": (ctypes.c_int, [vp, i32]),
            "bvhcd_learner_cut": (ctypes.c_int, [vp, vp, i32, ctypes.POINTER(i32), vp]),
            "bvhcd_learner_features": (ctypes.c_int, [vp, vp, i32, ctypes.POINTER(i32), vp]),
            "bvhcd_learner_work": (ctypes.c_int, [vp, vp, vp, i32, vp]),
            "bvhcd_mlp_gradient": (ctypes.c_int, [vp, vp, vp, i32, vp, vp, vp, vp]),
            "bvhcd_mlp_train": (ctypes.c_int, [vp, vp, vp, i32, vp, i32, i32, ctypes.c_float, ctypes.c_uint32,
                                               vp, vp]),
            "bvhcd_mlp_predict": (ctypes.c_int, [vp, vp, i32, vp, vp, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def _check(status, what):
    if status != 0:
        raise BvhcdError(status, what)


def _stream_ptr(stream):
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        except ImportError:
            pass
        return ctypes.c_void_p(0)
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


def schedule(frame: int, start: int = 0):
    """(bvh_op, front_op) of BenchmarkLogic::maintainScheme, STATIC_MANDATORY
    with divergent marks (Mine/system/Logic/BenchmarkLogic.hpp:102-117)."""
    b, f = ctypes.c_int32(), ctypes.c_int32()
    _check(lib().bvhcd_schedule_heuristic(frame, start, ctypes.byref(b), ctypes.byref(f)), "schedule")
    return b.value, f.value


def launch_count() -> int:
    n = ctypes.c_int64()
    _check(lib().bvhcd_launch_count(ctypes.byref(n)), "launch count")
    return n.value


def device_check(device: int = 0) -> bool:
    ok = ctypes.c_int32()
    _check(lib().bvhcd_device_check(device, ctypes.byref(ok)), "device check")
    return bool(ok.value)


class StagedPositions:
    """Positions copied to one of an LBvh's staging buffers by
    LBvh.stage_positions: pass it as `pos` (with faces on the GPU) to the
    next maintain / frame."""

    def __init__(self, ptr: int, num_vertices: int):
        self.ptr, self.num_vertices = int(ptr), int(num_vertices)


def _scene(pos, faces, faces_static=False):
    """Scene struct plus the objects that keep its buffers alive."""
    keep = []
    if isinstance(pos, StagedPositions):
        import torch
        assert isinstance(faces, torch.Tensor) and faces.is_cuda and faces.dtype == torch.int32, \
            "staged positions go with faces on the GPU"
        faces = faces.contiguous()
        keep.append(faces)
        return Scene(pos.ptr, faces.data_ptr(), pos.num_vertices, faces.shape[0], 1, int(faces_static)), keep
    try:
        import torch
        is_t = isinstance(pos, torch.Tensor)
    except ImportError:
        is_t = False
    if is_t:
        assert pos.is_cuda and faces.is_cuda, "tensors must live on the GPU"
        assert pos.dtype == torch.float32 and faces.dtype == torch.int32
        pos = pos.contiguous()
        faces = faces.contiguous()
        keep += [pos, faces]
        sc = Scene(pos.data_ptr(), faces.data_ptr(), pos.shape[0], faces.shape[0], 1, int(faces_static))
    else:
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        faces = np.ascontiguousarray(faces, dtype=np.int32)
        keep += [pos, faces]
        sc = Scene(pos.ctypes.data, faces.ctypes.data, pos.shape[0], faces.shape[0], 0, int(faces_static))
    return sc, keep


def _box_scene(boxes, faces, faces_static=False):
    """Box-scene struct (T x 6 boxes, FP32 or FP64; T x 3 faces) plus the
    objects that keep its buffers alive."""
    try:
        import torch
        is_t = isinstance(boxes, torch.Tensor)
    except ImportError:
        is_t = False
    if is_t:
        assert boxes.is_cuda and faces.is_cuda, "tensors must live on the GPU"
        assert boxes.dtype in (torch.float32, torch.float64) and faces.dtype == torch.int32
        boxes = boxes.contiguous()
        faces = faces.contiguous()
        f64 = int(boxes.dtype == torch.float64)
        return BoxScene(boxes.data_ptr(), faces.data_ptr(), faces.shape[0], f64, 1, int(faces_static)), [boxes, faces]
    boxes = np.asarray(boxes)
    f64 = int(boxes.dtype == np.float64)
    boxes = np.ascontiguousarray(boxes, dtype=np.float64 if f64 else np.float32).reshape(-1, 6)
    faces = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 3)
    assert boxes.shape[0] == faces.shape[0]
    return BoxScene(boxes.ctypes.data, faces.ctypes.data, faces.shape[0], f64, 0, int(faces_static)), [boxes, faces]


class LBvh:
    """LBvhFixedDeformable: maintain(BUILD | REFIT | UPDATE, scene) per frame."""

    def __init__(self, prim_capacity: int, vert_capacity: int = 0, enable_restr: bool = True,
                 node_box_fp16: bool = False):
        cfg = BvhConfig(int(prim_capacity), int(vert_capacity), int(enable_restr), int(node_box_fp16))
        h = ctypes.c_void_p()
        _check(lib().bvhcd_bvh_create(ctypes.byref(cfg), ctypes.byref(h)), "bvh create")
        self._h = h
        self._keep = []

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().bvhcd_bvh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def maintain(self, op: int, pos, faces, stream=None, faces_static=False):
        sc, keep = _scene(pos, faces, faces_static)
        self._keep = keep
        _check(lib().bvhcd_bvh_maintain(self._h, int(op), ctypes.byref(sc), _stream_ptr(stream)),
               "bvh maintain")

    def maintain_boxes(self, op: int, boxes, faces, stream=None, faces_static=False):
        """maintain(scheme, ARCSimSceneData): the primitives given as boxes
        (T x 6: min xyz, max xyz; FP64 boxes are rounded outward to FP32)."""
        sc, keep = _box_scene(boxes, faces, faces_static)
        self._keep = keep
        _check(lib().bvhcd_bvh_maintain_boxes(self._h, int(op), ctypes.byref(sc), _stream_ptr(stream)),
               "bvh maintain boxes")

    def stage_positions(self, pos, copy_stream=None) -> "StagedPositions":
        """bvhcd_bvh_stage_positions: copy the next frame's positions (a
        host array; pinned for an asynchronous copy) to a staging buffer on
        copy_stream; pass the result as the next maintain / frame's `pos`."""
        try:
            import torch
            is_t = isinstance(pos, torch.Tensor)
        except ImportError:
            is_t = False
        if is_t:
            assert not pos.is_cuda and pos.dtype == torch.float32 and pos.is_contiguous()
            ptr, nv = pos.data_ptr(), pos.shape[0]
        else:
            pos = np.ascontiguousarray(pos, dtype=np.float32)
            ptr, nv = pos.ctypes.data, pos.shape[0]
        self._stage_keep = pos
        out = ctypes.c_void_p()
        _check(lib().bvhcd_bvh_stage_positions(self._h, ctypes.c_void_p(ptr), int(nv), _stream_ptr(copy_stream),
                                               ctypes.byref(out)), "stage positions")
        return StagedPositions(out.value, nv)

    def profile(self, on: bool = True):
        """Record CUDA events around every stage (Logger::recordSection)."""
        _check(lib().bvhcd_profile_enable(self._h, int(on)), "profile enable")

    def stage_times(self, reset: bool = False) -> dict:
        ms = np.zeros(len(STAGES), np.float64)
        calls = np.zeros(len(STAGES), np.int64)
        _check(lib().bvhcd_profile_read(self._h, ms.ctypes.data, calls.ctypes.data, int(reset)),
               "profile read")
        return {k: (float(ms[i]), int(calls[i])) for i, k in enumerate(STAGES)}

    def sizes(self):
        a, b, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _check(lib().bvhcd_bvh_sizes(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "sizes")
        return a.value, b.value, c.value

    def opt_tag(self) -> int:
        t = ctypes.c_int32()
        _check(lib().bvhcd_bvh_opt_tag(self._h, ctypes.byref(t)), "opt tag")
        return t.value

    def set_scenes(self, tri_offsets):
        """Batched scenes: scene s owns triangles [tri_offsets[s], tri_offsets[s+1])
        of every scene passed to maintain; each gets its own tree and no pair
        crosses scenes (bvhcd_bvh_set_scenes)."""
        off = np.ascontiguousarray(tri_offsets, dtype=np.int32)
        _check(lib().bvhcd_bvh_set_scenes(self._h, off.size - 1, off.ctypes.data), "set scenes")
        self._offsets = off

    def request_restructure(self, roots, stream=None):
        """Mark subtrees (DFS ids) as degraded; the next maintain restructures."""
        r = np.ascontiguousarray(roots, dtype=np.int32)
        _check(lib().bvhcd_bvh_request_restructure(self._h, r.ctypes.data, r.size, _stream_ptr(stream)),
               "request restructure")

    def export(self, stream=None):
        T, _, I = self.sizes()
        inode = np.zeros((max(T - 1, 1), 6), np.int32)
        ibox = np.zeros((max(T - 1, 1), 6), np.float32)
        leaf = np.zeros((max(T, 1), 4), np.int32)
        lbox = np.zeros((max(T, 1), 6), np.float32)
        lca = np.zeros(T + 1, np.int32)
        codes = np.zeros(max(T, 1), np.uint32)
        primmap = np.zeros(max(T, 1), np.int32)
        _check(lib().bvhcd_bvh_export(self._h, inode.ctypes.data, ibox.ctypes.data, leaf.ctypes.data,
                                      lbox.ctypes.data, lca.ctypes.data, codes.ctypes.data,
                                      primmap.ctypes.data, _stream_ptr(stream)), "bvh export")
        return dict(inode=inode[:I], ibox=ibox[:I], leaf=leaf[:T], lbox=lbox[:T], lca=lca,
                    codes=codes[:T], primmap=primmap[:T])


class BvttFront:
    """BvttFrontLooseIntra over a borrowed LBvh: maintain(op) per frame.
    With rigid= another LBvh, BvttFrontLooseInter: the rigid BVH's triangles
    traverse `bvh` (the deformable one); pairs are (deformable id, rigid id)."""

    def __init__(self, bvh: LBvh, int_front_capacity: int = 2_300_000,
                 ext_front_capacity: int = 2_300_000, pair_capacity: int = 1_600_000,
                 cull_adjacent: bool = True, narrow_phase: bool = True, auto_grow: int = 0,
                 precision: int = 0, rigid: "LBvh" = None):
        """auto_grow: 0 off, 1 (or True) grow and replay in the same call
        (synchronises every maintain), 2 deferred (no synchronisation; a later
        maintain grows and regenerates)."""
        cfg = FrontConfig(int(int_front_capacity), int(ext_front_capacity), int(pair_capacity),
                          int(cull_adjacent), int(narrow_phase), int(auto_grow), int(precision))
        h = ctypes.c_void_p()
        if rigid is None:
            _check(lib().bvhcd_front_create(bvh.handle, ctypes.byref(cfg), ctypes.byref(h)), "front create")
        else:
            _check(lib().bvhcd_front_create_inter(bvh.handle, rigid.handle, ctypes.byref(cfg), ctypes.byref(h)),
                   "inter front create")
        self._h = h
        self._bvh = bvh
        self._rigid = rigid

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().bvhcd_front_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def maintain(self, op: int, stream=None):
        _check(lib().bvhcd_front_maintain(self._h, int(op), _stream_ptr(stream)), "front maintain")

    def stats(self, stream=None) -> dict:
        st = FrontStats()
        _check(lib().bvhcd_front_stats_get(self._h, ctypes.byref(st), _stream_ptr(stream)), "stats")
        return st.as_dict()

    def pairs(self, narrow: bool = False, stream=None) -> np.ndarray:
        """Broad-phase pairs (applyCpResults) or intersecting pairs, original ids."""
        n = ctypes.c_int64()
        st = lib().bvhcd_front_pairs(self._h, int(narrow), None, 0, ctypes.byref(n), 0, _stream_ptr(stream))
        if st not in (0, 3):
            _check(st, "pairs")
        out = np.zeros((max(n.value, 1), 2), np.int32)
        st = lib().bvhcd_front_pairs(self._h, int(narrow), out.ctypes.data, n.value, ctypes.byref(n), 0,
                                     _stream_ptr(stream))
        _check(st, "pairs")
        return out[:n.value]

    def export(self, which: int, stream=None) -> np.ndarray:
        n = ctypes.c_int64()
        st = lib().bvhcd_front_export(self._h, int(which), None, 0, ctypes.byref(n), _stream_ptr(stream))
        if st not in (0, 3):
            _check(st, "front export")
        out = np.zeros((max(n.value, 1), 2), np.int32)
        _check(lib().bvhcd_front_export(self._h, int(which), out.ctypes.data, n.value, ctypes.byref(n),
                                        _stream_ptr(stream)), "front export")
        return out[:n.value]

    def pairs_async(self, dst: "HostPairs", narrow: bool = False, stream=None):
        """Enqueues the pairs' copy into `dst` (bvhcd_front_pairs_async); no
        synchronisation."""
        _check(lib().bvhcd_front_pairs_async(self._h, int(narrow), ctypes.c_void_p(dst.pairs_ptr), dst.cap,
                                             ctypes.c_void_p(dst.count_ptr), _stream_ptr(stream)), "pairs async")

    def proximity(self, thickness: float, pos=None, stream=None) -> np.ndarray:
        """Vertex-face and edge-edge proximities of the broad pairs within
        `thickness` (bvhcd_front_proximity), a structured array of PROX_DTYPE
        records ordered by pair.  pos: CUDA tensor of positions, or None for
        the BVH's own."""
        ptr = None
        if pos is not None:
            import torch
            assert isinstance(pos, torch.Tensor) and pos.is_cuda and pos.dtype == torch.float32
            pos = pos.contiguous()
            ptr = pos.data_ptr()
        n = ctypes.c_int64()
        st = lib().bvhcd_front_proximity(self._h, ptr, float(thickness), None, 0, ctypes.byref(n), 0,
                                         _stream_ptr(stream))
        if st not in (0, 3):
            _check(st, "proximity")
        out = np.zeros(max(n.value, 1), dtype=PROX_DTYPE)
        _check(lib().bvhcd_front_proximity(self._h, ptr, float(thickness), out.ctypes.data, n.value, ctypes.byref(n),
                                           0, _stream_ptr(stream)), "proximity")
        return out[:n.value]

    def contacts(self, which: int = 0, stream=None):
        """which 0: (n, 4) contact midpoint xyz + segment length per hit (order
        of pairs(narrow=True)); 1: (n, 4) with the distance in column 3 per
        broad pair (order of pairs()).  Returns (array, items computed in FP64)."""
        n, fl = ctypes.c_int64(), ctypes.c_int64()
        st = lib().bvhcd_front_contacts(self._h, int(which), None, 0, ctypes.byref(n), ctypes.byref(fl), 0,
                                        _stream_ptr(stream))
        if st not in (0, 3):
            _check(st, "contacts")
        out = np.zeros((max(n.value, 1), 4), np.float32)
        _check(lib().bvhcd_front_contacts(self._h, int(which), out.ctypes.data, n.value, ctypes.byref(n),
                                          ctypes.byref(fl), 0, _stream_ptr(stream)), "contacts")
        return out[:n.value], int(fl.value)

    def contacts64(self, which: int = 0, stream=None) -> np.ndarray:
        """contacts() computed and returned in FP64: (n, 4) float64."""
        n = ctypes.c_int64()
        st = lib().bvhcd_front_contacts64(self._h, int(which), None, 0, ctypes.byref(n), 0, _stream_ptr(stream))
        if st not in (0, 3):
            _check(st, "contacts64")
        out = np.zeros((max(n.value, 1), 4), np.float64)
        _check(lib().bvhcd_front_contacts64(self._h, int(which), out.ctypes.data, n.value, ctypes.byref(n), 0,
                                            _stream_ptr(stream)), "contacts64")
        return out[:n.value]

    def shapes(self) -> dict:
        """Launch shape per front stage: {stage: (entries per thread step, threads per block)}."""
        sh = LaunchShapes()
        _check(lib().bvhcd_front_get_shapes(self._h, ctypes.byref(sh)), "get shapes")
        return sh.as_dict()

    def set_shapes(self, shapes: dict):
        sh = LaunchShapes()
        cur = self.shapes()
        cur.update(shapes)
        for i, k in enumerate(SHAPE_STAGES):
            sh.unroll[i], sh.block[i] = cur[k]
        _check(lib().bvhcd_front_set_shapes(self._h, ctypes.byref(sh)), "set shapes")

    def autotune(self, repeats: int = 3, stream=None):
        """Times every candidate launch shape of every front stage on the
        current front and keeps the fastest (bvhcd_front_autotune).  Returns
        ({stage: shape}, {stage: best mean ms per run})."""
        sh = LaunchShapes()
        best = np.zeros(6, np.float64)
        _check(lib().bvhcd_front_autotune(self._h, int(repeats), ctypes.byref(sh), best.ctypes.data,
                                          _stream_ptr(stream)), "autotune")
        return sh.as_dict(), {k: float(best[i]) for i, k in enumerate(SHAPE_STAGES)}

    def device_results(self):
        hits, counts = ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib().bvhcd_front_device_results(self._h, ctypes.byref(hits), ctypes.byref(counts)),
               "device results")
        return hits.value, counts.value


class HostPairs:
    """Mapped pinned host memory for `cap` pairs and their count, the target
    of BvttFront.pairs_async (bvhcd_host_alloc)."""

    def __init__(self, cap: int):
        self.cap = int(cap)
        p = ctypes.c_void_p()
        _check(lib().bvhcd_host_alloc(8 * self.cap + 64, ctypes.byref(p)), "host alloc")
        self._p = p
        buf = (ctypes.c_char * (8 * self.cap + 64)).from_address(p.value)
        self._count = np.frombuffer(buf, dtype=np.int64, count=1, offset=0)
        self._pairs = np.frombuffer(buf, dtype=np.int32, count=2 * self.cap, offset=64).reshape(-1, 2)

    @property
    def count_ptr(self):
        return self._p.value

    @property
    def pairs_ptr(self):
        return self._p.value + 64

    def read(self) -> np.ndarray:
        """The pairs written by the last completed pairs_async (the caller
        synchronises first)."""
        return self._pairs[:min(int(self._count[0]), self.cap)].copy()

    @property
    def count(self) -> int:
        return int(self._count[0])

    def close(self):
        if self._p:
            lib().bvhcd_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_obj(path: str):
    """(positions V x 3 float32, faces T x 3 int32) of a Wavefront OBJ file
    (bvhcd_obj_read: polygons fan-triangulated, vertex ids as the file
    shares them)."""
    V, T = ctypes.c_int32(), ctypes.c_int32()
    p = os.fsencode(path)
    _check(lib().bvhcd_obj_read(p, None, 0, None, 0, ctypes.byref(V), ctypes.byref(T)), f"read {path}")
    pos = np.zeros((max(V.value, 1), 3), np.float32)
    faces = np.zeros((max(T.value, 1), 3), np.int32)
    _check(lib().bvhcd_obj_read(p, pos.ctypes.data, V.value, faces.ctypes.data, T.value, ctypes.byref(V),
                                ctypes.byref(T)), f"read {path}")
    return pos[:V.value], faces[:T.value]


def obj_frames(pattern: str, start: int, count: int):
    """The frames of a benchmark sequence, one OBJ file per frame named by a
    printf pattern (CDBenchmarkSettings::file_name: pattern % frame for
    frames start .. start + count - 1); yields (positions, faces)."""
    for f in range(start, start + count):
        yield load_obj(pattern % f)


def frame(bvh: LBvh, front: BvttFront, f: int, start: int, pos, faces, stream=None, faces_static=False):
    """One frame of the reference app loop (CudaProjectApp.cpp:49-52)."""
    sc, keep = _scene(pos, faces, faces_static)
    _check(lib().bvhcd_frame(bvh.handle, front.handle, int(f), int(start), ctypes.byref(sc),
                             _stream_ptr(stream)), "frame")
    bvh._keep = keep


def frame_graph(bvh: LBvh, front: BvttFront, pos, faces, bvh_op: int, front_op: int, stream=None):
    """One frame through bvhcd_frame_graph: captured as a CUDA graph on first
    use of its key, replayed afterwards.  pos / faces are CUDA tensors whose
    storage stays the same from call to call (write each frame's positions
    into `pos` in place)."""
    sc, keep = _scene(pos, faces, True)
    _check(lib().bvhcd_frame_graph(bvh.handle, front.handle, ctypes.byref(sc), int(bvh_op), int(front_op),
                                   _stream_ptr(stream)), "frame graph")
    bvh._keep = keep


def copy_state(dst_bvh: LBvh, src_bvh: LBvh, dst_front: "BvttFront" = None, src_front: "BvttFront" = None,
               stream=None):
    """dst becomes a copy of src (bvhcd_bvh_copy_state / bvhcd_front_copy_state)."""
    _check(lib().bvhcd_bvh_copy_state(dst_bvh.handle, src_bvh.handle, _stream_ptr(stream)), "bvh copy")
    if dst_front is not None:
        _check(lib().bvhcd_front_copy_state(dst_front.handle, src_front.handle, _stream_ptr(stream)), "front copy")
    dst_bvh._keep = src_bvh._keep


def _dev_ptr(t):
    import torch
    assert isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()
    return ctypes.c_void_p(t.data_ptr())


class Learner:
    """The learned scheduler over a BVH (enable_restr) and its front
    (bvhcd_learner_*, bvhcd_mlp_*)."""

    def __init__(self, bvh: LBvh, front: BvttFront, max_subtree_leaves: int = 512):
        h = ctypes.c_void_p()
        _check(lib().bvhcd_learner_create(bvh.handle, front.handle, int(max_subtree_leaves), ctypes.byref(h)),
               "learner create")
        self._h = h
        self._bvh, self._front = bvh, front

    def close(self):
        if self._h:
            lib().bvhcd_learner_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_decide_every(self, frames: int):
        _check(lib().bvhcd_learner_set_decide_every(self._h, int(frames)), "decide every")

    def set_front_cycle(self, frames: int):
        """0: keep the front between decisions; c: the reference's front cycle of c frames."""
        _check(lib().bvhcd_learner_set_front_cycle(self._h, int(frames)), "front cycle")

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == MLP_PARAMS
        _check(lib().bvhcd_learner_set_params(self._h, p.ctypes.data), "set params")

    def params(self) -> np.ndarray:
        p = np.zeros(MLP_PARAMS, np.float32)
        _check(lib().bvhcd_learner_get_params(self._h, p.ctypes.data), "get params")
        return p

    def frame(self, pos, faces, frame: int, stream=None):
        sc, keep = _scene(pos, faces, True)
        tag, fop = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().bvhcd_learner_frame(self._h, ctypes.byref(sc), int(frame), ctypes.byref(tag),
                                         ctypes.byref(fop), _stream_ptr(stream)), "learner frame")
        self._bvh._keep = keep
        return tag.value, fop.value

    def observe(self, tree_changed: bool, generated: bool, stream=None):
        _check(lib().bvhcd_learner_observe(self._h, int(tree_changed), int(generated), _stream_ptr(stream)),
               "observe")

    def cut(self, stream=None) -> np.ndarray:
        n = ctypes.c_int32()
        _check(lib().bvhcd_learner_cut(self._h, None, 0, ctypes.byref(n), _stream_ptr(stream)), "cut")
        out = np.zeros(max(n.value, 1), np.int32)
        _check(lib().bvhcd_learner_cut(self._h, out.ctypes.data, out.size, ctypes.byref(n), _stream_ptr(stream)),
               "cut")
        return out[:n.value]

    def features(self, stream=None) -> np.ndarray:
        n = ctypes.c_int32()
        _check(lib().bvhcd_learner_features(self._h, None, 0, ctypes.byref(n), _stream_ptr(stream)), "features")
        X = np.zeros((max(n.value, 1), 16), np.float32)
        _check(lib().bvhcd_learner_features(self._h, X.ctypes.data, X.shape[0], ctypes.byref(n),
                                            _stream_ptr(stream)), "features")
        return X[:n.value]

    def work(self, front: BvttFront, n: int, stream=None) -> np.ndarray:
        out = np.zeros(max(n, 1), np.int64)
        _check(lib().bvhcd_learner_work(self._h, front.handle, out.ctypes.data, out.size, _stream_ptr(stream)),
               "work")
        return out[:n]

    def gradient(self, X, y, class_weight=(1.0, 1.0, 1.0), stream=None):
        """X: (n, 16) float32 CUDA tensor, y: (n,) int32 CUDA tensor."""
        cw = np.ascontiguousarray(class_weight, dtype=np.float32)
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        _check(lib().bvhcd_mlp_gradient(self._h, _dev_ptr(X), _dev_ptr(y), int(X.shape[0]), cw.ctypes.data,
                                        g.ctypes.data, loss.ctypes.data, _stream_ptr(stream)), "mlp gradient")
        return g, float(loss[0])

    def train(self, X, y, class_weight=(1.0, 1.0, 1.0), epochs=10, batch=4096, lr=1e-3, seed=0, stream=None):
        cw = np.ascontiguousarray(class_weight, dtype=np.float32)
        loss = np.zeros(1, np.float32)
        _check(lib().bvhcd_mlp_train(self._h, _dev_ptr(X), _dev_ptr(y), int(X.shape[0]), cw.ctypes.data,
                                     int(epochs), int(batch), float(lr), int(seed), loss.ctypes.data,
                                     _stream_ptr(stream)), "mlp train")
        return float(loss[0])

    def predict(self, X, stream=None):
        import torch
        n = int(X.shape[0])
        logits = torch.empty((max(n, 1), 3), dtype=torch.float32, device=X.device)
        vote = torch.empty(max(n, 1), dtype=torch.int32, device=X.device)
        _check(lib().bvhcd_mlp_predict(self._h, _dev_ptr(X), n, _dev_ptr(logits), _dev_ptr(vote),
                                       _stream_ptr(stream)), "mlp predict")
        torch.cuda.synchronize()
        return logits[:n].cpu().numpy(), vote[:n].cpu().numpy()
