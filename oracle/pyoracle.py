"""ctypes front end of the CPU oracle (liborc.so) and of oracle/_ref.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product library.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

BVH_BUILD, BVH_REFIT, BVH_UPDATE = 0, 1, 2
FRONT_PURE_BVH_CD, FRONT_GENERATE, FRONT_UPDATE, FRONT_REORDER, FRONT_KEEP, FRONT_RESTRUCTURE = range(6)

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build():
    """Compile liborc.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liborc.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_pipe_create.restype = ctypes.c_void_p
        L.orc_pipe_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_pipe_destroy.argtypes = [ctypes.c_void_p]
        L.orc_pipe_frame.restype = ctypes.c_int
        L.orc_pipe_frame.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, ctypes.c_int, _f32p,
                                     ctypes.c_int, ctypes.c_int]
        L.orc_pipe_info.argtypes = [ctypes.c_void_p, _i64p]
        L.orc_pipe_pairs.restype = ctypes.c_int64
        L.orc_pipe_pairs.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64]
        L.orc_pipe_front.restype = ctypes.c_int64
        L.orc_pipe_front.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64]
        L.orc_pipe_tree.restype = ctypes.c_int
        L.orc_pipe_tree.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 7
        L.orc_pipe_log.restype = ctypes.c_int
        L.orc_pipe_log.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_pipe_mark_restructure.argtypes = [ctypes.c_void_p, _i32p, ctypes.c_int]
        L.orc_pipe_set_reference_permutation.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_precision_pairs.argtypes = [ctypes.c_int64, _i32p, _i32p, _f32p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p]
        L.orc_proximity.restype = ctypes.c_int64
        L.orc_proximity.argtypes = [ctypes.c_int64, _i32p, _i32p, _f32p, _i32p, _f32p, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_void_p, ctypes.c_int64]
        L.orc_tritri_sat64.restype = ctypes.c_int
        L.orc_tritri_sat64.argtypes = [_f32p, _f32p]
        L.orc_contact64.restype = ctypes.c_int
        L.orc_contact64.argtypes = [_f32p, _f32p, ctypes.c_void_p]
        L.orc_tri_distance64.restype = ctypes.c_double
        L.orc_tri_distance64.argtypes = [_f32p, _f32p]
        L.orc_scene_box.argtypes = [ctypes.c_int, _i32p, _f32p, _f32p]
        L.orc_morton_codes.argtypes = [ctypes.c_int, _i32p, _f32p, _f32p, _u32p]
        L.orc_brute_pairs.restype = ctypes.c_int64
        L.orc_brute_pairs.argtypes = [ctypes.c_int, _i32p, _f32p, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_int64]
        L.orc_tritri_sat32.restype = ctypes.c_int
        L.orc_tritri_sat32.argtypes = [_f32p, _f32p]
        L.orc_tritri_exact.restype = ctypes.c_int
        L.orc_tritri_exact.argtypes = [_f32p, _f32p]
        L.orc_narrow_sat32.argtypes = [ctypes.c_int64, _i32p, _i32p, _f32p, _u8p]
        L.orc_narrow_exact.argtypes = [ctypes.c_int64, _i32p, _i32p, _f32p, _u8p]
        L.orc_schedule.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_int)]
        _LIB = L
    return _LIB


def ref_lib():
    """oracle/_ref/libref_tritri.so (the reference's own predicate), or None."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libref_tritri.so")
        if not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        R.ref_tritri.restype = ctypes.c_int
        R.ref_tritri.argtypes = [_f32p, _f32p]
        R.ref_narrow.argtypes = [ctypes.c_longlong, _i32p, _i32p, _f32p, _u8p]
        _REF = R
    return _REF


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def schedule(frame: int, start: int = 0):
    b, f = ctypes.c_int(), ctypes.c_int()
    lib().orc_schedule(frame, start, ctypes.byref(b), ctypes.byref(f))
    return b.value, f.value


def canon_pairs(p: np.ndarray) -> np.ndarray:
    """Unordered pairs as sorted (min, max) rows, lexicographically sorted."""
    p = np.asarray(p, dtype=np.int64).reshape(-1, 2)
    if p.size == 0:
        return np.zeros((0, 2), dtype=np.int64)
    q = np.sort(p, axis=1)
    order = np.lexsort((q[:, 1], q[:, 0]))
    return q[order]


def brute_pairs(faces: np.ndarray, pos: np.ndarray, cull: bool) -> np.ndarray:
    L = lib()
    faces = np.ascontiguousarray(faces, dtype=np.int32)
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    T = faces.shape[0]
    n = L.orc_brute_pairs(T, faces, pos, int(cull), None, 0)
    out = np.empty((max(n, 1), 2), dtype=np.int32)
    L.orc_brute_pairs(T, faces, pos, int(cull), out.ctypes.data, n)
    return canon_pairs(out[:n])


def narrow(pairs, faces, pos, exact=False):
    L = lib()
    pairs = np.ascontiguousarray(np.asarray(pairs).reshape(-1, 2), dtype=np.int32)
    hit = np.zeros(pairs.shape[0], dtype=np.uint8)
    fn = L.orc_narrow_exact if exact else L.orc_narrow_sat32
    fn(pairs.shape[0], pairs, np.ascontiguousarray(faces, dtype=np.int32),
       np.ascontiguousarray(pos, dtype=np.float32), hit)
    return hit


def _joined(fa, va, fb, vb):
    fa = np.asarray(fa, dtype=np.int32).reshape(-1, 3)
    fb = np.asarray(fb, dtype=np.int32).reshape(-1, 3)
    va = np.asarray(va, dtype=np.float32).reshape(-1, 3)
    vb = np.asarray(vb, dtype=np.float32).reshape(-1, 3)
    return np.concatenate([fa, fb + va.shape[0]]), np.concatenate([va, vb])


def brute_inter_pairs(fa, va, fb, vb) -> np.ndarray:
    """Every (a, b), a a triangle of mesh A and b one of mesh B, whose FP32
    AABBs overlap (touching counts), as sorted rows.  This is the pair set of
    an inter front over a deformable mesh A and an obstacle mesh B: the
    obstacle's primitives traverse A's BVH from the root and report each
    overlapping leaf, with no adjacency culling between the two meshes
    (genLooseInterFrontsWithLog, Mine/collision/bvtt_front/
    BvttFrontGenerateKernels.cu:92-124; pureBvhInterCD, BvhCDKernels.cu:51-76).
    Sweep and prune over the two meshes joined, keeping the pairs across."""
    faces, pos = _joined(fa, va, fb, vb)
    ta = np.asarray(fa).reshape(-1, 3).shape[0]
    p = brute_pairs(faces, pos, False)
    q = p[(p[:, 0] < ta) & (p[:, 1] >= ta)].copy()
    q[:, 1] -= ta
    return q


def inter_narrow(pairs, fa, va, fb, vb) -> np.ndarray:
    """FP32 SAT hit mask over (a, b) pairs of an inter front, the obstacle's
    triangle b as the first operand, as the inter front's narrow phase calls
    the test (the traversing primitive first)."""
    faces, pos = _joined(fa, va, fb, vb)
    ta = np.asarray(fa).reshape(-1, 3).shape[0]
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    q = np.stack([pairs[:, 1] + ta, pairs[:, 0]], axis=1)
    return narrow(q, faces, pos)


PROX_DTYPE = np.dtype([("pair", np.int32), ("kind", np.int32), ("fa", np.int32), ("fb", np.int32),
                       ("dist", np.float64), ("n", np.float64, 3), ("w", np.float64, 4)], align=True)


def proximity(pairs, fa, va, fb=None, vb=None, h=0.0):
    """Proximity records of a pair list (first triangle from (fa, va), second
    from (fb, vb); one mesh when fb is None), in the kernel's order."""
    same = fb is None
    if same:
        fb, vb = fa, va
    pairs = np.ascontiguousarray(np.asarray(pairs).reshape(-1, 2), dtype=np.int32)
    args = [np.ascontiguousarray(fa, dtype=np.int32), np.ascontiguousarray(va, dtype=np.float32),
            np.ascontiguousarray(fb, dtype=np.int32), np.ascontiguousarray(vb, dtype=np.float32)]
    L = lib()
    n = L.orc_proximity(pairs.shape[0], pairs, *args, int(same), float(h), None, 0)
    out = np.zeros(max(n, 1), dtype=PROX_DTYPE)
    L.orc_proximity(pairs.shape[0], pairs, *args, int(same), float(h), out.ctypes.data, n)
    return out[:n]


def ref_narrow(pairs, faces, pos):
    R = ref_lib()
    if R is None:
        return None
    pairs = np.ascontiguousarray(np.asarray(pairs).reshape(-1, 2), dtype=np.int32)
    hit = np.zeros(pairs.shape[0], dtype=np.uint8)
    R.ref_narrow(pairs.shape[0], pairs, np.ascontiguousarray(faces, dtype=np.int32),
                 np.ascontiguousarray(pos, dtype=np.float32), hit)
    return hit


class Pipeline:
    """CPU restatement of LBvhFixedDeformable + BvttFrontLooseIntra."""

    def __init__(self, restructure=True, cull_adjacent=True, narrow=True,
                 reference_permutation=False):
        """reference_permutation: restructure with the reference's own
        primitive-map update run in thread order (test pinning only; see
        orc_pipe_set_reference_permutation)."""
        self._p = ctypes.c_void_p(lib().orc_pipe_create(int(restructure), int(cull_adjacent),
                                                        int(narrow)))
        if reference_permutation:
            lib().orc_pipe_set_reference_permutation(self._p, 1)

    def close(self):
        if self._p:
            lib().orc_pipe_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def frame(self, faces, pos, bvh_op, front_op):
        self._faces = np.ascontiguousarray(faces, dtype=np.int32)
        self._pos = np.ascontiguousarray(pos, dtype=np.float32)
        rc = lib().orc_pipe_frame(self._p, self._faces.shape[0], self._faces,
                                  self._pos.shape[0], self._pos, int(bvh_op), int(front_op))
        if rc != 0:
            raise RuntimeError("oracle frame failed")

    def mark_restructure(self, roots):
        r = np.ascontiguousarray(roots, dtype=np.int32)
        lib().orc_pipe_mark_restructure(self._p, r, r.size)

    def info(self):
        a = np.zeros(16, dtype=np.int64)
        lib().orc_pipe_info(self._p, a)
        keys = ["T", "F_int", "F_ext", "P", "H", "opt_tag", "updated", "num_rt_subtree",
                "num_rt_int", "front_op", "narrow_ran"]
        return {k: int(a[i]) for i, k in enumerate(keys)}

    def pairs(self, narrow=False):
        L = lib()
        n = L.orc_pipe_pairs(self._p, int(narrow), None, 0)
        out = np.empty((max(n, 1), 2), dtype=np.int32)
        L.orc_pipe_pairs(self._p, int(narrow), out.ctypes.data, n)
        return out[:n]

    def front(self, which):
        L = lib()
        n = L.orc_pipe_front(self._p, which, None, 0)
        out = np.empty((max(n, 1), 2), dtype=np.int32)
        L.orc_pipe_front(self._p, which, out.ctypes.data, n)
        return out[:n]

    def tree(self):
        T = self.info()["T"]
        inode = np.zeros((max(T - 1, 1), 6), dtype=np.int32)
        ibox = np.zeros((max(T - 1, 1), 6), dtype=np.float32)
        leaf = np.zeros((max(T, 1), 4), dtype=np.int32)
        lbox = np.zeros((max(T, 1), 6), dtype=np.float32)
        lca = np.zeros(T + 1, dtype=np.int32)
        codes = np.zeros(max(T, 1), dtype=np.uint32)
        primmap = np.zeros(max(T, 1), dtype=np.int32)
        lib().orc_pipe_tree(self._p, inode.ctypes.data, ibox.ctypes.data, leaf.ctypes.data,
                            lbox.ctypes.data, lca.ctypes.data, codes.ctypes.data,
                            primmap.ctypes.data)
        return dict(inode=inode[:max(T - 1, 0)], ibox=ibox[:max(T - 1, 0)], leaf=leaf[:T],
                    lbox=lbox[:T], lca=lca, codes=codes[:T], primmap=primmap[:T])

    def log(self):
        T = self.info()["T"]
        arrs = [np.zeros(T + 1, dtype=np.uint32) for _ in range(4)]
        lib().orc_pipe_log(self._p, *[a.ctypes.data for a in arrs])
        return dict(zip(["intcnt", "extcnt", "intbeg", "extbeg"], arrs))


def precision_pairs(pairs, faces, verts):
    """FP64 references of the precision mode over a pair list of original
    triangle ids: (FP64 SAT hit mask, contact midpoint + segment length per
    pair -- NaN where not a hit or coplanar, distance per pair -- 0 for hits)."""
    pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    faces = np.ascontiguousarray(faces, dtype=np.int32)
    verts = np.ascontiguousarray(verts, dtype=np.float32)
    n = pairs.shape[0]
    hit = np.zeros(max(n, 1), np.uint8)
    con = np.zeros((max(n, 1), 4), np.float64)
    dist = np.zeros(max(n, 1), np.float64)
    lib().orc_precision_pairs(n, pairs, faces, verts, hit.ctypes.data, con.ctypes.data, dist.ctypes.data)
    return hit[:n].astype(bool), con[:n], dist[:n]


def tritri_sat64(p9, q9):
    return bool(lib().orc_tritri_sat64(np.ascontiguousarray(p9, np.float32), np.ascontiguousarray(q9, np.float32)))


def contact64(p9, q9):
    out = np.zeros(4, np.float64)
    st = lib().orc_contact64(np.ascontiguousarray(p9, np.float32), np.ascontiguousarray(q9, np.float32),
                             out.ctypes.data)
    return st, out


def tri_distance64(p9, q9):
    return float(lib().orc_tri_distance64(np.ascontiguousarray(p9, np.float32), np.ascontiguousarray(q9, np.float32)))
