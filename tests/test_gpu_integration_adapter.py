"""The reference-side binding that INTEGRATION.md shows, compiled and run.

tests/cpp/Makefile extracts the adapter classes (LBvhB200, BvttFrontB200,
LBvhRigidB200, BvttFrontInterB200) from INTEGRATION.md, compiles them with
nvcc against the reference's own headers (Mine/world/Scene.h,
Mine/setting/BvhSettings.h and the module headers that declare the
maintenance enums) and links them with libbvhcd.so, together with a frame
loop that is the reference app's (Mine/Frameworks/CudaProject/
CudaProjectApp.cpp:49-52) driven by the reference's own BenchmarkLogic
(maintainScheme / next, Mine/system/Logic/BenchmarkLogic.hpp:16-156).  This
test runs that binary on the 20-frame 128x128 folding cloth and holds every
frame to the fixture the reference pipeline itself produced
(tests/golden/ref_cloth_fold_128.json): the schedule, the BVH's opt tag, the
front sizes and pair counts inspectResults prints, and the SHA-256 of the
broad pair set applyCpResults returns.  The binary is built where the
reference tree exists (__graft_entry__.build()); on a machine without it the
prebuilt binary is used."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from test_reference_golden import _inputs, _load, comparable, digest

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "tests", "cpp", "_build", "adapter_c1")
FIXTURE = os.path.join(ROOT, "tests", "golden", "ref_cloth_fold_128.json")
LINE = re.compile(r"frame (\d+) bvh_op (\d+) front_op (\d+) opt_tag (\d+) front \((\d+), (\d+)\) cpNum (\d+) "
                  r"actualCpNum (\d+)")


def test_integration_adapters_match_reference_pipeline(cuda, lib_built, oracle, tmp_path):
    assert os.path.exists(BIN), "tests/cpp/_build/adapter_c1 is not built (make -C tests/cpp with the reference tree)"
    fx = _load(FIXTURE)
    faces, frames = _inputs(fx)
    T, V, F = faces.shape[0], frames[0].shape[0], len(frames)
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(src, "wb") as f:
        np.array([T, V, F], np.int32).tofile(f)
        np.ascontiguousarray(faces, np.int32).tofile(f)
        np.ascontiguousarray(np.stack(frames), np.float32).tofile(f)
    r = subprocess.run([BIN, str(src), str(dst)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    rows = [tuple(int(x) for x in m.groups()) for m in LINE.finditer(r.stdout)]
    assert len(rows) == F, r.stdout[-2000:]
    raw = np.fromfile(dst, dtype=np.int32)
    pairs, o = [], 0
    for _ in range(F):
        n = int(raw[o])
        pairs.append(raw[o + 1:o + 1 + 2 * n].reshape(-1, 2))
        o += 1 + 2 * n
    assert o == raw.size
    checked = 0
    for e, kind in comparable(fx["frames"], False):
        f = e["frame"]
        _, bop, fop, tag, fi, fe, P, H = rows[f]
        # the schedule the reference's BenchmarkLogic produced is the fixture's
        assert (bop, fop) == (e["bvh_op"], e["front_op"]), f
        if kind == "none":
            continue
        assert tag == e["opt_tag"], f
        if kind != "full":
            continue
        assert (fi, fe, P) == (e["int_front"], e["ext_front"], e["broad_pairs"]), f
        if e["opt_tag"] != 1:
            assert H == e["narrow_hits"], f
        assert digest(oracle.canon_pairs(pairs[f])) == e["pairs_sha256"], f
        checked += 1
    assert checked >= 15
