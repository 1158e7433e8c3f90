"""The learned scheduler on the GPU: its training kernels against the CPU
network (oracle/mlp_oracle.py), and learned frames against the exact pair
sets whatever the network votes."""
import numpy as np
import pytest

import mlp_oracle as m

pytestmark = pytest.mark.gpu


def _learner(lib, T, V, smax=256, caps=(2_000_000, 2_000_000, 1_000_000)):
    bvh = lib.LBvh(T, V, enable_restr=True)
    front = lib.BvttFront(bvh, *caps, cull_adjacent=True, narrow_phase=True)
    return bvh, front, lib.Learner(bvh, front, smax)


def test_gradient_and_forward_match_cpu_network(cuda, lib_built, cloth_c1):
    torch = cuda
    faces, frames = cloth_c1
    bvh, front, lrn = _learner(lib_built, faces.shape[0], frames[0].shape[0])
    rng = np.random.default_rng(5)
    p = rng.normal(0, 0.25, m.N_PARAMS).astype(np.float32)
    lrn.set_params(p)
    assert np.array_equal(lrn.params(), p)
    X = rng.normal(size=(1000, 16)).astype(np.float32)
    y = rng.integers(0, 3, 1000).astype(np.int32)
    cw = (1.0, 3.0, 2.0)
    g, loss = lrn.gradient(torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda(), cw)
    loss_ref, g_ref = m.loss_and_grad(p, X, y, cw, quantize=True)
    assert abs(loss - loss_ref) <= 1e-4 * abs(loss_ref)
    scale = np.abs(g_ref).max()
    assert np.max(np.abs(g - g_ref)) <= 2e-4 * scale, (np.max(np.abs(g - g_ref)), scale)
    logits, vote = lrn.predict(torch.from_numpy(X).cuda())
    z, _ = m.forward(p, X, quantize=True)
    assert np.max(np.abs(logits - z)) <= 1e-4 * max(1.0, np.abs(z).max())
    agree = np.mean(vote == np.argmax(z, axis=1))
    assert agree > 0.999


def test_training_fits_a_rule(cuda, lib_built, cloth_c1):
    """Adam on the GPU learns a rule of the features: class = which of three
    feature sums is largest."""
    torch = cuda
    faces, frames = cloth_c1
    bvh, front, lrn = _learner(lib_built, faces.shape[0], frames[0].shape[0])
    rng = np.random.default_rng(9)
    X = rng.normal(size=(60_000, 16)).astype(np.float32)
    y = np.argmax(np.stack([X[:, 0] + X[:, 1], X[:, 2] - X[:, 3], 0.5 * X[:, 4]], 1), 1).astype(np.int32)
    Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
    _, l0 = lrn.gradient(Xd, yd)
    last = lrn.train(Xd, yd, epochs=8, batch=2048, lr=3e-3, seed=1)
    assert last < 0.3 * l0, (l0, last)
    _, vote = lrn.predict(Xd)
    assert np.mean(vote == y) > 0.95


@pytest.mark.parametrize("bias", [(8.0, 0.0, 0.0), (0.0, 8.0, 0.0), (0.0, 0.0, 8.0), None],
                         ids=["refit", "restructure", "regenerate", "random"])
def test_learned_frames_keep_exact_pairs(cuda, lib_built, oracle, cloth_c1, bias):
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    bvh, front, lrn = _learner(lib_built, T, V)
    lrn.set_decide_every(2)
    lrn.set_front_cycle(6)  # the reference's front cycle between decisions (the default keeps)
    rng = np.random.default_rng(11)
    if bias is None:
        p = rng.normal(0, 0.3, m.N_PARAMS).astype(np.float32)
    else:
        p = np.zeros(m.N_PARAMS, np.float32)
        p[5440:5443] = bias
    lrn.set_params(p)
    ref = oracle.Pipeline(restructure=False, cull_adjacent=True, narrow=True)
    tags = []
    for f in range(14):
        tag, fop = lrn.frame(frames[f], faces, f)
        tags.append((tag, fop))
        ref.frame(faces, frames[f], 0 if f == 0 else 1, 1 if f == 0 else 4)
        assert front.stats()["overflow"] == 0
        got = oracle.canon_pairs(front.pairs())
        assert np.array_equal(got, oracle.canon_pairs(ref.pairs())), (f, tag, fop)
        assert np.array_equal(oracle.canon_pairs(front.pairs(narrow=True)),
                              oracle.canon_pairs(ref.pairs(narrow=True))), f
    if bias == (0.0, 0.0, 8.0):
        # decisions are applied a frame or more after they are queued
        assert sum(fop == lib_built.FRONT_GENERATE for _, fop in tags[1:]) >= 4
    if bias == (0.0, 8.0, 0.0):
        assert any(tag in (1, 2) for tag, _ in tags[1:])    # the marks reached the BVH
    if bias == (8.0, 0.0, 0.0):
        assert all(tag == 0 for tag, _ in tags[1:])
        assert [fop for _, fop in tags[1:7]] == [4, 4, 4, 4, 3, 2]


def test_features_and_work_at_a_build(cuda, lib_built, cloth_c1):
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    bvh, front, lrn = _learner(lib_built, T, V, smax=512)
    lrn.frame(frames[0], faces, 0)
    roots = lrn.cut()
    X = lrn.features()
    assert X.shape == (len(roots), 16) and len(roots) > 30
    inode = bvh.export()["inode"]
    size = inode[roots, 5] - inode[roots, 4] + 1
    assert size.max() <= 512 and size.sum() <= T
    assert np.allclose(X[:, 0], np.log2(size) / 16, atol=1e-6)
    assert np.allclose(X[:, 2], 1.0, atol=1e-5) and np.allclose(X[:, 4], 1.0, atol=1e-6)   # just built
    assert np.allclose(X[:, 5], 0.0) and np.allclose(X[:, 7], 1.0, atol=1e-6)
    w = lrn.work(front, len(roots))
    fi, fe = front.export(0), front.export(1)
    for c in range(0, len(roots), 7):
        r = roots[c]
        x0, x1 = inode[r, 4], inode[r, 5]
        exp = np.sum((fi[:, 1] >= r) & (fi[:, 1] < r + x1 - x0)) + np.sum((fe[:, 1] >= x0) & (fe[:, 1] <= x1))
        assert w[c] == exp, c
