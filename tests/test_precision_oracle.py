"""The precision mode's FP64 references (oracle/precision_oracle.c) on cases
with known answers, and against the exact predicate on random pairs."""
import numpy as np


def _tri(*v):
    return np.array(v, dtype=np.float32)


def test_contact_point_of_crossing_triangles(oracle):
    P = _tri(0, 0, 0, 1, 0, 0, 0, 1, 0)
    Q = _tri(0.2, 0.25, -1, 0.6, 0.25, -1, 0.4, 0.25, 1)     # cuts z = 0 along x in [0.3, 0.5]
    assert oracle.tritri_sat64(P, Q)
    st, c = oracle.contact64(P, Q)
    assert st == 1
    assert np.allclose(c, [0.4, 0.25, 0.0, 0.2], atol=1e-7)
    st, _ = oracle.contact64(P, _tri(0.2, 0.2, 0, 0.6, 0.2, 0, 0.4, 0.4, 0))   # coplanar
    assert st == 2


def test_distances_with_known_values(oracle):
    P = _tri(0, 0, 0, 1, 0, 0, 0, 1, 0)
    R = P.copy()
    R[2::3] = 0.5
    assert not oracle.tritri_sat64(P, R)
    assert abs(oracle.tri_distance64(P, R) - 0.5) < 1e-12
    # an edge-edge closest pair: two skew segments 0.25 apart
    A = _tri(0, 0, 0, 1, 0, 0, 0.5, -1, 0)
    B = _tri(0.5, -0.5, 0.25, 0.5, 0.5, 0.25, 0.5, 0.0, 1.25)
    assert abs(oracle.tri_distance64(A, B) - 0.25) < 1e-12


def test_sat64_agrees_with_exact_predicate(oracle):
    """On random non-degenerate pairs the FP64 SAT and the exact-arithmetic
    predicate agree everywhere."""
    rng = np.random.default_rng(17)
    n = 4000
    P = rng.uniform(0, 1, (n, 3, 3))
    Q = P + rng.normal(0, 0.3, (n, 3, 3))
    verts = np.concatenate([P, Q], axis=1).reshape(-1, 3).astype(np.float32)
    faces = np.arange(6 * n, dtype=np.int32).reshape(-1, 3)
    pairs = np.stack([np.arange(0, 2 * n, 2), np.arange(1, 2 * n, 2)], 1).astype(np.int32)
    exact = oracle.narrow(pairs, faces, verts, exact=True)
    hit, _, _ = oracle.precision_pairs(pairs, faces, verts)
    assert np.array_equal(np.asarray(exact, bool), hit)
    assert 0.1 < hit.mean() < 0.9


def test_precision_pairs_matches_per_pair_calls(oracle):
    import scenes
    faces, frames = scenes.stacked_layers_frames(24, 3, 2, z_noise=0.8)
    pairs = oracle.brute_pairs(faces, frames[1], 1)
    hit, con, dist = oracle.precision_pairs(pairs, faces, frames[1])
    assert hit.any() and (~hit).any()
    v = frames[1]
    for q in range(0, len(pairs), max(1, len(pairs) // 50)):
        a, b = pairs[q]
        P, Q = v[faces[a]].ravel(), v[faces[b]].ravel()
        assert hit[q] == oracle.tritri_sat64(P, Q)
        if hit[q]:
            st, c = oracle.contact64(P, Q)
            assert (st != 1 and np.isnan(con[q, 0])) or np.array_equal(c, con[q])
            assert dist[q] == 0.0
        else:
            assert dist[q] == oracle.tri_distance64(P, Q)
