"""The learned start guess's CPU oracle, checked on its own (no GPU).

The reference has no learned component, so the oracle (oracle/mlp.py) is
pinned by mathematics instead: its analytic gradient against central finite
differences, its BF16 rounding against the C oracle's, its features against a
per-vertex loop, and its subdomain composition against a direct sum.
"""
from __future__ import annotations

import numpy as np
import pytest

import cases
from oracle import mlp as OM
from oracle import oracle as O
from sgmas import synth


def random_params(seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, scale, OM.N_PARAMS)


def test_layout_matches_header():
    import re
    hdr = open(__file__.replace("tests/test_learned_oracle.py", "include/sgmas.h")).read()
    n = int(re.search(r"#define SGMAS_MLP_PARAMS (\d+)", hdr).group(1))
    assert n == OM.N_PARAMS == 16 * 128 + 128 + 128 * 128 + 128 + 128 * 6 + 6


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    P = random_params(1)
    X = rng.normal(size=(32, 16))
    T = rng.normal(size=(32, 3))
    mask = (rng.uniform(size=32) > 0.2).astype(np.float64)
    mask[16:20] = 0.0
    inv_n = 1.0 / mask.sum()
    loss, g = OM.loss_grad(P, X, T, mask, inv_n)
    idx = np.concatenate([rng.choice(OM.N_PARAMS, 60, replace=False),
                          [OM.O_B1, OM.O_W2 + 5, OM.O_B2 + 3, OM.O_W3 + 4, OM.O_B3 + 1, OM.O_B3 + 4]])
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (OM.loss_grad(Pp, X, T, mask, inv_n)[0] - OM.loss_grad(Pm, X, T, mask, inv_n)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_coarse_term_is_a_subdomain_mean():
    rng = np.random.default_rng(2)
    Y = rng.normal(size=(32, 6))
    mask = np.ones(32)
    mask[[3, 17, 18]] = 0
    pred = OM.prediction(Y, mask)
    for r in range(32):
        b = r // 16
        rows = [u for u in range(16 * b, 16 * b + 16) if mask[u] > 0]
        np.testing.assert_allclose(pred[r], Y[r, :3] + Y[rows, 3:6].mean(0), rtol=1e-14)


def test_bf16_rounding_matches_c_oracle():
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(size=4000) * 10.0 ** rng.integers(-8, 8, 4000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.005859375, 65504.0]])
    c = O.bf16_round(x) if hasattr(O, "bf16_round") else None
    mine = OM.bf16(x.astype(np.float32))
    if c is not None:
        np.testing.assert_array_equal(mine.view(np.uint32), np.asarray(c, np.float32).view(np.uint32))
    # ties to even at the BF16 boundary: 1 + 2^-8 is halfway between 1 and 1 + 2^-7
    assert OM.bf16(np.float32(1.0 + 2.0 ** -8)) == np.float32(1.0)
    assert OM.bf16(np.float32(1.0 + 3 * 2.0 ** -8)) == np.float32(1.0 + 2.0 ** -6)
    assert np.all(np.abs(mine - x.astype(np.float32)) <= np.abs(x.astype(np.float32)) * 2.0 ** -8 + 1e-45)


def test_features_match_per_vertex_formula():
    case = cases.build("c1")
    s = case.s
    rng = np.random.default_rng(4)
    prev = rng.normal(size=3 * case.n) * 1e-3
    pairs = np.array([[-(5 + 1), 6, 7, 8], [10, 11, 12, 13], [-(5 + 1), 14, -1, -1]], np.int32)
    X, mask, T, (sc, sb) = OM.features(s.vals, s.rows, s.cols, s.b, case.part_map, case.n, prev=prev,
                                       pairs=pairs, dx=prev)
    A = synth.full_matrix(s).toarray()
    Dk = {v: A[3 * v:3 * v + 3, 3 * v:3 * v + 3] for v in range(case.n)}
    b = s.b.reshape(-1, 3)
    Sk = {v: sum(A[3 * v:3 * v + 3, 3 * j:3 * j + 3] for j in range(case.n)) for v in range(case.n)}
    us = np.array([np.linalg.solve(Sk[v], b[v]) for v in range(case.n)])
    ys = np.array([np.linalg.solve(Dk[v], b[v]) for v in range(case.n)])
    assert abs(sc - np.sqrt((us ** 2).sum() / case.n)) <= 1e-10 * sc
    counts = {5: 2, 6: 1, 7: 1, 8: 1, 10: 1, 11: 1, 12: 1, 13: 1, 14: 1}
    for slot in rng.choice(len(case.part_map), 50, replace=False):
        v = case.part_map[slot]
        if v < 0:
            assert mask[slot] == 0 and not X[slot].any()
            continue
        D, t = Dk[v], np.trace(Dk[v]) / 3
        f = np.concatenate([us[v] / sc, prev.reshape(-1, 3)[v] / sc, ys[v] / sc, np.diag(D) / t - 1,
                            [D[0, 1] / t, D[0, 2] / t, D[1, 2] / t], [min(counts.get(v, 0), 32) / 8]])
        np.testing.assert_allclose(X[slot], f.astype(np.float32), rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(T[slot], ((prev.reshape(-1, 3)[v] - us[v]) / sc).astype(np.float32),
                                   rtol=1e-6, atol=1e-6)


def test_lumped_step_is_exact_for_translations():
    """Elastic terms are translation invariant: for b = A t of a rigid
    translation t of a mesh without anchors or contact regularisation,
    u = S^-1 b = t at every vertex."""
    case = cases.build("c1")
    s = case.s
    A = synth.full_matrix(s)
    t = np.tile([1e-3, -2e-3, 5e-4], case.n)
    u, _ = OM.lumped_step(s.vals, s.rows, s.cols, A @ t, case.n)
    np.testing.assert_allclose(u.ravel(), t, rtol=1e-9)


def test_compose_places_vertices_by_slot():
    case = cases.build("c1")
    rng = np.random.default_rng(5)
    Y = rng.normal(size=(len(case.part_map), 6))
    u = rng.normal(size=(case.n, 3))
    x0 = OM.compose(Y, case.part_map, case.n, 2.0, case.n + 3, u, fem_offset=3)
    mask = (case.part_map >= 0).astype(float)
    pred = OM.prediction(Y, mask)
    v = case.part_map[7]
    assert v >= 0
    np.testing.assert_allclose(x0.reshape(-1, 3)[3 + v], u[v] + 2.0 * pred[7])
    assert not x0[:9].any()


def test_bf16_inference_tracks_fp64_forward():
    rng = np.random.default_rng(6)
    P = random_params(6, 0.1)
    X = rng.normal(size=(64, 16)).astype(np.float32)
    y64 = OM.forward(P, X)
    y16 = OM.infer_bf16(P, X)
    assert np.max(np.abs(y16 - y64)) <= 0.05 * np.max(np.abs(y64)) + 1e-3
