"""CPU tests: the oracle against the reference's golden data and small
independent restatements, and the library's host-side set-up functions
(no GPU needed) against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

import cases
from oracle import oracle as O
from sgmas import synth


# ---------------------------------------------------------------- set-up data
@pytest.mark.parametrize("name", ["cube", "bar", "bunny2"])
def test_golden_partitions_give_monotone_slot_maps(name):
    """setMAS_partition on the reference's METIS partitions (SG/main.cu:47-75):
    parts are contiguous in the sorted meshes, no part exceeds 16 vertices,
    and slots follow vertex order inside every bank."""
    g = cases.golden(name)
    part = g["part"]
    assert np.all(np.diff(part) >= 0)
    assert np.bincount(part).max() <= 16
    pm, rm = O.mas_partition(part, 16)
    assert len(pm) == (part[-1] + 1) * 16
    np.testing.assert_array_equal(pm[rm], np.arange(len(part)))
    for b in range(len(pm) // 16):
        real = pm[16 * b:16 * b + 16]
        real = real[real >= 0]
        assert np.all(np.diff(real) > 0)


@pytest.mark.parametrize("name", ["cube", "bar", "bunny2"])
def test_library_part_maps_match_oracle(name):
    import sgmas
    part = cases.golden(name)["part"]
    pm, rm = sgmas.part_maps(part, 16)
    pm_o, rm_o = O.mas_partition(part, 16)
    np.testing.assert_array_equal(pm, pm_o)
    np.testing.assert_array_equal(rm, rm_o)


def _neighbors_python(tets, n, tris=()):
    """getVertNeighbors (SG/load_mesh.cpp:894-999) with a Python set, as written."""
    seen = set()
    order = []
    def insert(a, b):
        if (a, b) not in seen and (b, a) not in seen:
            seen.add((a, b))
            order.append((a, b))
    for t in tets:
        for i, j in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)):
            insert(int(t[i]), int(t[j]))
    for x, y, z in tris:
        for _ in range(3):
            insert(int(x), int(y)); insert(int(y), int(z)); insert(int(z), int(x))
    lists = [[] for _ in range(n)]
    for a, b in sorted(seen):
        lists[a].append(b)
        lists[b].append(a)
    return lists


@pytest.mark.parametrize("name", ["cube", "bar"])
def test_neighbors_oracle_and_library_match_python(name):
    import sgmas
    g = cases.golden(name)
    n = len(g["pos"])
    ref = _neighbors_python(g["tets"], n)
    for st, nn, nl in (O.vert_neighbors(g["tets"], n), sgmas.vert_neighbors(g["tets"], n)):
        got = [list(nl[st[v]:st[v] + nn[v]]) for v in range(n)]
        assert got == ref


def test_neighbors_with_triangles():
    import sgmas
    g = cases.golden("cloth_high")
    n = len(g["pos"])
    tris = g["tris"]
    ref = _neighbors_python(np.zeros((0, 4), np.int32), n, tris)
    for st, nn, nl in (O.vert_neighbors(np.zeros((0, 4), np.int32), n, tris),
                       sgmas.vert_neighbors(np.zeros((0, 4), np.int32), n, tris)):
        got = [list(nl[st[v]:st[v] + nn[v]]) for v in range(n)]
        assert got == ref


def test_num_levels():
    # computeNumLevels (SG/MASPreconditioner.cu:1720-1739)
    assert O.lib().or_num_levels(1008, 16) == 4
    assert O.lib().or_num_levels(16, 16) == 2
    assert O.lib().or_num_levels(17, 16) == 3
    assert O.lib().or_num_levels(10 ** 8, 16) == 6


# ---------------------------------------------------------------- Morton
def _expand(v):
    out = 0
    for i in range(10):
        out |= ((v >> i) & 1) << (3 * i)
    return out


def _hash_python(x, y, z, res=1024.0):
    c = [min(max(v * res, 0.0), res - 1.0) for v in (x, y, z)]
    xi, yi, zi = (int(v) for v in c)
    return ((_expand(xi) << 2) + (_expand(yi) << 1) + _expand(zi)) & 0xffffffff


def test_morton_hash_matches_bit_interleave():
    rng = np.random.default_rng(0)
    for x, y, z in rng.uniform(-0.1, 1.1, size=(500, 3)):
        assert O.lib().or_hash_code(x, y, z, 1024.0) == _hash_python(x, y, z)


def test_morton_codes_pack_index_and_sort():
    pos = cases.build("c1").s.pos
    codes = O.morton_codes(pos)
    np.testing.assert_array_equal(codes & np.uint64(0xffffffff), np.arange(len(pos), dtype=np.uint64))
    pm, rm = O.morton_partition(pos)
    assert len(pm) % 16 == 0 and np.all(pm[rm] == np.arange(len(pos)))


# ---------------------------------------------------------------- kernels
def test_spmv_matches_scipy():
    s = cases.build("c1").s
    A = synth.full_matrix(s)
    x = np.random.default_rng(1).normal(size=3 * s.n_verts)
    y0 = np.random.default_rng(2).normal(size=3 * s.n_verts)
    y = O.spmv_sym(-2.0, s.vals, s.rows, s.cols, x, 0.5, y0)
    np.testing.assert_allclose(y, -2.0 * (A @ x) + 0.5 * y0, rtol=1e-12, atol=1e-14)


def test_convert_matches_numpy_merge():
    s = synth.config1(seed=3, keep_raw=True)
    r, c, v = O.convert(s.raw_vals, s.raw_rows, s.raw_cols)
    r2, c2, v2 = synth.merge_triplets(s.raw_rows, s.raw_cols, s.raw_vals)
    np.testing.assert_array_equal(r, r2)
    np.testing.assert_array_equal(c, c2)
    np.testing.assert_allclose(v, v2, rtol=1e-13, atol=1e-18)


def test_upper_blocks_write_rule():
    rng = np.random.default_rng(4)
    H = rng.normal(size=(12, 12))
    nodes = np.array([7, 2, 9, 2], np.int32)
    vals = np.zeros((10, 9)); rows = np.zeros(10, np.int32); cols = np.zeros(10, np.int32)
    O.lib().or_write_upper_blocks(H.reshape(-1), 4, nodes, vals.reshape(-1), rows, cols)
    r2, c2, v2 = synth.upper_triplets(H[None], nodes[None].astype(np.int64))
    np.testing.assert_array_equal(rows, r2)
    np.testing.assert_array_equal(cols, c2)
    np.testing.assert_array_equal(vals, v2)
    assert np.all(rows <= cols)


def test_gauss_jordan_inverse_of_spd_blocks():
    rng = np.random.default_rng(5)
    bs = 136
    packed = np.zeros((2, bs, 9))
    for k in range(2):
        M = rng.normal(size=(48, 48))
        A = M @ M.T + 48 * np.eye(48)
        idx = 0
        for r in range(16):
            for c in range(r, 16):
                packed[k, idx] = A[3 * r:3 * r + 3, 3 * c:3 * c + 3].T.reshape(-1)  # column-major
                idx += 1
        inv = O.invert_blocks(packed.reshape(-1), 2).reshape(2, bs, 9)
        Ainv = np.linalg.inv(A)
        idx = 0
        for r in range(16):
            for c in range(r, 16):
                got = inv[k, idx].reshape(3, 3).T
                want = Ainv[3 * r:3 * r + 3, 3 * c:3 * c + 3]
                if r == c:  # the reference symmetrises the diagonal blocks from their upper part
                    want = np.triu(want) + np.triu(want, 1).T
                np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12)
                idx += 1


def test_factored_inverse_of_spd_blocks_with_padding():
    """W = L^-1 (the library's factored storage): W^T W = A^-1, W lower
    triangular; padding rows (zero diagonal) become identity rows."""
    rng = np.random.default_rng(6)
    bs = 136
    M = rng.normal(size=(48, 48))
    A = M @ M.T + 48 * np.eye(48)
    A[42:, :] = 0.0  # two padding slots (vertices 14, 15)
    A[:, 42:] = 0.0
    packed = np.zeros((bs, 9))
    idx = 0
    for r in range(16):
        for c in range(r, 16):
            packed[idx] = A[3 * r:3 * r + 3, 3 * c:3 * c + 3].T.reshape(-1)
            idx += 1
    w = O.factor_blocks(packed.reshape(-1), 1).reshape(bs, 9)
    W = np.zeros((48, 48))
    idx = 0
    for r in range(16):
        for c in range(r, 16):
            W[3 * c:3 * c + 3, 3 * r:3 * r + 3] = w[idx].reshape(3, 3).T  # slot (r, c) = block (c, r) of W
            idx += 1
    Ap = A.copy()
    Ap[np.arange(42, 48), np.arange(42, 48)] = 1.0
    assert np.allclose(np.triu(W, 1), 0.0)
    np.testing.assert_allclose(W.T @ W, np.linalg.inv(Ap), rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(W[42:, 42:], np.eye(6), atol=0)


@pytest.mark.parametrize("precision", [1, 3])
def test_factored_mas_apply_is_symmetric_positive(precision):
    """With factored tiles the MAS is W^T W per subdomain: symmetric (to FP32
    accumulation) and positive even in BF16."""
    case = cases.build("c1")
    m = case.oracle_mas(pairs=False, precision=precision)
    rng = np.random.default_rng(8)
    u, v = rng.normal(size=(2, 3 * case.n))
    Mu, Mv = m.apply(u), m.apply(v)
    assert abs(u @ Mv - v @ Mu) <= 1e-5 * np.sqrt((u @ Mu) * (v @ Mv))
    assert u @ Mu > 0 and v @ Mv > 0


# ---------------------------------------------------------------- MAS + PCG
@pytest.mark.parametrize("name", ["c1", "bar"])
def test_mas_hierarchy_invariants(name):
    case = cases.build(name)
    m = O.MAS(case.n, case.nb_start, case.nb_num, case.nb_list, case.part_map, case.real_map)
    m.reorder(case.s.pairs if len(case.s.pairs) else None)
    t = m.tables()
    ls = t["level_size"]
    L = m.levelnum
    assert ls[1, 1] == len(case.part_map)
    for lvl in range(1, L):
        cnt = ls[lvl, 0]
        ids = t["coarse_space"][lvl - 1]
        assert ids.min() >= 0 and ids.max() < cnt
        assert len(np.unique(ids)) == cnt          # every coarse node has a member
        assert ls[lvl + 1, 1] == ls[lvl, 1] + (cnt + 15) // 16 * 16
        assert ls[lvl + 1, 0] <= cnt
    assert m.total == ls[L, 1]
    # the coarse table is the goingNext chain
    v = np.arange(case.n)
    chain = t["going_next"][v]
    for lvl in range(L - 1):
        np.testing.assert_array_equal(t["coarse_table"][:, lvl], chain)
        chain = t["going_next"][chain]


@pytest.mark.parametrize("precond", [0, 1])
def test_oracle_pcg_converges_and_matches_direct(precond):
    import scipy.sparse.linalg as spl
    s = cases.build("c1").s
    x, rep = O.pcg(s.vals, s.rows, s.cols, s.n_verts, s.b, precond=precond, rel_tol=1e-10)
    xs = spl.spsolve(synth.full_matrix(s), s.b)
    assert rep["rel_residual"] <= 1e-10
    assert rep["iterations"] % 10 == 0
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) <= 1e-6


def test_oracle_mas_pcg_beats_block_jacobi():
    # the stiff contact case (cond ~ 2e10); on mass-dominated systems block-Jacobi
    # alone already converges in one check interval
    case = cases.build("c2s")
    s = case.s
    mas = case.oracle_mas(pairs=True, precision=2)
    _, rj = O.pcg(s.vals, s.rows, s.cols, s.n_verts, s.b, precond=1, rel_tol=1e-4)
    _, rm = O.pcg(s.vals, s.rows, s.cols, s.n_verts, s.b, precond=2, rel_tol=1e-4, mas=mas)
    assert rm["rel_residual"] <= 1e-4 and rj["rel_residual"] <= 1e-4
    assert rm["iterations"] < rj["iterations"]


def test_oracle_preconditioned_norm_and_max_iter():
    s = cases.build("c1").s
    _, r = O.pcg(s.vals, s.rows, s.cols, s.n_verts, s.b, precond=1, rel_tol=1e-30, max_iter=7)
    assert r["iterations"] == 7
    _, r2 = O.pcg(s.vals, s.rows, s.cols, s.n_verts, s.b, precond=1, rel_tol=1e-3, use_preconditioned_norm=True)
    assert r2["iterations"] % 10 == 0 and r2["iterations"] > 0


def test_oracle_start_guess_rule():
    """Start guess: scaled by x0.b / x0.A x0, kept when it lowers ||r||, and
    the convergence test is relative to ||b||; a guess with x0.b <= 0 or no
    finite scale is rejected and the solve equals the cold one."""
    import scipy.sparse.linalg as spl
    s = cases.build("c1").s
    xs = spl.spsolve(synth.full_matrix(s), s.b)
    _, cold = O.pcg(s.vals, s.rows, s.cols, s.n_verts, s.b, precond=1, rel_tol=1e-6)
    x, near = O.pcg(s.vals, s.rows, s.cols, s.n_verts, s.b, precond=1, rel_tol=1e-6, x0=2.0 * xs)
    assert near["x0_rejected"] == 0 and abs(near["x0_scale"] - 0.5) < 1e-9
    assert near["iterations"] == 10 and near["rel_residual"] <= 1e-6
    assert abs(near["rr0"] - float(s.b @ s.b)) <= 1e-12 * float(s.b @ s.b)
    xc, _ = O.pcg(s.vals, s.rows, s.cols, s.n_verts, s.b, precond=1, rel_tol=1e-6)
    for bad in (-xs, np.zeros_like(xs), np.full_like(xs, np.nan)):
        xr, rr = O.pcg(s.vals, s.rows, s.cols, s.n_verts, s.b, precond=1, rel_tol=1e-6, x0=bad)
        assert rr["x0_rejected"] == 1 and rr["iterations"] == cold["iterations"]
        np.testing.assert_array_equal(xr, xc)


def test_mas_apply_is_symmetric_positive():
    case = cases.build("c1")
    m = case.oracle_mas(pairs=False, precision=2)
    rng = np.random.default_rng(7)
    u, v = rng.normal(size=(2, 3 * case.n))
    Mu, Mv = m.apply(u), m.apply(v)
    assert abs(u @ Mv - v @ Mu) <= 1e-10 * abs(u @ Mv)
    assert u @ Mu > 0
