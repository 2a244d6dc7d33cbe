"""MatrixMarket boundary (host functions of libsgmas, no GPU needed): the
library writes the reference's export format byte for byte and reads it (and
symmetric files) back into the upper BCOO bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from sgmas import synth


@pytest.fixture(scope="module")
def sgm():
    import sgmas
    return sgmas


@pytest.fixture(scope="module")
def small():
    return synth.config1(seed=4)


def reference_export(path_A, path_b, s):
    """export_matrix_market_files (SG/linear_system/linear_system/
    global_linear_system.cu:98-261) restated: b as an M x 1 array, A general
    coordinate with each stored block and, off the diagonal, its transpose."""
    M = 3 * s.n_verts
    with open(path_b, "w") as f:
        f.write("%%MatrixMarket matrix array real general\n" + "%d %d\n" % (M, 1))
        for v in s.b:
            f.write("%.17g\n" % v)
    nnz = sum(9 if r == c else 18 for r, c in zip(s.rows, s.cols))
    with open(path_A, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n" + "%d %d %d\n" % (M, M, nnz))
        for k in range(len(s.rows)):
            bi, bj = int(s.rows[k]), int(s.cols[k])
            B = s.vals[k].reshape(3, 3).T  # column-major -> B[i, j]
            for i in range(3):
                for j in range(3):
                    f.write("%d %d %.17g\n" % (3 * bi + i + 1, 3 * bj + j + 1, B[i, j]))
            if bi != bj:
                for i in range(3):
                    for j in range(3):
                        f.write("%d %d %.17g\n" % (3 * bj + i + 1, 3 * bi + j + 1, B[j, i]))


def test_write_matches_reference_export_bytes(sgm, small, tmp_path):
    ra, rb = tmp_path / "ref_A.mtx", tmp_path / "ref_b.mtx"
    la, lb = tmp_path / "lib_A.mtx", tmp_path / "lib_b.mtx"
    reference_export(ra, rb, small)
    sgm.mtx_write(la, small.vals, small.rows, small.cols, small.n_verts, small.b, path_b=lb)
    assert la.read_bytes() == ra.read_bytes()
    assert lb.read_bytes() == rb.read_bytes()


def test_round_trip_is_bit_exact(sgm, small, tmp_path):
    a, b = tmp_path / "A.mtx", tmp_path / "b.mtx"
    sgm.mtx_write(a, small.vals, small.rows, small.cols, small.n_verts, small.b, path_b=b)
    vals, rows, cols, n, bb = sgm.mtx_read(a, b)
    assert n == small.n_verts
    np.testing.assert_array_equal(rows, small.rows)
    np.testing.assert_array_equal(cols, small.cols)
    np.testing.assert_array_equal(vals.view(np.uint64), small.vals.view(np.uint64))
    np.testing.assert_array_equal(bb.view(np.uint64), small.b.view(np.uint64))


def test_read_symmetric_file(sgm, small, tmp_path):
    """A symmetric file stores one scalar triangle; lower blocks are
    transposed into the upper triangle and diagonal blocks mirrored."""
    A = synth.full_matrix(small).tocoo()
    low = A.row >= A.col
    p = tmp_path / "sym.mtx"
    with open(p, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n% a comment\n")
        f.write("%d %d %d\n" % (A.shape[0], A.shape[1], int(low.sum())))
        for r, c, v in zip(A.row[low], A.col[low], A.data[low]):
            f.write("%d %d %.17g\n" % (r + 1, c + 1, v))
    vals, rows, cols, n, _ = sgm.mtx_read(p)
    np.testing.assert_array_equal(rows, small.rows)
    np.testing.assert_array_equal(cols, small.cols)
    # the diagonal blocks of the synthetic system are symmetric only to rounding;
    # a symmetric file carries their lower triangle
    np.testing.assert_allclose(vals, small.vals, rtol=1e-12, atol=1e-300)


def test_missing_diagonal_and_bad_banner(sgm, tmp_path):
    p = tmp_path / "bad.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n6 6 1\n1 4 2.0\n")
    with pytest.raises(sgm.SgmasError, match="diagonal block 0 missing"):
        sgm.mtx_read(p)
    q = tmp_path / "arr.mtx"
    q.write_text("%%MatrixMarket matrix array real general\n6 1\n")
    with pytest.raises(sgm.SgmasError, match="coordinate real"):
        sgm.mtx_read(q)
