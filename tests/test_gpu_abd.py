"""The affine-body coupling kernels (sgmas_abd_body_blocks, _pair_blocks,
_fem_blocks) against the oracle (oracle/abd.py), bit for bit: random bodies,
some fixed, pairs within a body and across bodies, FEM points with and
without a boundary type."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import abd as A

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def colmajor(blocks):  # [n][3][3] -> [n][9] column-major, as the library stores blocks
    return np.ascontiguousarray(np.asarray(blocks).transpose(0, 2, 1).reshape(-1, 9))


@pytest.fixture(scope="module")
def ctx():
    import sgmas
    c = sgmas.Context(0)
    c.set_stream(torch.cuda.current_stream().cuda_stream)
    yield c
    c.close()


def scene(seed=0, n_bodies=40, per_body=8):
    rng = np.random.default_rng(seed)
    nv = n_bodies * per_body
    body_of = np.repeat(np.arange(n_bodies), per_body).astype(np.int32)  # vertices numbered body by body
    xbar = rng.normal(size=(nv, 3)) * 0.1
    fixed = (rng.uniform(size=n_bodies) < 0.2).astype(np.int32)
    return rng, nv, body_of, xbar, fixed


def test_body_blocks(ctx):
    rng = np.random.default_rng(1)
    H12 = rng.normal(size=(37, 12, 12))
    H12 = H12 + H12.transpose(0, 2, 1)
    v = torch.zeros((370, 9), dtype=torch.float64, device="cuda")
    r = torch.zeros(370, dtype=torch.int32, device="cuda")
    c = torch.zeros(370, dtype=torch.int32, device="cuda")
    # 12x12 column-major per body
    ctx.abd_body_blocks(dev(np.ascontiguousarray(H12.transpose(0, 2, 1)).reshape(37, 144)), v, r, c)
    torch.cuda.synchronize()
    vo, ro, co = A.body_blocks(H12)
    np.testing.assert_array_equal(r.cpu().numpy(), ro)
    np.testing.assert_array_equal(c.cpu().numpy(), co)
    np.testing.assert_array_equal(v.cpu().numpy().view(np.uint64), colmajor(vo).view(np.uint64))


def test_pair_blocks(ctx):
    rng, nv, body_of, xbar, fixed = scene(2)
    n = 500
    i = rng.integers(0, nv, n)
    j = rng.integers(0, nv, n)
    rows, cols = np.minimum(i, j).astype(np.int32), np.maximum(i, j).astype(np.int32)  # upper vertex pairs
    H = rng.normal(size=(n, 3, 3))
    v = torch.zeros((16 * n, 9), dtype=torch.float64, device="cuda")
    r = torch.zeros(16 * n, dtype=torch.int32, device="cuda")
    c = torch.zeros(16 * n, dtype=torch.int32, device="cuda")
    ctx.abd_pair_blocks(dev(colmajor(H)), dev(rows), dev(cols), dev(xbar.ravel()), dev(body_of), dev(fixed), v, r, c)
    torch.cuda.synchronize()
    vo, ro, co = A.pair_blocks(H, rows, cols, xbar, body_of, fixed)
    np.testing.assert_array_equal(r.cpu().numpy(), ro)
    np.testing.assert_array_equal(c.cpu().numpy(), co)
    np.testing.assert_array_equal(v.cpu().numpy().view(np.uint64), colmajor(vo).view(np.uint64))
    assert (body_of[rows] == body_of[cols]).any() and fixed.any()  # both kinds of pair and a fixed body seen


def test_fem_blocks(ctx):
    rng, nv, body_of, xbar, fixed = scene(3)
    n_fem, n, off = 90, 400, nv
    fem_boundary = (rng.uniform(size=n_fem) < 0.15).astype(np.int32)
    rows = rng.integers(0, nv, n).astype(np.int32)
    cols = (off + rng.integers(0, n_fem, n)).astype(np.int32)
    H = rng.normal(size=(n, 3, 3))
    nb = int(body_of.max()) + 1
    v = torch.zeros((4 * n, 9), dtype=torch.float64, device="cuda")
    r = torch.zeros(4 * n, dtype=torch.int32, device="cuda")
    c = torch.zeros(4 * n, dtype=torch.int32, device="cuda")
    ctx.abd_fem_blocks(dev(colmajor(H)), dev(rows), dev(cols), dev(xbar.ravel()), dev(body_of), dev(fixed),
                       dev(fem_boundary), off, nb, v, r, c)
    torch.cuda.synchronize()
    vo, ro, co = A.fem_blocks(H, rows, cols, xbar, body_of, fixed, fem_boundary, off, nb)
    np.testing.assert_array_equal(r.cpu().numpy(), ro)
    np.testing.assert_array_equal(c.cpu().numpy(), co)
    np.testing.assert_array_equal(v.cpu().numpy().view(np.uint64), colmajor(vo).view(np.uint64))
