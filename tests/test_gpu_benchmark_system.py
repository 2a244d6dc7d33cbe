"""Parity on the benchmark system itself: the contact workload bench.py times
(two 40x20x20-vertex tet blocks 1e-4 m apart, 50,000 point-triangle barrier
pairs; 32,000 vertices, 96,000 DOF, 287,660 upper blocks, cond ~ 1e10), solved
by the persistent kernel in each MAS storage precision the bench reports.

Three checks per precision:
  * the reference's stopping rule at 1e-4: the true relative residual
    ||b - A x|| / ||b|| (computed here from the scipy matrix) is <= 1e-4;
  * the iteration count lies in the band the oracle port itself spans when b
    moves in its last bit (see below), widened by that band's width (at least
    one check interval);
  * at 1e-10, the solution is within 1e-6 relative of an FP64 direct solve
    (banded Cholesky in reverse Cuthill-McKee order, sgmas.synth.direct_solve),
    and at 1e-4 within 1e-5.

Why a band and not one fixed count: on this system CG's iteration count moves
with the last bit of any sum.  The oracle port (the same algorithm, serial or
OpenMP sums) run on b scaled by (1 + k * 2^-52), k = 0..3, spans a range of
counts by itself (measured in the test, printed on failure); the device's
count must fall inside that range, widened on each side by its own width
(at least one check interval, 10): a few samples under-read the spread.
"""
from __future__ import annotations

import functools

import numpy as np
import pytest

import cases
from oracle import oracle as O
from sgmas import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

PREC = {"fp32": 0, "bf16": 1, "fp64": 2, "fp32f": 3}


@functools.lru_cache(maxsize=None)
def bench_system():
    s = synth.config2(seed=0, scale=1.0)
    pm, rm = O.morton_partition(s.pos)
    st, nn, nl = O.vert_neighbors(s.tets, s.n_verts)
    return s, pm, rm, st, nn, nl


@functools.lru_cache(maxsize=None)
def direct():
    s = bench_system()[0]
    return synth.direct_solve(s)


@functools.lru_cache(maxsize=None)
def full():
    return synth.full_matrix(bench_system()[0])


@functools.lru_cache(maxsize=None)
def oracle_band(precision):
    """(min, max) iteration counts of the oracle port's MAS-PCG (1e-4,
    reference stopping rule) over b moved in its last bit
    (cases.oracle_iteration_band)."""
    s, pm, rm, st, nn, nl = bench_system()
    m = O.MAS(s.n_verts, st, nn, nl, pm, rm)
    m.reorder(s.pairs)
    m.assemble(s.vals, s.rows, s.cols, precision=PREC[precision])
    return cases.oracle_iteration_band(s, 2, mas=m, n_perturb=4, max_iter=5000)


def solve_gpu(precision, rel_tol):
    import sgmas
    s, pm, rm, st, nn, nl = bench_system()
    ctx = sgmas.Context(0, bank=16, precision=precision)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    ctx.set_pcg_mode("persistent")
    ctx.mas_init(s.n_verts, st, nn, nl, pm, rm)
    pairs = torch.from_numpy(s.pairs).cuda()
    ctx.mas_set_contacts(pairs, len(s.pairs))
    d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (s.vals, s.rows, s.cols, s.b)]
    x = torch.zeros(3 * s.n_verts, dtype=torch.float64, device="cuda")
    rep = ctx.pcg_solve(*d[:3], s.n_verts, d[3], x, rel_tol=rel_tol, max_iter=5000, preconditioner="mas")
    xg = x.cpu().numpy()
    ctx.close()
    return xg, rep


def rel_err(x, xs):
    return float(np.linalg.norm(x - xs) / np.linalg.norm(xs))


def test_direct_solve_is_exact_enough():
    """The reference solution itself: relative residual at FP64 round-off."""
    s = bench_system()[0]
    xs = direct()
    assert np.linalg.norm(s.b - full() @ xs) / np.linalg.norm(s.b) <= 1e-10


@pytest.mark.parametrize("precision", ["bf16", "fp32", "fp32f", "fp64"])
def test_benchmark_solve_matches_oracle(precision):
    s = bench_system()[0]
    xg, rep = solve_gpu(precision, 1e-4)
    assert rep["kernel_launches"] == 1, "the persistent form must take the benchmark system"
    assert rep["converged"] == 1
    res = np.linalg.norm(s.b - full() @ xg) / np.linalg.norm(s.b)
    assert res <= 1e-4 * 1.0001, res
    assert rep["iterations"] % 10 == 0
    band = oracle_band(precision)
    assert cases.band_ok(rep["iterations"], band), (rep["iterations"], band)
    # solution error at the benchmark tolerance (the oracle's is ~1e-6 here)
    assert rel_err(xg, direct()) <= 1e-5, rel_err(xg, direct())


@pytest.mark.parametrize("precision", ["bf16", "fp32", "fp32f", "fp64"])
def test_benchmark_tight_solve_matches_direct(precision):
    """At 1e-10 every storage precision gives the FP64 direct solution to
    1e-6 relative (measured: ~5e-12 for the oracle port in every precision).
    1e-10 and not tighter: with the reference's stopping rule (true residual
    every 10th iteration) CG on this system stops improving near 1e-11 and
    is not asked for more."""
    s = bench_system()[0]
    xg, rep = solve_gpu(precision, 1e-10)
    assert rep["converged"] == 1
    res = np.linalg.norm(s.b - full() @ xg) / np.linalg.norm(s.b)
    assert res <= 1e-10 * 1.0001, res
    assert rel_err(xg, direct()) <= 1e-6, rel_err(xg, direct())
