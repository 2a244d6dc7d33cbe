"""Failure paths of the solve, each made on the host and each reported as a
status (the reference aborts or prints instead): no GPU fault, trap or hang
is ever caused.

  * a device-side wait that runs out: the persistent kernel's grid barriers
    are told to expect one arrival more than the grid has CTAs (host-side
    fault injection, sgmas_set_wait_limit), with a short poll limit; every
    CTA gives up at its first barrier, the kernel returns, and the solve
    reports SGMAS_ERR_DEVICE ("bounded wait expired");
  * a NaN in the right-hand side: SGMAS_ERR_NUMERIC;
  * a diagonal block that is not positive definite: CG breaks down
    (p.A p <= 0) or its residual turns non-finite: SGMAS_ERR_NUMERIC;
  * sizes beyond a stated capacity: SGMAS_ERR_CAPACITY before any work.
After each failure the same context solves a valid system correctly.
"""
from __future__ import annotations

import numpy as np
import pytest

import cases
from sgmas import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ERR_CAPACITY, ERR_DEVICE, ERR_NUMERIC = -4, -5, -6


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def make(case, precision="fp32", mode="persistent"):
    import sgmas
    ctx = sgmas.Context(0, bank=16, precision=precision)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    ctx.set_pcg_mode(mode)
    ctx.mas_init(case.n, case.nb_start, case.nb_num, case.nb_list, case.part_map, case.real_map)
    return ctx


def good_solve(ctx, case, d, **kw):
    x = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda")
    rep = ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, d["b"], x, rel_tol=1e-4, **kw)
    A = synth.full_matrix(case.s)
    res = np.linalg.norm(case.s.b - A @ x.cpu().numpy()) / np.linalg.norm(case.s.b)
    assert rep["converged"] == 1 and res <= 1e-4 * 1.0001
    return rep


def upload(case):
    s = case.s
    return dict(vals=dev(s.vals), rows=dev(s.rows), cols=dev(s.cols), b=dev(s.b))


@pytest.mark.parametrize("precond", ["mas", "jacobi"])
def test_grid_barrier_timeout_is_reported(precond):
    import sgmas
    case = cases.build("c1")
    d = upload(case)
    ctx = make(case)
    ctx.set_wait_limit(spin_limit=2000, phantom_arrivals=1)
    x = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda")
    with pytest.raises(sgmas.SgmasError) as ei:
        ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, d["b"], x, rel_tol=1e-4, preconditioner=precond)
    assert ei.value.code == ERR_DEVICE and "bounded wait expired" in str(ei.value)
    ctx.set_wait_limit(0, 0)   # back to normal: the context is still usable
    rep = good_solve(ctx, case, d, preconditioner=precond)
    assert rep["kernel_launches"] == 1
    ctx.close()


@pytest.mark.parametrize("mode", ["persistent", "graph"])
def test_nan_rhs_is_reported(mode):
    import sgmas
    case = cases.build("c1")
    d = upload(case)
    ctx = make(case, mode=mode)
    b = case.s.b.copy()
    b[17] = np.nan
    x = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda")
    with pytest.raises(sgmas.SgmasError) as ei:
        ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, dev(b), x, rel_tol=1e-4, preconditioner="mas")
    assert ei.value.code == ERR_NUMERIC
    good_solve(ctx, case, d, preconditioner="mas")
    ctx.close()


@pytest.mark.parametrize("mode", ["persistent", "graph"])
@pytest.mark.parametrize("precond,precision", [("jacobi", "fp32"), ("mas", "fp32"), ("mas", "bf16")])
def test_non_spd_block_breaks_down(mode, precond, precision):
    """One vertex's diagonal block made strongly negative definite, b
    concentrated on that vertex: the first p.A p is negative."""
    import sgmas
    case = cases.build("c1")
    s = case.s
    d = upload(case)
    v = 123
    k = int(np.flatnonzero((s.rows == v) & (s.cols == v))[0])
    vals = s.vals.copy()
    vals[k] = -1e3 * np.abs(vals[k]).max() * np.eye(3).ravel()
    b = np.zeros_like(s.b)
    b[3 * v:3 * v + 3] = 1.0
    ctx = make(case, precision=precision, mode=mode)
    x = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda")
    with pytest.raises(sgmas.SgmasError) as ei:
        ctx.pcg_solve(dev(vals), d["rows"], d["cols"], case.n, dev(b), x, rel_tol=1e-4, preconditioner=precond)
    # CG breaks down (p.A p <= 0), or -- when the factored inverse of the
    # indefinite subdomain overflows -- the residual turns non-finite first
    assert ei.value.code == ERR_NUMERIC
    assert "breakdown" in str(ei.value) or "non-finite" in str(ei.value), str(ei.value)
    good_solve(ctx, case, d, preconditioner=precond)
    ctx.close()


def test_zero_rhs_is_solved_by_zero():
    """b = 0: r = 0 exactly, p.A p = 0 -- a solution, not a breakdown."""
    case = cases.build("c1")
    d = upload(case)
    ctx = make(case)
    x = torch.ones(3 * case.n, dtype=torch.float64, device="cuda")
    rep = ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, torch.zeros_like(d["b"]), x, rel_tol=1e-4,
                        preconditioner="mas")
    assert rep["converged"] == 1 and float(x.abs().max()) == 0.0
    ctx.close()


def test_capacity_limits_are_refused():
    import sgmas
    case = cases.build("c1")
    ctx = make(case)
    pos = dev(case.s.pos)
    with pytest.raises(sgmas.SgmasError) as ei:   # part_map array smaller than the partition needs
        ctx.morton_partition(pos, part_map_cap=16)
    assert ei.value.code == ERR_CAPACITY
    ctx.close()
