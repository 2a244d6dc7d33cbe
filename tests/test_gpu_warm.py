"""Start-guess (warm-start) solves on the GPU against the oracle's rule.

With ``initial_guess`` the solve scales x0 by alpha = x0.b / x0.A x0 (0
unless positive), rejects it (x0 = 0) when ||b - alpha A x0|| > ||b||, and
tests convergence against ||b||.  The oracle (or_pcg with initial_guess)
restates the same rule on the CPU.
"""
from __future__ import annotations

import numpy as np
import pytest

import cases
from oracle import oracle as O
from sgmas import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

PREC = {"fp32": 0, "bf16": 1, "fp64": 2, "fp32f": 3}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def sgm():
    import sgmas
    return sgmas


def make_ctx(sgm, case, precision="fp32"):
    ctx = sgm.Context(0, bank=16, precision=precision)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    ctx.mas_init(case.n, case.nb_start, case.nb_num, case.nb_list, case.part_map, case.real_map)
    d = dict(vals=dev(case.s.vals), rows=dev(case.s.rows), cols=dev(case.s.cols), b=dev(case.s.b),
             pairs=dev(case.s.pairs.reshape(-1, 4) if len(case.s.pairs) else np.zeros((1, 4), np.int32)))
    ctx.mas_set_contacts(d["pairs"], len(case.s.pairs))
    return ctx, d


def direct_solve(s):
    import scipy.sparse.linalg as spl
    return spl.spsolve(synth.full_matrix(s), s.b)


def solve(ctx, d, case, x0, precond):
    x = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda") if x0 is None else dev(x0)
    rep = ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, d["b"], x, rel_tol=1e-4,
                        preconditioner=precond, initial_guess=x0 is not None)
    torch.cuda.synchronize()
    return x.cpu().numpy(), rep


@pytest.mark.parametrize("mode", ["persistent", "graph"])
@pytest.mark.parametrize("name,precond", [("c1", "mas"), ("bar", "mas"), ("c1", "jacobi")])
def test_warm_start_matches_oracle(sgm, name, precond, mode):
    case = cases.build(name)
    s = case.s
    ctx, d = make_ctx(sgm, case)
    ctx.set_pcg_mode(mode)
    xs = direct_solve(s)
    rng = np.random.default_rng(3)
    x0 = xs + 1e-3 * np.linalg.norm(xs) / np.sqrt(len(xs)) * rng.normal(size=len(xs))
    xg, rep = solve(ctx, d, case, x0, precond)
    _, cold = solve(ctx, d, case, None, precond)
    mas = case.oracle_mas(pairs=bool(len(s.pairs)), precision=0) if precond == "mas" else None
    xo, ro = O.pcg(s.vals, s.rows, s.cols, case.n, s.b, precond=2 if precond == "mas" else 1, rel_tol=1e-4,
                   mas=mas, x0=x0)
    A = synth.full_matrix(s)
    res = np.linalg.norm(s.b - A @ xg) / np.linalg.norm(s.b)
    assert rep["converged"] == 1 and res <= 1e-4 * 1.0001, res
    assert rep["x0_rejected"] == 0 and ro["x0_rejected"] == 0
    assert abs(rep["x0_scale"] - ro["x0_scale"]) <= 1e-12 * abs(ro["x0_scale"])
    assert abs(rep["bb"] - float(s.b @ s.b)) <= 1e-12 * float(s.b @ s.b)
    assert abs(rep["iterations"] - ro["iterations"]) <= 10, (rep["iterations"], ro["iterations"])
    # a guess within 1e-3 of the solution saves iterations over x0 = 0
    assert rep["iterations"] < cold["iterations"], (rep["iterations"], cold["iterations"])
    ctx.close()


@pytest.mark.parametrize("mode", ["persistent", "graph"])
@pytest.mark.parametrize("bad", ["negated", "nan", "zero"])
def test_warm_start_rejected(sgm, mode, bad):
    """x0 = -x* has x0.b < 0 (alpha = 0), a NaN guess has no finite scale and a
    zero guess no direction: each is rejected and the solve is the cold one."""
    case = cases.build("c1")
    s = case.s
    ctx, d = make_ctx(sgm, case)
    ctx.set_pcg_mode(mode)
    xs = direct_solve(s)
    x0 = {"negated": -xs, "nan": np.where(np.arange(len(xs)) == 7, np.nan, xs), "zero": np.zeros_like(xs)}[bad]
    xg, rep = solve(ctx, d, case, x0, "mas")
    xc, cold = solve(ctx, d, case, None, "mas")
    assert rep["x0_rejected"] == 1 and rep["converged"] == 1
    assert rep["iterations"] == cold["iterations"]
    np.testing.assert_array_equal(xg, xc)
    if bad != "nan":
        _, ro = O.pcg(s.vals, s.rows, s.cols, case.n, s.b, precond=2, rel_tol=1e-4,
                      mas=case.oracle_mas(pairs=False, precision=0), x0=x0)
        assert ro["x0_rejected"] == 1
    ctx.close()


def test_warm_start_host_api(sgm):
    """sgmas_pcg_solve_host carries the start guess in x (uploaded with b)."""
    case = cases.build("c1")
    s = case.s
    ctx, _ = make_ctx(sgm, case)
    xs = direct_solve(s)
    x, rep = ctx.pcg_solve_host(s.vals, s.rows, s.cols, case.n, s.b, x0=xs * (1 + 1e-6), rel_tol=1e-4)
    assert rep["x0_rejected"] == 0 and rep["converged"] == 1
    assert rep["iterations"] == 10  # converged at the first test (k % 10 == 0)
    assert abs(rep["x0_scale"] - 1.0) < 1e-3
    ctx.close()
