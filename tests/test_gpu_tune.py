"""The launch-shape autotuner (sgmas_autotune_pcg): trial solves of the
persistent form on candidate grids and of the graph form, the choice by the
objective, and that solves with the tuned shape give the untuned result."""
from __future__ import annotations

import numpy as np
import pytest

import cases
from sgmas import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def sgm():
    import sgmas
    return sgmas


def setup(sgm, name, precision="bf16"):
    case = cases.build(name)
    s = case.s
    ctx = sgm.Context(0, bank=16, precision=precision)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    ctx.mas_init(case.n, case.nb_start, case.nb_num, case.nb_list, case.part_map, case.real_map)
    d = dict(vals=dev(s.vals), rows=dev(s.rows), cols=dev(s.cols), b=dev(s.b))
    if len(s.pairs):
        d["pairs"] = dev(s.pairs.reshape(-1, 4))
        ctx.mas_set_contacts(d["pairs"], len(s.pairs))
    return case, ctx, d


@pytest.mark.parametrize("objective,concurrency", [("latency", 1), ("throughput", 1), ("throughput", 8)])
def test_choice_follows_the_objective(sgm, objective, concurrency):
    case, ctx, d = setup(sgm, "c2s")
    t = ctx.autotune(d["vals"], d["rows"], d["cols"], case.n, d["b"], objective=objective, concurrency=concurrency,
                     trial_iters=20, reps=2)
    c = t["candidates"]
    sms = t["sms"]
    assert len(c) >= 2 and 0 <= t["chosen"] < len(c)
    assert not c[-1]["persistent"] and c[-1]["ctas"] == 0  # the graph form, tried last
    assert all(k["persistent"] and 1 <= k["ctas"] <= sms for k in c[:-1])
    assert [k["ctas"] for k in c[:-1]] == sorted({k["ctas"] for k in c[:-1]})
    assert c[-2]["ctas"] == sms  # every SM is always a candidate (the system fits it)
    for k in c:
        assert np.isfinite(k["us_per_iter"]) and k["us_per_iter"] > 0
        used = max(k["ctas"] if k["persistent"] else sms, sms / concurrency)
        want = k["us_per_iter"] if objective == "latency" else k["us_per_iter"] * used
        assert k["cost"] == pytest.approx(want, rel=1e-12)
    assert t["chosen"] == int(np.argmin([k["cost"] for k in c]))
    ctx.close()


def test_tuned_solve_matches_default(sgm):
    case, ctx, d = setup(sgm, "c2s")
    x_def = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda")
    rep_def = ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, d["b"], x_def, rel_tol=1e-6)
    t = ctx.autotune(d["vals"], d["rows"], d["cols"], case.n, d["b"], objective="throughput", trial_iters=20)
    ch = t["candidates"][t["chosen"]]
    x = torch.zeros_like(x_def)
    rep = ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, d["b"], x, rel_tol=1e-6)
    torch.cuda.synchronize()
    assert rep["converged"] == 1 and rep_def["converged"] == 1
    assert rep["kernel_launches"] == (1 if ch["persistent"] else rep["kernel_launches"])
    # another grid sums the CTA partials of the dot products in other groups:
    # the same method up to rounding, so a few per cent more or fewer iterations
    assert abs(rep["iterations"] - rep_def["iterations"]) <= 0.1 * rep_def["iterations"]
    A = synth.full_matrix(case.s)
    b = case.s.b
    xt, xd = x.cpu().numpy(), x_def.cpu().numpy()
    for xv in (xt, xd):
        assert np.linalg.norm(b - A @ xv) <= 1e-6 * 1.0001 * np.linalg.norm(b)
    assert np.linalg.norm(xt - xd) <= 1e-3 * np.linalg.norm(xd)
    ctx.close()


def test_bad_arguments(sgm):
    case, ctx, d = setup(sgm, "c1")
    with pytest.raises(sgm.SgmasError):
        ctx.autotune(d["vals"], d["rows"], d["cols"], case.n, d["b"], trial_iters=1)
    with pytest.raises(sgm.SgmasError):
        ctx.autotune(d["vals"], d["rows"], d["cols"], case.n, d["b"], reps=0)
    with pytest.raises(sgm.SgmasError):
        ctx.autotune(d["vals"], d["rows"], d["cols"], case.n, d["b"], concurrency=0)
    # the context still solves after a refused call
    x = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda")
    assert ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, d["b"], x)["converged"] == 1
    ctx.close()


def test_system_beyond_every_persistent_grid(sgm):
    """82,944 vertices need more than 32 level-0 subdomains per CTA on every
    grid: no persistent candidate survives, the graph form is the choice, and
    the solve with it converges."""
    case, ctx, d = setup(sgm, "g80k")
    t = ctx.autotune(d["vals"], d["rows"], d["cols"], case.n, d["b"], objective="latency", trial_iters=10, reps=1)
    c = t["candidates"]
    assert len(c) == 1 and not c[0]["persistent"] and t["chosen"] == 0
    x = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda")
    rep = ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, d["b"], x, rel_tol=1e-4)
    assert rep["converged"] == 1 and rep["kernel_launches"] > 1
    A = synth.full_matrix(case.s)
    res = np.linalg.norm(case.s.b - A @ x.cpu().numpy()) / np.linalg.norm(case.s.b)
    assert res <= 1e-4 * 1.0001, res
    ctx.close()
