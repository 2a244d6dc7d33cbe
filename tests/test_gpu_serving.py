"""Batched serving: the persistent solve on a capped number of CTAs, and
several such solves running side by side on their own streams."""
from __future__ import annotations

import threading

import numpy as np
import pytest

import cases

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def sgm():
    import sgmas
    return sgmas


def make_ctx(sgm, case, precision="bf16", ctas=0, stream=None):
    ctx = sgm.Context(0, bank=16, precision=precision)
    ctx.set_stream((stream or torch.cuda.current_stream()).cuda_stream)
    ctx.mas_init(case.n, case.nb_start, case.nb_num, case.nb_list, case.part_map, case.real_map)
    ctx.set_pcg_ctas(ctas)
    return ctx


@pytest.mark.parametrize("precision", ["bf16"])
def test_capped_ctas_give_the_same_preconditioner(sgm, precision):
    """z = M^-1 b of a solve stopped after the first apply is bit-identical on
    8 CTAs and on every SM (subdomain sums do not depend on the ownership).
    BF16-factored storage: the explicit FP32 inverse of two separate
    assemblies already differs in its last bits (FP64 atomics in the
    subdomain-matrix scatter, amplified by Gauss-Jordan)."""
    case = cases.build("c2s")
    s = case.s
    d = dict(vals=dev(s.vals), rows=dev(s.rows), cols=dev(s.cols), b=dev(s.b), pairs=dev(s.pairs.reshape(-1, 4)))
    out = []
    for ctas in (0, 8):
        ctx = make_ctx(sgm, case, precision, ctas)
        ctx.mas_set_contacts(d["pairs"], len(s.pairs))
        x = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda")
        rep = ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, d["b"], x, max_iter=1)
        assert rep["kernel_launches"] == 1
        z = torch.zeros_like(x)
        ctx.pcg_last_vectors(None, z)
        torch.cuda.synchronize()
        out.append(z.cpu().numpy())
        ctx.close()
    np.testing.assert_array_equal(out[0], out[1])


def test_capped_ctas_solve_matches(sgm):
    case = cases.build("c1")
    s = case.s
    d = dict(vals=dev(s.vals), rows=dev(s.rows), cols=dev(s.cols), b=dev(s.b))
    res = []
    for ctas in (0, 4):
        ctx = make_ctx(sgm, case, "bf16", ctas)
        x = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda")
        rep = ctx.pcg_solve(d["vals"], d["rows"], d["cols"], case.n, d["b"], x, rel_tol=1e-8)
        torch.cuda.synchronize()
        res.append((rep["iterations"], x.cpu().numpy()))
        ctx.close()
    assert abs(res[0][0] - res[1][0]) <= 10
    np.testing.assert_allclose(res[1][1], res[0][1], rtol=0, atol=1e-6 * np.abs(res[0][1]).max())


def test_concurrent_solves_on_streams_match_sequential(sgm):
    """Four contexts on four streams, each on at most 16 CTAs, solving from
    four host threads at once: every result equals the same solve run alone
    (same iterations, solution to the last bits of the reassembled matrices)."""
    case = cases.build("c1")
    s = case.s
    rng = np.random.default_rng(0)
    bs = [s.b * (1.0 + 0.1 * k) + rng.normal(size=len(s.b)) * np.abs(s.b).max() * 0.01 for k in range(4)]
    d = dict(vals=dev(s.vals), rows=dev(s.rows), cols=dev(s.cols))
    streams = [torch.cuda.Stream() for _ in range(4)]
    ctxs = [make_ctx(sgm, case, "bf16", 16, st) for st in streams]
    bd = [dev(b) for b in bs]
    xs = [torch.zeros(3 * case.n, dtype=torch.float64, device="cuda") for _ in range(4)]
    torch.cuda.synchronize()
    reps = [None] * 4
    errs = []

    def work(k):
        try:
            with torch.cuda.stream(streams[k]):
                reps[k] = ctxs[k].pcg_solve(d["vals"], d["rows"], d["cols"], case.n, bd[k], xs[k], rel_tol=1e-6)
        except Exception as e:  # surfaced below
            errs.append(e)

    th = [threading.Thread(target=work, args=(k,)) for k in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    torch.cuda.synchronize()
    assert not errs, errs
    for k in range(4):
        x_alone = torch.zeros_like(xs[k])
        rep = ctxs[k].pcg_solve(d["vals"], d["rows"], d["cols"], case.n, bd[k], x_alone, rel_tol=1e-6)
        torch.cuda.synchronize()
        assert reps[k]["converged"] == 1 and rep["iterations"] == reps[k]["iterations"]
        # each solve reassembles the subdomain matrices (FP64 atomics: last-bit differences)
        xa = x_alone.cpu().numpy()
        np.testing.assert_allclose(xs[k].cpu().numpy(), xa, rtol=0, atol=1e-7 * np.abs(xa).max())
    for c in ctxs:
        c.close()
