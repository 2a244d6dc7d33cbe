"""The learned start guess on the GPU against its CPU oracle (oracle/mlp.py),
and the gain it brings to the solve on held-out steps of drop sequences."""
from __future__ import annotations

import numpy as np
import pytest

import cases
from oracle import mlp as OM

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def sgm():
    import sgmas
    return sgmas


def ctx_for(sgm, case, precision="bf16", pairs=None):
    ctx = sgm.Context(0, bank=16, precision=precision)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    ctx.mas_init(case.n, case.nb_start, case.nb_num, case.nb_list, case.part_map, case.real_map)
    if pairs is not None and len(pairs):
        ctx._pairs_dev = dev(np.asarray(pairs, np.int32).reshape(-1, 4))
        ctx.mas_set_contacts(ctx._pairs_dev, len(pairs))
    return ctx


def params(seed, scale=0.15):
    return np.random.default_rng(seed).normal(0.0, scale, OM.N_PARAMS).astype(np.float32)


@pytest.mark.parametrize("name", ["c1", "c2s"])
def test_features_match_oracle(sgm, name):
    case = cases.build(name)
    s = case.s
    ctx = ctx_for(sgm, case, pairs=s.pairs)
    rng = np.random.default_rng(0)
    prev = rng.normal(size=3 * case.n) * 1e-3
    dx = rng.normal(size=3 * case.n) * 1e-3
    Mm = len(case.part_map)
    X = torch.zeros(Mm * 16, dtype=torch.float32, device="cuda")
    M = torch.zeros(Mm, dtype=torch.float32, device="cuda")
    T = torch.zeros(Mm * 3, dtype=torch.float32, device="cuda")
    sy, sb = ctx.mlp_features(dev(s.vals), dev(s.rows), dev(s.cols), case.n, dev(s.b), X, M, prev=dev(prev),
                              dx=dev(dx), T=T)
    Xo, Mo, To, (syo, sbo) = OM.features(s.vals, s.rows, s.cols, s.b, case.part_map, case.n, prev=prev,
                                         pairs=s.pairs if len(s.pairs) else None, dx=dx)
    # stiff contact blocks cancel in the row sums S, so S (and the RMS of
    # S^-1 b) carries summation-order rounding of ~1e-10 relative
    assert abs(sy - syo) <= 1e-7 * syo and abs(sb - sbo) <= 1e-12 * sbo
    np.testing.assert_array_equal(M.cpu().numpy(), Mo)
    # FP32 features of FP64 quantities; the lumped step of contact vertices
    # inherits the row-sum cancellation above (a few 1e-6 relative)
    np.testing.assert_allclose(X.cpu().numpy().reshape(Mm, 16), Xo, rtol=2e-5, atol=1e-5)
    np.testing.assert_allclose(T.cpu().numpy().reshape(Mm, 3), To, rtol=2e-5, atol=1e-5)
    if len(s.pairs):
        assert Xo[:, 15].max() > 0  # contact counts reached the features
    ctx.close()


def test_fp32_forward_and_gradient_match_oracle(sgm):
    case = cases.build("c1")
    ctx = ctx_for(sgm, case)
    P = params(1)
    ctx.mlp_set_params(P)
    rng = np.random.default_rng(2)
    n = 16 * 7  # two tiles of 64 rows, the second partial
    X = rng.normal(size=(n, 16)).astype(np.float32)
    T = rng.normal(size=(n, 3)).astype(np.float32)
    mask = (rng.uniform(size=n) > 0.15).astype(np.float32)
    mask[32:48] = 0
    inv_n = 1.0 / mask.sum()
    Y = torch.zeros(n * 6, dtype=torch.float32, device="cuda")
    ctx.mlp_forward(dev(X), n, Y, bf16=False)
    Yo = OM.forward(P, X)
    np.testing.assert_allclose(Y.cpu().numpy().reshape(n, 6), Yo, rtol=1e-4, atol=1e-4 * np.abs(Yo).max())
    g = torch.zeros(OM.N_PARAMS, dtype=torch.float32, device="cuda")
    loss = ctx.mlp_gradient(dev(X), dev(T), dev(mask), n, inv_n, g)
    lo, go = OM.loss_grad(P, X, T, mask, inv_n)
    assert abs(loss - lo) <= 1e-4 * lo
    gg = g.cpu().numpy()
    assert np.linalg.norm(gg - go) <= 1e-4 * np.linalg.norm(go)
    np.testing.assert_allclose(gg, go, rtol=0, atol=2e-4 * np.abs(go).max())
    # the gradient call does not move the parameters
    np.testing.assert_array_equal(ctx.mlp_get_params(), P)
    # one Adam step = the oracle's Adam on the oracle's gradient (|g| large enough to fix the step)
    lr = 1e-3
    ctx.mlp_train_step(dev(X), dev(T), dev(mask), n, inv_n, lr)
    P1 = ctx.mlp_get_params().astype(np.float64)
    Po, _, _ = OM.adam(P.astype(np.float64), np.zeros(OM.N_PARAMS), np.zeros(OM.N_PARAMS), go, 1, lr)
    big = np.abs(go) > 1e-3 * np.abs(go).max()
    np.testing.assert_allclose(P1[big], Po[big], rtol=0, atol=2e-3 * lr + 1e-7)
    ctx.close()


def test_bf16_inference_matches_oracle(sgm):
    case = cases.build("c1")
    ctx = ctx_for(sgm, case)
    P = params(3)
    ctx.mlp_set_params(P)
    rng = np.random.default_rng(4)
    n = 16 * 37
    X = rng.normal(size=(n, 16)).astype(np.float32)
    Y = torch.zeros(n * 6, dtype=torch.float32, device="cuda")
    ctx.mlp_forward(dev(X), n, Y, bf16=True)
    Yg = Y.cpu().numpy().reshape(n, 6)
    Yo = OM.infer_bf16(P, X)
    scale = np.abs(Yo).max()
    assert np.max(np.abs(Yg - Yo)) <= 2e-2 * scale, np.max(np.abs(Yg - Yo)) / scale
    assert np.median(np.abs(Yg - Yo)) <= 2e-3 * scale
    # and it tracks the FP64 network within BF16 accuracy
    assert np.max(np.abs(Yg - OM.forward(P, X))) <= 6e-2 * np.abs(OM.forward(P, X)).max()
    ctx.close()


def test_bf16_inference_many_tiles(sgm):
    """160,016 rows: 1,251 tiles of 128 rows on at most two CTAs per SM (each CTA
    runs several tiles through the same TMEM accumulator and mbarrier phases),
    the last tile holding 16 rows."""
    case = cases.build("c1")
    ctx = ctx_for(sgm, case)
    P = params(5)
    ctx.mlp_set_params(P)
    rng = np.random.default_rng(6)
    n = 16 * 10001
    X = rng.normal(size=(n, 16)).astype(np.float32)
    Y = torch.full((n * 6,), float("nan"), dtype=torch.float32, device="cuda")
    ctx.mlp_forward(dev(X), n, Y, bf16=True)
    Yg = Y.cpu().numpy().reshape(n, 6)
    Yo = OM.infer_bf16(P, X)
    scale = np.abs(Yo).max()
    assert np.isfinite(Yg).all()
    assert np.max(np.abs(Yg - Yo)) <= 2e-2 * scale, np.max(np.abs(Yg - Yo)) / scale
    assert np.median(np.abs(Yg - Yo)) <= 2e-3 * scale
    # every tile as accurate as the first (no stale accumulator or phase slip)
    err = np.abs(Yg - Yo).max(axis=1).reshape(-1, 16).max(axis=1)
    assert err[-1] <= 2e-2 * scale and np.percentile(err, 99) <= 1e-2 * scale
    ctx.close()


def test_warm_start_is_galerkin_optimal(sgm):
    """x0 is the A-norm-best combination of its candidates: with zero network
    parameters it equals the oracle's Galerkin combination of the previous
    step and the lumped step; with a network it is no worse (A-norm) than
    either alone, and the coefficients come back."""
    from sgmas import synth
    case = cases.build("c2s")
    s = case.s
    ctx = ctx_for(sgm, case, pairs=s.pairs)
    A = synth.full_matrix(s)
    xs = np.linalg.solve(A.toarray(), s.b)
    prev = xs * (1.0 + 0.05 * np.random.default_rng(6).normal(size=len(xs)))
    u, _ = OM.lumped_step(s.vals, s.rows, s.cols, s.b, case.n)
    u = u.ravel()
    V = np.stack([prev, u], 1)
    c_o = np.linalg.solve(V.T @ (A @ V), V.T @ s.b)
    x0 = torch.zeros(3 * case.n, dtype=torch.float64, device="cuda")
    ctx.mlp_set_params(np.zeros(OM.N_PARAMS, np.float32))
    c = ctx.mlp_warm_start(dev(s.vals), dev(s.rows), dev(s.cols), case.n, dev(s.b), x0, prev=dev(prev), coef=True)
    np.testing.assert_allclose(c[:2], c_o, rtol=1e-6, atol=1e-9 * np.abs(c_o).max())
    assert c[2] == 0 and c[3] == 0   # zero network outputs: skipped candidates
    np.testing.assert_allclose(x0.cpu().numpy(), V @ c_o, rtol=1e-6, atol=1e-9 * np.abs(xs).max())
    enorm = lambda x: float(np.sqrt((xs - x) @ (A @ (xs - x))))
    best1 = lambda v: enorm(v * (v @ s.b) / (v @ (A @ v)))
    ctx.mlp_set_params(params(5))
    c = ctx.mlp_warm_start(dev(s.vals), dev(s.rows), dev(s.cols), case.n, dev(s.b), x0, prev=dev(prev), coef=True)
    e = enorm(x0.cpu().numpy())
    assert np.all(np.isfinite(c))
    assert e <= best1(prev) * (1 + 1e-9) and e <= best1(u) * (1 + 1e-9), (e, best1(prev), best1(u))
    # without a previous step the candidate is skipped
    c = ctx.mlp_warm_start(dev(s.vals), dev(s.rows), dev(s.cols), case.n, dev(s.b), x0, coef=True)
    assert c[0] == 0 and enorm(x0.cpu().numpy()) <= best1(u) * (1 + 1e-9)
    ctx.close()


def test_training_is_deterministic(sgm):
    case = cases.build("c1")
    rng = np.random.default_rng(7)
    n = 16 * 40
    X = dev(rng.normal(size=(n, 16)).astype(np.float32))
    T = dev(rng.normal(size=(n, 3)).astype(np.float32))
    M = dev(np.ones(n, np.float32))
    out = []
    for _ in range(2):
        ctx = ctx_for(sgm, case)
        ctx.mlp_set_params(params(8))
        for _ in range(5):
            ctx.mlp_train_step(X, T, M, n, 1.0 / n, 1e-3, want_loss=False)
        out.append(ctx.mlp_get_params())
        ctx.close()
    np.testing.assert_array_equal(out[0], out[1])


def solve_ms(ctx, args, x, **cfg):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rep = ctx.pcg_solve(*args, x, rel_tol=1e-4, **cfg)
    e1.record()
    torch.cuda.synchronize()
    return rep, e0.elapsed_time(e1)


def test_learned_start_saves_iterations_on_held_out_steps(sgm):
    """Train on the solver's own solves of small drop sequences; on held-out
    sequences the learned start guess must cut the mean iteration count of
    BF16 MAS-PCG against x0 = 0, every solve still reaching 1e-4 of ||b||.
    (The same start with a zero network is reported beside it: on these
    sequences most of the gain comes from the previous step in the Galerkin
    combination.)"""
    from sgmas import learned
    from sgmas.sequence import DropScene
    from sgmas import synth

    def scene_ctx(sc):
        ctx = sgm.Context(0, bank=16, precision="bf16")
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        pm, rm = ctx.morton_partition(torch.as_tensor(sc.X, device="cuda"))
        ctx.mas_init(sc.n, *sgm.vert_neighbors(sc.tets, sc.n), pm, rm)
        ctx.mas_set_contacts(sc.t_pairs, len(sc.pairs))
        sc.ctx = ctx
        return ctx, pm

    ts = learned.TrainingSet("cuda")
    for seed in range(6):
        sc = DropScene(seed=seed, scale=0.25, device="cuda")
        ctx, pm = scene_ctx(sc)
        for _ in range(20):
            vals, rows, cols, b = sc.system()
            x = torch.zeros_like(b)
            ctx.pcg_solve(vals, rows, cols, sc.n, b, x, rel_tol=1e-6)
            ts.add(ctx, vals, rows, cols, sc.n, b, x, prev=sc.prev, part_map=pm)
            sc.advance(x)
        ctx.close()
    ts.finalize()
    trainer = sgm.Context(0, bank=16, precision="bf16")
    trainer.set_stream(torch.cuda.current_stream().cuda_stream)
    trainer.mlp_set_params(learned.init_params(0))
    hist = learned.train(trainer, ts, epochs=40, batch_banks=64, lr=2e-3, lr_final=2e-4, seed=0, log_every=100)
    assert hist[-1][1] < 0.5 * hist[0][1], hist
    P = trainer.mlp_get_params()
    trainer.close()
    it_plain, it_learn, it_zero = [], [], []
    for seed in (100, 101):
        sc = DropScene(seed=seed, scale=0.25, device="cuda")
        ctx, _ = scene_ctx(sc)
        ctx.mlp_set_params(P)
        for _ in range(20):
            vals, rows, cols, b = sc.system()
            args = (vals, rows, cols, sc.n, b)
            x = torch.zeros_like(b)
            rp, _ = solve_ms(ctx, args, x)
            x0 = torch.zeros_like(b)
            ctx.mlp_warm_start(*args, x0, prev=sc.prev)
            rl, _ = solve_ms(ctx, args, x0, initial_guess=True)
            assert rp["converged"] == 1 and rl["converged"] == 1
            s = synth.System(n_verts=sc.n, rows=rows.cpu().numpy(), cols=cols.cpu().numpy(),
                             vals=vals.cpu().numpy(), b=b.cpu().numpy(), pos=sc.X, tets=sc.tets, pairs=sc.pairs)
            A = synth.full_matrix(s)
            res = np.linalg.norm(s.b - A @ x0.cpu().numpy()) / np.linalg.norm(s.b)
            assert res <= 1e-4 * 1.0001
            ctx.mlp_set_params(np.zeros(len(P), np.float32))
            xz = torch.zeros_like(b)
            ctx.mlp_warm_start(*args, xz, prev=sc.prev)
            rz, _ = solve_ms(ctx, args, xz, initial_guess=True)
            ctx.mlp_set_params(P)
            it_plain.append(rp["iterations"])
            it_learn.append(rl["iterations"])
            it_zero.append(rz["iterations"])
            sc.advance(x)
        ctx.close()
    print(f"mean iterations: plain {np.mean(it_plain):.1f}, learned {np.mean(it_learn):.1f}, "
          f"zero network {np.mean(it_zero):.1f}")
    assert np.mean(it_learn) <= 0.85 * np.mean(it_plain), (it_learn, it_plain)


def test_energy_fine_tuning(sgm):
    """learned.anorm_loss_grad: L = e^T A e / (dx^T b) for the start error
    e = s (y - T) on the MAS rows, against a scipy product of the full
    matrix; learned.train_anorm lowers the mean of L over its systems."""
    import types
    from sgmas import learned, synth
    from sgmas.sequence import DropScene

    sc = DropScene(seed=3, scale=0.25, device="cuda")
    ctx = sgm.Context(0, bank=16, precision="bf16")
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    pm, rm = ctx.morton_partition(torch.as_tensor(sc.X, device="cuda"))
    ctx.mas_init(sc.n, *sgm.vert_neighbors(sc.tets, sc.n), pm, rm)
    ctx.mas_set_contacts(sc.t_pairs, len(sc.pairs))
    sc.ctx = ctx
    ts = learned.TrainingSet("cuda")
    for _ in range(10):
        vals, rows, cols, b = sc.system()
        x = torch.zeros_like(b)
        ctx.pcg_solve(vals, rows, cols, sc.n, b, x, rel_tol=1e-8)
        ts.add(ctx, vals, rows, cols, sc.n, b, x, prev=sc.prev, part_map=pm, keep_system=True)
        sc.advance(x)
    ts.finalize()
    ctx.mlp_set_params(learned.init_params(0))
    learned.train(ctx, ts, epochs=10, batch_banks=64, lr=2e-3, lr_final=2e-4, seed=0)
    sysd = ts.systems[-1]
    L, y, g = learned.anorm_loss_grad(ctx, sysd)
    A = synth.full_matrix(types.SimpleNamespace(vals=sysd["vals"].cpu().numpy(), rows=sysd["rows"].cpu().numpy(),
                                                cols=sysd["cols"].cpu().numpy(), n_verts=sysd["n"]))
    Mm = ctx.part_map_size
    pmn = np.asarray(pm)[:Mm]
    ok = pmn >= 0
    e = np.zeros((sysd["n"], 3))
    e[pmn[ok]] = sysd["s"] * (y.cpu().numpy()[ok].astype(np.float64) - sysd["T"].view(Mm, 3).cpu().numpy()[ok])
    e = e.ravel()
    dx, b = sysd["dx"].cpu().numpy(), sysd["b"].cpu().numpy()
    L_ref = float(e @ (A @ e)) / float(dx @ b)
    assert abs(L - L_ref) <= 1e-9 * abs(L_ref), (L, L_ref)
    g_ref = 2.0 * sysd["s"] * (A @ e).reshape(-1, 3)[pmn[ok]] / float(dx @ b)
    np.testing.assert_allclose(g.cpu().numpy()[ok], g_ref, rtol=1e-9, atol=1e-12 * np.abs(g_ref).max())
    before = np.mean([learned.anorm_loss_grad(ctx, q)[0] for q in ts.systems])
    learned.train_anorm(ctx, ts, epochs=4, lr=2e-4, seed=0)
    after = np.mean([learned.anorm_loss_grad(ctx, q)[0] for q in ts.systems])
    assert np.isfinite(after) and after < before, (before, after)
    ctx.close()
