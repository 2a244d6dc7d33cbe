"""Seeded time sequences of Newton systems: the training and evaluation data
of the learned start guess.

A scene is the contact workload's geometry (two stacked tet blocks,
point-triangle barrier pairs between the top block's bottom face and the
bottom block's top face).  The top block is released from rest h ~ U(0.01,
0.1) m above its resting place (1e-4 m above the bottom block) and falls onto
it; the bottom block's base layer is held by stiff springs.  Each time step
is one linearly implicit Euler (Newton) step of the incremental potential

    E(x) = 1/2 (x - xh)^T M (x - xh) + dt^2 (E_elastic(x) + E_barrier(x) + E_base(x)),
    xh = x_t + dt v_t + dt^2 g,

so A = M + dt^2 (K_elastic + H_barrier + k_base I) in the reference scaling,
b = -grad E(x_t).  The solver's dx is applied with the step filter of an IPC
line search: the largest fraction beta <= 1 that keeps every barrier pair at
least 10 % of its current distance (distances linear along the step), so
x_{t+1} = x_t + beta dx, v_{t+1} = beta dx / dt.
The elastic term is the stable Neo-Hookean energy with its per-element
Hessian projected to PSD (as sgmas.synth); a barrier pair at plane distance d
contributes kappa b(d) with b(d) = -(d - dhat)^2 ln(d / dhat) for d < dhat,
its gradient kappa b'(d) g and the SPD Hessian kappa b''(d) g g^T + kappa eps I.

Torch holds the state (any device).  On a CUDA device the element and pair
matrices go through the library's own triplet writer and converter
(sgmas_write_upper_blocks, sgmas_convert); on the CPU through numpy.  All
sums are deterministic (fixed-order gathers, no atomics).
"""
from __future__ import annotations

import numpy as np

from . import synth


def _incidence(index, n):
    """[n, maxdeg] positions (-1 = none) of each target id in `index`, stable order."""
    index = np.asarray(index, np.int64)
    order = np.argsort(index, kind="stable")
    counts = np.bincount(index, minlength=n)
    maxdeg = max(int(counts.max()) if len(counts) else 0, 1)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
    pos = np.full((n, maxdeg), -1, np.int64)
    sorted_ids = index[order]
    pos[sorted_ids, np.arange(len(index)) - starts[sorted_ids]] = order
    return pos


def two_block_scene(nx, ny, nz, h, gap, n_pairs, rng):
    """Rest positions (jittered 1e-4 m), tets and interface point-triangle
    pairs (reference int4 PT encoding) of two stacked nx*ny*nz tet grids:
    each point of the top block's bottom face is paired with triangles of the
    bottom block's top face whose centre lies within 3.5 cells."""
    P, T = [], []
    off = 0
    for k in range(2):
        p, t = synth.tet_grid(nx, ny, nz, h, (0.0, k * ((ny - 1) * h + gap), 0.0))
        P.append(p)
        T.append(t + off)
        off += len(p)
    X = np.concatenate(P)
    X = X + rng.normal(0.0, 1e-4, X.shape)
    tets = np.concatenate(T).astype(np.int64)
    nv1 = nx * ny * nz
    vid = lambda x_, y_, z_, o: o + x_ + nx * (y_ + ny * z_)
    gx, gz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    pts = vid(gx.ravel(), 0, gz.ravel(), nv1)
    qx, qz = np.meshgrid(np.arange(nx - 1), np.arange(nz - 1), indexing="ij")
    qx, qz = qx.ravel(), qz.ravel()
    a = vid(qx, ny - 1, qz, 0)
    b1 = vid(qx + 1, ny - 1, qz, 0)
    c1 = vid(qx, ny - 1, qz + 1, 0)
    d1 = vid(qx + 1, ny - 1, qz + 1, 0)
    tris = np.concatenate([np.stack([a, b1, d1], 1), np.stack([a, d1, c1], 1)])
    tri_c = np.concatenate([np.stack([qx + 2 / 3, qz + 1 / 3], 1), np.stack([qx + 1 / 3, qz + 2 / 3], 1)])
    pxz = np.stack([gx.ravel(), gz.ravel()], 1).astype(np.float64)
    cand = []
    for i in range(len(pts)):
        js = np.nonzero(np.abs(tri_c - pxz[i]).max(1) <= 3.5)[0]
        cand.append(np.stack([np.full(len(js), i), js], 1))
    cand = np.concatenate(cand)
    pick = np.sort(rng.choice(len(cand), size=min(n_pairs, len(cand)), replace=False))
    cand = cand[pick]
    nodes = np.stack([pts[cand[:, 0]], tris[cand[:, 1], 0], tris[cand[:, 1], 1], tris[cand[:, 1], 2]], 1)
    pairs = np.stack([-(nodes[:, 0] + 1), nodes[:, 1], nodes[:, 2], nodes[:, 3]], 1).astype(np.int32)
    return X, tets, pairs


class DropScene:
    G = (0.0, -9.81, 0.0)

    def __init__(self, seed=0, scale=1.0, drop_height=None, device="cpu", dt=0.01, E=1e6, nu=0.45, rho=1000.0,
                 kappa=1e5, dhat=1e-3, eps=1e-6, h=0.01, gap=1e-4, k_base=1e7, ctx=None):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        self.ctx = ctx
        rng = np.random.default_rng(seed)
        nx, ny, nz = max(2, int(round(40 * scale))), max(2, int(round(20 * scale))), max(2, int(round(20 * scale)))
        n_pairs = int(round(50000 * (nx * nz) / 800.0))
        X, self.tets, self.pairs = two_block_scene(nx, ny, nz, h, gap, n_pairs, rng)
        self.n = len(X)
        self.X = X
        self.info = dict(nx=nx, ny=ny, nz=nz, n_pairs=len(self.pairs), seed=seed, scale=scale)
        self.drop_height = float(rng.uniform(0.01, 0.1)) if drop_height is None else float(drop_height)
        self.dt, self.kappa, self.dhat, self.eps, self.k_base = dt, kappa, dhat, eps, k_base
        mu = E / (2 * (1 + nu))
        lam = E * nu / ((1 + nu) * (1 - 2 * nu))
        self.mu, self.lam, self.alpha = mu, lam, 1 + mu / lam
        t = torch.as_tensor
        X = self.X
        Xt = X[self.tets]
        Dm = np.stack([Xt[:, 1] - Xt[:, 0], Xt[:, 2] - Xt[:, 0], Xt[:, 3] - Xt[:, 0]], -1)
        vol = np.abs(np.linalg.det(Dm)) / 6.0
        Dminv = np.linalg.inv(Dm)
        dFdx = np.zeros((len(self.tets), 9, 12))
        for col in range(3):
            for k in range(3):
                c = Dminv[:, k, col]
                for d in range(3):
                    dFdx[:, col * 3 + d, (k + 1) * 3 + d] += c
                    dFdx[:, col * 3 + d, d] -= c
        mass = np.zeros(self.n)
        np.add.at(mass, self.tets.ravel(), np.repeat(rho * vol / 4.0, 4))
        nv1 = nx * ny * nz
        base_mask = np.zeros(self.n)
        base_mask[np.arange(nv1)[(np.arange(nv1) // nx) % ny == 0]] = 1.0   # y = 0 layer of the bottom block
        self.nodes_pair = np.stack([-self.pairs[:, 0] - 1, self.pairs[:, 1], self.pairs[:, 2], self.pairs[:, 3]], 1).astype(np.int64)
        d64 = dict(dtype=torch.float64, device=self.dev)
        self.t_vol = t(vol, **d64)
        self.t_dFdx = t(dFdx, **d64)
        self.t_mass = t(mass, **d64)
        self.t_base = t(base_mask, **d64)
        self.t_X = t(X, **d64)
        self.t_tets = t(self.tets, device=self.dev)
        self.t_pn = t(self.nodes_pair, device=self.dev)
        # fixed-order gathers for the gradient: vertex <- (element, corner), vertex <- (pair, corner)
        self.t_inc_e = t(_incidence(self.tets.ravel(), self.n), device=self.dev)
        self.t_inc_p = t(_incidence(self.nodes_pair.ravel(), self.n), device=self.dev)
        self.t_nodes32 = t(self.tets.astype(np.int32), device=self.dev)
        self.t_pn32 = t(self.nodes_pair.astype(np.int32), device=self.dev)
        self.t_pairs = t(np.ascontiguousarray(self.pairs, np.int32), device=self.dev)
        # state: the top block at rest, drop_height above its resting place
        x0 = X.copy()
        x0[nv1:, 1] += self.drop_height
        self.x = t(x0, **d64)
        self.v = torch.zeros(self.n, 3, **d64)
        self.prev = torch.zeros(3 * self.n, **d64)
        self.step_index = 0

    # ---- energy terms at the current state -------------------------------------------
    def _elastic(self, x):
        torch = self.torch
        vecx = x[self.t_tets].reshape(-1, 12)
        F = (self.t_dFdx @ vecx[:, :, None])[:, :, 0].reshape(-1, 3, 3).transpose(1, 2)  # vec(F) is column-major
        f0, f1, f2 = F[:, :, 0], F[:, :, 1], F[:, :, 2]
        J = torch.linalg.det(F)
        g = torch.cat([torch.cross(f1, f2, dim=1), torch.cross(f2, f0, dim=1), torch.cross(f0, f1, dim=1)], 1)
        vecF = torch.cat([f0, f1, f2], 1)
        mu, lam, alpha = self.mu, self.lam, self.alpha
        P = mu * vecF + (lam * (J - alpha))[:, None] * g

        def hat(v):
            z = torch.zeros_like(v[:, 0])
            return torch.stack([torch.stack([z, -v[:, 2], v[:, 1]], 1), torch.stack([v[:, 2], z, -v[:, 0]], 1),
                                torch.stack([-v[:, 1], v[:, 0], z], 1)], 1)
        z3 = torch.zeros(len(F), 3, 3, dtype=F.dtype, device=F.device)
        HJ = torch.cat([torch.cat([z3, -hat(f2), hat(f1)], 2), torch.cat([hat(f2), z3, -hat(f0)], 2),
                        torch.cat([-hat(f1), hat(f0), z3], 2)], 1)
        HF = mu * torch.eye(9, dtype=F.dtype, device=F.device)[None] + lam * g[:, :, None] * g[:, None, :] + \
            (lam * (J - alpha))[:, None, None] * HJ
        # PSD projection, in chunks (the batched eigensolver limits the batch size)
        parts = []
        for i0 in range(0, len(HF), 16384):
            w, V = torch.linalg.eigh(HF[i0:i0 + 16384])
            parts.append((V * torch.clamp(w, min=0.0)[:, None, :]) @ V.transpose(1, 2))
        HF = torch.cat(parts)
        He = self.t_vol[:, None, None] * (self.t_dFdx.transpose(1, 2) @ HF @ self.t_dFdx)
        ge = self.t_vol[:, None] * (self.t_dFdx.transpose(1, 2) @ P[:, :, None])[:, :, 0]
        return He, ge

    def _plane_distance(self, x):
        torch = self.torch
        p, a, b, c = (x[self.t_pn[:, i]] for i in range(4))
        n = torch.cross(b - a, c - a, dim=1)
        n = n / torch.linalg.norm(n, dim=1, keepdim=True)
        n = torch.where(n[:, 1:2] < 0, -n, n)
        return ((p - a) * n).sum(1), n, p, a, b, c

    def _barrier(self, x):
        torch = self.torch
        d, n, p, a, b, c = self._plane_distance(x)
        # barycentric weights of p's projection, clamped to the triangle
        q = p - d[:, None] * n
        v0, v1, v2 = b - a, c - a, q - a
        d00, d01, d11 = (v0 * v0).sum(1), (v0 * v1).sum(1), (v1 * v1).sum(1)
        d20, d21 = (v2 * v0).sum(1), (v2 * v1).sum(1)
        den = d00 * d11 - d01 * d01
        wb = torch.clamp((d11 * d20 - d01 * d21) / den, 0.0, 1.0)
        wc = torch.clamp((d00 * d21 - d01 * d20) / den, 0.0, 1.0)
        s = torch.clamp(wb + wc, min=1.0)
        wb, wc = wb / s, wc / s
        wa = 1.0 - wb - wc
        dh = self.dhat
        de = torch.clamp(d, min=1e-2 * dh)
        act = de < dh
        lg = torch.log(de / dh)
        bp = torch.where(act, -2.0 * (de - dh) * lg - (de - dh) ** 2 / de, torch.zeros_like(de))
        bpp = torch.where(act, -2.0 * lg - 4.0 * (de - dh) / de + (de - dh) ** 2 / de ** 2, torch.zeros_like(de))
        gv = torch.cat([n, -wa[:, None] * n, -wb[:, None] * n, -wc[:, None] * n], 1)
        H = (self.kappa * bpp)[:, None, None] * gv[:, :, None] * gv[:, None, :]
        H = H + self.kappa * self.eps * torch.eye(12, dtype=x.dtype, device=x.device)[None]
        grad = (self.kappa * bp)[:, None] * gv
        return H, grad, int(act.sum())

    def system(self):
        """(vals [nb,9], rows, cols, b [3n]) of the current step, on the scene's device."""
        torch = self.torch
        dt = self.dt
        x = self.x
        xh = x + dt * self.v + dt * dt * torch.tensor(self.G, dtype=x.dtype, device=x.device)[None]
        He, ge = self._elastic(x)
        Hc, gc, self.n_active = self._barrier(x)
        ve = torch.cat([ge.reshape(-1, 3), ge.new_zeros(1, 3)], 0)[self.t_inc_e].sum(1)
        vc = torch.cat([gc.reshape(-1, 3), gc.new_zeros(1, 3)], 0)[self.t_inc_p].sum(1)
        gbase = self.k_base * self.t_base[:, None] * (x - self.t_X)
        grad = self.t_mass[:, None] * (x - xh) + dt * dt * (ve + vc + gbase)
        b = (-grad).reshape(-1).contiguous()
        He = (dt * dt) * He
        Hc = (dt * dt) * Hc
        diag = self.t_mass + dt * dt * self.k_base * self.t_base
        vm = torch.zeros(self.n, 9, dtype=x.dtype, device=x.device)
        vm[:, 0] = vm[:, 4] = vm[:, 8] = diag
        if self.dev.type == "cuda" and self.ctx is not None:
            vals, rows, cols = self._merge_device(He.contiguous(), Hc.contiguous(), vm)
        else:
            r_e, c_e, v_e = synth.upper_triplets(He.cpu().numpy(), self.tets)
            r_c, c_c, v_c = synth.upper_triplets(Hc.cpu().numpy(), self.nodes_pair)
            ar = np.arange(self.n)
            mr, mc, mv = synth.merge_triplets(np.concatenate([ar, r_e, r_c]).astype(np.int32),
                                              np.concatenate([ar, c_e, c_c]).astype(np.int32),
                                              np.concatenate([vm.cpu().numpy(), v_e, v_c]))
            vals, rows, cols = (torch.as_tensor(a, device=self.dev) for a in (mv, mr, mc))
        return vals, rows, cols, b

    def _merge_device(self, He, Hc, vm):
        torch = self.torch
        ctx = self.ctx
        ne, nc = len(He), len(Hc)
        n_raw = self.n + 10 * ne + 10 * nc
        if getattr(self, "_raw", None) is None or self._raw[0].shape[0] != n_raw:
            dev = self.dev
            self._raw = (torch.empty(n_raw, 9, dtype=torch.float64, device=dev),
                         torch.empty(n_raw, dtype=torch.int32, device=dev),
                         torch.empty(n_raw, dtype=torch.int32, device=dev),
                         torch.empty(n_raw, 9, dtype=torch.float64, device=dev),
                         torch.empty(n_raw, dtype=torch.int32, device=dev),
                         torch.empty(n_raw, dtype=torch.int32, device=dev))
        rv, rr, rc, ov, orr, oc = self._raw
        rv[: self.n] = vm
        rr[: self.n] = torch.arange(self.n, dtype=torch.int32, device=self.dev)
        rc[: self.n] = rr[: self.n]
        o = self.n
        ctx.write_upper_blocks(He, self.t_nodes32, rv[o:o + 10 * ne], rr[o:o + 10 * ne], rc[o:o + 10 * ne])
        o += 10 * ne
        ctx.write_upper_blocks(Hc, self.t_pn32, rv[o:], rr[o:], rc[o:])
        nu = ctx.convert(rv, rr, rc, ov, orr, oc)
        return ov[:nu], orr[:nu], oc[:nu]

    def step_fraction(self, dx):
        """Largest beta <= 1 keeping every pair at >= 10 % of its current distance."""
        torch = self.torch
        d0 = self._plane_distance(self.x)[0]
        d1 = self._plane_distance(self.x + dx.reshape(-1, 3))[0]
        lim = 0.1 * d0
        hit = d1 < lim
        if not bool(hit.any()):
            return 1.0
        frac = (d0[hit] - lim[hit]) / (d0[hit] - d1[hit])
        return float(torch.clamp(frac.min(), 0.0, 1.0))

    def advance(self, dx):
        """x += beta dx, v = beta dx / dt (beta from step_fraction); the
        applied step is the next system's previous Newton step."""
        beta = self.step_fraction(dx)
        step = beta * dx.reshape(-1, 3)
        self.x = self.x + step
        self.v = step / self.dt
        self.prev = step.reshape(-1).clone()
        self.step_index += 1
        self.last_beta = beta
        return beta
