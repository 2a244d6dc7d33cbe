"""Host driver of the learned start guess (csrc/mlp.cu through the C-ABI).

* init_params: seeded initial FP32 parameters (uniform +-1/sqrt(fan_in), the
  output layer scaled by 0.1 so an untrained network predicts a small step).
* TrainingSet: slot-ordered features and targets of solved steps, kept on the
  device; whole 16-slot subdomains are sampled, since the coarse term is a
  subdomain mean.
* train: minibatch Adam on the GPU (sgmas_mlp_train_step), batches of whole
  subdomains drawn by a seeded permutation each epoch.
* train_anorm: fine-tuning on the energy norm of the start error instead
  of its per-vertex squares: for a stored system, L = (x0 - dx)^T A
  (x0 - dx) / (dx^T b) with x0 = u + s y (lumped step plus the network's
  prediction); its gradient needs A (x0 - dx), one SpMV of the library per
  step (sgmas_spmv), and enters the FP32 training kernels through a
  pseudo-target T' = y - (n / 2) dL/dy.
* warm_start: the start guess of a new system (sgmas_mlp_warm_start): the
  A-norm-best combination of the previous step, the lumped step and the
  network's step and coarse term, to be passed to sgmas_pcg_solve with
  initial_guess = 1, which rejects it when it raises the residual.

The reference has no learned component; this is the library's own addition.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 16, 128, 6
N_PARAMS = N_IN * N_HID + N_HID + N_HID * N_HID + N_HID + N_HID * N_OUT + N_OUT
BANK = 16


def init_params(seed=0):
    rng = np.random.default_rng(seed)

    def layer(fan_in, fan_out, scale=1.0):
        bound = 1.0 / np.sqrt(fan_in)
        return (scale * rng.uniform(-bound, bound, (fan_in, fan_out)), scale * rng.uniform(-bound, bound, fan_out))

    W1, b1 = layer(N_IN, N_HID)
    W2, b2 = layer(N_HID, N_HID)
    W3, b3 = layer(N_HID, N_OUT, 0.1)
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, W3.ravel(), b3]).astype(np.float32)


class TrainingSet:
    """Features X [R,16], targets T [R,3] and masks [R] (R = 16 x subdomains) on the device."""

    def __init__(self, device="cuda", keep=1.0, seed=0):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        self.keep = keep
        self.rng = np.random.default_rng(seed)
        self._X, self._T, self._M, self._cnt = [], [], [], []
        self.X = self.T = self.M = None
        self.counts = None
        self.systems = []

    def add(self, ctx, vals, rows, cols, n_block_rows, b, dx, prev=None, part_map=None, fem_offset=0,
            keep_system=False):
        """Features and targets (dx / s_y) of one solved system, a `keep`
        fraction of its subdomains (seeded), appended.  keep_system: also
        keep the whole system (matrix, b, dx, all slots) for train_anorm."""
        torch = self.torch
        Mm = ctx.part_map_size
        X = torch.empty(Mm * N_IN, dtype=torch.float32, device=self.dev)
        M = torch.empty(Mm, dtype=torch.float32, device=self.dev)
        T = torch.empty(Mm * 3, dtype=torch.float32, device=self.dev)
        sc = ctx.mlp_features(vals, rows, cols, n_block_rows, b, X, M, prev=prev, dx=dx, T=T, fem_offset=fem_offset)
        if keep_system:
            pm = torch.as_tensor(np.asarray(part_map, np.int64), device=self.dev)
            self.systems.append(dict(vals=vals.clone(), rows=rows.clone(), cols=cols.clone(), n=n_block_rows,
                                     b=b.clone(), dx=dx.clone(), X=X.clone(), M=M.clone(), T=T.clone(), s=sc[0],
                                     part_map=pm, fem_offset=fem_offset))
        nb = Mm // BANK
        banks = np.arange(nb)
        if self.keep < 1.0:
            banks = np.sort(self.rng.choice(nb, max(1, int(round(self.keep * nb))), replace=False))
        idx = torch.as_tensor((banks[:, None] * BANK + np.arange(BANK)).ravel(), device=self.dev)
        self._X.append(X.view(Mm, N_IN)[idx])
        self._T.append(T.view(Mm, 3)[idx])
        self._M.append(M[idx])
        if part_map is None:
            cnt = np.full(len(banks), BANK)
        else:
            cnt = (np.asarray(part_map).reshape(nb, BANK)[banks] >= 0).sum(1)
        self._cnt.append(cnt)

    def finalize(self):
        torch = self.torch
        self.X = torch.cat(self._X).contiguous()
        self.T = torch.cat(self._T).contiguous()
        self.M = torch.cat(self._M).contiguous()
        self.counts = np.concatenate(self._cnt)
        self._X, self._T, self._M = [], [], []
        return self

    @property
    def n_banks(self):
        return len(self.counts)


def train(ctx, ts, epochs=4, batch_banks=512, lr=1e-3, seed=0, lr_final=1e-4, log_every=0):
    """Adam over minibatches of whole subdomains; lr decays geometrically from
    lr to lr_final over the run.  Returns [(step, loss)] of the logged steps."""
    torch = ts.torch
    rng = np.random.default_rng(seed)
    nb = ts.n_banks
    steps = epochs * ((nb + batch_banks - 1) // batch_banks)
    decay = (lr_final / lr) ** (1.0 / max(steps - 1, 1))
    hist = []
    step = 0
    ar = torch.arange(BANK, device=ts.dev)
    for _ in range(epochs):
        perm = rng.permutation(nb)
        for s0 in range(0, nb, batch_banks):
            banks = np.sort(perm[s0:s0 + batch_banks])
            rows = (torch.as_tensor(banks, device=ts.dev)[:, None] * BANK + ar).reshape(-1)
            n_valid = int(ts.counts[banks].sum())
            if n_valid == 0:
                continue
            want = log_every > 0 and (step % log_every == 0 or step == steps - 1)
            loss = ctx.mlp_train_step(ts.X[rows].contiguous(), ts.T[rows].contiguous(), ts.M[rows].contiguous(),
                                      int(rows.numel()), 1.0 / n_valid, float(lr * decay ** step), want_loss=want)
            if want:
                hist.append((step, loss))
            step += 1
    return hist


def anorm_loss_grad(ctx, sysd):
    """(L, y, dL/dy) of one stored system for the current parameters:
    y [Mm, 3] the combined prediction (step + subdomain mean of the coarse
    term, as the training kernel forms it), L = e^T A e / (dx^T b) with
    e = s (y - T) on the MAS rows, dL/dy = 2 s (A e) / (dx^T b) per slot."""
    import torch
    X, M, T, s = sysd["X"], sysd["M"], sysd["T"], sysd["s"]
    Mm = M.numel()
    Y = torch.empty(Mm * N_OUT, dtype=torch.float32, device=X.device)
    ctx.mlp_forward(X, Mm, Y, bf16=False)
    Y = Y.view(Mm, N_OUT)
    Mb = M.view(-1, BANK)
    cnt = Mb.sum(1).clamp(min=1.0)
    cm = (Y[:, 3:6].view(-1, BANK, 3) * Mb[..., None]).sum(1) / cnt[:, None]
    y = Y[:, 0:3] + cm.repeat_interleave(BANK, 0)
    valid = sysd["part_map"] >= 0
    rows_of = sysd["fem_offset"] + sysd["part_map"][valid]
    n = sysd["n"]
    e = torch.zeros(n, 3, dtype=torch.float64, device=X.device)
    e[rows_of] = s * (y[valid].double() - T.view(Mm, 3)[valid].double())
    g = torch.zeros_like(e)
    ctx.spmv(1.0, sysd["vals"], sysd["rows"], sysd["cols"], n, e.view(-1), 0.0, g.view(-1))
    lam = 1.0 / float(torch.dot(sysd["dx"], sysd["b"]))
    L = lam * float(torch.dot(e.view(-1), g.view(-1)))
    dLdy = torch.zeros(Mm, 3, dtype=torch.float64, device=X.device)
    dLdy[valid] = 2.0 * lam * s * g[rows_of]
    return L, y, dLdy


def train_anorm(ctx, ts, epochs=2, lr=2e-4, seed=0):
    """Fine-tune on the energy norm of the start error over the stored
    systems (ts.systems), one system per Adam step, seeded order.  Returns
    [(step, L)]."""
    rng = np.random.default_rng(seed)
    hist = []
    step = 0
    for _ in range(epochs):
        for q in rng.permutation(len(ts.systems)):
            sysd = ts.systems[q]
            L, y, dLdy = anorm_loss_grad(ctx, sysd)
            n_valid = float(sysd["M"].sum())
            Tp = (y.double() - dLdy * (n_valid / 2.0)).float().contiguous()
            ctx.mlp_train_step(sysd["X"], Tp.view(-1), sysd["M"], int(sysd["M"].numel()), 1.0 / n_valid, float(lr),
                               want_loss=False)
            hist.append((step, L))
            step += 1
    return hist


def warm_start(ctx, vals, rows, cols, n_block_rows, b, x0, prev=None, fem_offset=0):
    """x0 <- the learned start guess of (A, b) (device arrays)."""
    ctx.mlp_warm_start(vals, rows, cols, n_block_rows, b, x0, prev=prev, fem_offset=fem_offset)
    return x0
