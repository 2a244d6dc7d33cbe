"""Seeded synthetic IPC Newton systems in the reference's BCOO layout.

The reference builds its Hessian from Stable Neo-Hookean tets
(SG/femEnergy.cu:1789-1927), IPC barrier pairs (SG/GIPC.cu:3108-4947) and a
lumped mass diagonal (SG/GIPC.cu:10201-10220).  The physics producers are not
part of the solve; this module stands in for them with seeded inputs of the
same shapes, sizes and value ranges:

* a structured tet grid (6 tets per cube, Freudenthal split), vertex
  positions jittered, a random deformation of the given scale;
* the element Hessian of the stable Neo-Hookean energy
  psi = mu/2 (tr F^T F - 3) + lam/2 (J - 1 - mu/lam)^2, projected to PSD per
  element, scaled by volume * dt^2 (reference scaling: A = M + dt^2 K);
* b = dt^2 * gradient of the elastic energy at the deformed state;
* synthetic point-triangle barrier pairs between two stacked blocks, each an
  SPD 12x12 matrix kappa*b''(d) g g^T + kappa*eps*I written as 10 upper blocks
  and encoded as the reference's PT int4 (-(p+1), t0, t1, t2).

Element matrices are written into upper 3x3 triplets exactly like
write_triplet_fem (SG/femEnergy.cu:14-62): row <= col, the (jj, ii) block
transposed when the vertex order is reversed.  Values are column-major 3x3.
"""
from __future__ import annotations

import dataclasses

import numpy as np

_TET_SPLIT = np.array([  # Freudenthal/Kuhn split of the unit cube along (0,0,0)-(1,1,1)
    [0, 1, 3, 7], [0, 1, 5, 7], [0, 2, 3, 7],
    [0, 2, 6, 7], [0, 4, 5, 7], [0, 4, 6, 7]], dtype=np.int64)

# corner c of a cube -> (dx, dy, dz) with c = dx + 2 dy + 4 dz
_CORNER = np.array([[c & 1, (c >> 1) & 1, (c >> 2) & 1] for c in range(8)], dtype=np.int64)

UPPER_PAIRS_4 = [(ii, jj) for ii in range(4) for jj in range(ii, 4)]


@dataclasses.dataclass
class System:
    """An upper-triangular 3x3 BCOO system A x = b (reference scaling)."""
    n_verts: int
    rows: np.ndarray          # int32 [nb]
    cols: np.ndarray          # int32 [nb]
    vals: np.ndarray          # float64 [nb, 9], column-major 3x3
    b: np.ndarray             # float64 [3 n]
    pos: np.ndarray           # float64 [n, 3] (rest positions)
    tets: np.ndarray          # int32 [ntet, 4]
    pairs: np.ndarray         # int32 [cp, 4] contact pairs (reference int4 encoding)
    # raw triplets before merging (the scatter-assembly input)
    raw_rows: np.ndarray = None
    raw_cols: np.ndarray = None
    raw_vals: np.ndarray = None
    elem_groups: list = None
    info: dict = dataclasses.field(default_factory=dict)


def tet_grid(nx: int, ny: int, nz: int, h: float, origin=(0.0, 0.0, 0.0)):
    """Vertices (x fastest) and 6 tets per cube of an nx*ny*nz vertex grid."""
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    vid = lambda x, y, z: x + nx * (y + ny * z)
    pos = np.stack([ix.ravel(order="F"), iy.ravel(order="F"), iz.ravel(order="F")], 1).astype(np.float64)
    pos = pos * h + np.asarray(origin, dtype=np.float64)
    cx, cy, cz = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), np.arange(nz - 1), indexing="ij")
    cx, cy, cz = cx.ravel(order="F"), cy.ravel(order="F"), cz.ravel(order="F")
    corners = np.stack([vid(cx + d[0], cy + d[1], cz + d[2]) for d in _CORNER], 1)  # [ncube, 8]
    tets = corners[:, _TET_SPLIT].reshape(-1, 4)
    return pos, tets.astype(np.int64)


def _hat(v):
    z = np.zeros(v.shape[:-1])
    return np.stack([np.stack([z, -v[..., 2], v[..., 1]], -1),
                     np.stack([v[..., 2], z, -v[..., 0]], -1),
                     np.stack([-v[..., 1], v[..., 0], z], -1)], -2)


def neo_hookean_elements(X, x, tets, E, nu):
    """Per-tet volume-weighted PSD Hessian [ntet,12,12] and gradient [ntet,12]."""
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    alpha = 1.0 + mu / lam
    Xt = X[tets]                                         # [t,4,3]
    Dm = np.stack([Xt[:, 1] - Xt[:, 0], Xt[:, 2] - Xt[:, 0], Xt[:, 3] - Xt[:, 0]], -1)
    vol = np.abs(np.linalg.det(Dm)) / 6.0
    Dminv = np.linalg.inv(Dm)
    xt = x[tets]
    Ds = np.stack([xt[:, 1] - xt[:, 0], xt[:, 2] - xt[:, 0], xt[:, 3] - xt[:, 0]], -1)
    F = Ds @ Dminv
    f0, f1, f2 = F[:, :, 0], F[:, :, 1], F[:, :, 2]
    J = np.linalg.det(F)
    g = np.concatenate([np.cross(f1, f2), np.cross(f2, f0), np.cross(f0, f1)], -1)  # vec(dJ/dF), column-major
    vecF = np.concatenate([f0, f1, f2], -1)
    P = mu * vecF + (lam * (J - alpha))[:, None] * g
    z3 = np.zeros((len(tets), 3, 3))
    HJ = np.block([[z3, -_hat(f2), _hat(f1)],
                   [_hat(f2), z3, -_hat(f0)],
                   [-_hat(f1), _hat(f0), z3]])
    HF = mu * np.eye(9)[None] + lam * g[:, :, None] * g[:, None, :] + (lam * (J - alpha))[:, None, None] * HJ
    w, V = np.linalg.eigh(HF)
    HF = (V * np.maximum(w, 0.0)[:, None, :]) @ np.swapaxes(V, 1, 2)
    # dvec(F)/dx: vec(F) = (Dminv^T kron I3) vec(Ds); Ds columns x_k - x_0
    dFdx = np.zeros((len(tets), 9, 12))
    for col in range(3):          # column of F
        for k in range(3):        # Ds column k = x_{k+1} - x_0
            c = Dminv[:, k, col]
            for d in range(3):
                dFdx[:, col * 3 + d, (k + 1) * 3 + d] += c
                dFdx[:, col * 3 + d, d] -= c
    He = vol[:, None, None] * (np.swapaxes(dFdx, 1, 2) @ HF @ dFdx)
    ge = vol[:, None] * np.einsum("tij,ti->tj", dFdx, P)
    return He, ge, vol


def upper_triplets(H, nodes):
    """write_triplet_fem (SG/femEnergy.cu:14-62) for a batch: H [m,3k,3k], nodes [m,k]."""
    m, k = nodes.shape
    pairs = [(ii, jj) for ii in range(k) for jj in range(ii, k)]
    rows = np.empty((m, len(pairs)), np.int64)
    cols = np.empty((m, len(pairs)), np.int64)
    vals = np.empty((m, len(pairs), 9))
    for q, (ii, jj) in enumerate(pairs):
        r, c = nodes[:, ii], nodes[:, jj]
        swap = r > c
        blk = H[:, 3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3]          # (a, c) = H[ii*3+a, jj*3+c]
        blkT = np.swapaxes(H[:, 3 * jj:3 * jj + 3, 3 * ii:3 * ii + 3], 1, 2)
        # when swapped the stored block is (jj,ii) block: element (a,c) = H[jj*3+a, ii*3+c]
        blk_sw = H[:, 3 * jj:3 * jj + 3, 3 * ii:3 * ii + 3]
        use = np.where(swap[:, None, None], blk_sw, blk)
        rows[:, q] = np.where(swap, c, r)
        cols[:, q] = np.where(swap, r, c)
        vals[:, q] = np.swapaxes(use, 1, 2).reshape(m, 9)           # column-major
        del blkT
    return rows.ravel(), cols.ravel(), vals.reshape(-1, 9)


def merge_triplets(rows, cols, vals):
    """Stable sort by (row, col) and sum duplicates (Converter::convert)."""
    key = (rows.astype(np.uint64) << np.uint64(32)) + cols.astype(np.uint64)
    order = np.argsort(key, kind="stable")
    ks = key[order]
    head = np.ones(len(ks), bool)
    head[1:] = ks[1:] != ks[:-1]
    seg = np.cumsum(head) - 1
    out = np.zeros((int(seg[-1]) + 1, 9))
    np.add.at(out, seg, vals[order])
    uk = ks[head]
    return (uk >> np.uint64(32)).astype(np.int32), (uk & np.uint64(0xffffffff)).astype(np.int32), out


def barrier_hessian(d, dhat, kappa, eps, normal, bary, rng):
    """kappa*b''(d) g g^T + kappa*eps*I12 for point-triangle pairs (SPD)."""
    bpp = (-2.0 * np.log(d / dhat) - 4.0 * (d - dhat) / d + (d - dhat) ** 2 / d ** 2)
    g = np.concatenate([normal, -bary[:, 0:1] * normal, -bary[:, 1:2] * normal, -bary[:, 2:3] * normal], 1)
    H = (kappa * bpp)[:, None, None] * g[:, :, None] * g[:, None, :]
    H += kappa * eps * np.eye(12)[None]
    return H


def make_grid_system(nx=10, ny=10, nz=10, h=0.01, E=1e5, nu=0.4, rho=1000.0, dt=0.01,
                     jitter=1e-4, deform=0.05, seed=0, blocks=1, gap=1e-4,
                     n_pairs=0, dhat=1e-3, kappa=1e5, eps=1e-6, keep_raw=False):
    """One or two stacked tet grids (+ barrier pairs between them)."""
    rng = np.random.default_rng(seed)
    P, T = [], []
    off = 0
    for k in range(blocks):
        origin = (0.0, k * ((ny - 1) * h + gap), 0.0)
        p, t = tet_grid(nx, ny, nz, h, origin)
        P.append(p)
        T.append(t + off)
        off += len(p)
    X = np.concatenate(P)
    tets = np.concatenate(T)
    n = len(X)
    X = X + rng.normal(0.0, jitter, X.shape)
    G = rng.normal(0.0, 1.0, (3, 3))
    x = X + deform * (X - X.mean(0)) @ G.T + deform * h * rng.normal(0.0, 1.0, X.shape)
    He, ge, vol = neo_hookean_elements(X, x, tets, E, nu)
    He *= dt * dt
    ge *= dt * dt
    r_el, c_el, v_el = upper_triplets(He, tets)
    mass = np.zeros(n)
    np.add.at(mass, tets.ravel(), np.repeat(rho * vol / 4.0, 4))
    b = np.zeros(3 * n)
    np.add.at(b, (3 * tets[:, :, None] + np.arange(3)).ravel(), ge.ravel())
    # mass diagonal (SG/GIPC.cu:10201-10220): m * I
    r_m = np.arange(n)
    v_m = np.zeros((n, 9))
    v_m[:, 0] = v_m[:, 4] = v_m[:, 8] = mass
    rows = [r_m, r_el]
    cols = [r_m, c_el]
    vals = [v_m, v_el]
    H_m = np.zeros((n, 3, 3))
    H_m[:, 0, 0] = H_m[:, 1, 1] = H_m[:, 2, 2] = mass
    groups = [(H_m, np.arange(n, dtype=np.int32)[:, None]), (He, tets.astype(np.int32))]
    pairs = np.zeros((0, 4), np.int32)
    if n_pairs and blocks == 2:
        nv1 = nx * ny * nz
        vid = lambda x_, y_, z_, o: o + x_ + nx * (y_ + ny * z_)
        # points: bottom face (y = 0) of the top block
        gx, gz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
        pts = vid(gx.ravel(), 0, gz.ravel(), nv1)
        # triangles: top face (y = ny-1) of the bottom block, 2 per quad
        qx, qz = np.meshgrid(np.arange(nx - 1), np.arange(nz - 1), indexing="ij")
        qx, qz = qx.ravel(), qz.ravel()
        a = vid(qx, ny - 1, qz, 0); b1 = vid(qx + 1, ny - 1, qz, 0)
        c1 = vid(qx, ny - 1, qz + 1, 0); d1 = vid(qx + 1, ny - 1, qz + 1, 0)
        tris = np.concatenate([np.stack([a, b1, d1], 1), np.stack([a, d1, c1], 1)])
        tri_c = np.concatenate([np.stack([qx + 2 / 3, qz + 1 / 3], 1), np.stack([qx + 1 / 3, qz + 2 / 3], 1)])
        pxz = np.stack([gx.ravel(), gz.ravel()], 1).astype(np.float64)
        # candidate (point, triangle) pairs within 3.5 cells
        cand = []
        for i in range(len(pts)):
            dd = np.abs(tri_c - pxz[i]).max(1)
            js = np.nonzero(dd <= 3.5)[0]
            cand.append(np.stack([np.full(len(js), i), js], 1))
        cand = np.concatenate(cand)
        pick = rng.choice(len(cand), size=min(n_pairs, len(cand)), replace=False)
        cand = cand[np.sort(pick)]
        pi, tj = cand[:, 0], cand[:, 1]
        m = len(cand)
        d = rng.uniform(0.0, dhat, m)
        d = np.maximum(d, dhat * 1e-3)
        normal = np.tile([0.0, 1.0, 0.0], (m, 1)) + rng.normal(0.0, 0.05, (m, 3))
        normal /= np.linalg.norm(normal, axis=1, keepdims=True)
        bary = rng.dirichlet(np.ones(3), m)
        Hc = barrier_hessian(d, dhat, kappa, eps, normal, bary, rng) * dt * dt
        nodes = np.stack([pts[pi], tris[tj, 0], tris[tj, 1], tris[tj, 2]], 1)
        r_c, c_c, v_c = upper_triplets(Hc, nodes)
        rows.append(r_c); cols.append(c_c); vals.append(v_c)
        groups.append((Hc, nodes.astype(np.int32)))
        pairs = np.stack([-(nodes[:, 0] + 1), nodes[:, 1], nodes[:, 2], nodes[:, 3]], 1).astype(np.int32)
    raw_r = np.concatenate(rows).astype(np.int32)
    raw_c = np.concatenate(cols).astype(np.int32)
    raw_v = np.concatenate(vals)
    mr, mc, mv = merge_triplets(raw_r, raw_c, raw_v)
    sysm = System(n_verts=n, rows=mr, cols=mc, vals=mv, b=b, pos=X, tets=tets.astype(np.int32),
                  pairs=pairs,
                  info=dict(nx=nx, ny=ny, nz=nz, blocks=blocks, n_pairs=len(pairs), E=E, nu=nu,
                            dt=dt, h=h, eps=eps, kappa=kappa, dhat=dhat, seed=seed, n_tets=len(tets),
                            n_raw=len(raw_r), n_blocks=len(mr)))
    if keep_raw:  # raw triplets, and the element groups (matrices [m, 3k, 3k], nodes [m, k]) they come from
        sysm.raw_rows, sysm.raw_cols, sysm.raw_vals = raw_r, raw_c, raw_v
        sysm.elem_groups = groups
    return sysm


def mesh_system(X, tets, E=1e5, nu=0.4, rho=1000.0, dt=0.01, deform=0.05, seed=0):
    """A Neo-Hookean system on a given tet mesh (positions X [n,3], tets [t,4])."""
    rng = np.random.default_rng(seed)
    X = np.asarray(X, np.float64)
    tets = np.asarray(tets, np.int64)
    n = len(X)
    h = float(np.median(np.linalg.norm(X[tets[:, 1]] - X[tets[:, 0]], axis=1)))
    G = rng.normal(0.0, 1.0, (3, 3))
    x = X + deform * (X - X.mean(0)) @ G.T + deform * h * rng.normal(0.0, 1.0, X.shape)
    He, ge, vol = neo_hookean_elements(X, x, tets, E, nu)
    He *= dt * dt
    ge *= dt * dt
    r_el, c_el, v_el = upper_triplets(He, tets)
    mass = np.zeros(n)
    np.add.at(mass, tets.ravel(), np.repeat(rho * vol / 4.0, 4))
    mass = np.maximum(mass, 1e-12)
    b = np.zeros(3 * n)
    np.add.at(b, (3 * tets[:, :, None] + np.arange(3)).ravel(), ge.ravel())
    v_m = np.zeros((n, 9))
    v_m[:, 0] = v_m[:, 4] = v_m[:, 8] = mass
    raw_r = np.concatenate([np.arange(n), r_el]).astype(np.int32)
    raw_c = np.concatenate([np.arange(n), c_el]).astype(np.int32)
    raw_v = np.concatenate([v_m, v_el])
    mr, mc, mv = merge_triplets(raw_r, raw_c, raw_v)
    return System(n_verts=n, rows=mr, cols=mc, vals=mv, b=b, pos=X, tets=tets.astype(np.int32),
                  pairs=np.zeros((0, 4), np.int32), raw_rows=raw_r, raw_cols=raw_c, raw_vals=raw_v,
                  info=dict(n_tets=len(tets), n_blocks=len(mr), E=E, nu=nu, dt=dt, seed=seed))


def config1(seed=0, **kw):
    """10x10x10 tet grid, Neo-Hookean E=1e5 nu=0.4, no contact (3,000 DOF)."""
    return make_grid_system(10, 10, 10, 0.01, E=1e5, nu=0.4, seed=seed, **kw)


def config2(seed=0, scale=1.0, **kw):
    """Two 40x20x20 grids stacked 1e-4 m apart with 50k point-triangle pairs."""
    nx, ny, nz = max(2, int(round(40 * scale))), max(2, int(round(20 * scale))), max(2, int(round(20 * scale)))
    npairs = int(round(50000 * (nx * nz) / 800.0))
    return make_grid_system(nx, ny, nz, 0.01, E=1e6, nu=0.45, seed=seed, blocks=2,
                            n_pairs=npairs, **kw)


def full_matrix(s: System):
    """Dense (small) or scipy-sparse full symmetric matrix for direct solves."""
    import scipy.sparse as sp
    n = s.n_verts
    r3 = (3 * s.rows[:, None, None] + np.arange(3)[None, :, None]) + 0 * np.arange(3)[None, None, :]
    c3 = (3 * s.cols[:, None, None] + np.arange(3)[None, None, :]) + 0 * np.arange(3)[None, :, None]
    v3 = s.vals.reshape(-1, 3, 3).transpose(0, 2, 1)   # column-major -> (a, c)
    A = sp.coo_matrix((v3.ravel(), (r3.ravel(), c3.ravel())), shape=(3 * n, 3 * n)).tocsr()
    off = s.rows != s.cols
    AT = sp.coo_matrix((v3[off].ravel(), (r3[off].ravel(), c3[off].ravel())), shape=(3 * n, 3 * n)).tocsr().T
    return (A + AT).tocsc()


def direct_solve(s: System, band_bytes_max: float = 8e9):
    """FP64 direct solve of A x = b, the accuracy reference for the PCG
    results.  Vertices are put in reverse Cuthill-McKee order of the block
    graph (3 DOF each), so A becomes a band; LAPACK's banded Cholesky
    (dpbtrf/dpbtrs) factors and solves it, and one step of iterative
    refinement with the FP64 residual follows.  On the 96,000-DOF contact
    benchmark the band is ~5,800 wide (4.5 GB) and the solve takes ~20 s on 8
    cores, against ~2 min for SuperLU (COLAMD); the two agree to ~1e-11.
    Falls back to SuperLU when the band would need more than band_bytes_max."""
    import scipy.linalg as sl
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    A = full_matrix(s).tocsr()
    n = s.n_verts
    G = sp.csr_matrix((np.ones(len(s.rows)), (s.rows, s.cols)), shape=(n, n))
    p = reverse_cuthill_mckee((G + G.T).tocsr(), symmetric_mode=True)
    P = (3 * p[:, None] + np.arange(3)[None, :]).ravel()
    Ap = A[P][:, P].tocoo()
    bw = int(np.max(np.abs(Ap.row - Ap.col))) if Ap.nnz else 0
    if (bw + 1) * 3.0 * n * 8 > band_bytes_max:
        lu = spl.splu(A.tocsc(), permc_spec="COLAMD")
        x = lu.solve(s.b)
        return x + lu.solve(s.b - A @ x)
    up = Ap.row <= Ap.col
    ab = np.zeros((bw + 1, 3 * n))
    ab[bw + Ap.row[up] - Ap.col[up], Ap.col[up]] = Ap.data[up]
    c = sl.cholesky_banded(ab, overwrite_ab=True, lower=False, check_finite=False)
    del ab
    y = sl.cho_solve_banded((c, False), s.b[P], check_finite=False)
    x = np.empty_like(y)
    x[P] = y
    r = s.b - A @ x
    d = sl.cho_solve_banded((c, False), r[P], check_finite=False)
    x[P] += d
    return x


def hybrid_system(n_bodies=8, fem=(8, 8, 8), n_contacts=200, body_ratio=1e3, kappa_ratio=10.0, seed=0):
    """Affine bodies + FEM mesh, as the reference's hybrid scenes lay them out:
    each body is 12 DOF = 4 block rows, the bodies' rows come first
    (SG/GIPC.cu:10082-10083, :10217), the FEM vertices follow at
    fem_offset = 4 * n_bodies.  Body blocks: a dense SPD 12x12 (shape
    stiffness) per body, scaled body_ratio times the FEM diagonal.
    Couplings: body point x = t + A xbar against an FEM vertex, with
    J = [I | xbar1 I | xbar2 I | xbar3 I] (3x12); the pair's 15x15 block is
    kappa g g^T + eps I, g = [J^T n; -n], written as upper 3x3 blocks over
    the body's 4 rows and the vertex's row.  pos / tets describe the FEM part
    only (the MAS covers the FEM range)."""
    rng = np.random.default_rng(seed + 17)
    fs = make_grid_system(*fem, seed=seed)
    off = 4 * n_bodies
    N = fs.n_verts
    diag = fs.vals[fs.rows == fs.cols]
    dscale = float(np.mean(diag[:, [0, 4, 8]]))
    G = rng.normal(size=(n_bodies, 12, 12))
    Hb = (np.einsum("bij,bkj->bik", G, G) / 12.0 + 0.5 * np.eye(12)[None]) * dscale * body_ratio
    nodes_b = off * 0 + 4 * np.arange(n_bodies)[:, None] + np.arange(4)[None, :]
    rb, cb, vb = upper_triplets(Hb, nodes_b)
    bod = rng.integers(0, n_bodies, n_contacts)
    ver = rng.integers(0, N, n_contacts)
    xbar = rng.uniform(-1.0, 1.0, (n_contacts, 3))
    nrm = rng.normal(size=(n_contacts, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    J = np.zeros((n_contacts, 3, 12))
    J[:, :, 0:3] = np.eye(3)
    for k in range(3):
        J[:, :, 3 + 3 * k:6 + 3 * k] = xbar[:, k, None, None] * np.eye(3)[None]
    g = np.concatenate([np.einsum("pij,pi->pj", J, nrm), -nrm], 1)        # [p, 15]
    Hc = dscale * kappa_ratio * (g[:, :, None] * g[:, None, :] + 1e-3 * np.eye(15)[None])
    nodes_c = np.concatenate([4 * bod[:, None] + np.arange(4)[None, :], (off + ver)[:, None]], 1)
    rc, cc, vc = upper_triplets(Hc, nodes_c)
    rows = np.concatenate([fs.rows.astype(np.int64) + off, rb, rc])
    cols = np.concatenate([fs.cols.astype(np.int64) + off, cb, cc])
    vals = np.concatenate([fs.vals, vb, vc])
    mr, mc, mv = merge_triplets(rows, cols, vals)
    b = np.concatenate([rng.normal(size=3 * off) * float(np.abs(fs.b).mean()), fs.b])
    return System(n_verts=off + N, rows=mr, cols=mc, vals=mv, b=b, pos=fs.pos, tets=fs.tets,
                  pairs=np.zeros((0, 4), np.int32), raw_rows=rows, raw_cols=cols, raw_vals=vals,
                  info=dict(abd_bodies=n_bodies, fem_offset=off, fem_n=N))


def cst_membrane(X, tris, E, nu, thickness):
    """Linear (StVK at rest) constant-strain membrane Hessians of triangles
    lying in the x-z plane: 9x9 per triangle, in-plane (x, z) stiffness only
    (PSD; the out-of-plane direction is carried by the mass)."""
    P = X[tris][:, :, [0, 2]]                         # [t, 3, 2] in-plane coordinates
    e1, e2 = P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]
    area = 0.5 * np.abs(e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0])
    # shape-function gradients of the 3 nodes
    Dm = np.stack([e1, e2], 2)                        # [t, 2, 2]
    Dinv = np.linalg.inv(Dm)
    grads = np.zeros((len(tris), 3, 2))
    grads[:, 1] = Dinv[:, 0, :]
    grads[:, 2] = Dinv[:, 1, :]
    grads[:, 0] = -grads[:, 1] - grads[:, 2]
    # strain-displacement B [t, 3, 9] over (x, y, z) of 3 nodes; y (out of plane) unused
    Bm = np.zeros((len(tris), 3, 9))
    for a in range(3):
        gx, gz = grads[:, a, 0], grads[:, a, 1]
        Bm[:, 0, 3 * a + 0] = gx                      # eps_xx
        Bm[:, 1, 3 * a + 2] = gz                      # eps_zz
        Bm[:, 2, 3 * a + 0] = gz                      # gamma_xz
        Bm[:, 2, 3 * a + 2] = gx
    D = E / (1.0 - nu * nu) * np.array([[1.0, nu, 0.0], [nu, 1.0, 0.0], [0.0, 0.0, 0.5 * (1.0 - nu)]])
    K = np.einsum("tij,jk,tkl->til", Bm.transpose(0, 2, 1), D, Bm) * (thickness * area)[:, None, None]
    return K, area


def config3(seed=0, scale=1.0, n_bodies=200, cloth_side=200, n_pairs=80000, E_body=1e10, E_cloth=1e5,
            nu=0.3, thickness=1e-3, rho=1000.0, dt=0.01, dhat=1e-3, kappa=1e5, eps=1e-6, dmin=1e-3, chunk=8000):
    """Stiff hybrid (config 3): affine bodies resting on a cloth sheet.

    Bodies: 12-DOF affine bodies (4 block rows each, rows 0 .. 4 n_bodies,
    before the FEM rows as SG/GIPC.cu:10082-10083 places ABD), cubes of
    8x8x8 vertices; mass matrix int rho J^T J dV in the body's centroid
    frame (m I3 for the translation, m s^2/12 I9 for the affine part) plus
    dt^2 x the shape stiffness E_body * V on the symmetric part of the
    affine map.  Cloth: cloth_side^2 vertices in the x-z plane, lumped mass,
    constant-strain membrane (E_cloth, thickness).  Contacts: n_pairs barrier
    pairs between a point of a body's bottom face, x = t + A xbar
    (J = [I | xbar1 I | xbar2 I | xbar3 I]), and a cloth triangle under the
    body: 21x21 kappa b''(d) g g^T + kappa eps I, g = [J^T n; -b_k n], drawn
    as the contact benchmark's pairs: kappa = 1e5, d ~ U(0, dhat) floored at
    dmin dhat = 1e-3 dhat.  The barrier terms of a body's pairs then outweigh
    the light cloth under it by orders of magnitude: block-Jacobi and MAS
    with the bodies' 12x12 blocks stall on this matrix, the body patches
    (body_patches) converge.  scale shrinks the cloth side, the bodies and
    the pairs together."""
    rng = np.random.default_rng(seed)
    side = max(8, int(round(cloth_side * np.sqrt(scale))))
    nbod = max(1, int(round(n_bodies * scale)))
    npr = int(round(n_pairs * scale))
    hc = 0.01
    gx, gz = np.meshgrid(np.arange(side), np.arange(side), indexing="ij")
    Xc = np.stack([gx.ravel() * hc, np.zeros(side * side), gz.ravel() * hc], 1)
    Xc += rng.normal(0.0, 1e-5, Xc.shape) * np.array([1.0, 0.0, 1.0])
    vid = lambda i, k: i * side + k
    qi, qk = np.meshgrid(np.arange(side - 1), np.arange(side - 1), indexing="ij")
    qi, qk = qi.ravel(), qk.ravel()
    a, b1, c1, d1 = vid(qi, qk), vid(qi + 1, qk), vid(qi, qk + 1), vid(qi + 1, qk + 1)
    tris = np.concatenate([np.stack([a, b1, d1], 1), np.stack([a, d1, c1], 1)])
    nc = side * side
    off = 4 * nbod
    K, area = cst_membrane(Xc, tris, E_cloth, nu, thickness)
    rows, cols, vals = [], [], []
    r_el, c_el, v_el = upper_triplets(K * dt * dt, tris + off)
    rows.append(r_el); cols.append(c_el); vals.append(v_el)
    mass = np.zeros(nc)
    np.add.at(mass, tris.ravel(), np.repeat(rho * thickness * area / 3.0, 3))
    v_m = np.zeros((nc, 9))
    v_m[:, 0] = v_m[:, 4] = v_m[:, 8] = mass
    rows.append(np.arange(nc) + off); cols.append(np.arange(nc) + off); vals.append(v_m)
    # bodies: side s, centred over random cloth cells
    s_b = 0.07
    m_b = rho * s_b ** 3
    Mb = np.zeros((12, 12))
    Mb[:3, :3] = m_b * np.eye(3)
    Mb[3:, 3:] = m_b * s_b * s_b / 12.0 * np.eye(9)
    # shape stiffness on the symmetric part of A (9 affine dofs, A row-major in q[3:12])
    Psym = np.zeros((9, 9))
    for i in range(3):
        for j in range(3):
            Psym[3 * i + j, 3 * i + j] += 0.5
            Psym[3 * i + j, 3 * j + i] += 0.5
    Kb = np.zeros((12, 12))
    Kb[3:, 3:] = 4.0 * E_body * s_b ** 3 * Psym
    Ab = Mb + dt * dt * Kb
    Hb = np.repeat(Ab[None], nbod, 0) * (1.0 + 0.05 * rng.uniform(-1, 1, (nbod, 1, 1)))
    nodes_b = 4 * np.arange(nbod)[:, None] + np.arange(4)[None, :]
    rb, cb, vb = upper_triplets(Hb, nodes_b)
    rows.append(rb); cols.append(cb); vals.append(vb)
    foot = int(round(s_b / hc))                      # footprint in cells
    cx = rng.integers(0, max(1, side - 1 - foot), nbod)
    cz = rng.integers(0, max(1, side - 1 - foot), nbod)
    # contacts, in chunks (21x21 blocks)
    done = 0
    while done < npr:
        m = min(chunk, npr - done)
        bod = rng.integers(0, nbod, m)
        ti = cx[bod] + rng.integers(0, foot, m)
        tk = cz[bod] + rng.integers(0, foot, m)
        which = rng.integers(0, 2, m)
        qid = ti * (side - 1) + tk
        tri = tris[which * (side - 1) * (side - 1) + qid]
        xbar = np.stack([rng.uniform(-0.5, 0.5, m) * s_b, np.full(m, -0.5 * s_b), rng.uniform(-0.5, 0.5, m) * s_b], 1)
        J = np.zeros((m, 3, 12))
        J[:, :, 0:3] = np.eye(3)
        for k in range(3):
            J[:, :, 3 + 3 * k:6 + 3 * k] = xbar[:, k, None, None] * np.eye(3)[None]
        nrm = np.tile([0.0, 1.0, 0.0], (m, 1)) + rng.normal(0.0, 0.05, (m, 3))
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        bary = rng.dirichlet(np.ones(3), m)
        d = np.maximum(rng.uniform(0.0, dhat, m), dhat * dmin)
        bpp = (-2.0 * np.log(d / dhat) - 4.0 * (d - dhat) / d + (d - dhat) ** 2 / d ** 2)
        g = np.concatenate([np.einsum("pij,pi->pj", J, nrm), -bary[:, 0:1] * nrm, -bary[:, 1:2] * nrm,
                            -bary[:, 2:3] * nrm], 1)
        H = (kappa * bpp)[:, None, None] * g[:, :, None] * g[:, None, :] + kappa * eps * np.eye(21)[None]
        H *= dt * dt
        nodes = np.concatenate([4 * bod[:, None] + np.arange(4)[None, :], tri + off], 1)
        r_c, c_c, v_c = upper_triplets(H, nodes)
        rows.append(r_c); cols.append(c_c); vals.append(v_c)
        done += m
    raw_r = np.concatenate(rows).astype(np.int64)
    raw_c = np.concatenate(cols).astype(np.int64)
    raw_v = np.concatenate(vals)
    mr, mc, mv = merge_triplets(raw_r, raw_c, raw_v)
    n = off + nc
    grav = np.zeros((n, 3))
    grav[:off:4, 1] = -9.8 * m_b * dt                 # body translation rows
    grav[off:, 1] = -9.8 * mass * dt
    b = grav.ravel() + rng.normal(0.0, 1e-6, 3 * n)
    return System(n_verts=n, rows=mr, cols=mc, vals=mv, b=b, pos=Xc, tets=np.zeros((0, 4), np.int32),
                  pairs=np.zeros((0, 4), np.int32),
                  info=dict(abd_bodies=nbod, fem_offset=off, fem_n=nc, tris=tris.astype(np.int32),
                            n_pairs=npr, n_blocks=len(mr), side=side, dt=dt))


def stencil_grid_system(nx, ny, nz, h=0.01, E=1e5, nu=0.4, rho=1000.0, dt=0.01, n_pairs=0, dhat=1e-3,
                        kappa=1e5, eps=1e-6, seed=0):
    """A tet grid system assembled directly in merged (stencil) form.

    The grid is regular, so each of the 6 tets of a cube has the same
    rest-state stiffness (the Neo-Hookean Hessian at F = I, PSD-projected):
    each tet type's 3x3 blocks are added into per-offset block arrays by
    slicing, and the sorted upper BCOO is read off the stencil -- no element
    loop, no triplet sort (used for the many large systems of config 5).
    n_pairs barrier pairs couple top-face points to nearby top-face
    triangles (12x12 blocks, merged in), with their reference int4 encoding."""
    rng = np.random.default_rng(seed)
    # one cube's 6 tets at rest
    Xc, tc = tet_grid(2, 2, 2, h)
    He, _, vol = neo_hookean_elements(Xc, Xc, tc, E, nu)
    He = He * dt * dt
    n = nx * ny * nz
    strides = np.array([1, nx, nx * ny])
    cub = (nx - 1, ny - 1, nz - 1)
    blocks = {}   # offset delta >= 0 -> [nz, ny, nx, 3, 3] (row vertex grid)

    def add(delta, dr, blk):
        a = blocks.setdefault(delta, np.zeros((nz, ny, nx, 3, 3)))
        a[dr[2]:dr[2] + cub[2], dr[1]:dr[1] + cub[1], dr[0]:dr[0] + cub[0]] += blk

    for t in range(6):
        cs = _TET_SPLIT[t]
        for ii in range(4):
            for jj in range(ii, 4):
                da, db = _CORNER[cs[ii]], _CORNER[cs[jj]]
                va, vb = int(da @ strides), int(db @ strides)
                B = He[t, 3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3]
                if va <= vb:
                    add(vb - va, da, B if va != vb else B)
                else:
                    add(va - vb, db, B.T)
    # lumped mass on the diagonal
    m_cube = rho * vol.sum() / 4.0   # each tet gives vol/4 to each of its 4 vertices
    mass = np.zeros((nz, ny, nx))
    for t in range(6):
        for ii in range(4):
            d = _CORNER[_TET_SPLIT[t][ii]]
            mass[d[2]:d[2] + cub[2], d[1]:d[1] + cub[1], d[0]:d[0] + cub[0]] += rho * vol[t] / 4.0
    del m_cube
    blocks[0] = blocks[0] + mass[..., None, None] * np.eye(3)
    # read the upper BCOO off the stencil: rows ascending, then offsets ascending
    deltas = sorted(blocks)
    vidx = np.arange(n)
    rows, cols, vals = [], [], []
    touched = {d: np.abs(blocks[d]).reshape(n, 9).max(1) > 0 for d in deltas}
    for d in deltas:
        ok = touched[d]
        rows.append(vidx[ok])
        cols.append(vidx[ok] + d)
        vals.append(np.swapaxes(blocks[d].reshape(n, 3, 3)[ok], 1, 2).reshape(-1, 9))  # column-major
    r = np.concatenate(rows); c = np.concatenate(cols); v = np.concatenate(vals)
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    X = tet_grid(nx, ny, nz, h)[0]
    pairs = np.zeros((0, 4), np.int32)
    if n_pairs > 0:
        # top face (y = ny - 1): points against triangles of nearby quads
        gx, gz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
        top = lambda x_, z_: x_ + nx * ((ny - 1) + ny * z_)
        pi = rng.integers(0, nx * nz, n_pairs)
        px, pz = gx.ravel()[pi], gz.ravel()[pi]
        qx = np.clip(px + rng.integers(-2, 2, n_pairs), 0, nx - 2)
        qz = np.clip(pz + rng.integers(-2, 2, n_pairs), 0, nz - 2)
        a0, b0, c0, d0 = top(qx, qz), top(qx + 1, qz), top(qx, qz + 1), top(qx + 1, qz + 1)
        w = rng.integers(0, 2, n_pairs)
        tri = np.where(w[:, None] == 0, np.stack([a0, b0, d0], 1), np.stack([a0, d0, c0], 1))
        pt = top(px, pz)
        keep = (pt != tri[:, 0]) & (pt != tri[:, 1]) & (pt != tri[:, 2])
        pt, tri = pt[keep], tri[keep]
        m = len(pt)
        d_ = np.maximum(rng.uniform(0.0, dhat, m), dhat * 1e-2)
        normal = np.tile([0.0, 1.0, 0.0], (m, 1)) + rng.normal(0.0, 0.05, (m, 3))
        normal /= np.linalg.norm(normal, axis=1, keepdims=True)
        bary = rng.dirichlet(np.ones(3), m)
        Hc = barrier_hessian(d_, dhat, kappa, eps, normal, bary, rng) * dt * dt
        nodes = np.stack([pt, tri[:, 0], tri[:, 1], tri[:, 2]], 1)
        r_c, c_c, v_c = upper_triplets(Hc, nodes)
        r, c, v = merge_triplets(np.concatenate([r, r_c]), np.concatenate([c, c_c]), np.concatenate([v, v_c]))
        pairs = np.stack([-(nodes[:, 0] + 1), nodes[:, 1], nodes[:, 2], nodes[:, 3]], 1).astype(np.int32)
    b = rng.normal(0.0, 1.0, 3 * n) * float(np.median(v[r == c][:, 0])) * 1e-3
    _, tets = tet_grid(nx, ny, nz, h)
    return System(n_verts=n, rows=r.astype(np.int32), cols=c.astype(np.int32), vals=v, b=b, pos=X,
                  tets=tets.astype(np.int32), pairs=pairs,
                  info=dict(nx=nx, ny=ny, nz=nz, E=E, n_pairs=len(pairs), n_blocks=len(r)))


def config5(seed=0, n_scenes=64, nmin=2000, nmax=200000, scale=1.0):
    """Batched serving of uneven scenes (config 5): n_scenes tet grids with
    vertex counts log-uniform in [nmin, nmax] * scale, E log-uniform in
    [1e4, 1e8], barrier pairs 0 to 20 % of the vertices."""
    rng = np.random.default_rng(seed)
    scenes = []
    for k in range(n_scenes):
        N = float(np.exp(rng.uniform(np.log(nmin * scale), np.log(nmax * scale))))
        # box with aspect 2:1:1
        side = (N / 2.0) ** (1.0 / 3.0)
        nx, ny, nz = max(3, int(round(2 * side))), max(3, int(round(side))), max(3, int(round(side)))
        E = float(np.exp(rng.uniform(np.log(1e4), np.log(1e8))))
        npairs = int(rng.uniform(0.0, 0.2) * nx * ny * nz)
        scenes.append(stencil_grid_system(nx, ny, nz, E=E, n_pairs=min(npairs, 4 * nx * nz), seed=seed * 1000 + k))
    return scenes
