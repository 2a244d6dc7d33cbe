"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs as the checker.  The product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


class PCGCfg(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("rel_tol", C.c_double), ("abs_tol", C.c_double),
                ("use_preconditioned_norm", C.c_int), ("precond", C.c_int),
                ("abd_bodies", C.c_int), ("fem_offset", C.c_int), ("nthreads", C.c_int),
                ("initial_guess", C.c_int)]


class PCGReport(C.Structure):
    _fields_ = [("iterations", C.c_int), ("rel_residual", C.c_double), ("rz0", C.c_double),
                ("rr0", C.c_double), ("ms", C.c_double), ("x0_scale", C.c_double), ("x0_rejected", C.c_int)]


def build():
    """Compile the oracle with gcc (no FMA contraction; OpenMP for the timed arm)."""
    src = os.path.join(_HERE, "sgmas_oracle.c")
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-o", _LIB_PATH, src, "-lm"]
    subprocess.check_call(cmd)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(_HERE, "sgmas_oracle.c")
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        build()
    L = C.CDLL(_LIB_PATH)
    L.or_mas_partition.argtypes = [i32p, C.c_int, C.c_int, C.POINTER(C.c_int), i32p, C.c_int, i32p]
    L.or_vert_neighbors.argtypes = [i32p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, u32p, u32p, u32p, C.c_int]
    L.or_num_levels.argtypes = [C.c_int, C.c_int]
    L.or_hash_code.argtypes = [C.c_double] * 4
    L.or_hash_code.restype = C.c_uint32
    L.or_vert_morton.argtypes = [f64p, C.c_int, u64p]
    L.or_spmv_sym.argtypes = [C.c_double, f64p, i32p, i32p, C.c_int, f64p, C.c_double, f64p, C.c_int]
    L.or_dot.argtypes = [f64p, f64p, C.c_int]
    L.or_dot.restype = C.c_double
    L.or_convert.argtypes = [f64p, i32p, i32p, C.c_int, f64p, i32p, i32p]
    L.or_write_upper_blocks.argtypes = [f64p, C.c_int, i32p, f64p, i32p, i32p]
    L.or_mas_create.argtypes = [C.c_int, C.c_int, C.c_int, u32p, C.c_int, u32p, u32p, i32p, C.c_int, i32p]
    L.or_mas_create.restype = C.c_void_p
    L.or_mas_destroy.argtypes = [C.c_void_p]
    L.or_mas_reorder.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    L.or_mas_levelnum.argtypes = [C.c_void_p]
    L.or_mas_total_clusters.argtypes = [C.c_void_p]
    L.or_mas_get_tables.argtypes = [C.c_void_p, u32p, i32p, i32p, C.c_int, i32p, i32p, i32p]
    L.or_mas_assemble.argtypes = [C.c_void_p, f64p, i32p, i32p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    L.or_mas_get_matrices.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.or_mas_invert_blocks.argtypes = [f64p, C.c_int, C.c_int, f64p]
    L.or_mas_factor_blocks.argtypes = [f64p, C.c_int, C.c_int, f64p]
    L.or_mas_set_hess.argtypes = [C.c_void_p, f64p, C.c_int]
    L.or_mas_apply.argtypes = [C.c_void_p, f64p, f64p]
    L.or_pcg.argtypes = [f64p, i32p, i32p, C.c_int, C.c_int, f64p, f64p, C.POINTER(PCGCfg),
                         C.c_void_p, C.POINTER(PCGReport)]
    L.or_bf16_round.argtypes = [f64p, C.c_int, f32p]
    L.or_omp_max_threads.argtypes = []
    _lib = L
    return L


def c32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def cf64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def mas_partition(part_id, bank=16):
    """setMAS_partition: part ids -> (part_map, real_map); raises on bad input."""
    part_id = c32(part_id)
    n = len(part_id)
    cap = (int(part_id.max()) + 1) * bank
    pm = np.empty(cap, np.int32)
    rm = np.empty(n, np.int32)
    po = C.c_int(0)
    rc = lib().or_mas_partition(part_id, n, bank, C.byref(po), pm, cap, rm)
    if rc != 0:
        raise ValueError(f"or_mas_partition failed: {rc}")
    return pm[: po.value * bank].copy(), rm


def vert_neighbors(tets, n_verts, tris=None, abd_vert_offset=0):
    tets = c32(tets).reshape(-1)
    ntet = len(tets) // 4
    if tris is not None and len(tris):
        tris = c32(tris).reshape(-1)
        ntri = len(tris) // 3
        tris_p = tris.ctypes.data_as(C.c_void_p)
    else:
        ntri, tris_p = 0, None
    cap = 12 * ntet + 6 * ntri + 16
    st = np.zeros(n_verts, np.uint32)
    nn = np.zeros(n_verts, np.uint32)
    nl = np.zeros(cap, np.uint32)
    size = lib().or_vert_neighbors(tets, ntet, tris_p, ntri, n_verts, abd_vert_offset, st, nn, nl, cap)
    if size < 0:
        raise ValueError(f"or_vert_neighbors failed: {size}")
    return st, nn, nl[:size].copy()


def morton_codes(pos):
    pos = cf64(pos).reshape(-1)
    n = len(pos) // 3
    out = np.zeros(n, np.uint64)
    lib().or_vert_morton(pos, n, out)
    return out


def morton_partition(pos, bank=16):
    """Morton order -> contiguous chunks of `bank` vertices -> (part_map, real_map)."""
    codes = morton_codes(pos)
    order = np.argsort(codes, kind="stable").astype(np.int32)
    n = len(order)
    nparts = (n + bank - 1) // bank
    pm = np.full(nparts * bank, -1, np.int32)
    pm[:n] = order
    rm = np.empty(n, np.int32)
    rm[order] = np.arange(n, dtype=np.int32)
    return pm, rm


def spmv_sym(a, vals, rows, cols, x, b=0.0, y=None):
    x = cf64(x)
    y = np.zeros_like(x) if y is None else cf64(y).copy()
    lib().or_spmv_sym(a, cf64(vals).reshape(-1), c32(rows), c32(cols), len(rows), x, b, y, len(x))
    return y


def convert(vals, rows, cols):
    n = len(rows)
    ov = np.zeros((n, 9))
    orr = np.zeros(n, np.int32)
    oc = np.zeros(n, np.int32)
    u = lib().or_convert(cf64(vals).reshape(-1), c32(rows), c32(cols), n, ov.reshape(-1), orr, oc)
    return orr[:u].copy(), oc[:u].copy(), ov[:u].copy()


def bf16_round(x):
    x = cf64(x).reshape(-1)
    out = np.empty(len(x), np.float32)
    lib().or_bf16_round(x, len(x), out)
    return out


class MAS:
    """The oracle MAS preconditioner over one FEM range."""

    def __init__(self, n_verts, nb_start, nb_num, nb_list, part_map, real_map, bank=16, node_offset=0):
        L = lib()
        self.n = n_verts
        self.bank = bank
        self.Mm = len(part_map)
        self.h = L.or_mas_create(bank, n_verts, node_offset, np.ascontiguousarray(nb_list, np.uint32),
                                 len(nb_list), np.ascontiguousarray(nb_start, np.uint32),
                                 np.ascontiguousarray(nb_num, np.uint32), c32(part_map), len(part_map),
                                 c32(real_map))
        if not self.h:
            raise ValueError("or_mas_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_mas_destroy(self.h)
            self.h = None

    @property
    def levelnum(self):
        return lib().or_mas_levelnum(self.h)

    @property
    def total(self):
        return lib().or_mas_total_clusters(self.h)

    def reorder(self, pairs=None):
        if pairs is not None and len(pairs):
            p = c32(pairs).reshape(-1)
            self._pairs = p
            return lib().or_mas_reorder(self.h, p.ctypes.data_as(C.c_void_p), len(p) // 4)
        return lib().or_mas_reorder(self.h, None, 0)

    def tables(self):
        Ln = self.levelnum
        fm = np.zeros(self.n, np.uint32)
        cs = np.zeros(self.n * Ln, np.int32)
        gn = np.zeros(max(self.total, self.n) + 1, np.int32)
        ls = np.zeros(2 * (Ln + 1), np.int32)
        po = np.zeros(self.Mm // self.bank, np.int32)
        ct = np.zeros(self.n * 6, np.int32)
        lib().or_mas_get_tables(self.h, fm, cs, gn, len(gn), ls, po, ct)
        return dict(fine_mask=fm, coarse_space=cs.reshape(Ln, self.n), going_next=gn,
                    level_size=ls.reshape(Ln + 1, 2), prefix_orig=po, coarse_table=ct.reshape(self.n, 6))

    def assemble(self, vals, rows, cols, offset=0, indices=None, precision=0):
        ip = None
        if indices is not None:
            self._idx = np.ascontiguousarray(indices, np.uint32)
            ip = self._idx.ctypes.data_as(C.c_void_p)
        self._vals = cf64(vals).reshape(-1)
        n = len(rows) if indices is None else len(self._idx)  # with indices: their count (as the reference's triplet_num)
        rc = lib().or_mas_assemble(self.h, self._vals, c32(rows), c32(cols), ip, offset, n, precision)
        if rc != 0:
            raise ValueError("or_mas_assemble failed")

    def matrices(self):
        nblk = self.total // self.bank
        bs = self.bank * (self.bank + 1) // 2
        h = np.zeros(nblk * bs * 9)
        i64 = np.zeros(nblk * bs * 9)
        i32 = np.zeros(nblk * bs * 9, np.float32)
        lib().or_mas_get_matrices(self.h, h.ctypes.data_as(C.c_void_p), i64.ctypes.data_as(C.c_void_p),
                                  i32.ctypes.data_as(C.c_void_p))
        return h, i64, i32

    def set_hess(self, hess, precision=0):
        if lib().or_mas_set_hess(self.h, cf64(hess), precision) != 0:
            raise ValueError("assemble first")

    def apply(self, r):
        r = cf64(r)
        z = np.zeros_like(r)
        lib().or_mas_apply(self.h, r, z)
        return z


def invert_blocks(hess, nblocks, bank=16):
    out = np.zeros_like(cf64(hess))
    lib().or_mas_invert_blocks(cf64(hess), nblocks, bank, out)
    return out


def factor_blocks(hess, nblocks, bank=16):
    """W = L^-1 per subdomain matrix, in the tile slots (the library's factored storage)."""
    out = np.zeros_like(cf64(hess))
    lib().or_mas_factor_blocks(cf64(hess), nblocks, bank, out)
    return out


def pcg(s_vals, rows, cols, nrows, b, precond=1, rel_tol=1e-4, abs_tol=0.0, max_iter=0,
        use_preconditioned_norm=False, mas=None, fem_offset=0, abd_bodies=0, nthreads=1, x0=None):
    """x0: a start guess (scaled by x0.b / x0.A x0, rejected when it raises
    the residual, convergence against ||b||); None = x0 = 0 (the reference)."""
    cfg = PCGCfg(max_iter, rel_tol, abs_tol, int(use_preconditioned_norm), precond, abd_bodies,
                 fem_offset, nthreads, int(x0 is not None))
    rep = PCGReport()
    b = cf64(b)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64, copy=True)
    lib().or_pcg(cf64(s_vals).reshape(-1), c32(rows), c32(cols), len(rows), nrows, b, x,
                 C.byref(cfg), mas.h if mas is not None else None, C.byref(rep))
    return x, dict(iterations=rep.iterations, rel_residual=rep.rel_residual, ms=rep.ms,
                   rz0=rep.rz0, rr0=rep.rr0, x0_scale=rep.x0_scale, x0_rejected=rep.x0_rejected)
