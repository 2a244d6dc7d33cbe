"""Python binding of libsgmas (the C-ABI in include/sgmas.h) via ctypes.

Device arrays are passed as objects with ``data_ptr()`` (torch tensors) or as
raw integer addresses; host arrays are numpy.  Torch is used only for device
memory and streams.  There is no CPU fallback: if the library is missing or no
GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

LIB_PATH = _build.LIB_PATH
_lib = None

SGMAS_MAS_FP32, SGMAS_MAS_BF16, SGMAS_MAS_FP64, SGMAS_MAS_FP32_FACTORED = 0, 1, 2, 3
# fp32: explicit inverses as the reference; bf16 / fp32f: factored inverses W = L^-1
PRECISION = {"fp32": 0, "bf16": 1, "fp64": 2, "fp32f": 3}


class SgmasError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"sgmas error {code}: {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("bank_size", C.c_int), ("mas_precision", C.c_int)]


class PcgConfig(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("rel_tol", C.c_double), ("abs_tol", C.c_double),
                ("use_preconditioned_norm", C.c_int), ("preconditioner", C.c_int),
                ("abd_bodies", C.c_int), ("fem_offset", C.c_int), ("check_every", C.c_int),
                ("initial_guess", C.c_int), ("body_patches", C.c_int)]


class PcgReport(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("rz0", C.c_double), ("rr0", C.c_double),
                ("rr_last", C.c_double), ("solve_ms", C.c_float), ("precond_ms", C.c_float),
                ("kernel_launches", C.c_int), ("build_launches", C.c_int), ("x0_rejected", C.c_int),
                ("x0_scale", C.c_double), ("rr_x0", C.c_double), ("bb", C.c_double)]


TUNE_MAX = 16  # SGMAS_TUNE_MAX_CANDIDATES in include/sgmas.h


class TuneReport(C.Structure):
    _fields_ = [("n_candidates", C.c_int), ("ctas", C.c_int * TUNE_MAX), ("persistent", C.c_int * TUNE_MAX),
                ("us_per_iter", C.c_double * TUNE_MAX), ("cost", C.c_double * TUNE_MAX), ("chosen", C.c_int),
                ("sms", C.c_int)]


class ElementGroup(C.Structure):
    _fields_ = [("d_H", C.c_void_p), ("d_nodes", C.c_void_p), ("n_elem", C.c_int), ("nodes_per_elem", C.c_int)]


class Bcoo(C.Structure):
    _fields_ = [("d_values", C.c_void_p), ("d_rows", C.c_void_p), ("d_cols", C.c_void_p),
                ("n_blocks", C.c_int), ("n_block_rows", C.c_int)]


EXPORTS = [
    "sgmas_create", "sgmas_destroy", "sgmas_last_error", "sgmas_set_stream", "sgmas_synchronize",
    "sgmas_mas_init", "sgmas_mas_set_contacts", "sgmas_mas_assemble", "sgmas_mas_apply", "sgmas_mas_info",
    "sgmas_mas_download_tables", "sgmas_mas_download_matrices", "sgmas_mas_invert_host",
    "sgmas_pcg_solve", "sgmas_pcg_solve_host", "sgmas_spmv", "sgmas_convert", "sgmas_write_upper_blocks",
    "sgmas_morton_codes", "sgmas_morton_partition", "sgmas_pcg_profile", "sgmas_vert_neighbors",
    "sgmas_part_maps", "sgmas_morton_codes_noalloc", "sgmas_set_pcg_mode", "sgmas_pcg_last_vectors",
    "sgmas_mtx_write", "sgmas_mtx_read", "sgmas_set_pcg_ctas", "sgmas_set_wait_limit", "sgmas_mlp_set_params", "sgmas_mlp_get_params", "sgmas_mlp_features",
    "sgmas_mlp_gradient", "sgmas_mlp_train_step", "sgmas_mlp_forward", "sgmas_mlp_warm_start",
    "sgmas_autotune_pcg", "sgmas_assembly_plan", "sgmas_assemble", "sgmas_element_plan", "sgmas_element_assemble", "sgmas_append_triplets", "sgmas_abd_body_blocks",
    "sgmas_abd_pair_blocks", "sgmas_abd_fem_blocks",
]
MLP_PARAMS = 19462  # SGMAS_MLP_PARAMS in include/sgmas.h

MORTON_NOALLOC_MAX_VERTS = 2097152  # SGMAS_MORTON_NOALLOC_MAX_VERTS in include/sgmas.h


def lib(build_if_missing: bool = False):
    """Load libsgmas.so (built in-tree by sgmas.build / __graft_entry__.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise SgmasError(-2, f"{LIB_PATH} is missing: run __graft_entry__.build()")
        _build.build()
    L = C.CDLL(LIB_PATH)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.sgmas_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
    L.sgmas_destroy.argtypes = [vp]
    L.sgmas_destroy.restype = None
    L.sgmas_last_error.argtypes = [vp]
    L.sgmas_last_error.restype = C.c_char_p
    L.sgmas_set_stream.argtypes = [vp, vp]
    L.sgmas_synchronize.argtypes = [vp]
    L.sgmas_mas_init.argtypes = [vp, i, i, i, vp, vp, vp, vp, i, vp]
    L.sgmas_mas_set_contacts.argtypes = [vp, vp, i]
    L.sgmas_mas_assemble.argtypes = [vp, vp, vp, vp, vp, i, i, i]
    L.sgmas_mas_apply.argtypes = [vp, vp, vp]
    L.sgmas_mas_info.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
    L.sgmas_mas_download_tables.argtypes = [vp, vp, vp, vp, i, vp, vp, vp]
    L.sgmas_mas_download_matrices.argtypes = [vp, vp, vp]
    L.sgmas_mas_invert_host.argtypes = [vp, vp, i, vp]
    L.sgmas_pcg_solve.argtypes = [vp, C.POINTER(Bcoo), vp, vp, C.POINTER(PcgConfig), C.POINTER(PcgReport)]
    L.sgmas_pcg_solve_host.argtypes = [vp, vp, vp, vp, i, i, vp, vp, C.POINTER(PcgConfig), C.POINTER(PcgReport)]
    L.sgmas_spmv.argtypes = [vp, d, C.POINTER(Bcoo), vp, d, vp]
    L.sgmas_convert.argtypes = [vp, vp, vp, vp, i, vp, vp, vp, C.POINTER(i)]
    L.sgmas_write_upper_blocks.argtypes = [vp, vp, i, i, vp, vp, vp, vp]
    L.sgmas_morton_codes.argtypes = [vp, vp, i, vp, vp]
    L.sgmas_morton_partition.argtypes = [vp, vp, i, vp, i, C.POINTER(i), vp]
    L.sgmas_pcg_profile.argtypes = [vp, i, vp, i]
    L.sgmas_vert_neighbors.argtypes = [vp, i, vp, i, i, i, vp, vp, vp, i]
    L.sgmas_part_maps.argtypes = [vp, i, i, vp, i, C.POINTER(i), vp]
    L.sgmas_morton_codes_noalloc.argtypes = [vp, i, vp, vp, vp]
    L.sgmas_set_pcg_mode.argtypes = [vp, i]
    L.sgmas_set_pcg_ctas.argtypes = [vp, i]
    L.sgmas_set_wait_limit.argtypes = [vp, i, i]
    L.sgmas_autotune_pcg.argtypes = [vp, C.POINTER(Bcoo), vp, C.POINTER(PcgConfig), i, i, i, i, C.POINTER(TuneReport)]
    L.sgmas_pcg_last_vectors.argtypes = [vp, vp, vp]
    L.sgmas_assembly_plan.argtypes = [vp, vp, vp, i, vp, vp, C.POINTER(i)]
    L.sgmas_assemble.argtypes = [vp, vp, i, vp]
    L.sgmas_element_plan.argtypes = [vp, C.POINTER(ElementGroup), i, vp, vp, C.POINTER(i)]
    L.sgmas_append_triplets.argtypes = [vp, vp, vp, vp, i, vp, vp, vp, i, vp, vp, vp, C.POINTER(i)]
    L.sgmas_element_assemble.argtypes = [vp, C.POINTER(ElementGroup), i, vp]
    L.sgmas_abd_body_blocks.argtypes = [vp, vp, i, vp, vp, vp]
    L.sgmas_abd_pair_blocks.argtypes = [vp, vp, vp, vp, i, vp, vp, vp, vp, vp, vp]
    L.sgmas_abd_fem_blocks.argtypes = [vp, vp, vp, vp, i, vp, vp, vp, vp, i, i, vp, vp, vp]
    L.sgmas_mtx_write.argtypes = [C.c_char_p, C.c_char_p, vp, vp, vp, i, i, vp]
    L.sgmas_mtx_read.argtypes = [C.c_char_p, C.c_char_p, vp, vp, vp, i, vp, i, C.POINTER(i), C.POINTER(i)]
    f = C.c_float
    L.sgmas_mlp_set_params.argtypes = [vp, vp, i]
    L.sgmas_mlp_get_params.argtypes = [vp, vp, i]
    L.sgmas_mlp_features.argtypes = [vp, C.POINTER(Bcoo), vp, vp, vp, i, vp, vp, vp, vp]
    L.sgmas_mlp_gradient.argtypes = [vp, vp, vp, vp, i, f, vp, C.POINTER(f)]
    L.sgmas_mlp_train_step.argtypes = [vp, vp, vp, vp, i, f, f, C.POINTER(f)]
    L.sgmas_mlp_forward.argtypes = [vp, vp, i, i, vp]
    L.sgmas_mlp_warm_start.argtypes = [vp, C.POINTER(Bcoo), vp, vp, i, vp, vp]
    _lib = L
    return L


def morton_codes_noalloc(pos, codes, aabb=None, stream=None, n=None):
    """Morton codes without any device allocation (sgmas_morton_codes_noalloc).

    For callers that may not allocate device memory (a host whose device
    memory comes from its own pool, a loop that must not allocate once it
    runs).  Runs on the current device; returns the C status code (0 = ok,
    SGMAS_ERR_CAPACITY = -4 when n exceeds MORTON_NOALLOC_MAX_VERTS)."""
    box = None if aabb is None else _h(aabb, np.float64)
    count = int(pos.shape[0]) if n is None else n
    return lib().sgmas_morton_codes_noalloc(_ptr(pos), count, _ptr(box), _ptr(codes), stream)


def mtx_write(path_A, vals, rows, cols, n_block_rows, b=None, path_b=None):
    """Write a host BCOO (and b) in the reference's MatrixMarket export format."""
    vals, rows, cols = _h(vals, np.float64), _h(rows, np.int32), _h(cols, np.int32)
    bb = None if b is None else _h(b, np.float64)
    rc = lib().sgmas_mtx_write(str(path_A).encode(), None if path_b is None else str(path_b).encode(), _ptr(vals),
                               _ptr(rows), _ptr(cols), len(rows), n_block_rows, _ptr(bb))
    if rc != 0:
        raise SgmasError(rc, lib().sgmas_last_error(None).decode())


def mtx_read(path_A, path_b=None):
    """Read MatrixMarket A (and b) into an upper sorted BCOO: (vals, rows, cols, n_block_rows, b)."""
    L = lib()
    nb, nr = C.c_int(), C.c_int()
    pa, pb = str(path_A).encode(), None if path_b is None else str(path_b).encode()
    rc = L.sgmas_mtx_read(pa, pb, None, None, None, 0, None, 0, C.byref(nb), C.byref(nr))
    if rc not in (0, -4):
        raise SgmasError(rc, L.sgmas_last_error(None).decode())
    vals = np.zeros((nb.value, 9))
    rows = np.zeros(nb.value, np.int32)
    cols = np.zeros(nb.value, np.int32)
    b = np.zeros(3 * nr.value) if path_b is not None else None
    rc = L.sgmas_mtx_read(pa, pb, _ptr(vals), _ptr(rows), _ptr(cols), nb.value, _ptr(b), 0 if b is None else len(b),
                          C.byref(nb), C.byref(nr))
    if rc != 0:
        raise SgmasError(rc, L.sgmas_last_error(None).decode())
    return vals, rows, cols, nr.value, b


def vert_neighbors(tets, n_verts, tris=None, abd_vert_offset=0):
    """Neighbour CSR of a tet (+ triangle) mesh (host; getVertNeighbors)."""
    tets = _h(tets, np.int32).reshape(-1)
    tris = None if tris is None or len(tris) == 0 else _h(tris, np.int32).reshape(-1)
    ntet, ntri = len(tets) // 4, 0 if tris is None else len(tris) // 3
    cap = 12 * ntet + 6 * ntri + 16
    st = np.zeros(n_verts, np.uint32)
    nn = np.zeros(n_verts, np.uint32)
    nl = np.zeros(cap, np.uint32)
    rc = lib().sgmas_vert_neighbors(_ptr(tets), ntet, _ptr(tris), ntri, n_verts, abd_vert_offset, _ptr(st),
                                    _ptr(nn), _ptr(nl), cap)
    if rc < 0:
        raise SgmasError(rc, "sgmas_vert_neighbors failed")
    return st, nn, nl[:rc].copy()


def part_maps(part_id, bank=16):
    """Slot maps from per-vertex part ids (host; setMAS_partition)."""
    part_id = _h(part_id, np.int32)
    cap = (int(part_id[-1]) + 1) * bank
    pm = np.zeros(cap, np.int32)
    rm = np.zeros(len(part_id), np.int32)
    size = C.c_int()
    rc = lib().sgmas_part_maps(_ptr(part_id), len(part_id), bank, _ptr(pm), cap, C.byref(size), _ptr(rm))
    if rc != 0:
        raise SgmasError(rc, "sgmas_part_maps: parts must be contiguous, <= bank vertices each")
    return pm[: size.value], rm


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return x.data_ptr()


def _h(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def pcg_config(max_iter=0, rel_tol=1e-4, abs_tol=0.0, use_preconditioned_norm=False, preconditioner="mas",
               abd_bodies=0, fem_offset=0, check_every=10, initial_guess=False, body_patches=False):
    """initial_guess=True: x holds a start guess x0 on entry (scaled by
    x0.b / x0.A x0, rejected when it raises the residual; convergence is then
    tested against ||b||).  body_patches=True: each affine body's block is
    widened to the body plus the FEM vertices it touches (sgmas.h)."""
    pc = {"jacobi": 0, "mas": 1, 0: 0, 1: 1}[preconditioner]
    return PcgConfig(max_iter, rel_tol, abs_tol, int(use_preconditioned_norm), pc, abd_bodies, fem_offset,
                     check_every, int(bool(initial_guess)), int(bool(body_patches)))


class Context:
    """One sgmas_context: a MAS preconditioner + PCG solver on one GPU."""

    def __init__(self, device=0, bank=16, precision="fp32"):
        self.L = lib()
        self.h = C.c_void_p()
        cfg = Config(device, bank, PRECISION.get(precision, precision))
        rc = self.L.sgmas_create(C.byref(cfg), C.byref(self.h))
        if rc != 0:
            raise SgmasError(rc, "sgmas_create failed (no CUDA device?)")
        self.bank = bank
        self.precision = precision
        self._keep = {}

    def close(self):
        if self.h:
            self.L.sgmas_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise SgmasError(rc, self.L.sgmas_last_error(self.h).decode())

    def set_stream(self, stream_ptr):
        self._check(self.L.sgmas_set_stream(self.h, stream_ptr))

    def pcg_last_vectors(self, r=None, z=None):
        """Copy the last solve's residual r and z = M^-1 r into device arrays."""
        self._check(self.L.sgmas_pcg_last_vectors(self.h, _ptr(r), _ptr(z)))

    def set_pcg_mode(self, mode):
        """'persistent' (one cooperative kernel, default) or 'graph' (a kernel per phase)."""
        self._check(self.L.sgmas_set_pcg_mode(self.h, {"graph": 0, "persistent": 1}[mode]))

    def set_pcg_ctas(self, max_ctas):
        """Cap the persistent kernel's CTAs (0 = one per SM): small systems on a
        few SMs leave the rest to concurrent solves on other streams."""
        self._check(self.L.sgmas_set_pcg_ctas(self.h, int(max_ctas)))

    def set_wait_limit(self, spin_limit=0, phantom_arrivals=0):
        """Polls per device-side wait of the persistent kernel (0 = default);
        phantom_arrivals > 0 injects a grid barrier that never completes
        (tests of the timeout path)."""
        self._check(self.L.sgmas_set_wait_limit(self.h, int(spin_limit), int(phantom_arrivals)))

    def autotune(self, vals, rows, cols, n_block_rows, b, objective="throughput", concurrency=1, trial_iters=30,
                 reps=2, **cfg):
        """Time trial solves of the persistent form on candidate grids and of the
        graph form; keep the best for `objective` ('latency': least time per
        iteration; 'throughput': least SM-time per iteration with `concurrency`
        solves sharing the GPU, each charged at least SMs / concurrency) on this context.
        Returns the candidates: a list of dicts (ctas, persistent, us_per_iter,
        cost) and the index of the choice."""
        A = self.bcoo(vals, rows, cols, n_block_rows)
        c = pcg_config(**cfg)
        rep = TuneReport()
        obj = {"latency": 0, "throughput": 1}[objective]
        self._check(self.L.sgmas_autotune_pcg(self.h, C.byref(A), _ptr(b), C.byref(c), obj, int(concurrency),
                                              int(trial_iters), int(reps), C.byref(rep)))
        cands = [dict(ctas=rep.ctas[i], persistent=bool(rep.persistent[i]), us_per_iter=rep.us_per_iter[i],
                      cost=rep.cost[i]) for i in range(rep.n_candidates)]
        return {"candidates": cands, "chosen": rep.chosen, "sms": rep.sms}

    def synchronize(self):
        self._check(self.L.sgmas_synchronize(self.h))

    # ---- MAS ----
    def mas_init(self, n_verts, nb_start, nb_num, nb_list, part_map, real_map, node_offset=0):
        nb_start, nb_num = _h(nb_start, np.uint32), _h(nb_num, np.uint32)
        nb_list, part_map, real_map = _h(nb_list, np.uint32), _h(part_map, np.int32), _h(real_map, np.int32)
        self.n_verts = n_verts
        self.part_map_size = len(part_map)
        self._check(self.L.sgmas_mas_init(self.h, n_verts, node_offset, len(nb_list), _ptr(nb_list),
                                          _ptr(nb_start), _ptr(nb_num), _ptr(part_map), len(part_map),
                                          _ptr(real_map)))

    def mas_set_contacts(self, pairs, cp_num=None):
        n = 0 if pairs is None else (cp_num if cp_num is not None else pairs.shape[0])
        self._keep["pairs"] = pairs
        self._check(self.L.sgmas_mas_set_contacts(self.h, _ptr(pairs) if n else None, n))
        self.cp_num = n

    def mas_assemble(self, vals, rows, cols, indices=None, offset=0, cp_num=None):
        """setPreconditioner_bcoo: with indices (device uint32), the triplet
        count is the number of indices, as calculate_subsystem_bcoo_indices
        returns it; without, every block of the BCOO."""
        if cp_num is None:
            cp_num = getattr(self, "cp_num", 0)
        n = int(rows.shape[0]) if indices is None else int(indices.shape[0])
        self._check(self.L.sgmas_mas_assemble(self.h, _ptr(vals), _ptr(rows), _ptr(cols), _ptr(indices), offset,
                                              n, cp_num))

    def mas_apply(self, r, z):
        self._check(self.L.sgmas_mas_apply(self.h, _ptr(r), _ptr(z)))

    def mas_info(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._check(self.L.sgmas_mas_info(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return dict(levelnum=a.value, total=b.value, n_mas_blocks=c.value)

    def mas_tables(self):
        info = self.mas_info()
        Ln, n = info["levelnum"], self.n_verts
        fm = np.zeros(n, np.uint32)
        cs = np.zeros(Ln * n, np.int32)
        gn = np.zeros(max(info["total"], n) + 1, np.int32)
        ls = np.zeros(2 * (Ln + 1), np.int32)
        po = np.zeros(self.part_map_size // self.bank, np.int32)
        ct = np.zeros(6 * n, np.int32)
        self._check(self.L.sgmas_mas_download_tables(self.h, _ptr(fm), _ptr(cs), _ptr(gn), len(gn), _ptr(ls),
                                                     _ptr(po), _ptr(ct)))
        return dict(fine_mask=fm, coarse_space=cs.reshape(Ln, n), going_next=gn, level_size=ls.reshape(Ln + 1, 2),
                    prefix_orig=po, coarse_table=ct.reshape(n, 6))

    def mas_matrices(self):
        info = self.mas_info()
        nval = info["n_mas_blocks"] * (self.bank * (self.bank + 1) // 2) * 9
        h = np.zeros(nval)
        inv = np.zeros(nval)
        self._check(self.L.sgmas_mas_download_matrices(self.h, _ptr(h), _ptr(inv)))
        return h, inv

    def mas_invert_host(self, hess64, nblocks):
        hess64 = _h(hess64, np.float64)
        out = np.zeros_like(hess64)
        self._check(self.L.sgmas_mas_invert_host(self.h, _ptr(hess64), nblocks, _ptr(out)))
        return out

    # ---- PCG ----
    @staticmethod
    def bcoo(vals, rows, cols, n_block_rows):
        return Bcoo(_ptr(vals), _ptr(rows), _ptr(cols), int(rows.shape[0]), n_block_rows)

    def pcg_solve(self, vals, rows, cols, n_block_rows, b, x, **cfg):
        A = self.bcoo(vals, rows, cols, n_block_rows)
        c = pcg_config(**cfg)
        rep = PcgReport()
        self._check(self.L.sgmas_pcg_solve(self.h, C.byref(A), _ptr(b), _ptr(x), C.byref(c), C.byref(rep)))
        return {k: getattr(rep, k) for k, _ in PcgReport._fields_}

    def pcg_solve_host(self, vals, rows, cols, n_block_rows, b, x0=None, out=None, **cfg):
        """Host arrays in, x out (sgmas_pcg_solve_host).  out: a host float64
        array for x (e.g. pinned memory); x0: a start guess (copied into x)."""
        vals, rows, cols, b = _h(vals, np.float64), _h(rows, np.int32), _h(cols, np.int32), _h(b, np.float64)
        if out is not None:
            x = out
            if x0 is not None:
                x[...] = np.asarray(x0, np.float64)
        else:
            x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64, copy=True)
        if x0 is not None:
            cfg["initial_guess"] = True
        c = pcg_config(**cfg)
        rep = PcgReport()
        self._check(self.L.sgmas_pcg_solve_host(self.h, _ptr(vals), _ptr(rows), _ptr(cols), len(rows),
                                                n_block_rows, _ptr(b), _ptr(x), C.byref(c), C.byref(rep)))
        return x, {k: getattr(rep, k) for k, _ in PcgReport._fields_}

    # ---- learned start guess ----
    def mlp_set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        self._check(self.L.sgmas_mlp_set_params(self.h, _ptr(p), len(p)))

    def mlp_get_params(self):
        p = np.zeros(MLP_PARAMS, np.float32)
        self._check(self.L.sgmas_mlp_get_params(self.h, _ptr(p), MLP_PARAMS))
        return p

    def mlp_features(self, vals, rows, cols, n_block_rows, b, X, mask, prev=None, dx=None, T=None, fem_offset=0):
        """Slot-ordered features into device arrays X [Mm*16], mask [Mm] (+ T [Mm*3] from dx); returns (s_y, s_b)."""
        A = self.bcoo(vals, rows, cols, n_block_rows)
        sc = np.zeros(2)
        self._check(self.L.sgmas_mlp_features(self.h, C.byref(A), _ptr(b), _ptr(prev), _ptr(dx), fem_offset, _ptr(X),
                                              _ptr(mask), _ptr(T), _ptr(sc)))
        return float(sc[0]), float(sc[1])

    def mlp_gradient(self, X, T, mask, n_rows, inv_n, grad):
        loss = C.c_float()
        self._check(self.L.sgmas_mlp_gradient(self.h, _ptr(X), _ptr(T), _ptr(mask), n_rows, inv_n, _ptr(grad),
                                              C.byref(loss)))
        return loss.value

    def mlp_train_step(self, X, T, mask, n_rows, inv_n, lr, want_loss=True):
        loss = C.c_float()
        self._check(self.L.sgmas_mlp_train_step(self.h, _ptr(X), _ptr(T), _ptr(mask), n_rows, inv_n, lr,
                                                C.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def mlp_forward(self, X, n_rows, Y, bf16=True):
        self._check(self.L.sgmas_mlp_forward(self.h, _ptr(X), n_rows, int(bool(bf16)), _ptr(Y)))

    def mlp_warm_start(self, vals, rows, cols, n_block_rows, b, x0, prev=None, fem_offset=0, coef=False):
        """x0 <- the learned start guess; with coef=True also returns the Galerkin
        coefficients of (previous step, lumped step, network step, network coarse term)."""
        A = self.bcoo(vals, rows, cols, n_block_rows)
        c = np.zeros(4) if coef else None
        self._check(self.L.sgmas_mlp_warm_start(self.h, C.byref(A), _ptr(b), _ptr(prev), fem_offset, _ptr(x0),
                                                _ptr(c)))
        return c

    def pcg_profile(self, reps=20):
        """Per-phase device ms of one iteration of the last solve (sgmas_pcg_profile)."""
        ms = np.zeros(24, np.float32)
        self._check(self.L.sgmas_pcg_profile(self.h, reps, _ptr(ms), 24))
        if ms[5] == 0:  # graph form: kernel replays
            return dict(spmv=float(ms[0]), update_l0=float(ms[1]), coarse=float(ms[2]), collect=float(ms[3]))
        out = dict(spmv=float(ms[0]), update_levels01=float(ms[1]), levels2_collect=float(ms[2]),
                   loop_ms=float(ms[4]), stamped_iterations=int(ms[5]))
        names = ("spmv", "x_refresh", "r_refresh", "levels01", "unused", "end")
        out["barriers"] = {nm: dict(work_mean=float(ms[6 + 3 * i]), work_max=float(ms[7 + 3 * i]),
                                    wait_mean=float(ms[8 + 3 * i])) for i, nm in enumerate(names)}
        return out

    # ---- path kernels ----
    def spmv(self, a, vals, rows, cols, n_block_rows, x, b, y):
        A = self.bcoo(vals, rows, cols, n_block_rows)
        self._check(self.L.sgmas_spmv(self.h, a, C.byref(A), _ptr(x), b, _ptr(y)))

    def convert(self, vals, rows, cols, out_vals, out_rows, out_cols):
        nu = C.c_int()
        self._check(self.L.sgmas_convert(self.h, _ptr(vals), _ptr(rows), _ptr(cols), int(rows.shape[0]),
                                         _ptr(out_vals), _ptr(out_rows), _ptr(out_cols), C.byref(nu)))
        return nu.value

    def assembly_plan(self, rows, cols, out_rows, out_cols):
        """Sort and merge a fixed triplet structure once (sgmas_assembly_plan); returns the merged count."""
        nu = C.c_int()
        self._check(self.L.sgmas_assembly_plan(self.h, _ptr(rows), _ptr(cols), int(rows.shape[0]), _ptr(out_rows),
                                               _ptr(out_cols), C.byref(nu)))
        return nu.value

    def assemble(self, vals, out_vals):
        """Merge one step's raw values in the planned structure (sgmas_assemble)."""
        self._check(self.L.sgmas_assemble(self.h, _ptr(vals), int(vals.shape[0]), _ptr(out_vals)))

    # ---- affine-body coupling (vertex blocks -> 12-DOF body rows) ----
    def abd_body_blocks(self, H12, vals, rows, cols):
        """Each body's 12x12 Hessian (column-major) -> its 10 upper 3x3 blocks."""
        self._check(self.L.sgmas_abd_body_blocks(self.h, _ptr(H12), int(H12.shape[0]), _ptr(vals), _ptr(rows),
                                                 _ptr(cols)))

    def abd_pair_blocks(self, in_vals, in_rows, in_cols, xbar, body_of, fixed, vals, rows, cols):
        """Body-body vertex-pair blocks -> 16 blocks each of J_i^T H J_j."""
        self._check(self.L.sgmas_abd_pair_blocks(self.h, _ptr(in_vals), _ptr(in_rows), _ptr(in_cols),
                                                 int(in_rows.shape[0]), _ptr(xbar), _ptr(body_of), _ptr(fixed),
                                                 _ptr(vals), _ptr(rows), _ptr(cols)))

    def abd_fem_blocks(self, in_vals, in_rows, in_cols, xbar, body_of, fixed, fem_boundary, fem_point_offset,
                       n_bodies, vals, rows, cols):
        """Body-vertex / FEM-vertex blocks -> 4 blocks each of J^T H."""
        self._check(self.L.sgmas_abd_fem_blocks(self.h, _ptr(in_vals), _ptr(in_rows), _ptr(in_cols),
                                                int(in_rows.shape[0]), _ptr(xbar), _ptr(body_of), _ptr(fixed),
                                                _ptr(fem_boundary), int(fem_point_offset), int(n_bodies), _ptr(vals),
                                                _ptr(rows), _ptr(cols)))

    def append_triplets(self, base_vals, base_rows, base_cols, n_base, vals, rows, cols, out_vals, out_rows,
                        out_cols):
        """Sorted append (sgmas_append_triplets): raw triplets merged into a
        sorted merged block list; returns the output count."""
        no = C.c_int()
        n = int(rows.shape[0]) if rows is not None else 0
        self._check(self.L.sgmas_append_triplets(self.h, _ptr(base_vals), _ptr(base_rows), _ptr(base_cols),
                                                 int(n_base), _ptr(vals), _ptr(rows), _ptr(cols), n, _ptr(out_vals),
                                                 _ptr(out_rows), _ptr(out_cols), C.byref(no)))
        return no.value

    def element_plan(self, nodes_list, out_rows, out_cols):
        """Plan the merged structure of element groups (sgmas_element_plan):
        nodes_list = [int32 [n_elem, k] device arrays], group after group;
        out_rows / out_cols need room for all raw triplets.  Returns the
        merged count."""
        G = (ElementGroup * len(nodes_list))()
        for g, nd in enumerate(nodes_list):
            G[g] = ElementGroup(None, _ptr(nd), int(nd.shape[0]), int(nd.shape[1]))
        nu = C.c_int()
        self._check(self.L.sgmas_element_plan(self.h, G, len(nodes_list), _ptr(out_rows), _ptr(out_cols),
                                              C.byref(nu)))
        return nu.value

    def element_assemble(self, H_list, out_vals):
        """One step's element matrices (float64 [n_elem, 3k, 3k] device
        arrays, the planned groups in order) -> merged values
        (sgmas_element_assemble)."""
        G = (ElementGroup * len(H_list))()
        for g, H in enumerate(H_list):
            G[g] = ElementGroup(_ptr(H), None, int(H.shape[0]), int(H.shape[1]) // 3)
        self._check(self.L.sgmas_element_assemble(self.h, G, len(H_list), _ptr(out_vals)))

    def write_upper_blocks(self, H, nodes, vals, rows, cols):
        n_elem, k = int(nodes.shape[0]), int(nodes.shape[1])
        self._check(self.L.sgmas_write_upper_blocks(self.h, _ptr(H), n_elem, k, _ptr(nodes), _ptr(vals),
                                                    _ptr(rows), _ptr(cols)))

    def morton_codes(self, pos, codes, aabb=None):
        box = None if aabb is None else _h(aabb, np.float64)
        self._check(self.L.sgmas_morton_codes(self.h, _ptr(pos), int(pos.shape[0]), _ptr(box), _ptr(codes)))

    def morton_partition(self, pos, part_map_cap=None):
        n = int(pos.shape[0])
        cap = (n + self.bank - 1) // self.bank * self.bank if part_map_cap is None else int(part_map_cap)
        pm = np.zeros(max(cap, 1), np.int32)
        rm = np.zeros(n, np.int32)
        size = C.c_int()
        self._check(self.L.sgmas_morton_partition(self.h, _ptr(pos), n, _ptr(pm), cap, C.byref(size), _ptr(rm)))
        return pm[: size.value], rm
