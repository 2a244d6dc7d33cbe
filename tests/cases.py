"""Parity cases shared by the CPU and GPU tests: synthetic systems of the
benchmark shapes (scaled to oracle-friendly sizes) and the reference's own
METIS-partitioned meshes from tests/golden/."""
from __future__ import annotations

import functools
import os

import numpy as np

from oracle import oracle as O
from sgmas import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


class Case:
    def __init__(self, name, sysm, part_map, real_map, nb_start, nb_num, nb_list):
        self.name = name
        self.s = sysm
        self.part_map = part_map
        self.real_map = real_map
        self.nb_start, self.nb_num, self.nb_list = nb_start, nb_num, nb_list

    @property
    def n(self):
        return self.s.n_verts

    def oracle_mas(self, pairs=True, precision=0, bank=16):
        m = O.MAS(self.n, self.nb_start, self.nb_num, self.nb_list, self.part_map, self.real_map, bank=bank)
        m.reorder(self.s.pairs if pairs else None)
        m.assemble(self.s.vals, self.s.rows, self.s.cols, precision=precision)
        return m


@functools.lru_cache(maxsize=None)
def build(name, bank=16):
    if name == "c1":
        s = synth.config1(seed=0)
        pm, rm = O.morton_partition(s.pos, bank)
    elif name == "c2s":
        s = synth.config2(seed=1, scale=0.3)
        pm, rm = O.morton_partition(s.pos, bank)
    elif name == "g80k":  # large enough for more than 32 subdomains at levels >= 2
        s = synth.stencil_grid_system(64, 36, 36, E=1e5, n_pairs=2000, seed=3)
        pm, rm = O.morton_partition(s.pos, bank)
    elif name == "g221k":  # block CSR of both triangles about twice the 126 MB L2
        s = synth.stencil_grid_system(96, 48, 48, E=1e5, n_pairs=4000, seed=4)
        pm, rm = O.morton_partition(s.pos, bank)
    elif name in ("bar", "bunny2", "cube"):
        g = golden(name)
        s = synth.mesh_system(g["pos"], g["tets"], seed=2)
        pm, rm = O.mas_partition(g["part"], bank)
    else:
        raise KeyError(name)
    st, nn, nl = O.vert_neighbors(s.tets, s.n_verts)
    return Case(name, s, pm, rm, st, nn, nl)


def oracle_iteration_band(s, precond, mas=None, rel_tol=1e-4, n_perturb=10, **kw):
    """(min, max) iteration counts of the oracle port's PCG on b scaled by
    (1 + k 2^-52), k = 0 .. n_perturb - 1, serial and on every host thread.
    On ill-conditioned systems CG's count moves with the last bit of any sum;
    this measured spread (not a guess) is the band a device solve must fall
    in (see band_ok)."""
    its = []
    nth = O.lib().or_omp_max_threads()
    for k in range(n_perturb):
        b = s.b * (1.0 + k * 2.0 ** -52)
        for nt in ((1, nth) if k < 2 else (nth,)):
            _, r = O.pcg(s.vals, s.rows, s.cols, s.n_verts, b, precond=precond, rel_tol=rel_tol, mas=mas,
                         nthreads=nt, **kw)
            its.append(r["iterations"])
    return min(its), max(its)


def band_ok(iterations, band):
    """The device's count lies in the oracle's measured band, widened on both
    sides by that band's own width (a handful of samples under-reads the
    spread) and by at least one check interval."""
    lo, hi = band
    w = max(10, hi - lo)
    return lo - w <= iterations <= hi + w
