"""Generate the golden fixtures under tests/golden/ from the reference's own
data files (run once in a container that has the reference checkout; the
fixtures are committed, the tests never read the reference tree).

Sources (paths inside the StiffGIPC project):
  * examples/bar_width_15_1_1_num_75_5_5_sorted.16_sorted.16.{msh,part}
      METIS-sorted tet bar (2736 vertices) and its partition;
  * examples/bar_width_15_1_1_num_75_5_5_sorted.16.msh
      the input mesh that partition was computed from;
  * Assets/sorted_mesh/bunny2_sorted.16.{msh,part}, Assets/tetMesh/bunny2.msh
  * Assets/sorted_mesh/cube_sorted.16.{msh,part}, Assets/tetMesh/cube.msh
  * Assets/sorted_mesh/cloth_high_sorted.16.{obj,part}, Assets/triMesh/cloth_high.obj

Each .npz holds int32 tets/triangles (0-based), float64 positions and the
int32 part ids exactly as the reference shipped them.

Usage: python tests/golden/make_fixtures.py /path/to/StiffGIPC-checkout
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_msh(path):
    """Gmsh ASCII 2.2 / 4.1 reader: nodes and 4-node tetrahedra (type 4)."""
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    ver = float(lines[lines.index("$MeshFormat") + 1].split()[0])
    i = lines.index("$Nodes") + 1
    if ver < 4:
        n = int(lines[i]); i += 1
        ids, pos = [], []
        for k in range(n):
            t = lines[i + k].split()
            ids.append(int(t[0])); pos.append([float(v) for v in t[1:4]])
        tag = {t: j for j, t in enumerate(ids)}
        i = lines.index("$Elements") + 1
        m = int(lines[i]); i += 1
        tets = []
        for k in range(m):
            t = [int(v) for v in lines[i + k].split()]
            if t[1] == 4:
                ntag = t[2]
                tets.append([tag[v] for v in t[3 + ntag:3 + ntag + 4]])
        return np.array(pos, np.float64), np.array(tets, np.int32)
    nblocks, nnodes = [int(v) for v in lines[i].split()[:2]]; i += 1
    tags, pos = [], []
    for _ in range(nblocks):
        _, _, _, nb = [int(v) for v in lines[i].split()]; i += 1
        blk_tags = [int(lines[i + k]) for k in range(nb)]; i += nb
        for k in range(nb):
            pos.append([float(v) for v in lines[i + k].split()[:3]])
        i += nb
        tags += blk_tags
    tag = {t: j for j, t in enumerate(tags)}
    i = lines.index("$Elements") + 1
    nblocks = int(lines[i].split()[0]); i += 1
    tets = []
    for _ in range(nblocks):
        _, _, etype, ne = [int(v) for v in lines[i].split()]; i += 1
        for k in range(ne):
            t = [int(v) for v in lines[i + k].split()]
            if etype == 4:
                tets.append([tag[v] for v in t[1:5]])
        i += ne
    return np.array(pos, np.float64), np.array(tets, np.int32)


def read_obj(path):
    pos, tris = [], []
    with open(path) as f:
        for ln in f:
            t = ln.split()
            if not t:
                continue
            if t[0] == "v":
                pos.append([float(v) for v in t[1:4]])
            elif t[0] == "f":
                tris.append([int(v.split("/")[0]) - 1 for v in t[1:4]])
    return np.array(pos, np.float64), np.array(tris, np.int32)


def read_part(path):
    return np.loadtxt(path, dtype=np.int64).astype(np.int32).reshape(-1)


def main(ref):
    jobs = {
        "bar": ("examples/bar_width_15_1_1_num_75_5_5_sorted.16_sorted.16.msh",
                "examples/bar_width_15_1_1_num_75_5_5_sorted.16_sorted.16.part",
                "examples/bar_width_15_1_1_num_75_5_5_sorted.16.msh"),
        "bunny2": ("Assets/sorted_mesh/bunny2_sorted.16.msh", "Assets/sorted_mesh/bunny2_sorted.16.part",
                   "Assets/tetMesh/bunny2.msh"),
        "cube": ("Assets/sorted_mesh/cube_sorted.16.msh", "Assets/sorted_mesh/cube_sorted.16.part",
                 "Assets/tetMesh/cube.msh"),
    }
    for name, (msh, part, src) in jobs.items():
        pos, tets = read_msh(os.path.join(ref, msh))
        spos, stets = read_msh(os.path.join(ref, src))
        pid = read_part(os.path.join(ref, part))
        assert len(pid) == len(pos), (name, len(pid), len(pos))
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), pos=pos, tets=tets, part=pid,
                            src_pos=spos, src_tets=stets)
        print(name, pos.shape, tets.shape, pid.max() + 1)
    pos, tris = read_obj(os.path.join(ref, "Assets/sorted_mesh/cloth_high_sorted.16.obj"))
    spos, stris = read_obj(os.path.join(ref, "Assets/triMesh/cloth_high.obj"))
    pid = read_part(os.path.join(ref, "Assets/sorted_mesh/cloth_high_sorted.16.part"))
    np.savez_compressed(os.path.join(HERE, "cloth_high.npz"), pos=pos, tris=tris, part=pid, src_pos=spos,
                        src_tris=stris)
    print("cloth_high", pos.shape, tris.shape, pid.max() + 1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <path of the StiffGIPC checkout>")
    main(sys.argv[1])
