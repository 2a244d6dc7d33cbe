"""The C++ host mirror (stiff-gipc_b200/host/sgmas.hpp) compiles against the
C-ABI header, links libsgmas.so and runs its host-only paths (no GPU): a
MatrixMarket round trip and the neighbour CSR of one tet."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "stiff-gipc_b200")

PROGRAM = r'''
#include <cstdio>
#include <cmath>
#include "host/sgmas.hpp"

int main(int argc, char** argv) {
    sgmas::HostSystem s;
    s.n_block_rows = 2;
    s.rows = {0, 0, 1};
    s.cols = {0, 1, 1};
    s.values.assign(27, 0.0);
    for (int k = 0; k < 27; ++k) s.values[k] = 0.5 + k;   // arbitrary blocks
    s.b = {1, 2, 3, 4, 5, 6};
    const std::string a = std::string(argv[1]) + "/A.mtx", b = std::string(argv[1]) + "/b.mtx";
    sgmas::mtx_write(a, b, s);
    sgmas::HostSystem t = sgmas::mtx_read(a, b);
    if (t.rows != s.rows || t.cols != s.cols || t.values != s.values || t.b != s.b || t.n_block_rows != 2) return 2;
    try {
        sgmas::mtx_read(std::string(argv[1]) + "/missing.mtx");
        return 3;
    } catch (const sgmas::Error& e) {
        if (e.code != SGMAS_ERR_ARG) return 4;
    }
    // getVertNeighbors of one tet: 4 vertices, each linked to the 3 others
    const int tet[4] = {0, 1, 2, 3};
    unsigned st[4], nn[4], nl[32];
    const int n = sgmas_vert_neighbors(tet, 1, nullptr, 0, 4, 0, st, nn, nl, 32);
    if (n != 12 || nn[0] != 3 || nn[3] != 3) return 5;
    std::printf("ok\n");
    return 0;
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ missing")
def test_cpp_mirror_compiles_links_and_runs(tmp_path):
    import sgmas
    sgmas.lib()  # built in-tree
    src = tmp_path / "mirror.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "mirror"
    cmd = ["g++", "-std=c++17", "-O1", "-I" + PKG, "-I/usr/local/cuda/include", str(src), "-L" + PKG, "-lsgmas",
           "-Wl,-rpath," + PKG, "-o", str(exe)]
    subprocess.check_call(cmd)
    out = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert out.stdout.strip() == "ok"
