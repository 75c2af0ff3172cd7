"""A plain C11 program builds against include/mela.h, links to the library and
runs on a machine without a GPU, as long as it only reaches checks that come
before any device work (here: a product whose inner dimensions disagree)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mex_linear_algebra_b200")

PROGRAM = r"""
#include <stdio.h>
#include "mela.h"
int main(void)
{
    double a[6] = {1, 0, 1, 1, 0, 1};        /* 2 x 3, column-major */
    unsigned char b[6] = {1, 1, 0, 1, 0, 1}; /* 2 x 3: inner dimensions 3 and 2 disagree */
    mela_host_matrix A = {MELA_KIND_DOUBLE, 0, 2, 3, a};
    mela_host_matrix B = {MELA_KIND_LOGICAL, 0, 2, 3, b};
    unsigned char C[6];
    mela_status st = mela_matmul_gf2(&A, &B, C);
    printf("%d|%s\n", (int)st, mela_status_string(st));
    return st == MELA_ERR_DIM ? 0 : 1;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_program_builds_links_and_runs(tmp_path):
    from mex_linear_algebra_b200 import lib
    lib()  # the library is built
    src = tmp_path / "use_mela.c"
    exe = tmp_path / "use_mela"
    src.write_text(PROGRAM)
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
                    str(src), "-L" + PKG, "-lmela_b200", "-Wl,-rpath," + PKG, "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "inner dimensions must agree" in r.stdout
