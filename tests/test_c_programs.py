"""C programs against the C ABI: a translator-free user program (varargs
PSStencilMap/PSStencilRun/PSReduce), the same program with its stencil
written in the DSL and compiled by the front end, and a program in the shape
of the reference's generated CUDA code. Each must compile against
include/physis_b200.h, link with libphysis_rt_b200.so, and (on a GPU)
reproduce the oracle bit for bit."""
import os
import subprocess

import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
CDIR = os.path.join(ROOT, "tests", "c")
LIBDIR = os.path.dirname(ps.LIB_PATH)


def build(name, tmp):
    src = os.path.join(CDIR, name)
    exe = os.path.join(str(tmp), name.split(".")[0])
    extra = []
    if name == "dsl_diffusion.c":
        # The stencil comes from the DSL front end as a kernel library.
        import sys
        so = os.path.join(str(tmp), "libdsl_kernels.so")
        r = subprocess.run([sys.executable, "-m", "physis_b200.dsl",
                            os.path.join(CDIR, "dsl_kernels.c"), "-o", so],
                           capture_output=True, text=True, cwd=ROOT)
        assert r.returncode == 0, r.stdout + r.stderr
        extra = ["-L" + str(tmp), "-ldsl_kernels", "-Wl,-rpath," + str(tmp)]
    if name.endswith(".cu"):
        cmd = ["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a",
               "-fmad=false", "-O2", "-I" + os.path.join(ROOT, "include"), src, "-o", exe,
               "-L" + LIBDIR, "-lphysis_rt_b200", "-Xlinker", "-rpath=" + LIBDIR]
    else:
        cmd = ["gcc", "-O2", "-std=gnu11", "-I" + os.path.join(ROOT, "include"), src, "-o", exe,
               *extra, "-L" + LIBDIR, "-lphysis_rt_b200", "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


PROGRAMS = ["user_diffusion.c", "generated_diffusion.cu", "dsl_diffusion.c"]


@pytest.mark.parametrize("name", PROGRAMS)
def test_programs_compile_and_link(name, tmp_path):
    build(name, tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("name", PROGRAMS)
def test_programs_match_oracle(name, tmp_path):
    exe = build(name, tmp_path)
    nx, ny, nz, count = 37, 20, 24, 10
    f = np.random.default_rng(31).random((nz, ny, nx), dtype=np.float32)
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    f.tofile(fin)
    r = subprocess.run([exe, str(nx), str(ny), str(nz), str(count), str(fin), str(fout),
                        "--physis-trace"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.fromfile(fout, dtype=np.float32).reshape(f.shape)
    want = oracle.diffusion7(f, count, np.asarray([0.1] * 6 + [0.4], np.float32))
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    s64, abss = oracle.sum_f64(want)
    assert abs(float(r.stdout.split()[0]) - s64) <= 1e-6 * abss
