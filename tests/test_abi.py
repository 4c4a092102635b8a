"""The C-ABI library: it loads and exports every symbol the header declares
(CPU only: nothing here launches GPU work)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _strip_inline_bodies(text):
    """Drop the bodies of static inline helpers (they are not exports)."""
    out, i = [], 0
    while True:
        j = text.find("static inline", i)
        if j < 0:
            out.append(text[i:])
            return "".join(out)
        out.append(text[i:j])
        k = text.find("{", j)
        depth, m = 0, k
        while m < len(text):
            depth += text[m] == "{"
            depth -= text[m] == "}"
            m += 1
            if depth == 0:
                break
        i = m


def declared_functions():
    names = set()
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not hdr.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = _strip_inline_bodies(text)
        text = re.sub(r"#(?:\\\n|[^\n])*", "", text)  # directives, with continuations
        for m in re.finditer(r"([A-Za-z_][A-Za-z_0-9]*)\s*\(([^;{}]*)\)\s*;", text):
            name = m.group(1)
            pre = text[max(0, m.start() - 200):m.start()]
            if "typedef" in pre.split(";")[-1]:
                continue
            names.add(name)
    return sorted(names)


def test_header_declares_the_reference_abi():
    names = set(declared_functions())
    for n in ["PSInit", "PSFinalize", "__PSGridNew", "__PSGridFree", "__PSGridCopyin",
              "__PSGridCopyout", "__PSGridSwap", "__PSGridGetID", "__PSGridSet",
              "PSDomain1DNew", "PSDomain2DNew", "PSDomain3DNew", "__PSReduceGridFloat",
              "__PSReduceGridDouble", "__PSCheckCudaError", "__PSRandomInit",
              "PSGrid3DFloatNew", "PSGrid3DDoubleNew", "PSGridCopyin", "PSGridCopyout",
              "PSGridFree", "__PSStencilMap", "PSReduce"]:
        assert n in names, n


def test_library_exports_every_declared_symbol():
    import physis_b200
    lib = ctypes.CDLL(physis_b200.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert hasattr(lib, "__ps_trace")


def test_struct_layouts_match_reference_abi():
    import physis_b200 as ps
    # __PSGrid: void *p0; int dim[3]; int elm_size; int num_dims; int64 num_elms; dev*
    assert ctypes.sizeof(ps.PSGridStruct) == 48
    assert ps.PSGridStruct.num_elms.offset == 32 and ps.PSGridStruct.dev.offset == 40
    assert ctypes.sizeof(ps.PSDomain) == 48


def test_ctypes_structs_match_header(tmp_path):
    """Sizes and field offsets of the ctypes mirrors equal the C header's."""
    import physis_b200 as ps
    structs = {"psb_request": ps.Request, "psb_result": ps.Result,
               "psb_tune_config": ps.TuneConfig, "psb_generic_stencil": ps.GenericStencilStruct,
               "psb_user_type": ps.UserType, "psb_grid_view": ps.GridViewStruct,
               "psb_launch_args": ps.LaunchArgs, "psb_compiled_stencil": ps.CompiledStencilStruct}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include <stdint.h>',
             '#include "physis_b200.h"',
             'int main(void) {']
    for cname, cls in structs.items():
        lines.append('printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for f in cls._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines += ['return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True,
                               text=True).stdout.splitlines():
        c, f, v = line.split()
        got[(c, f)] = int(v)
    for cname, cls in structs.items():
        assert got[(cname, "sizeof")] == ctypes.sizeof(cls), cname
        for f in cls._fields_:
            assert got[(cname, f[0])] == getattr(cls, f[0]).offset, (cname, f[0])


def test_domain_constructors_need_no_gpu():
    import physis_b200 as ps
    d = ps.PSDomain3DNew(1, 31, 2, 30, 3, 29)
    assert list(d.min) == [1, 2, 3] and list(d.max) == [31, 30, 29]
    assert list(d.local_min) == [1, 2, 3] and list(d.local_max) == [31, 30, 29]
    d2 = ps.PSDomain2DNew(0, 5, 1, 6)
    assert list(d2.local_max)[:2] == [5, 6]


def test_status_strings():
    import physis_b200 as ps
    for code, text in ps.STATUS.items():
        assert ps.lib.psb_status_string(code).decode() == text


def test_tune_cache_roundtrip(tmp_path, monkeypatch):
    """The autotuner's cache is host-only state: set/get without a GPU."""
    import subprocess
    import sys
    path = tmp_path / "tune.json"
    code = (
        "import physis_b200 as ps\n"
        "ps.tune_set(ps.DIFFUSION7, ps.PS_FLOAT, (64, 64, 64), impl=2, tile_x=128, tile_y=4,"
        " z_chunk=32, stages=8, t_depth=1)\n"
        "print(ps.tune_get(ps.DIFFUSION7, ps.PS_FLOAT, (64, 64, 64)))\n")
    env = dict(os.environ, PHYSIS_B200_TUNE_CACHE=str(path), PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert "'tile_x': 128" in out.stdout


def test_batch_tune_entries_use_the_header_base_and_buckets():
    """ps.batch_tune_set writes the entry a batch member of that stencil and
    size bucket reads: kernel id PSB_BATCH_TUNE_BASE + kernel_id - 1 (the
    header's value), extents rounded up to powers of two, at least 8."""
    import sys
    import physis_b200 as ps
    with open(os.path.join(ROOT, "include", "physis_b200.h")) as f:
        base = int(re.search(r"#define PSB_BATCH_TUNE_BASE (\d+)", f.read()).group(1))
    assert base == ps.PSB_BATCH_TUNE_BASE
    assert ps.batch_bucket((3, 100, 257)) == [8, 128, 512]
    assert ps.batch_bucket((8, 128, 512)) == [8, 128, 512]
    code = (
        "import physis_b200 as ps\n"
        "ps.batch_tune_set(ps.HIMENO19, (100, 70, 33), impl=2, tile_x=64, tile_y=8,"
        " z_chunk=0, stages=6, t_depth=2)\n"
        "print(ps.tune_get(%d + ps.HIMENO19 - 1, ps.PS_FLOAT, (128, 128, 64)))\n" % base)
    env = dict(os.environ, PHYSIS_B200_TUNE_CACHE=os.devnull, PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert "'t_depth': 2" in out.stdout and "'tile_x': 64" in out.stdout


def test_tune_cache_reads_a_list_on_one_line(tmp_path):
    """The cache reader takes entries in any layout: here json.dump's whole
    list on one line, with two entries."""
    import json
    import sys
    path = tmp_path / "tune.json"
    ents = [{"kernel": 3, "type": 2, "n": [128, 128, 128], "impl": 2, "tile_x": 64, "tile_y": 8,
             "z_chunk": 64, "stages": 6, "t_depth": 2, "ms": 0},
            {"kernel": 1, "type": 2, "n": [96, 96, 96], "impl": 2, "tile_x": 64, "tile_y": 4,
             "z_chunk": 8, "stages": 6, "t_depth": 1, "ms": 0}]
    path.write_text(json.dumps(ents))
    code = ("import physis_b200 as ps\n"
            "print(ps.tune_get(ps.HIMENO19, ps.PS_FLOAT, (128, 128, 128)))\n"
            "print(ps.tune_get(ps.DIFFUSION7, ps.PS_FLOAT, (96, 96, 96)))\n")
    env = dict(os.environ, PHYSIS_B200_TUNE_CACHE=str(path), PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    assert "'t_depth': 2" in lines[0] and "'z_chunk': 64" in lines[0]
    assert "'tile_y': 4" in lines[1] and "'z_chunk': 8" in lines[1]
