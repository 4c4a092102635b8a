"""The tune table that ships beside the library (physis_b200/tune_b200.json):
entries measured on B200 by the autotuner (single-grid kernels and batch
member size buckets). Every entry must be one the kernels accept, written
in the layout the library's reader parses, and the library must load it."""
import json
import os
import re
import subprocess
import sys

import physis_b200 as ps

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
TABLE = os.path.join(ROOT, "physis_b200", "tune_b200.json")
KEYS = ["kernel", "type", "n", "impl", "tile_x", "tile_y", "z_chunk", "stages", "t_depth", "ms"]
# The line layout the library's reader (tune.cu, parse_cache_file) scans.
LINE = re.compile(r'\{"kernel": -?\d+, "type": -?\d+, "n": \[\d+, \d+, \d+\], "impl": -?\d+, '
                  r'"tile_x": -?\d+, "tile_y": -?\d+, "z_chunk": -?\d+, "stages": -?\d+, '
                  r'"t_depth": -?\d+, "ms": [0-9.]+\},?$')
SINGLE = (ps.DIFFUSION7, ps.DIFFUSION7_PERIODIC, ps.HIMENO19)
BATCH = tuple(ps.PSB_BATCH_TUNE_BASE + k - 1 for k in SINGLE)
# Batch tile widths the batch autotuner times (consumer threads along x x 4
# points; 0 keeps the member's fewest-tiles shape).
BATCH_TILE_X = (0, 32, 44, 64, 84, 128)


def _entries():
    with open(TABLE) as f:
        return json.load(f)


def test_table_lines_parse_as_the_library_reads_them():
    with open(TABLE) as f:
        lines = [l.strip() for l in f if l.strip() not in ("", "[", "]")]
    assert lines and all(LINE.match(l) for l in lines), [l for l in lines if not LINE.match(l)]
    assert len(lines) == len(_entries())


def test_entries_are_valid_configurations():
    seen = set()
    for e in _entries():
        assert list(e) == KEYS, e
        key = (e["kernel"], e["type"], tuple(e["n"]))
        assert key not in seen, key
        seen.add(key)
        assert e["type"] in (ps.PS_FLOAT, ps.PS_DOUBLE) and all(v > 0 for v in e["n"]), e
        assert e["t_depth"] in (1, 2), e
        if e["kernel"] in SINGLE:
            assert e["impl"] in (ps.IMPL_PLAIN, ps.IMPL_TMA), e
            assert e["tile_x"] > 0 and e["tile_y"] > 0 and e["z_chunk"] > 0, e
            assert 2 <= e["stages"] <= 8, e
            if e["t_depth"] == 2:
                assert e["kernel"] in (ps.DIFFUSION7, ps.HIMENO19), e
        else:
            assert e["kernel"] in BATCH, e
            assert e["type"] == ps.PS_FLOAT, e
            # size buckets: each extent a power of two, at least 8
            assert list(e["n"]) == ps.batch_bucket(e["n"]), e
            assert e["tile_x"] in BATCH_TILE_X, e
            if e["t_depth"] == 2:  # two sweeps per pass: Himeno on 64 x 8 tiles
                assert e["kernel"] == ps.PSB_BATCH_TUNE_BASE + ps.HIMENO19 - 1, e
                assert e["tile_x"] in (0, 64), e


def test_library_loads_the_shipped_table(tmp_path):
    """With the shipped table on (the default outside the tests) every entry
    is what psb_tune_get returns; with PHYSIS_B200_TUNE_SHIPPED=0 none is."""
    code = (
        "import json, sys\n"
        "import physis_b200 as ps\n"
        "out = []\n"
        "for e in json.load(open(sys.argv[1])):\n"
        "    c = ps.tune_get(e['kernel'], e['type'], e['n'])\n"
        "    out.append(all(c[k] == e[k] for k in ('impl', 'tile_x', 'tile_y', 'z_chunk',\n"
        "                                           'stages', 't_depth')))\n"
        "print(json.dumps(out))\n")
    for shipped in ("1", "0"):
        env = dict(os.environ, PHYSIS_B200_TUNE_SHIPPED=shipped,
                   PHYSIS_B200_TUNE_CACHE=str(tmp_path / ("cache%s.json" % shipped)))
        r = subprocess.run([sys.executable, "-c", code, TABLE], env=env, cwd=ROOT,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        got = json.loads(r.stdout.strip().splitlines()[-1])
        if shipped == "1":
            assert all(got), got
        else:
            assert not all(got)
