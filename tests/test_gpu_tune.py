"""The autotuner (psb_autotune) on the GPU: it times the candidate tile
configurations of a (kernel, type, shape) key, keeps the fastest, caches it
in the JSON file and makes PSStencilRun use it. The chosen configuration
must be one of the candidates, survive a reload of the cache, and the run
with it must stay bit-exact against the oracle (the reference tunes at
translation time by trial, translator/reference_translator.cc:749-1223)."""
import json
import os

import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U

pytestmark = pytest.mark.gpu

COEF = [0.1, 0.1, 0.1, 0.1, 0.1, 0.1, 0.4]
CASES = [(ps.DIFFUSION7, ps.PS_FLOAT, (96, 80, 40)),
         (ps.DIFFUSION7_PERIODIC, ps.PS_FLOAT, (64, 48, 32)),
         (ps.DIFFUSION7, ps.PS_DOUBLE, (64, 40, 36)),
         (ps.HIMENO19, ps.PS_FLOAT, (65, 49, 33))]


def _valid(kernel, type_, dims, c):
    if c["impl"] == ps.IMPL_PLAIN:
        return True
    if c["impl"] != ps.IMPL_TMA or c["stages"] not in (4, 6, 8):
        return False
    if c["t_depth"] == 2:
        return kernel == ps.DIFFUSION7 and type_ == ps.PS_FLOAT and c["z_chunk"] in (32, 64, 128)
    txs = (16, 32, 64) if type_ == ps.PS_DOUBLE else (32, 64, 128)
    tys = (4, 8, 16) if kernel == ps.HIMENO19 else (4, 8, 16, 32)
    return (c["t_depth"] == 1 and c["tile_x"] in txs and c["tile_y"] in tys
            and c["z_chunk"] in (2, 4, 8, 16, 32, 64, 128) and c["z_chunk"] <= 2 * dims[2])


@pytest.mark.parametrize("kernel,type_,dims", CASES)
def test_autotune_picks_a_candidate_and_stays_bit_exact(kernel, type_, dims):
    ps.PSInit()
    cfg = ps.autotune(kernel, type_, dims, force=True)
    assert _valid(kernel, type_, dims, cfg), cfg
    assert ps.tune_get(kernel, type_, dims) == cfg
    # The choice is in the cache file under its key.
    with open(os.environ["PHYSIS_B200_TUNE_CACHE"]) as f:
        entries = json.load(f)
    hit = [e for e in entries if e["kernel"] == kernel and e["type"] == type_
           and e["n"] == list(dims)]
    assert len(hit) == 1
    assert {k: hit[0][k] for k in cfg} == cfg
    # Not forced: the cached entry comes back without tuning again.
    assert ps.autotune(kernel, type_, dims) == cfg
    nx, ny, nz = dims
    if kernel == ps.HIMENO19:
        p, coef = U.himeno_inputs((nz, ny, nx), 3)
        got, gosa = U.himeno_gpu(p, coef, 0.8, 6)
        want, wgosa = oracle.himeno(p, coef, 0.8, 6)
        assert U.bits_equal(got, want)
        assert np.allclose(gosa, wgosa, rtol=1e-12, atol=0)
    else:
        dt = np.float32 if type_ == ps.PS_FLOAT else np.float64
        f = np.random.default_rng(4).random((nz, ny, nx)).astype(dt)
        periodic = kernel == ps.DIFFUSION7_PERIODIC
        got = U.diffusion_gpu(f, 10, COEF, periodic=periodic)
        want = oracle.diffusion7(f, 10, np.asarray(COEF, dt), periodic=periodic)
        assert U.bits_equal(got, want)


def test_tune_set_overrides_and_every_candidate_shape_runs():
    """psb_tune_set installs a configuration that PSStencilRun then uses; a
    sweep of explicit shapes (all bit-exact) covers the tuner's candidate
    space beyond the one it picked."""
    ps.PSInit()
    dims = (72, 40, 24)
    f = np.random.default_rng(8).random(tuple(reversed(dims)), dtype=np.float32)
    want = oracle.diffusion7(f, 4, np.asarray(COEF, np.float32))
    try:
        for tx in (32, 64, 128):
            for ty in (4, 8, 16, 32):
                for zc, st in ((2, 4), (16, 6), (64, 8)):
                    cfg = dict(impl=ps.IMPL_TMA, tile_x=tx, tile_y=ty, z_chunk=zc, stages=st,
                               t_depth=1)
                    ps.tune_set(ps.DIFFUSION7, ps.PS_FLOAT, dims, **cfg)
                    assert ps.tune_get(ps.DIFFUSION7, ps.PS_FLOAT, dims) == cfg
                    got = U.diffusion_gpu(f, 4, COEF)
                    assert U.bits_equal(got, want), cfg
    finally:
        ps.tune_set(ps.DIFFUSION7, ps.PS_FLOAT, dims, impl=ps.IMPL_PLAIN, tile_x=32, tile_y=16,
                    z_chunk=16, stages=6, t_depth=1)


def _pow2(n):
    b = 8
    while b < n:
        b <<= 1
    return b


def test_batch_autotune_caches_per_bucket_and_stays_bit_exact():
    """psb_batch_autotune times the fewest-tiles rule, fixed tile widths and
    (Himeno) two sweeps per pass for each member size bucket on scratch
    grids, caches the winners (kernel id 100 + member kind, extents rounded
    up to powers of two), and later runs use them: each member's item shape
    is its bucket's entry (or its own rule where the rule won) and every
    result is bit-exact against the oracle (the members' own grids were not
    touched)."""
    from physis_b200.workloads import himeno_inputs
    ps.PSInit()
    spec = [("diff", (100, 90, 70), 6), ("diffp", (64, 48, 80), 5), ("him", (90, 66, 50), 4),
            ("diff", (120, 70, 100), 3)]  # the last shares the first one's bucket
    kinds = {"diff": (ps.DIFFUSION7, 0), "diffp": (ps.DIFFUSION7_PERIODIC, 1),
             "him": (ps.HIMENO19, 2)}
    data, grids = [], []
    for i, (kind, dims, steps) in enumerate(spec):
        nx, ny, nz = dims
        if kind == "him":
            p, coef = himeno_inputs((nz, ny, nx), 30 + i)
            gs = [ps.grid_new(ps.PS_FLOAT, dims) for _ in range(14)]
            ps.PSGridCopyin(gs[0], p)
            ps.PSGridCopyin(gs[1], p)
            for k in range(12):
                ps.PSGridCopyin(gs[2 + k], coef[k])
            data.append((p, coef))
        else:
            f = np.random.default_rng(30 + i).random((nz, ny, nx), dtype=np.float32)
            gs = [ps.grid_new(ps.PS_FLOAT, dims) for _ in range(2)]
            ps.PSGridCopyin(gs[0], f)
            data.append((f, None))
        grids.append(gs)
    b = ps.Batch()
    try:
        for (kind, dims, steps), gs in zip(spec, grids):
            b.add(kinds[kind][0], gs, [0.8] if kind == "him" else COEF, steps)
        b.autotune(force=True)
        with open(os.environ["PHYSIS_B200_TUNE_CACHE"]) as f:
            entries = json.load(f)
        tuned = {}
        for e in entries:
            if e["kernel"] >= 100:
                tuned[(e["kernel"] - 100, tuple(e["n"]))] = e
        b.run(0)
        for i, (kind, dims, steps) in enumerate(spec):
            key = (kinds[kind][1], tuple(_pow2(v) for v in dims))
            assert key in tuned, key
            e = tuned[key]
            lay = b.layout(i)
            if e["tile_x"] > 0:  # a fixed width won
                assert (lay["tile_x"], lay["tile_y"]) == (e["tile_x"], e["tile_y"]), (lay, e)
            else:  # the batch's rule won: the member fits its own extents
                assert lay["tile_x"] > 0, (lay, e)
            assert lay["t_depth"] == e["t_depth"], (lay, e)
            assert lay["tuned"] == 1  # (the z chunk follows the batch's own rule)
            done, _, g = b.result(i)
            assert done == steps
            f, coef = data[i]
            if kind == "him":
                want = oracle.himeno(f, coef, 0.8, steps)[0]
            else:
                want = oracle.diffusion7(f, steps, np.asarray(COEF, np.float32),
                                         periodic=kind == "diffp")
            assert U.bits_equal(ps.PSGridCopyout(g), want), (i, kind, lay)
    finally:
        b.free()
        for gs in grids:
            for g in gs:
                ps.PSGridFree(g)
