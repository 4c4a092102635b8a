"""Batched solves (psb_batch_*): many uneven grids in one persistent launch,
per-step graph launches, and the per-grid loops. Every member's result must
equal the oracle bit for bit in every mode, alone or in the mix."""
import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U

COEF = [0.1, 0.1, 0.1, 0.1, 0.1, 0.1, 0.4]

# (kind, (nx, ny, nz), steps)
MEMBERS = [
    ("diff", (64, 64, 64), 6),
    ("diffp", (32, 32, 32), 7),
    ("him", (33, 33, 65), 4),
    ("diff", (33, 17, 40), 3),
    ("diffp", (48, 20, 9), 10),
    ("him", (20, 9, 70), 5),
    ("diff", (100, 7, 5), 1),
    ("him", (65, 12, 4), 2),
    ("diffp", (70, 66, 33), 12),
]


def _inputs(kind, dims, seed):
    nx, ny, nz = dims
    if kind == "him":
        return U.himeno_inputs((nz, ny, nx), seed)
    return np.random.default_rng(seed).random((nz, ny, nx), dtype=np.float32), None


def _want(kind, data, steps):
    f, coef = data
    if kind == "him":
        return oracle.himeno(f, coef, 0.8, steps)[0]
    return oracle.diffusion7(f, steps, np.asarray(COEF, np.float32), periodic=kind == "diffp")


class Members:
    def __init__(self, spec):
        self.spec = spec
        self.data = [_inputs(k, d, 100 + i) for i, (k, d, _) in enumerate(spec)]
        self.grids = []
        for (kind, dims, _), (f, coef) in zip(spec, self.data):
            n = 14 if kind == "him" else 2
            gs = [ps.grid_new(ps.PS_FLOAT, dims) for _ in range(n)]
            self.grids.append(gs)
        self.load()

    def load(self):
        for (kind, dims, _), (f, coef), gs in zip(self.spec, self.data, self.grids):
            ps.PSGridCopyin(gs[0], f)
            ps.PSGridCopyin(gs[1], f)
            if kind == "him":
                for i in range(12):
                    ps.PSGridCopyin(gs[2 + i], coef[i])

    def batch(self, stop=None):
        b = ps.Batch()
        for i, ((kind, dims, steps), gs) in enumerate(zip(self.spec, self.grids)):
            k = {"diff": ps.DIFFUSION7, "diffp": ps.DIFFUSION7_PERIODIC, "him": ps.HIMENO19}[kind]
            params = [0.8] if kind == "him" else COEF
            tol, every = stop(i) if stop else (0.0, 0)
            b.add(k, gs, params, steps, tol=tol, check_every=every)
        return b

    def free(self):
        for gs in self.grids:
            for g in gs:
                ps.PSGridFree(g)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_batch_members_bit_exact(mode):
    M = Members(MEMBERS)
    try:
        b = M.batch()
        b.run(mode)
        st = b.stats()
        assert st["lattice_updates"] > 0 and st["launches"] >= 1
        if mode == 0:
            assert st["launches"] <= 2  # one persistent launch per stencil kind
        for i, (kind, dims, steps) in enumerate(MEMBERS):
            done, _, g = b.result(i)
            assert done == steps
            got = ps.PSGridCopyout(g)
            assert U.bits_equal(got, _want(kind, M.data[i], steps)), (mode, i, kind, dims)
        b.free()
    finally:
        M.free()


@pytest.mark.gpu
def test_batch_rerun_is_repeatable():
    """Running the same batch twice from the same inputs gives the same bits."""
    M = Members(MEMBERS[:5])
    try:
        b = M.batch()
        b.run(0)
        first = [ps.PSGridCopyout(b.result(i)[2]) for i in range(5)]
        M.load()
        b.run(0)
        second = [ps.PSGridCopyout(b.result(i)[2]) for i in range(5)]
        assert all(U.bits_equal(a, c) for a, c in zip(first, second))
        b.free()
    finally:
        M.free()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_batch_convergence_same_alone_and_in_mix(mode):
    """Members stop at their residual tolerance; the stop step and the field
    are the same whether a member runs alone or in the mix."""
    spec = [("diff", (40, 40, 40), 200), ("him", (33, 33, 33), 120), ("diffp", (24, 24, 24), 150),
            ("diff", (64, 30, 20), 90)]
    stop = lambda i: ((2e-3, 5), (0.4, 4), (3e-3, 3), (1e-2, 2))[i]
    M = Members(spec)
    try:
        b = M.batch(stop)
        b.run(mode)
        mixed = []
        for i in range(len(spec)):
            done, res, g = b.result(i)
            mixed.append((done, res, ps.PSGridCopyout(g)))
        b.free()
        for i, (kind, dims, steps) in enumerate(spec):
            done = mixed[i][0]
            assert 0 < done <= steps
            # the field after `done` steps is the oracle's field after `done` steps
            assert U.bits_equal(mixed[i][2], _want(kind, M.data[i], done)), (i, done)
        # each member alone
        for i in range(len(spec)):
            M.load()
            alone = Members.__new__(Members)
            alone.spec = [spec[i]]
            alone.data = [M.data[i]]
            alone.grids = [M.grids[i]]
            b1 = alone.batch(lambda _j: stop(i))
            b1.run(mode)
            done, res, g = b1.result(0)
            assert done == mixed[i][0] and res == mixed[i][1]
            assert U.bits_equal(ps.PSGridCopyout(g), mixed[i][2])
            b1.free()
    finally:
        M.free()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [ps.FILL_UNIFORM, ps.FILL_CONST, ps.FILL_BND, ps.FILL_ZPROFILE])
def test_grid_fill_matches_host_restatement(kind):
    dims = (37, 20, 11)
    for layout in (ps.LAYOUT_PITCHED, ps.LAYOUT_DENSE):
        g = ps.grid_new(ps.PS_FLOAT, dims, layout)
        try:
            ps.grid_fill(g, kind, 77, -0.5, 2.0)
            got = ps.PSGridCopyout(g)
            want = ps.fill_reference(dims, kind, 77, -0.5, 2.0)
            assert U.bits_equal(got, want)
        finally:
            ps.PSGridFree(g)


# Members large enough (>= 128 items per step) that an item waits only for
# the 27 items around it in the member's previous step, so consecutive steps
# overlap as a wavefront: clamped and periodic 7-point (a periodic member
# one tile wide in x, whose dependencies wrap onto itself) and Himeno.
WAVE_MEMBERS = [
    ("diff", (192, 192, 192), 24),
    ("diffp", (160, 160, 160), 30),
    ("him", (160, 160, 160), 20),
    ("diffp", (64, 48, 512), 25),
    ("him", (300, 40, 130), 16),
]

_WANT_CACHE = {}


def _want_cached(i, kind, data, steps):
    key = (i, kind, steps)
    if key not in _WANT_CACHE:
        _WANT_CACHE[key] = _want(kind, data, steps)
    return _WANT_CACHE[key]


@pytest.mark.gpu
@pytest.mark.parametrize("mix", ["alone", "mixed"])
def test_batch_wavefront_members_bit_exact(mix):
    """Large members take the per-tile (wavefront) dependency path; each is
    bit-exact against the oracle whether it runs alone or with every other
    large member and the small members of MEMBERS."""
    spec = WAVE_MEMBERS + (MEMBERS if mix == "mixed" else [])
    M = Members(spec)
    try:
        groups = [[i] for i in range(len(WAVE_MEMBERS))] if mix == "alone" else [list(range(len(spec)))]
        for ids in groups:
            sub = Members.__new__(Members)
            sub.spec = [spec[i] for i in ids]
            sub.data = [M.data[i] for i in ids]
            sub.grids = [M.grids[i] for i in ids]
            b = sub.batch()
            b.run(0)
            for j, i in enumerate(ids):
                kind, dims, steps = spec[i]
                lay = b.layout(j)
                done, _, g = b.result(j)
                assert done == steps
                if i < len(WAVE_MEMBERS):
                    assert lay["wavefront"] == 1 and lay["tiles"] >= 128, (i, lay)
                else:
                    assert lay["wavefront"] == 0, (i, lay)
                want = (_want_cached(i, kind, M.data[i], steps) if i < len(WAVE_MEMBERS)
                        else _want(kind, M.data[i], steps))
                assert U.bits_equal(ps.PSGridCopyout(g), want), (mix, i, kind, dims, lay)
            b.free()
    finally:
        M.free()


@pytest.mark.gpu
def test_batch_wavefront_with_residual_checks():
    """Wavefront members with residual checks: the step after a check waits
    for the whole step and its decision; stop steps and fields equal the
    oracle's after that many steps."""
    spec = [("diff", (192, 160, 96), 60), ("him", (160, 128, 96), 40)]
    stop = lambda i: ((3e-3, 7), (0.5, 5))[i]
    M = Members(spec)
    try:
        b = M.batch(stop)
        b.run(0)
        for i, (kind, dims, steps) in enumerate(spec):
            assert b.layout(i)["wavefront"] == 1
            done, res, g = b.result(i)
            assert 0 < done <= steps
            assert U.bits_equal(ps.PSGridCopyout(g), _want(kind, M.data[i], done)), (i, done)
        b.free()
    finally:
        M.free()


def _pow2(n):
    b = 8
    while b < n:
        b <<= 1
    return b


def _two_sweep_entries(spec, zc=8):
    """Tune entries that put every Himeno member of spec on two sweeps per pass
    (batch bucket entries: kernel 100 + 2, extents rounded up to powers of 2)."""
    for kind, dims, _ in spec:
        if kind == "him":
            ps.tune_set(102, ps.PS_FLOAT, tuple(_pow2(v) for v in dims), impl=ps.IMPL_TMA,
                        tile_x=64, tile_y=8, z_chunk=zc, stages=6, t_depth=2)


def _drop_entries(spec):
    for kind, dims, _ in spec:
        if kind == "him":
            ps.tune_set(102, ps.PS_FLOAT, tuple(_pow2(v) for v in dims), impl=ps.IMPL_TMA,
                        tile_x=64, tile_y=8, z_chunk=8, stages=6, t_depth=1)


TWO_SWEEP_MEMBERS = [
    ("him", (160, 160, 160), 20),   # wavefront path
    ("him", (70, 40, 33), 7),       # odd steps: a one-sweep last pass
    ("him", (33, 20, 65), 2),
    ("diffp", (48, 20, 9), 10),
    ("him", (130, 12, 18), 5),
    ("diff", (64, 64, 64), 6),
]


@pytest.mark.gpu
def test_batch_default_sweeps_per_pass():
    """Without tune entries a Himeno member runs two sweeps per pass when it
    is at least 120 inside on every axis and 64-wide tiles cover its x
    extent with at most 15% to spare (129^3: 127 of 128 columns), else one
    (160^3: 158 of 192; 96^3: too small); results equal the oracle's."""
    spec = [("him", (129, 129, 129), 6), ("him", (160, 160, 160), 3), ("him", (96, 96, 96), 4),
            ("diff", (64, 64, 64), 5)]
    M = Members(spec)
    try:
        b = M.batch()
        b.run(0)
        want_td = [2, 1, 1, 1]
        for i, (kind, dims, steps) in enumerate(spec):
            lay = b.layout(i)
            done, _, g = b.result(i)
            assert done == steps
            assert lay["t_depth"] == want_td[i] and lay["tuned"] == 0, (i, lay)
            assert U.bits_equal(ps.PSGridCopyout(g), _want(kind, M.data[i], steps)), (i, lay)
        b.free()
    finally:
        M.free()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_batch_two_sweep_himeno_bit_exact(mode):
    """Himeno members on two sweeps per pass (the autotuner's t_depth 2) give
    the oracle's fields bit for bit, in persistent and per-pass graph mode,
    next to diffusion members on the single-step lists."""
    spec = TWO_SWEEP_MEMBERS
    M = Members(spec)
    _two_sweep_entries(spec)
    try:
        b = M.batch()
        b.run(mode)
        for i, (kind, dims, steps) in enumerate(spec):
            lay = b.layout(i)
            done, _, g = b.result(i)
            assert done == steps
            if kind == "him":
                assert lay["t_depth"] == 2 and lay["units"] == (steps + 1) // 2, (i, lay)
            if i == 0:
                assert lay["wavefront"] == 1
            assert U.bits_equal(ps.PSGridCopyout(g), _want(kind, M.data[i], steps)), (mode, i, lay)
        b.free()
    finally:
        _drop_entries(spec)
        M.free()


@pytest.mark.gpu
def test_batch_two_sweep_himeno_checks_match_one_sweep():
    """With residual checks (every 4 steps, and the first sweep) a pass never
    straddles a check: stop steps, residuals and fields equal those of the
    one-sweep list."""
    spec = [("him", (96, 64, 40), 60), ("him", (40, 33, 33), 45), ("diff", (40, 40, 40), 30)]
    stop = lambda i: ((0.05, 4), (0.08, 4), (0.0, 0))[i]
    results = {}
    for td in (1, 2):
        M = Members(spec)
        if td == 2:
            _two_sweep_entries(spec)
        try:
            b = M.batch(stop)
            b.run(0)
            results[td] = []
            for i in range(len(spec)):
                done, res, g = b.result(i)
                results[td].append((done, res, ps.PSGridCopyout(g), b.layout(i)["t_depth"]))
            b.free()
        finally:
            _drop_entries(spec)
            M.free()
    for i, (kind, dims, steps) in enumerate(spec):
        d1, r1, f1, t1 = results[1][i]
        d2, r2, f2, t2 = results[2][i]
        if kind == "him":
            assert t1 == 1 and t2 == 2
        assert 0 < d1 <= steps
        assert d1 == d2 and r1 == pytest.approx(r2, rel=1e-12), (i, d1, d2, r1, r2)
        assert U.bits_equal(f1, f2), i
        assert U.bits_equal(f2, _want(kind, _inputs(kind, dims, 100 + i), d2)), i
