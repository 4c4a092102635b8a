"""Benchmark of the B200 Physis stencil path.

Default workload (one GPU): 7-point diffusion, 512^3 float, one "step" = one
solve of 1000 time steps run as PSStencilRun(m(g1->g2), m(g2->g1), 500) on
the seeded cos-product field + U[0,1e-3) noise. Metric: lattice updates per
second (GLUPS), whole job. Inputs (537 MB per grid) exceed the 126 MB L2, so
no flush is needed between steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                    [--workload c2|c2f64|c3|c1]

Under torchrun (N > 1) every rank runs an independent replica on its own
GPU (the path does not shard on one node: there is no data exchange), the
timed region is bracketed by barriers and device syncs, and rank 0 prints the
max over ranks. `--impl reference` times the reference's own CPU target
(libphysis_rt_ref built from the reference sources, oracle/_ref) on the host
cores for the same metric.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
COEF = [0.1, 0.1, 0.1, 0.1, 0.1, 0.1, 0.4]  # ce cw cn cs ct cb cc

WORKLOADS = {
    # name: (kernel, dtype, dims, time steps per solve, bytes per lattice update)
    "c2": ("diffusion7", np.float32, (512, 512, 512), 1000, 8),
    "c2f64": ("diffusion7", np.float64, (256, 256, 256), 1000, 16),
    "c3": ("himeno", np.float32, (257, 257, 513), 200, 56),
    "c1": ("diffusion7", np.float32, (64, 64, 64), 100, 8),
    # a user stencil through the generic term table: the 27-point box
    # average (each neighbour times 1/27), interior of 512^3
    "g27": ("generic27", np.float32, (512, 512, 512), 100, 8),
    # the C2 stencil written as a stencil function in the reference's DSL and
    # compiled by the translator-free front end (physis_b200/dsl.py)
    "dsl7": ("dsl7", np.float32, (512, 512, 512), 100, 8),
    # the g27 stencil written as a DSL stencil function (interior domain: the
    # front end's staged form runs it)
    "dsl27": ("dsl27", np.float32, (512, 512, 512), 100, 8),
    # batched: 256 members, see c4_members(); dims/steps are per member
    "c4": ("batch", np.float32, (0, 0, 0), 0, 0),
    # served: a Poisson trace of solve requests, see c5_trace()
    "c5": ("serve", np.float32, (0, 0, 0), 0, 0),
}


def describe(wl):
    k, dt, dims, steps, _ = WORKLOADS[wl]
    if k == "serve":
        return ("served: Poisson arrivals at 2000 req/s, 60% 7-point diffusion fp32 (clamped) / "
                "40% 19-point Himeno fp32 (C3 coefficient distributions), cubes of side "
                "32*12^U (32..384), each to relative residual 1e-5 (checked every 10 steps) or "
                "1000 steps, 150 GB device budget, continuous batching")
    if k == "batch":
        return ("batched: 256 grids, sides 32*8^U per axis (seeded), even members 7-point "
                "diffusion fp32 periodic, odd members 19-point Himeno fp32 (C3 coefficient "
                "distributions), 50-500 steps each (uniform), one persistent launch")
    if k == "himeno":
        return ("19-point Himeno Jacobi %dx%dx%d fp32, %d sweeps per solve, FP64 residual fused "
                "per sweep" % (dims + (steps,)))
    if k == "generic27":
        return ("generic (user) stencil: 27-point box average sum_{d in {-1,0,1}^3} (1/27)*u(p+d) "
                "as a psb_generic_stencil term table, %dx%dx%d fp32 interior [1,n-1)^3, %d time "
                "steps per solve (double-buffered PSStencilRun)" % (dims + (steps,)))
    if k == "dsl27":
        return ("27-point box average %dx%dx%d fp32 written as a DSL stencil function "
                "(physis_b200.workloads.BOX27_DSL: the g27 table's terms, order and "
                "coefficient) and compiled by the translator-free front end, interior "
                "[1,n-1)^3, %d time steps per solve (double-buffered PSStencilRun)"
                % (dims + (steps,)))
    if k == "dsl7":
        return ("7-point diffusion %dx%dx%d fp32 written as a DSL stencil function "
                "(physis_b200.workloads.DIFFUSION7_DSL) and compiled by the translator-free "
                "front end (the kernel form that ran is in config.generic_kernel), %d time "
                "steps per solve (double-buffered PSStencilRun), clamped faces"
                % (dims + (steps,)))
    return ("7-point diffusion %dx%dx%d %s, %d time steps per solve (double-buffered "
            "PSStencilRun), clamped faces" % (dims + ("fp32" if dt == np.float32 else "fp64", steps)))


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# Inputs
# ---------------------------------------------------------------------------
def c2_field(dims, dtype, seed=2024):
    """0.125(1-cos 2pi x/N)(1-cos 2pi y/N)(1-cos 2pi z/N) + U[0,1e-3), seeded."""
    nx, ny, nz = dims
    cx = (1 - np.cos(2 * np.pi * np.arange(nx) / nx)).astype(np.float64)
    cy = (1 - np.cos(2 * np.pi * np.arange(ny) / ny)).astype(np.float64)
    cz = (1 - np.cos(2 * np.pi * np.arange(nz) / nz)).astype(np.float64)
    rng = np.random.default_rng(seed)
    out = np.empty((nz, ny, nx), dtype=dtype)
    for z in range(nz):
        plane = 0.125 * cz[z] * np.outer(cy, cx) + 1e-3 * rng.random((ny, nx))
        out[z] = plane.astype(dtype)
    return out


def himeno_fields(dims, seed=77):
    from physis_b200.workloads import himeno_inputs
    nx, ny, nz = dims
    return himeno_inputs((nz, ny, nx), seed)


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
class Dist:
    """One process per GPU (torchrun env): barriers and max/sum over ranks.
    NCCL on GPU hosts; gloo where no GPU is visible (host-side tests)."""

    def __init__(self, gpus):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            timeout = datetime.timedelta(seconds=300)
            if torch.cuda.is_available():
                torch.cuda.set_device(self.local)
                self.device = "cuda"
                dist.init_process_group("nccl", timeout=timeout,
                                        device_id=torch.device("cuda", self.local))
            else:
                dist.init_process_group("gloo", timeout=timeout)
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def _reduce(self, v, op):
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=op)
        return float(t.item())

    def max(self, v):
        return self._reduce(v, self.pg.ReduceOp.MAX if self.pg else None)

    def sum(self, v):
        return self._reduce(v, self.pg.ReduceOp.SUM if self.pg else None)

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()
            self.pg = None


def load_traffic(kernel_name):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        return t.get(kernel_name)
    except Exception:
        return None


def cpu_baseline_sample(wl, field=None):
    """The reference CPU target (1 thread) on a bounded sample of the workload."""
    from oracle import oracle
    k, dt, dims, steps, bpl = WORKLOADS[wl]
    nx, ny, nz = dims
    use_ref = oracle.ref_available()
    if k == "himeno":
        p, coef = himeno_fields(dims)
        sweeps = 4
        if use_ref:
            _, secs = oracle.ref_himeno(p, coef, 0.8, sweeps)
        else:
            t0 = time.perf_counter()
            oracle.himeno(p, coef, 0.8, sweeps)
            secs = time.perf_counter() - t0
        pts = (nx - 2) * (ny - 2) * (nz - 2) * sweeps
        sample = "%dx%dx%d, %d sweeps" % (nx, ny, nz, sweeps)
    elif k == "generic27":
        f = field if field is not None else c2_field(dims, dt)
        count = 2
        c = float(np.float32(1.0 / 27.0))
        if use_ref:
            _, secs = oracle.ref_box27(f, count, c)
        else:
            from physis_b200.workloads import box27_struct
            import physis_b200 as ps
            w = [f.copy(), f.copy()]
            t0 = time.perf_counter()
            oracle.generic_apply(box27_struct(ps.PS_FLOAT), w, [1, 1, 1],
                                 [nx - 1, ny - 1, nz - 1])
            secs = (time.perf_counter() - t0) * count
        pts = (nx - 2) * (ny - 2) * (nz - 2) * count
        sample = "%dx%dx%d, %d time steps of the 27-point box average" % (nx, ny, nz, count)
    else:
        f = field if field is not None else c2_field(dims, dt)
        count = 12 if nx * ny * nz >= 1 << 26 else 100
        if use_ref:
            _, secs = oracle.ref_diffusion7(f, count, np.asarray(COEF, dt))
        else:
            t0 = time.perf_counter()
            oracle.diffusion7(f, count, np.asarray(COEF, dt))
            secs = time.perf_counter() - t0
        pts = nx * ny * nz * count
        sample = "%dx%dx%d %s, %d time steps" % (nx, ny, nz, np.dtype(dt).name, count)
    kind = "reference" if use_ref else "port"
    who = ("reference CPU target: libphysis_rt_ref built from the reference runtime sources + "
           "translator-shaped run loop" if use_ref else "oracle port (C restatement)")
    return {"value": pts / secs / 1e9, "unit": "GLUPS", "cores": 1, "kind": kind,
            "sample": sample + "; " + who + "; run loop only, copies excluded"}


# ---------------------------------------------------------------------------
# Numerics: every run states its error against the FP64 oracle
# ---------------------------------------------------------------------------
NUMERICS_SIDE = 96       # the full-length solve is checked at this size
NUMERICS_FULL_STEPS = 2  # the full-size grid is checked after this many steps


def _coef_sum(dt):
    return float(sum(np.float64(np.asarray(COEF, dt))))


def numerics_diffusion(ps, dt, dims, tsteps, grids, m1, m2, host, mass0, mass1, steps_done,
                       kernel_id=None):
    """Error of the 7-point path against the oracle, outside the timed
    region: (1) the full-size grid after NUMERICS_FULL_STEPS steps from the
    workload's field, against the oracle port (the reference CPU target bit
    for bit: `bit_exact_vs_reference`) and the FP64 oracle; (2) a full-length
    solve (tsteps steps) of the same field formula at NUMERICS_SIDE^3,
    likewise; (3) the timed solves themselves: the clamped scheme conserves
    sum(u) * (sum of coefficients)^steps exactly, so the drift of the device
    sum (FP64 reduction) from that value is the rounding of every step run."""
    from oracle import oracle
    coef = np.asarray(COEF, dt)
    out = {"vs": "FP64 oracle (the reference's algorithm and term order in double from the "
                 "same inputs); bit_exact_vs_reference: equality with the oracle port, which "
                 "equals the reference CPU target bit for bit"}
    # (3) mass after every warm-up and timed step
    expect = mass0 * _coef_sum(dt) ** steps_done
    out["timed_solves_mass"] = {"steps": steps_done, "sum_initial": mass0, "sum_final": mass1,
                                "sum_expected": expect, "rel_drift": abs(mass1 - expect) / abs(expect)}
    # (1) full size, a few steps
    ps.PSGridCopyin(grids[0], host)
    ps.PSStencilRun(m1, m2, NUMERICS_FULL_STEPS // 2)
    got = ps.PSGridCopyout(grids[0])
    want = oracle.diffusion7(host, NUMERICS_FULL_STEPS, coef)
    ref64 = oracle.diffusion7_fp64(host, NUMERICS_FULL_STEPS, coef)
    full = {"sample": "%dx%dx%d after %d steps" % (dims + (NUMERICS_FULL_STEPS,)),
            "bit_exact_vs_reference": bool(np.array_equal(got.view(np.uint8), want.view(np.uint8)))}
    full.update(oracle.error_norms(got, ref64))
    full["max_ulp_vs_reference"] = oracle.error_norms(got, want)["max_ulp_err"]
    if ps.get_fp_mode() == ps.FP_FMA:
        # the exact arithmetic on the same grid: equal to the reference bit for bit
        ps.set_fp_mode(ps.FP_EXACT)
        ps.PSGridCopyin(grids[0], host)
        ps.PSStencilRun(m1, m2, NUMERICS_FULL_STEPS // 2)
        ex = ps.PSGridCopyout(grids[0])
        ps.set_fp_mode(ps.FP_FMA)
        full["exact_mode_bit_exact_vs_reference"] = bool(
            np.array_equal(ex.view(np.uint8), want.view(np.uint8)))
        del ex
    del got, want, ref64
    out["full_size"] = full
    # (2) full-length solve, smaller grid
    n = NUMERICS_SIDE
    f = c2_field((n, n, n), dt)
    g = [ps.grid_new(ps.PS_FLOAT if dt == np.float32 else ps.PS_DOUBLE, (n, n, n))
         for _ in range(2)]
    ps.PSGridCopyin(g[0], f)
    d = ps.PSDomain3DNew(0, n, 0, n, 0, n)
    kid = ps.DIFFUSION7 if kernel_id is None else kernel_id
    a = ps.PSStencilMap(kid, d, g[0], g[1], *COEF)
    b = ps.PSStencilMap(kid, d, g[1], g[0], *COEF)
    ps.PSStencilRun(a, b, tsteps // 2)
    got = ps.PSGridCopyout(g[0])
    for x in g:
        ps.PSGridFree(x)
    want = oracle.diffusion7(f, tsteps, coef)
    ref64 = oracle.diffusion7_fp64(f, tsteps, coef)
    solve = {"sample": "%d^3, %d steps (the full solve length), same field formula" % (n, tsteps),
             "bit_exact_vs_reference": bool(np.array_equal(got.view(np.uint8), want.view(np.uint8)))}
    solve.update(oracle.error_norms(got, ref64))
    solve["reference_vs_fp64"] = oracle.error_norms(want, ref64)
    solve["max_ulp_vs_reference"] = oracle.error_norms(got, want)["max_ulp_err"]
    out["full_solve"] = solve
    out["bit_exact_vs_reference"] = full["bit_exact_vs_reference"] and solve["bit_exact_vs_reference"]
    out["max_abs_err"] = max(full["max_abs_err"], solve["max_abs_err"])
    out["rms_err"] = solve["rms_err"]
    return out


def numerics_himeno(ps, dims, tsteps, grids, m1, m2, p, coef):
    """Error of the Himeno path: the full-size grids after 2 sweeps and a
    full-length run (tsteps sweeps) at 65x65x129, each against the oracle
    port (bit-exact check, per-sweep residuals) and the FP64 oracle."""
    from oracle import oracle
    from physis_b200.workloads import himeno_gpu, himeno_inputs
    out = {"vs": "FP64 oracle (the reference's algorithm and term order in double from the "
                 "same inputs); bit_exact_vs_reference: equality with the oracle port, which "
                 "equals the reference CPU target bit for bit"}
    ps.PSGridCopyin(grids[0], p)
    ps.PSGridCopyin(grids[1], p)
    ps.PSStencilRun(m1, m2, 1)
    got = ps.PSGridCopyout(grids[0])
    want, wg = oracle.himeno(p, coef, 0.8, 2)
    ref64, g64 = oracle.himeno_fp64(p, coef, 0.8, 2)
    full = {"sample": "%dx%dx%d after 2 sweeps" % dims,
            "bit_exact_vs_reference": bool(np.array_equal(got.view(np.uint8), want.view(np.uint8)))}
    full.update(oracle.error_norms(got, ref64))
    del got, want, ref64
    out["full_size"] = full
    shape = (129, 65, 65)
    ps_, cf = himeno_inputs(shape, 5)
    got, gg = himeno_gpu(ps_, cf, 0.8, tsteps)
    want, wg = oracle.himeno(ps_, cf, 0.8, tsteps)
    ref64, g64 = oracle.himeno_fp64(ps_, cf, 0.8, tsteps)
    solve = {"sample": "65x65x129, %d sweeps (the full run length)" % tsteps,
             "bit_exact_vs_reference": bool(np.array_equal(got.view(np.uint8), want.view(np.uint8)))}
    solve.update(oracle.error_norms(got, ref64))
    gg = np.asarray(gg)
    solve["gosa_max_rel_diff_vs_reference"] = float(np.max(np.abs(gg - wg) / np.abs(wg)))
    solve["gosa_max_rel_err_vs_fp64"] = float(np.max(np.abs(gg - g64) / np.abs(g64)))
    out["full_solve"] = solve
    out["bit_exact_vs_reference"] = full["bit_exact_vs_reference"] and solve["bit_exact_vs_reference"]
    out["max_abs_err"] = max(full["max_abs_err"], solve["max_abs_err"])
    out["rms_err"] = solve["rms_err"]
    return out


def generic27_stencil(ps, accum=None):
    from physis_b200.workloads import box27_stencil
    return box27_stencil(accum if accum is not None else ps.PS_FLOAT)


def numerics_generic27(ps, dt, n=96, steps=10, kernel_id=None, params=()):
    """The generic 27-point path at n^3 for `steps` steps against the oracle
    port (bit-exact check) and the FP64 oracle (the same term table
    evaluated in double by the port)."""
    from oracle import oracle
    from physis_b200.workloads import box27_stencil, box27_struct
    f = c2_field((n, n, n), dt)
    kid = box27_stencil(ps.PS_FLOAT).kernel_id if kernel_id is None else kernel_id
    g = [ps.grid_new(ps.PS_FLOAT, (n, n, n)) for _ in range(2)]
    for x in g:
        ps.PSGridCopyin(x, f)
    d = ps.PSDomain3DNew(1, n - 1, 1, n - 1, 1, n - 1)
    a = ps.PSStencilMap(kid, d, g[0], g[1], *params)
    b = ps.PSStencilMap(kid, d, g[1], g[0], *params)
    ps.PSStencilRun(a, b, steps // 2)
    got = ps.PSGridCopyout(g[0])
    exact = None
    if ps.get_fp_mode() == ps.FP_FMA:
        # the exact arithmetic on the same field: the reference's bits
        ps.set_fp_mode(ps.FP_EXACT)
        for x in g:
            ps.PSGridCopyin(x, f)
        ps.PSStencilRun(a, b, steps // 2)
        exact = ps.PSGridCopyout(g[0])
        ps.set_fp_mode(ps.FP_FMA)
    for x in g:
        ps.PSGridFree(x)
    want = [f.copy(), f.copy()]
    ref = [f.astype(np.float64), f.astype(np.float64)]
    s32, s64 = box27_struct(ps.PS_FLOAT), box27_struct(ps.PS_DOUBLE)
    for i in range(steps):
        src, dst = (0, 1) if i % 2 == 0 else (1, 0)
        oracle.generic_apply(s32, [want[src], want[dst]], [1, 1, 1], [n - 1] * 3)
        oracle.generic_apply(s64, [ref[src], ref[dst]], [1, 1, 1], [n - 1] * 3)
    out = {"vs": "FP64 oracle (the same term table evaluated in double by the oracle port); "
                 "bit_exact_vs_reference: equality with the oracle port's float evaluation "
                 "(the reference CPU target's arithmetic)",
           "sample": "%d^3, %d steps of the same stencil and field formula" % (n, steps),
           "bit_exact_vs_reference": bool(np.array_equal(got.view(np.uint8),
                                                         want[0].view(np.uint8)))}
    if exact is not None:
        out["exact_mode_bit_exact_vs_reference"] = bool(
            np.array_equal(exact.view(np.uint8), want[0].view(np.uint8)))
        out["exact_mode_errors"] = oracle.error_norms(exact, ref[0])
    out.update(oracle.error_norms(got, ref[0]))
    return out


def run_ours(args):
    dist = Dist(args.gpus)
    os.environ["PHYSIS_B200_DEVICE"] = str(dist.local)
    import physis_b200 as ps
    ps.PSInit()
    wl = args.workload
    kname, dt, dims, tsteps, bpl = WORKLOADS[wl]
    nx, ny, nz = dims
    ptype = ps.PS_FLOAT if dt == np.float32 else ps.PS_DOUBLE
    kernel = ps.HIMENO19 if kname == "himeno" else ps.DIFFUSION7
    tune = None
    if kname not in ("generic27", "dsl7", "dsl27"):
        tune = ps.autotune(kernel, ptype, dims) if args.tune else ps.tune_get(kernel, ptype, dims)
        if args.t_depth and kname == "diffusion7" and dt == np.float32:
            # pin the temporal depth of this shape (profiling)
            tune = dict(tune, t_depth=args.t_depth)
            if args.t_depth == 2:
                tune.update(impl=ps.IMPL_TMA, tile_x=128, tile_y=16)
            if args.z_chunk:
                tune.update(z_chunk=args.z_chunk)
            ps.tune_set(kernel, ptype, dims, **tune)
    if args.plain:
        # the thread-per-point shape of the reference's generated kernels
        ps.set_impl(ps.IMPL_GENERIC if kname == "generic27" else ps.IMPL_PLAIN)
    # The 7-point workloads time the contracted (FMA) arithmetic by default
    # and report the exact (reference-identical) arithmetic beside it.
    fma = kname in ("diffusion7", "generic27") and not args.plain and \
        args.fp_mode in ("auto", "fma")
    ps.set_fp_mode(ps.FP_FMA if fma else ps.FP_EXACT)

    # Inputs, pinned host buffers for the end-to-end leg.
    if kname == "himeno":
        p, coef = himeno_fields(dims)
        host = p
        grids = [ps.PSGrid3DFloatNew(nx, ny, nz) for _ in range(14)]
        ps.PSGridCopyin(grids[0], p)
        ps.PSGridCopyin(grids[1], p)
        for i in range(12):
            ps.PSGridCopyin(grids[2 + i], coef[i])
        dom = ps.PSDomain3DNew(1, nx - 1, 1, ny - 1, 1, nz - 1)
        m1 = ps.PSStencilMap(ps.HIMENO19, dom, *grids, 0.8)
        m2 = ps.PSStencilMap(ps.HIMENO19, dom, *([grids[1], grids[0]] + grids[2:]), 0.8)
        if not args.no_residual:
            ps.himeno_residual_enable(m1, tsteps)
            ps.himeno_residual_enable(m2, tsteps)
        pts_per_step = (nx - 2) * (ny - 2) * (nz - 2) * tsteps
        g_io = grids[0]
    elif kname in ("generic27", "dsl27"):
        host = c2_field(dims, dt)
        grids = [ps.grid_new(ptype, dims), ps.grid_new(ptype, dims)]
        ps.PSGridCopyin(grids[0], host)
        ps.PSGridCopyin(grids[1], host)  # the boundary cells stay as they are
        kid, kparams = generic27_stencil(ps).kernel_id, ()
        if kname == "dsl27":
            from physis_b200 import dsl
            from physis_b200.workloads import BOX27_DSL
            kid = dsl.compile_stencils(BOX27_DSL)["box27"].kernel_id
            kparams = (float(np.float32(1.0 / 27.0)),)
        dom = ps.PSDomain3DNew(1, nx - 1, 1, ny - 1, 1, nz - 1)
        m1 = ps.PSStencilMap(kid, dom, grids[0], grids[1], *kparams)
        m2 = ps.PSStencilMap(kid, dom, grids[1], grids[0], *kparams)
        pts_per_step = (nx - 2) * (ny - 2) * (nz - 2) * tsteps
        g_io = grids[0]
    else:
        host = c2_field(dims, dt)
        grids = [ps.grid_new(ptype, dims), ps.grid_new(ptype, dims)]
        ps.PSGridCopyin(grids[0], host)
        dom = ps.PSDomain3DNew(0, nx, 0, ny, 0, nz)
        kid = ps.DIFFUSION7
        if kname == "dsl7":
            from physis_b200 import dsl
            from physis_b200.workloads import DIFFUSION7_DSL
            kid = dsl.compile_stencils(DIFFUSION7_DSL)["diffusion7"].kernel_id
        m1 = ps.PSStencilMap(kid, dom, grids[0], grids[1], *COEF)
        m2 = ps.PSStencilMap(kid, dom, grids[1], grids[0], *COEF)
        pts_per_step = nx * ny * nz * tsteps
        g_io = grids[0]

    def solve():
        ps.PSStencilRun(m1, m2, tsteps // 2)
        return ps.last_run_stats()

    # ---- device-resident timing ------------------------------------------
    mass0 = ps.reduce64(ps.PS_SUM, g_io) if kname in ("diffusion7", "dsl7") else None
    for _ in range(args.warmup):
        solve()
    ps.sync()
    sampler = ClockSampler(dist.local)
    dist.barrier()
    ps.sync()
    sampler.start()
    ms_list, launches = [], 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ms, n = solve()
        ms_list.append(ms)
        launches += n
    ps.sync()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    dist.barrier()
    mass1 = ps.reduce64(ps.PS_SUM, g_io) if kname in ("diffusion7", "dsl7") else None
    exact_mode = None
    if fma:
        # The same solves with the exact arithmetic (outside the headline's
        # timed region, same grids and launch configuration).
        ps.set_fp_mode(ps.FP_EXACT)
        solve()
        ms_e = [solve()[0] for _ in range(args.steps)]
        ps.sync()
        ps.set_fp_mode(ps.FP_FMA)
        t_e = dist.max(sum(ms_e) / 1e3)
        v_e = dist.sum(pts_per_step * args.steps) / t_e / 1e9
        peak_e = peaks()[0]
        exact_mode = {"value": v_e, "unit": "GLUPS", "ms_per_step": t_e / args.steps * 1e3,
                      "frac": bpl * pts_per_step / (t_e / args.steps) / 1e9 / peak_e,
                      "what": "the same solves with every product and sum rounded in the "
                              "reference's order (bit-identical to the reference CPU target)"}
    gimpl = None
    if kname in ("dsl7", "dsl27"):
        form = ps.compiled_last_staged()
        gimpl = ("staged form: the function body over the TMA plane ring (k_generic_tma's "
                 "kernel body)%s" % (", reads that leave the point checked against the grid"
                                      if form == 2 else "") if form else
                 "thread per (x, y) point with a z loop (the reference's generated-kernel shape)")
    if kname == "generic27":
        import ctypes
        v = ctypes.c_int()
        ps.check(ps.lib.psb_generic_last_impl(ctypes.byref(v)), "psb_generic_last_impl")
        gimpl = {ps.IMPL_TMA: "k_generic_tma (TMA z-streaming)",
                 ps.IMPL_GENERIC: "k_generic (thread per point)"}.get(v.value, str(v.value))
        if v.value == ps.IMPL_TMA:
            gimpl += (", compiled at run time for this table (psb_generic_tma_compiled)"
                      if ps.generic_last_compiled() else ", interpreting the table")
    dev_s = sum(ms_list) / 1e3
    dev_s_max = dist.max(dev_s)
    total_pts = dist.sum(pts_per_step * args.steps)
    value = total_pts / dev_s_max / 1e9
    per_launch_s = dev_s / launches
    alg_bytes = bpl * (pts_per_step / tsteps)
    hbm, peak_kind = peaks()
    # Compulsory bytes of every update over the device time (GLUPS x B/LUP):
    # the same as per-launch bytes over launch time when every launch is one
    # step; with two steps per launch (temporal blocking) it is the effective
    # bandwidth and may exceed the copy peak.
    achieved = bpl * pts_per_step * args.steps / dev_s / 1e9
    two_sweeps = kname == "himeno" and tune is not None and tune.get("t_depth") == 2
    two_steps = kname == "diffusion7" and tune is not None and tune.get("t_depth") == 2
    kname_traffic = ("k_himeno_tb2" if two_sweeps else "k_himeno_tma") if kname == "himeno" else \
        ("k_diff7_tb2_f32" + ("_fma" if fma else "")) if two_steps else \
        "k_generic_tma_f32" if kname == "generic27" else "k_dsl_diffusion7_f32" if kname == "dsl7" \
        else "k_dsl_box27_f32" if kname == "dsl27" else (
        "k_diff7_tma_f32" if dt == np.float32 else "k_diff7_tma_f64") + ("_fma" if fma else "")
    if args.plain:
        kname_traffic = kname_traffic.replace("tma", "plain")
    traffic = load_traffic("%s_%dx%dx%d" % (kname_traffic, nx, ny, nz))

    # ---- end to end through the C ABI, host buffers --------------------------
    import ctypes
    nbytes = host.nbytes
    hp = ctypes.c_void_p()
    ps.check(ps.lib.psb_host_alloc(nbytes, ctypes.byref(hp)), "psb_host_alloc")
    pinned = np.ctypeslib.as_array((ctypes.c_char * nbytes).from_address(hp.value))
    pinned = pinned.view(host.dtype).reshape(host.shape)
    pinned[...] = host
    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 3))
    e2e_value = None
    if e2e_steps:
        ps.PSGridCopyin(g_io, pinned)
        solve()
        ps.PSGridCopyout(g_io, pinned)
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ps.PSGridCopyin(g_io, pinned)
            solve()
            ps.PSGridCopyout(g_io, pinned)
        e2e_s = dist.max(time.perf_counter() - t0)
        e2e_value = dist.sum(pts_per_step * e2e_steps) / e2e_s / 1e9
    ps.check(ps.lib.psb_host_free(hp), "psb_host_free")

    numerics = None
    if dist.rank == 0 and not args.no_numerics:
        if kname == "himeno":
            numerics = numerics_himeno(ps, dims, tsteps, grids, m1, m2, p, coef)
        elif kname == "generic27":
            numerics = numerics_generic27(ps, dt)
        elif kname == "dsl27":
            numerics = numerics_generic27(ps, dt, kernel_id=kid, params=kparams)
        else:
            numerics = numerics_diffusion(ps, dt, dims, tsteps, grids, m1, m2, host, mass0, mass1,
                                          (args.warmup + args.steps) * tsteps,
                                          kernel_id=kid if kname == "dsl7" else None)
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(wl if kname != "dsl27" else "g27",
                                  host if kname in ("diffusion7", "generic27", "dsl7", "dsl27")
                                  else None)

    line = {
        "metric": "lattice_updates_per_s_" + wl,
        "value": value,
        "unit": "GLUPS",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_s_max / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if dt == np.float32 else "f64",
        "data": "synthetic",
        "config": {
            "workload": describe(wl),
            "step": "one solve of %d time steps (PSStencilRun of two maps x %d)" % (tsteps, tsteps // 2),
            "inputs_vs_l2": "%.0f MB per grid > 126 MB L2; no flush needed" % (host.nbytes / 1e6),
            "parallelism": "replicas (one independent solve per GPU, no exchange)",
            "impl": ("DSL stencil function compiled by physis_b200.dsl" if kname in ("dsl7", "dsl27")
                     else
                     "plain" if args.plain else "autotuned"),
            "fp_mode": (("fma: the reference's term order with fused multiply-adds (one "
                         "rounding per term; every point within 4 ulp of the exact step per "
                         "step; errors against the FP64 oracle in `numerics`)")
                        if fma and kname == "diffusion7" else
                        ("fma: the table's term order, each term after the first added by a "
                         "fused multiply-add in the kernel compiled for the table (errors "
                         "against the FP64 oracle, and the exact mode's bit-equality with the "
                         "reference, in `numerics`)") if fma else
                        "exact: every product and sum rounded in the reference's term order "
                        "(bit-identical to the reference CPU target)"),
            "exact_mode": exact_mode,
            "tune": tune,
            "generic_kernel": gimpl,
            "hbm_gbs_effective": value * bpl,
            "wall_s_timed": wall,
        },
        "roofline": {
            "bound": "hbm",
            "achieved": achieved,
            "peak": hbm,
            "unit": "GB/s",
            "frac": achieved / hbm,
            "traffic": traffic,
            "peak_source": peak_kind,
            "algorithmic_bytes_per_step": alg_bytes,
            "avg_launch_us": per_launch_s * 1e6,
            "steps_per_launch": (tsteps * args.steps) / launches,
            "achieved_is": "compulsory bytes per lattice update x updates / device time "
                           "(effective; with two steps per launch it may exceed the peak)",
        },
        "e2e": {"value": e2e_value, "unit": "GLUPS", "h2d_bytes_per_step": int(nbytes),
                "d2h_bytes_per_step": int(nbytes), "steps": e2e_steps,
                "path": "PSGridCopyin(pinned) + PSStencilRun + PSGridCopyout(pinned) via the C ABI"},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "cpu_baseline": cpu,
        "numerics": numerics,
    }
    for g in grids:
        ps.PSGridFree(g)
    dist.close()
    if dist.rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Reference arm
# ---------------------------------------------------------------------------
def _ref_worker(args):
    kind, dims, dt_name, count, seed = args
    sys.path.insert(0, ROOT)
    from oracle import oracle
    dt = np.dtype(dt_name)
    if kind == "himeno":
        p, coef = himeno_fields(dims, seed)
        _, secs = oracle.ref_himeno(p, coef, 0.8, count)
        nx, ny, nz = dims
        return (nx - 2) * (ny - 2) * (nz - 2) * count, secs
    if kind == "generic27":
        f = c2_field(dims, dt, seed)
        _, secs = oracle.ref_box27(f, count, float(np.float32(1.0 / 27.0)))
        nx, ny, nz = dims
        return (nx - 2) * (ny - 2) * (nz - 2) * count, secs
    f = c2_field(dims, dt, seed)
    _, secs = oracle.ref_diffusion7(f, count, np.asarray(COEF, dt), periodic=kind == "diffusion7p")
    return dims[0] * dims[1] * dims[2] * count, secs


def c4_members(seed=4242, count=256):
    """(kind, (nx, ny, nz), steps) of the batched workload, seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        dims = tuple(int(round(32 * 8 ** rng.random())) for _ in range(3))
        steps = int(rng.integers(50, 501))
        out.append(("diffp" if i % 2 == 0 else "him", dims, steps))
    return out


def c4_build(ps, members):
    """Grids of every member, filled on the device with the seeded fields."""
    grids = []
    for i, (kind, dims, steps) in enumerate(members):
        if kind == "diffp":
            g = [ps.grid_new(ps.PS_FLOAT, dims) for _ in range(2)]
            ps.grid_fill(g[0], ps.FILL_UNIFORM, 1000 + i, 0.0, 1.0)
        else:
            g = [ps.grid_new(ps.PS_FLOAT, dims) for _ in range(14)]
            ps.grid_fill(g[0], ps.FILL_ZPROFILE)
            ps.grid_fill(g[1], ps.FILL_ZPROFILE)
            ranges = [(0.9, 1.1)] * 3 + [(0.95 / 6, 1.05 / 6)] + [(-0.01, 0.01)] * 3 + [(0.9, 1.1)] * 3
            for k, (lo, hi) in enumerate(ranges):
                ps.grid_fill(g[2 + k], ps.FILL_UNIFORM, 100000 * (i + 1) + k, lo, hi)
            ps.grid_fill(g[12], ps.FILL_BND)
            ps.grid_fill(g[13], ps.FILL_CONST, 0, 0.0)
        grids.append(g)
    ps.sync()
    return grids


def c4_batch(ps, members, grids):
    b = ps.Batch()
    for (kind, dims, steps), g in zip(members, grids):
        if kind == "diffp":
            b.add(ps.DIFFUSION7_PERIODIC, g, COEF, steps)
        else:
            b.add(ps.HIMENO19, g, [0.8], steps)
    return b


def c4_traffic(alg_bytes):
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return alg_bytes * float(json.load(f)["k_batch_c4_traffic_per_algorithmic_byte"])
    except Exception:
        return None


def c4_e2e(ps, members, grids, b, lups, dist, reps=2):
    """The batch through the public API with host buffers: every member's
    input grids (7-point: the field; Himeno: both p grids and the twelve
    coefficient fields) copied in from pinned host memory, the batch run,
    every result grid copied back, all inside the timed region."""
    import ctypes
    ins, outs = [], []
    for (kind, dims, steps), g in zip(members, grids):
        ins += [g[0]] if kind == "diffp" else list(g)
        outs.append(g[steps & 1])
    n_in = sum(int(np.prod(g.dims)) for g in ins)
    n_out = sum(int(np.prod(g.dims)) for g in outs)
    hp = ctypes.c_void_p()
    ps.check(ps.lib.psb_host_alloc((n_in + n_out) * 4, ctypes.byref(hp)), "psb_host_alloc")
    host = np.ctypeslib.as_array((ctypes.c_float * (n_in + n_out)).from_address(hp.value))
    off, ptr_in, ptr_out = 0, [], []
    for g in ins:
        ptr_in.append(hp.value + off * 4)
        off += int(np.prod(g.dims))
    for g in outs:
        ptr_out.append(hp.value + off * 4)
        off += int(np.prod(g.dims))
    for g, p in zip(ins, ptr_in):  # the inputs as they are now, as host data
        ps.check(ps.lib.psb_grid_copyout_async(g.ptr, ctypes.c_void_p(p)), "copyout")
    ps.sync()

    def one():
        for g, p in zip(ins, ptr_in):
            ps.check(ps.lib.psb_grid_copyin_async(g.ptr, ctypes.c_void_p(p)), "copyin")
        b.run(0)
        for g, p in zip(outs, ptr_out):
            ps.check(ps.lib.psb_grid_copyout_async(g.ptr, ctypes.c_void_p(p)), "copyout")
        ps.sync()

    one()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(reps):
        one()
    secs = dist.max(time.perf_counter() - t0)
    ps.check(ps.lib.psb_host_free(hp), "psb_host_free")
    del host
    return {"value": dist.sum(lups * reps) / secs / 1e9, "unit": "GLUPS",
            "h2d_bytes_per_step": n_in * 4, "d2h_bytes_per_step": n_out * 4}


C4_HIMENO_RANGES = [(0.9, 1.1)] * 3 + [(0.95 / 6, 1.05 / 6)] + [(-0.01, 0.01)] * 3 + [(0.9, 1.1)] * 3


def c4_host_inputs(ps, kind, dims, i):
    """Host copies of member i's seeded inputs (the host restatement of the
    device fills of c4_build, equal to them bit for bit)."""
    if kind == "diffp":
        return ps.fill_reference(dims, ps.FILL_UNIFORM, 1000 + i, 0.0, 1.0), None
    p = ps.fill_reference(dims, ps.FILL_ZPROFILE)
    coef = [ps.fill_reference(dims, ps.FILL_UNIFORM, 100000 * (i + 1) + k, lo, hi)
            for k, (lo, hi) in enumerate(C4_HIMENO_RANGES)]
    coef += [ps.fill_reference(dims, ps.FILL_BND), np.zeros(tuple(reversed(dims)), np.float32)]
    return p, coef


def member_numerics(kind, data, steps, got):
    """One solve against the oracle port (bit-exact check) and the FP64
    oracle (error norms). kind: "diff", "diffp" or "him"."""
    from oracle import oracle
    f, coef = data
    if kind == "him":
        want = oracle.himeno(f, coef, 0.8, steps)[0]
        ref64 = oracle.himeno_fp64(f, coef, 0.8, steps)[0]
    else:
        per = kind == "diffp"
        want = oracle.diffusion7(f, steps, np.asarray(COEF, np.float32), periodic=per)
        ref64 = oracle.diffusion7_fp64(f, steps, COEF, periodic=per)
    out = {"bit_exact_vs_reference": bool(np.array_equal(got.view(np.uint8), want.view(np.uint8)))}
    out.update(oracle.error_norms(got, ref64))
    return out


def summarize_numerics(recs, what):
    return {"vs": "FP64 oracle (the reference's algorithm and term order in double from the "
                  "same inputs); bit_exact_vs_reference: equality with the oracle port, which "
                  "equals the reference CPU target bit for bit",
            "sample": what, "solves_checked": len(recs),
            "bit_exact_vs_reference": all(r["bit_exact_vs_reference"] for r in recs),
            "max_abs_err": max(r["max_abs_err"] for r in recs),
            "rms_err": float(np.sqrt(np.mean([r["rms_err"] ** 2 for r in recs]))),
            "max_rel_err": max(r["max_rel_err"] for r in recs),
            "per_solve": recs}


def c4_numerics(ps, members, grids, b, max_work=3e8):
    """After the timed runs: the sampled members' inputs are regenerated,
    the whole batch runs once more (mode 0), and each sampled member is
    compared with the oracle. Sample: the five cheapest members of each kind
    and the cheapest member of each kind that took the wavefront path."""
    def work(i):
        k, d, st = members[i]
        return d[0] * d[1] * d[2] * st
    sample = []
    for kind in ("diffp", "him"):
        ids = sorted((i for i, m in enumerate(members) if m[0] == kind), key=work)
        sample += ids[:5]
        wave = [i for i in ids if b.layout(i)["wavefront"] and work(i) <= max_work]
        if wave:
            sample.append(wave[0])
    for i in sample:
        kind, dims, steps = members[i]
        g = grids[i]
        if kind == "diffp":
            ps.grid_fill(g[0], ps.FILL_UNIFORM, 1000 + i, 0.0, 1.0)
        else:
            ps.grid_fill(g[0], ps.FILL_ZPROFILE)
            ps.grid_fill(g[1], ps.FILL_ZPROFILE)
    ps.sync()
    b.run(0)
    recs = []
    for i in sample:
        kind, dims, steps = members[i]
        done, _, g = b.result(i)
        got = ps.PSGridCopyout(g)
        r = member_numerics(kind, c4_host_inputs(ps, kind, dims, i), done, got)
        r.update({"member": i, "kind": kind, "dims": list(dims), "steps": done,
                  "wavefront": bool(b.layout(i)["wavefront"])})
        recs.append(r)
    return summarize_numerics(recs, "the five cheapest members of each kind and the cheapest "
                                    "wavefront-path member of each kind (<= %.0e updates), "
                                    "rerun from their seeded inputs in the whole batch" % max_work)


def run_c4(args, dist):
    os.environ["PHYSIS_B200_DEVICE"] = str(dist.local)
    import physis_b200 as ps
    ps.PSInit()
    members = c4_members(count=args.members)
    if args.c4_kind:
        members = [m for m in members if m[0] == args.c4_kind]
    if args.c4_cube:
        members = [(k, (args.c4_cube,) * 3, st) for k, _, st in members]
    if args.c4_steps:
        members = [(k, d, args.c4_steps) for k, d, _ in members]
    if args.him_two_sweeps:
        for k, d, _ in members:
            if k == "him":
                ps.batch_tune_set(ps.HIMENO19, d, impl=ps.IMPL_TMA, tile_x=64, tile_y=8, z_chunk=0,
                                  stages=6, t_depth=2)
    grids = c4_build(ps, members)
    b = c4_batch(ps, members, grids)
    if args.tune:
        b.autotune(force=True)  # tile shapes and z chunks per member size bucket, cached
    lups = sum(((d[0] - 2) * (d[1] - 2) * (d[2] - 2) if k == "him" else d[0] * d[1] * d[2]) * st
               for k, d, st in members)
    alg_bytes = sum(((d[0] - 2) * (d[1] - 2) * (d[2] - 2) * 56 if k == "him"
                     else d[0] * d[1] * d[2] * 8) * st for k, d, st in members)

    def timed(mode, reps, warm):
        for _ in range(warm):
            b.run(mode)
        ms = []
        for _ in range(reps):
            b.run(mode)
            ms.append(b.stats()["device_ms"])
        return ms

    res = {1: timed(1, 2, 1) if not args.skip_graph else [float("nan")]}  # per-step graph mode
    timed(0, 0, args.warmup)    # warm up the persistent mode (the headline)
    sampler = ClockSampler(dist.local)
    dist.barrier()
    sampler.start()
    ms_p = timed(0, args.steps, 0)
    clocks = sampler.stop()
    dev_s = dist.max(sum(ms_p) / 1e3)
    value = dist.sum(lups * args.steps) / dev_s / 1e9
    launches = b.stats()["launches"] * args.steps
    loop_plain = timed(2, 1, 0)[0] if not args.skip_loops else float("nan")
    loop_tuned = timed(3, 1, 0)[0] if not args.skip_loops else float("nan")
    per_run_s = dev_s / args.steps
    e2e = None if args.no_e2e else c4_e2e(ps, members, grids, b, lups, dist)
    numerics = None
    if dist.rank == 0 and not args.no_numerics:
        numerics = c4_numerics(ps, members, grids, b)
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        rate_d, rate_h, kind, sample = cpu_rates(periodic=True)
        lu_d = sum(d[0] * d[1] * d[2] * st for k, d, st in members if k == "diffp")
        lu_h = lups - lu_d
        cpu = {"value": lups / (lu_d / rate_d + lu_h / rate_h) / 1e9, "unit": "GLUPS",
               "cores": 1, "kind": kind,
               "sample": sample + "; GLUPS = the batch's updates / sum of updates / rate per kind"}
    line = {
        "metric": "lattice_updates_per_s_c4", "value": value, "unit": "GLUPS",
        "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_run_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": describe("c4"), "step": "one run of the whole batch (256 solves)",
                   "tiles": "per member size bucket from the batch autotuner's table "
                            "(psb_batch_autotune; shipped entries in physis_b200/tune_b200.json) "
                            "where it has an entry, else the fewest-tiles rule",
                   "tuned_members": sum(1 for i in range(len(members)) if b.tuned(i)),
                   "members": len(members), "lattice_updates_per_run": lups,
                   "parallelism": "replicas (one batch per GPU)",
                   "inputs_vs_l2": "all members' grids (~18 GB) resident; each run streams "
                                   "%.2f TB, far beyond the 126 MB L2" % (alg_bytes / 1e12)},
        "batch": {
            "solves_per_s": len(members) / per_run_s,
            "graph_mode_glups": lups / (min(res[1]) / 1e3) / 1e9,
            "plain_loop_glups": lups / (loop_plain / 1e3) / 1e9,
            "plain_loop_solves_per_s": len(members) / (loop_plain / 1e3),
            "tuned_loop_glups": lups / (loop_tuned / 1e3) / 1e9,
            "speedup_vs_plain_loop": (loop_plain / 1e3) / per_run_s,
            "speedup_vs_tuned_loop": (loop_tuned / 1e3) / per_run_s,
        },
        "roofline": {"bound": "hbm", "achieved": alg_bytes / per_run_s / 1e9, "peak": peaks()[0],
                     "unit": "GB/s", "frac": alg_bytes / per_run_s / 1e9 / peaks()[0],
                     "traffic": c4_traffic(alg_bytes), "algorithmic_bytes_per_launch": alg_bytes,
                     "avg_launch_us": per_run_s * 1e6,
                     "launch": "one run of the batch: the two kinds' persistent k_batch launches",
                     "traffic_note": "scaled from an ncu capture of the first 32 members "
                                     "(DRAM bytes per algorithmic byte)"},
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "numerics": numerics,
    }
    overrides = {k: v for k, v in (("members", args.members if args.members != 256 else None),
                                   ("kind", args.c4_kind), ("cube", args.c4_cube),
                                   ("steps", args.c4_steps),
                                   ("himeno_two_sweeps", args.him_two_sweeps or None))
                 if v is not None}
    if overrides:
        line["config"]["profiling_overrides"] = overrides
    b.free()
    for g in grids:
        for x in g:
            ps.PSGridFree(x)
    dist.close()
    if dist.rank == 0:
        print(json.dumps(line), flush=True)


C5_RATE = 2000.0
C5_BUDGET = 150 * 10 ** 9
C5_TOL, C5_MAX_STEPS, C5_CHECK = 1e-5, 1000, 10


def c5_trace(seed=5005, count=128):
    """(arrival_s, kind, side, seed) of the served workload, seeded."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for i in range(count):
        t += rng.exponential(1.0 / C5_RATE)
        kind = "diff" if rng.random() < 0.6 else "him"
        side = int(round(32 * 12 ** rng.random()))
        out.append((t, kind, side, 10000 + i))
    return out


def c5_points(kind, side):
    return (side - 2) ** 3 if kind == "him" else side ** 3


def serve_trace(ps, trace, mode, shared_init, out_arena):
    """Replay a trace open-loop against a server: a submitter thread submits
    each request at its arrival time, the caller collects completions.
    Diffusion requests carry their initial field from pinned host memory,
    every request's final field comes back to its own slice of a pinned
    host arena."""
    import threading
    srv = ps.Server(C5_BUDGET, 0, mode)
    index = {}
    h2d = d2h = 0
    t0 = time.monotonic() + 0.02
    errors = []

    offs = np.cumsum([0] + [side ** 3 for _, _, side, _ in trace])
    assert offs[-1] <= out_arena.size

    def submitter():
        for i, (t, kind, side, seed) in enumerate(trace):
            dt = t0 + t - time.monotonic()
            if dt > 0:
                time.sleep(dt)
            n = side ** 3
            out = out_arena[offs[i]:offs[i + 1]]
            try:
                if kind == "diff":
                    rid = srv.submit(ps.DIFFUSION7, (side,) * 3, COEF, C5_MAX_STEPS, C5_TOL, C5_CHECK,
                                     init=shared_init[:n], out=out, seed=seed)
                else:
                    rid = srv.submit(ps.HIMENO19, (side,) * 3, [0.8], C5_MAX_STEPS, C5_TOL, C5_CHECK,
                                     out=out, seed=seed)
            except Exception as e:  # reported after the run
                errors.append(e)
                return
            index[rid] = i

    th = threading.Thread(target=submitter)
    th.start()
    recs = []
    while len(recs) < len(trace) and not errors:
        try:
            recs.append(srv.wait(-1, 5.0))
        except ps.PhysisError as e:
            if e.status not in (ps.PSB_ERR_INVALID, ps.PSB_ERR_TIMEOUT):
                raise
            time.sleep(0.0005)
    th.join()
    stats = srv.stats()
    srv.destroy()
    if errors:
        raise errors[0]
    lups = alg = 0
    lat = []
    for r in recs:
        if r["status"] != ps.PSB_OK:
            raise RuntimeError("request %d failed with status %d" % (r["id"], r["status"]))
        t, kind, side, seed = trace[index[r["id"]]]
        pts = c5_points(kind, side)
        lups += pts * r["steps_done"]
        alg += pts * r["steps_done"] * (56 if kind == "him" else 8)
        lat.append(r["finish_s"] - r["submit_s"])
        d2h += side ** 3 * 4
        h2d += side ** 3 * 4 if kind == "diff" else 0
    makespan = max(r["finish_s"] for r in recs) - t0
    lat = np.array(lat)
    return {"solves_per_s": len(recs) / makespan, "makespan_s": makespan,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_steps": float(np.mean([r["steps_done"] for r in recs])),
            "converged": int(sum(r["steps_done"] < C5_MAX_STEPS for r in recs)),
            "lattice_updates": lups, "alg_bytes": alg, "h2d": h2d, "d2h": d2h,
            "steps_done": {index[r["id"]]: r["steps_done"] for r in recs},
            "wave_rounds": {index[r["id"]]: r["wave_rounds"] for r in recs}, **stats}


def c5_numerics(ps, trace, served, shared, arena, max_work=5e8):
    """Served results against the oracle: the four smallest requests of each
    kind and the cheapest one of each kind that ran on the wavefront path
    (<= max_work updates), each compared after the steps it was served."""
    offs = np.cumsum([0] + [side ** 3 for _, _, side, _ in trace])
    steps = served["steps_done"]
    waves = served["wave_rounds"]
    sample = []
    for kind in ("diff", "him"):
        ids = sorted((i for i, t in enumerate(trace) if t[1] == kind), key=lambda i: trace[i][2])
        sample += ids[:4]
        wave = [i for i in sorted(ids, key=lambda i: trace[i][2] ** 3 * steps[i])
                if waves[i] > 0 and trace[i][2] ** 3 * steps[i] <= max_work]
        if wave:
            sample.append(wave[0])
    recs = []
    for i in sample:
        _, kind, side, seed = trace[i]
        dims = (side, side, side)
        got = np.array(arena[offs[i]:offs[i + 1]]).reshape(side, side, side)
        if kind == "diff":
            data = (np.array(shared[:side ** 3]).reshape(side, side, side), None)
        else:
            p = ps.fill_reference(dims, ps.FILL_ZPROFILE)
            coef = [ps.fill_reference(dims, ps.FILL_UNIFORM, seed * 16 + 1 + k, lo, hi)
                    for k, (lo, hi) in enumerate(C4_HIMENO_RANGES)]
            coef += [ps.fill_reference(dims, ps.FILL_BND), np.zeros((side,) * 3, np.float32)]
            data = (p, coef)
        r = member_numerics(kind, data, steps[i], got)
        r.update({"request": i, "kind": kind, "side": side, "steps": steps[i],
                  "wave_rounds": waves[i]})
        recs.append(r)
    return summarize_numerics(recs, "the four smallest requests of each kind and the cheapest "
                                    "wavefront-path request of each kind (<= %.0e updates), "
                                    "after the steps each was served" % max_work)


def c5_tune(ps, trace):
    """Autotune the batch size buckets the trace's requests fall in: one
    representative member per (kind, bucket), on its own grids, through
    psb_batch_autotune (the entries are cached for the server's rounds)."""
    def bucket(side):
        return 1 << max(3, (side - 1).bit_length())
    seen, members = set(), []
    for _, kind, side, _ in trace:
        key = (kind, bucket(side))
        if key not in seen:
            seen.add(key)
            members.append((kind, side))
    b = ps.Batch()
    grids = []
    try:
        for kind, side in members:
            n = 14 if kind == "him" else 2
            gs = [ps.grid_new(ps.PS_FLOAT, (side,) * 3) for _ in range(n)]
            grids.append(gs)
            if kind == "him":
                b.add(ps.HIMENO19, gs, [0.8], 8)
            else:
                b.add(ps.DIFFUSION7, gs, COEF, 8)
        b.autotune(force=True)
    finally:
        b.free()
        for gs in grids:
            for g in gs:
                ps.PSGridFree(g)
    return len(members)


def run_c5(args, dist):
    os.environ["PHYSIS_B200_DEVICE"] = str(dist.local)
    import ctypes
    import physis_b200 as ps
    ps.PSInit()
    trace = c5_trace(count=args.c5_requests)
    tuned_buckets = c5_tune(ps, trace) if args.tune else None
    if args.him_two_sweeps:
        for side in sorted({side for _, kind, side, _ in trace if kind == "him"} |
                           {32 + 16 * i for i in range(6)}):
            ps.batch_tune_set(ps.HIMENO19, (side,) * 3, impl=ps.IMPL_TMA, tile_x=64, tile_y=8,
                              z_chunk=0, stages=6, t_depth=2)

    def pinned(n):
        hp = ctypes.c_void_p()
        ps.check(ps.lib.psb_host_alloc(n * 4, ctypes.byref(hp)), "psb_host_alloc")
        return hp, np.ctypeslib.as_array((ctypes.c_float * n).from_address(hp.value))

    nmax = 384 ** 3
    hp_in, shared = pinned(nmax)
    shared[:] = np.random.default_rng(7).random(nmax, dtype=np.float32)
    hp_out, arena = pinned(int(sum(side ** 3 for _, _, side, _ in trace)))
    warm = [(0.0005 * i, "diff" if i % 2 else "him", 32 + 16 * i, 50 + i) for i in range(6)]
    for mode in (ps.SERVE_BATCHED, ps.SERVE_FIFO):
        serve_trace(ps, warm, mode, shared, arena)
    sampler = ClockSampler(dist.local)
    dist.barrier()
    sampler.start()
    ours = serve_trace(ps, trace, ps.SERVE_BATCHED, shared, arena)
    clocks = sampler.stop()
    numerics = None
    if dist.rank == 0 and not args.no_numerics:
        numerics = c5_numerics(ps, trace, ours, shared, arena)
    fifo = None if args.c5_skip_fifo else serve_trace(ps, trace, ps.SERVE_FIFO, shared, arena)
    for hp in (hp_in, hp_out):
        ps.check(ps.lib.psb_host_free(hp), "psb_host_free")
    if fifo:
        same = fifo["steps_done"] == ours["steps_done"]
    n = len(trace)
    value = dist.sum(n) / dist.max(ours["makespan_s"])
    dev_s = ours["device_ms"] / 1e3
    achieved = ours["alg_bytes"] / dev_s / 1e9
    hbm, peak_kind = peaks()
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        cpu = c5_cpu_baseline(trace, ours["steps_done"])
    line = {
        "metric": "served_solves_per_s_c5", "value": value, "unit": "solves/s",
        "n_gpus": dist.world, "steps": n, "warmup": len(warm),
        "ms_per_step": ours["makespan_s"] / n * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": describe("c5"), "step": "one served solve (request)",
                   "requests": n, "trace_seed": 5005, "arrival_rate_per_s": C5_RATE,
                   "budget_bytes": C5_BUDGET,
                   "tiles": "per member size bucket from the batch autotuner's table where it "
                            "has an entry (tile shape, z chunk, Himeno sweeps per pass), else "
                            "the fewest-tiles rule",
                   "buckets_tuned_in_run": tuned_buckets,
                   "himeno_two_sweeps_pinned": bool(args.him_two_sweeps),
                   "inputs": "diffusion u0 from pinned host memory (U[0,1)); Himeno p and "
                             "coefficients generated on the device from per-request seeds; "
                             "every final field copied back to pinned host memory",
                   "parallelism": "replicas (one server per GPU)",
                   "inputs_vs_l2": "resident grids of all admitted requests (GBs) far exceed "
                                   "the 126 MB L2"},
        "latency_s": {"p50": ours["p50_s"], "p99": ours["p99_s"]},
        "served": {k: ours[k] for k in ("makespan_s", "mean_steps", "converged", "lattice_updates",
                                        "rounds", "launches", "peak_bytes", "device_ms")},
        "glups_device": ours["lattice_updates"] / dev_s / 1e9,
        "fifo_baseline": None if not fifo else {
            "solves_per_s": fifo["solves_per_s"], "p50_s": fifo["p50_s"], "p99_s": fifo["p99_s"],
            "makespan_s": fifo["makespan_s"], "launches": fifo["launches"],
            "glups_device": fifo["lattice_updates"] / (fifo["device_ms"] / 1e3) / 1e9,
            "same_steps_as_served": same,
            "what": "one request at a time in arrival order, one plain-kernel launch per step, "
                    "separate residual pass per check"},
        "speedup_vs_fifo": None if not fifo else ours["solves_per_s"] / fifo["solves_per_s"],
        "p99_vs_fifo": None if not fifo else fifo["p99_s"] / ours["p99_s"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": None,
                     "kernel": "k_batch, persistent (all rounds)",
                     "algorithmic_bytes": ours["alg_bytes"]},
        "e2e": {"value": value, "unit": "solves/s",
                "h2d_bytes_per_step": ours["h2d"] / n, "d2h_bytes_per_step": ours["d2h"] / n},
        "gpu_launches": ours["launches"],
        "clocks": clocks,
        "cpu_baseline": cpu,
        "numerics": numerics,
    }
    dist.close()
    if dist.rank == 0:
        print(json.dumps(line), flush=True)


def cpu_rates(periodic=False):
    """Rates (updates/s) of the reference CPU target, 1 thread, on bounded
    samples: 7-point diffusion 128^3 x 40 steps and Himeno 129^3 x 16 sweeps
    (about a second each), run loop only."""
    from oracle import oracle
    use_ref = oracle.ref_available()
    f = np.random.default_rng(3).random((128, 128, 128), dtype=np.float32)
    t0 = time.perf_counter()
    if use_ref:
        _, secs_d = oracle.ref_diffusion7(f, 40, np.asarray(COEF, np.float32), periodic=periodic)
    else:
        oracle.diffusion7(f, 40, np.asarray(COEF, np.float32), periodic=periodic)
        secs_d = time.perf_counter() - t0
    rate_d = 128 ** 3 * 40 / secs_d
    p, coef = himeno_fields((129, 129, 129))
    t0 = time.perf_counter()
    if use_ref:
        _, secs_h = oracle.ref_himeno(p, coef, 0.8, 16)
    else:
        oracle.himeno(p, coef, 0.8, 16)
        secs_h = time.perf_counter() - t0
    rate_h = 127 ** 3 * 16 / secs_h
    sample = ("%s 128^3 %s diffusion x 40 steps (%.3f GLUPS) and 129^3 Himeno x 16 sweeps "
              "(%.3f GLUPS), 1 thread, run loop only"
              % ("reference CPU target" if use_ref else "oracle port",
                 "periodic" if periodic else "clamped", rate_d / 1e9, rate_h / 1e9))
    return rate_d, rate_h, "reference" if use_ref else "port", sample


def c5_cpu_baseline(trace, steps_done):
    """Reference CPU target rates applied to the trace's lattice updates (the
    served steps of every request)."""
    rate_d, rate_h, kind, sample = cpu_rates(periodic=False)
    total = 0.0
    for i, (t, k, side, seed) in enumerate(trace):
        total += c5_points(k, side) * steps_done[i] / (rate_h if k == "him" else rate_d)
    return {"value": len(trace) / total, "unit": "solves/s", "cores": 1, "kind": kind,
            "sample": sample + "; solves/s = requests / sum over the trace of served steps x "
                               "points / rate (residual checks not counted)"}


def _ref_rate(pool, procs, kind, dims, dt, count, reps, warm):
    """Aggregate rate of the reference CPU target: `procs` processes, each
    running its own solve of `count` steps; lattice updates / slowest loop."""
    vals = []
    for i in range(warm + reps):
        jobs = [(kind, dims, np.dtype(dt).name, count, 1000 + j) for j in range(procs)]
        res = pool.map(_ref_worker, jobs)
        if i >= warm:
            vals.append((sum(r[0] for r in res), max(r[1] for r in res)))
    pts = sum(v[0] for v in vals)
    loop_s = sum(v[1] for v in vals)
    return pts / loop_s, loop_s / len(vals)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    wl = args.workload
    kname, dt, dims, tsteps, bpl = WORKLOADS[wl]
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU runtime (oracle/_ref) was not built: reference sources "
                          "absent at build time"}), flush=True)
        return
    import multiprocessing as mp
    ncpu = os.cpu_count() or 1
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except Exception:
        avail = 16 << 30
    ctx = mp.get_context("spawn")
    common = {"n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
              "data": "synthetic", "impl": "reference"}
    if kname in ("batch", "serve"):
        # Independent solves: sample each stencil's rate on all host cores and
        # apply it to the workload's lattice updates.
        sd, sh = (128, 128, 128), (129, 129, 129)
        per = 14 * int(np.prod(sh)) * 4
        procs = max(1, min(ncpu, int(avail * 0.6 // per), args.ref_procs))
        dkind = "diffusion7p" if kname == "batch" else "diffusion7"
        with ctx.Pool(procs) as pool:
            rate_d, _ = _ref_rate(pool, procs, dkind, sd, np.float32, 10, max(1, args.steps // 3), 1)
            rate_h, _ = _ref_rate(pool, procs, "himeno", sh, np.float32, 4, max(1, args.steps // 3), 1)
        if kname == "batch":
            members = c4_members(count=args.members)
            lu_d = sum(d[0] * d[1] * d[2] * st for k, d, st in members if k == "diffp")
            lu_h = sum((d[0] - 2) * (d[1] - 2) * (d[2] - 2) * st for k, d, st in members if k == "him")
            secs = lu_d / rate_d + lu_h / rate_h
            value, unit, metric = (lu_d + lu_h) / secs / 1e9, "GLUPS", "lattice_updates_per_s_c4"
            per_step = secs
            what = "the batch's %d members at their step counts" % len(members)
        else:
            trace = c5_trace(count=args.c5_requests)
            secs = sum(c5_points(k, side) * C5_MAX_STEPS / (rate_h if k == "him" else rate_d)
                       for _, k, side, _ in trace)
            value, unit, metric = len(trace) / secs, "solves/s", "served_solves_per_s_c5"
            per_step = secs / len(trace)
            what = ("the trace's %d requests at %d steps each (the reference has no residual "
                    "stop)" % (len(trace), C5_MAX_STEPS))
        sample = ("rates of %s 128^3 x 10 steps (%.2f GLUPS) and Himeno 129^3 x 4 sweeps "
                  "(%.2f GLUPS), each on %d processes at once, applied to %s"
                  % (dkind, rate_d / 1e9, rate_h / 1e9, procs, what))
        line = dict(common, metric=metric, value=value, unit=unit, ms_per_step=per_step * 1e3,
                    dtype="f32", config={"workload": describe(wl),
                                         "parallelism": "%d host processes" % procs},
                    cpu_baseline={"value": value, "unit": unit, "cores": procs,
                                  "kind": "reference", "sample": sample},
                    e2e={"value": value, "unit": unit, "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0})
        print(json.dumps(line), flush=True)
        return
    per = (14 if kname == "himeno" else 3) * int(np.prod(dims)) * np.dtype(dt).itemsize
    procs = max(1, min(ncpu, int(avail * 0.6 // per), args.ref_procs))
    count = 2
    with ctx.Pool(procs) as pool:
        rate, loop_s = _ref_rate(pool, procs, kname, dims, dt, count, args.steps, args.warmup)
    value = rate / 1e9
    sample = ("%d independent %dx%dx%d %s solves of %d %s each per step, one per process, "
              "run loop timed (copies excluded)" % (procs, dims[0], dims[1], dims[2],
                                                     np.dtype(dt).name, count,
                                                     "sweeps" if kname == "himeno" else "time steps"))
    line = dict(common, metric="lattice_updates_per_s_" + wl, value=value, unit="GLUPS",
                ms_per_step=loop_s * 1e3, dtype="f32" if dt == np.float32 else "f64",
                config={"workload": describe(wl), "parallelism": "%d host processes" % procs},
                cpu_baseline={"value": value, "unit": "GLUPS", "cores": procs, "kind": "reference",
                              "sample": sample},
                e2e={"value": value, "unit": "GLUPS", "h2d_bytes_per_step": 0,
                     "d2h_bytes_per_step": 0})
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--tune", action="store_true", help="autotune before timing")
    ap.add_argument("--t-depth", type=int, default=0, choices=[0, 1, 2],
                    help="7-point fp32: pin the time steps per launch (2: temporal blocking; "
                         "profiling)")
    ap.add_argument("--z-chunk", type=int, default=0,
                    help="with --t-depth: pin the z chunk as well (profiling)")
    ap.add_argument("--plain", action="store_true", help="time the plain one-launch kernel")
    ap.add_argument("--fp-mode", default="auto", choices=["auto", "exact", "fma"],
                    help="arithmetic of the 7-point TMA kernel (auto: fma, with the exact "
                         "arithmetic timed beside it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-procs", type=int, default=64)
    ap.add_argument("--dims", default=None, help="override grid extents nx,ny,nz (profiling)")
    ap.add_argument("--time-steps", type=int, default=None,
                    help="override time steps per solve (profiling)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-numerics", action="store_true",
                    help="skip the error report against the oracle (profiling runs)")
    ap.add_argument("--no-residual", action="store_true", help="c3: skip the fused residual")
    ap.add_argument("--members", type=int, default=256, help="c4: batch members (profiling)")
    ap.add_argument("--skip-loops", action="store_true", help="c4: skip the per-grid loops")
    ap.add_argument("--skip-graph", action="store_true", help="c4: skip the per-step graph mode")
    ap.add_argument("--c4-cube", type=int, default=None,
                    help="c4: every member a cube of this side (kinds and steps kept; profiling)")
    ap.add_argument("--c4-steps", type=int, default=None,
                    help="c4: every member this many steps (profiling)")
    ap.add_argument("--him-two-sweeps", action="store_true",
                    help="c4/c5: pin every Himeno bucket to two sweeps per pass (profiling)")
    ap.add_argument("--c4-kind", default=None, choices=["diffp", "him"],
                    help="c4: keep only one kind of member (profiling)")
    ap.add_argument("--c5-requests", type=int, default=128, help="c5: requests in the trace")
    ap.add_argument("--c5-skip-fifo", action="store_true", help="c5: skip the FIFO baseline")
    args = ap.parse_args()
    if args.dims or args.time_steps:
        k, dt, dims, ts, bpl = WORKLOADS[args.workload]
        if args.dims:
            dims = tuple(int(v) for v in args.dims.split(","))
        WORKLOADS[args.workload] = (k, dt, dims, args.time_steps or ts, bpl)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif WORKLOADS[args.workload][0] == "batch":
        run_c4(args, Dist(args.gpus))
    elif WORKLOADS[args.workload][0] == "serve":
        run_c5(args, Dist(args.gpus))
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
