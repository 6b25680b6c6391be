#!/usr/bin/env python
"""Throughput of the periodic-box clustering estimators: mocks/s for P_l (l = 0, 2, 4) plus
bispectrum multipoles B_{l1 l2 L} in {(000), (110), (202), (022)} over all (k1, k2) shell
pairs, on a 512^3 mesh with 10^7 particles (the clustered lognormal catalogue with
Zel'dovich RSD), TSC assignment, 25 k shells 0.01-0.26 h/Mpc.

One step = one mock through the whole pipeline (assignment, FFT, P_l binning, shell
transforms, bispectrum sums and shot noise).  `value` has the catalogue resident in HBM;
`e2e` copies it from host memory every step and reads the results back, through the
library's batch entry point hg_batch_run (the next mock's upload overlapping the current
one's statistics); `e2e.sequential_value` is hg_set_particles + the statistic calls, one
mock after another.  Three forms are measured: the chosen form (the headline: FP32 with the
density and the bispectrum signal in FP64, the fastest setting whose every bin is within
1e-5 of the FP64 form), the plain FP32 form and the plain FP64 form, with the per-bin
relative difference of each against FP64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--small]
  python bench.py --lean --forms fp32 [--n-mesh M --n-particles P]   (profiling runs)
  python bench.py --config {1,2,3,5} [--cpu]   (the other configurations; not the headline)
Under torchrun every rank runs its own mocks (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

CHOSEN = "fp32+density+bk_signal"
METRIC = "mocks/sec P_ℓ+B_ℓ @512³,1e7 pts: batched FP32 vs FP64 GPU, ≤1e-5 rel err"
UNIT = "mocks/s"
PK_ELLS = (0, 2, 4)
MULTIPOLES = ((0, 0, 0), (1, 1, 0), (2, 0, 2), (0, 2, 2))


def workload(small: bool, n_mesh: int = 0, n_part: int = 0):
    from hitomi_b200.api import Binning
    if small:
        return dict(name="box P_l+B_l, 64^3 mesh, 2e5 particles (reduced check size)", n_mesh=64, boxsize=1000.0,
                    n_part=200_000, ngrid=64, binning=Binning(0.015, 0.255, 25))
    if n_mesh or n_part:  # profiling cases: same statistics, other sizes (never the headline)
        nm, npart = n_mesh or 512, n_part or 10_000_000
        return dict(name=f"box P_l+B_l, {nm}^3 mesh, {npart} particles (profiling size)", n_mesh=nm,
                    boxsize=1000.0, n_part=npart, ngrid=min(256, nm), binning=Binning(0.015, 0.255, 25))
    return dict(name="box P_l(l=0,2,4)+B_l(000,110,202,022), all k1,k2; 512^3 mesh, 1e7 particles, TSC", n_mesh=512,
                boxsize=1000.0, n_part=10_000_000, ngrid=256, binning=Binning(0.015, 0.255, 25))


def workload_config(wl, world):
    """The bench line's `config`: the workload alone, identical in both arms (the precision
    form of our arm is reported beside it, in `form`)."""
    b = wl["binning"]
    return {"workload": wl["name"], "n_mesh": wl["n_mesh"], "n_particles": wl["n_part"], "boxsize": wl["boxsize"],
            "assignment": "TSC", "n_kbin": b.n_kbin, "kmin": b.kmin, "kmax": b.kmax, "pk_ells": list(PK_ELLS),
            "bk_multipoles": [list(m) for m in MULTIPOLES],
            "l2": ("inputs larger than L2 (mesh and catalogue > 126 MB)" if wl["n_mesh"] ** 3 * 4 > 126e6
                   else "inputs smaller than L2 (reduced check size)"),
            "parallelism": f"mocks sharded over {world} rank(s), one catalogue each, no collective on the data path"}


def catalogue(wl, seed):
    from hitomi_b200.synthetic import lognormal_box
    return lognormal_box(wl["n_part"], wl["boxsize"], ngrid=wl["ngrid"], seed=seed, exact_n=wl["n_part"])


def run_mock(ctx):
    """One mock: P_l for l in PK_ELLS and all B multipoles; returns results and launch count."""
    out = {}
    launches = 0
    for ell in PK_ELLS:
        pk, _, norm = ctx.pk_box(ell)
        out[("pk", ell)] = norm * pk
        launches += ctx.last_timing()[1]
    bk, sn, norm = ctx.bk_box_multi(MULTIPOLES)
    for q, mp in enumerate(MULTIPOLES):
        out[("bk",) + mp] = norm * (bk[q] - sn[q])
    launches += ctx.last_timing()[1]
    return out, launches


def result_bytes(res) -> int:
    return int(sum(v.size * 16 for v in res.values()))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms.  The sampler starts
    before the warm-up (nvidia-smi takes a few hundred ms to emit its first line) and the
    timed region is marked with host times; only samples stamped inside the timed region
    (widened by one sampling interval on each side) are summarised."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.p = None
        self.t0 = self.t1 = None
        self.path = os.path.join("/tmp", f"hg_clocks_{os.getpid()}_{device_index}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "100", "-i", str(self.dev)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def mark_start(self):
        import datetime
        self.t0 = datetime.datetime.now()

    def mark_stop(self):
        import datetime
        self.t1 = datetime.datetime.now()

    def stop(self):
        import datetime
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 10:
                    continue
                try:
                    ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f")
                    rows.append((ts, float(parts[2]), float(parts[3]), parts[6:10]))
                except ValueError:
                    continue
        os.unlink(self.path)
        if not rows:
            return None
        pad = datetime.timedelta(milliseconds=100)
        inside = [r for r in rows if self.t0 is not None and self.t1 is not None and self.t0 - pad <= r[0] <= self.t1 + pad]
        if not inside:  # the region was shorter than the sampling interval: the nearest sample after its start
            after = [r for r in rows if self.t0 is None or r[0] >= self.t0 - pad]
            inside = after[:1] if after else rows[-1:]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in inside:
            for nm, v in zip(names, r[3]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median([r[1] for r in inside]), "sm_max_mhz": inside[-1][2],
                "reasons": sorted(reasons), "samples": len(inside)}


def measured_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    p = os.path.join(HERE, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def max_rel_err(a, ref):
    floor = 1e-12 * float(np.max(np.abs(ref))) if np.size(ref) else 0.0
    return float(np.max(np.abs(a - ref) / np.maximum(np.abs(ref), floor))) if np.size(ref) else 0.0


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def reduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args, wl, world, rank):
    """Reference arm: the reference's own CPU code (oracle/_ref) on the host cores."""
    if rank != 0:
        return 0
    from oracle import cpu_baseline, ref_runner
    line = {"impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic"}
    if not ref_runner.available():
        line["unavailable"] = "oracle/_ref/ref_harness was not built on this machine"
        print(json.dumps(line), flush=True)
        return 0
    pos = catalogue(wl, 2)
    vals, per = [], []
    for s in range(args.warmup + args.steps):
        r = cpu_baseline.baseline(pos, wl["n_mesh"], wl["boxsize"], wl["binning"], PK_ELLS, MULTIPOLES)
        if s >= args.warmup:
            vals.append(r["mocks_per_s"])
            per.append(r["sample_wall_seconds"])
    v = statistics.median(vals)
    line.update({
        "value": v,
        "ms_per_step": 1000.0 * statistics.median(per),
        "config": workload_config(wl, world),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["cores"], "kind": "reference",
                         "sample": "each step: every building block of the reference's box P/B drivers timed once "
                                   f"at {wl['n_mesh']}^3 / {wl['n_part']} particles (one single-core process per "
                                   "block, concurrently); "
                                   "per-mock time extrapolated by the drivers' call counts; FFT is the project "
                                   "shim, not FFTW"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(line), flush=True)
    return 0


def cufft_reference(n_mesh, timing):
    """cuFFT (through torch.fft.rfftn) on the density transform's shape, timed beside the
    library's own transform as a reference point only: the real n^3 mesh to its
    [n][n][n/2+1] half spectrum, FP32 and FP64, CUDA events over 5 runs after 3 warm-ups.
    `ours_ms` is the library's fft_density (the same transform, its input scaled and
    offset on the fly) from the profiled step of each form."""
    import torch
    out = {"shape": [n_mesh] * 3, "what": "real-to-complex 3-D transform, mean ms per transform"}
    for name, dt in (("fp32", torch.float32), ("fp64", torch.float64)):
        x = torch.randn((n_mesh,) * 3, dtype=dt, device="cuda")
        for _ in range(3):
            y = torch.fft.rfftn(x)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(5):
            y = torch.fft.rfftn(x)
        e1.record()
        torch.cuda.synchronize()
        out[f"cufft_{name}_ms"] = e0.elapsed_time(e1) / 5
        del x, y
    torch.cuda.empty_cache()
    for form, t in timing.items():
        st = t.get("stats") or {}
        for key in ("fft_density", "fp64:fft_density"):
            if key in st and st[key]["launches"]:
                prec = "fp64" if (key.startswith("fp64:") or form == "fp64") else "fp32"
                out[f"ours_{prec}_ms"] = st[key]["ms"]
    return out


def run_config(args) -> int:
    """The other benchmark workloads (1: box P_l at 128^3, 2: box P_l at 512^3, 3: survey P_l,
    5: batched P_l + zeta at 256^3), measured end to end through the public API (the
    catalogue copied from host memory every mock), both forms, FP32-vs-FP64 error per
    statistic; with --cpu also the reference's own code (oracle/_ref) timed on this host:
    directly where a mock takes seconds, else extrapolated from timed parts (stated)."""
    import torch
    from hitomi_b200.api import Binning, Context
    from hitomi_b200.synthetic import lognormal_box, survey_shell, uniform_box
    from hitomi_b200 import survey
    cfg = args.config
    stats = {}
    if cfg == 1:
        name = "box P_l l=0,2,4: 2e5 uniform, 128^3, TSC+interlacing, k 0.005-0.295 (30 bins)"
        mocks = [uniform_box(200_000, 1000.0, seed=1 + i) for i in range(4)]
        setup = dict(n_mesh=128, boxsize=1000.0, b=Binning(0.005, 0.295, 30), assign="TSC", interlace=True)
    elif cfg == 2:
        name = "box P_l l=0,2,4: lognormal 1e7 (RSD f=0.7), 512^3, PCS+interlacing"
        mocks = [catalogue(workload(False), 2 + i) for i in range(2)]
        setup = dict(n_mesh=512, boxsize=1000.0, b=Binning(0.005, 0.295, 30), assign="PCS", interlace=True)
    elif cfg == 3:
        name = "survey P_l l=0,2,4 (local LOS): 1e6 data + 5e7 randoms, shell 1000-1800, 60x60 deg cap, 512^3, box 3500, TSC"
        d, r = survey_shell(1_000_000, 50_000_000, seed=3)
        mocks = [survey.prepare(d, r, 512, 3500.0)]
        setup = dict(n_mesh=512, boxsize=3500.0, b=Binning(0.005, 0.295, 30), assign="TSC", interlace=False)
    elif cfg == 5:
        name = "batched covariance: P_l l=0,2,4 + zeta (000,110,202), 20 r bins 4-156, 256^3, N_p ~ N(2e6, 4e5)"
        rng = np.random.default_rng(1000)
        mocks = [lognormal_box(max(int(rng.normal(2e6, 4e5)), 100_000), 1000.0, ngrid=128, seed=1000 + i)
                 for i in range(args.n_mocks)]
        setup = dict(n_mesh=256, boxsize=1000.0, b=Binning(0.015, 0.255, 25, 4.0, 156.0, 20), assign="TSC",
                     interlace=False)
    else:
        raise SystemExit("--config takes 1, 2, 3 or 5 (4 is the default headline run)")
    zmps = ((0, 0, 0), (1, 1, 0), (2, 0, 2))

    def load(ctx, m, dev):
        """host arrays through hg_set_particles, or device copies through hg_set_particles_device"""
        if cfg == 3:
            if dev is None:
                ctx.set_survey(*m)
            else:
                for slot, t in ((0, dev[0]), (1, dev[1])):
                    ctx.set_particles_device(slot, t.data_ptr(), t.shape[0], 56, 0, 3, 6, keep=t)
        elif dev is None:
            ctx.set_particles(0, m)
        else:
            ctx.set_particles_device(0, dev.data_ptr(), dev.shape[0], 24, keep=dev)

    def one(ctx, m, dev=None):
        out = {}
        load(ctx, m, dev)
        if cfg == 3:
            a, vs, *_ = ctx.survey_scalars()
            for ell in PK_ELLS:
                pk, _, norm = ctx.pk_survey(ell, a, vs)
                out[f"pk{ell}"] = norm * pk
            return out
        for ell in PK_ELLS:
            pk, _, norm = ctx.pk_box(ell)
            out[f"pk{ell}"] = norm * pk
        if cfg == 5:
            z, sn, norm = ctx.zeta_box_multi(zmps)
            for q, mp in enumerate(zmps):
                out["zeta" + "".join(map(str, mp))] = norm * (z[q] - sn[q]).real
        return out

    line = {"config": cfg, "workload": name, "unit": UNIT,
            "timing": "per mock; *_mocks_per_s with the catalogue resident on the device, *_e2e_mocks_per_s "
                      "copying it from (pageable) host arrays through hg_set_particles every mock",
            "n_mocks": len(mocks), "data": "synthetic"}
    devs = []
    for m in mocks:
        if cfg == 3:
            devs.append(tuple(torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in m))
        else:
            devs.append(torch.from_numpy(np.ascontiguousarray(m)).cuda())
    res = {}
    for form in ("fp64", "fp32"):
        with Context(setup["n_mesh"], setup["boxsize"], setup["b"], setup["assign"], form,
                     interlace=setup["interlace"]) as ctx:
            for m in mocks:  # warm-up over every mock: tables, splines, buffers sized for the largest
                one(ctx, m)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            outs = [one(ctx, m, d) for m, d in zip(mocks, devs)]
            torch.cuda.synchronize()
            dt = (time.perf_counter() - t0) / len(mocks)
            t0 = time.perf_counter()
            for m in mocks:
                one(ctx, m)
            torch.cuda.synchronize()
            de = (time.perf_counter() - t0) / len(mocks)
        res[form] = outs
        line[f"{form}_mocks_per_s"] = 1.0 / dt
        line[f"{form}_ms_per_mock"] = 1000.0 * dt
        line[f"{form}_e2e_mocks_per_s"] = 1.0 / de
    line["fp32_over_fp64"] = line["fp32_mocks_per_s"] / line["fp64_mocks_per_s"]
    errs = {}
    for k in res["fp64"][0]:
        errs[k] = max(max_rel_err(a[k], b[k]) for a, b in zip(res["fp32"], res["fp64"]))
        scale = max(float(np.max(np.abs(b[k]))) for b in res["fp64"])
        errs[k + "_rel_to_max"] = max(float(np.max(np.abs(a[k] - b[k]))) for a, b in zip(res["fp32"], res["fp64"])) / scale
    line["rel_err_fp32_vs_fp64"] = errs
    if args.cpu:
        line["cpu_reference"] = cpu_config(cfg, mocks, setup, zmps)
    print(json.dumps(line), flush=True)
    return 0


def cpu_config(cfg, mocks, setup, zmps):
    """The reference's own code (oracle/_ref/ref_harness) on this host's cores."""
    from oracle import cpu_baseline, ref_runner
    if not ref_runner.available():
        return {"unavailable": "oracle/_ref/ref_harness was not built on this machine"}
    cores = cpu_baseline.host_cores()
    b = setup["b"]
    if cfg in (1, 2):
        # the reference has neither PCS nor interlacing: its TSC path, one process per l
        t = 0.0
        for ell in PK_ELLS:
            with ref_runner.RefRun() as r:
                r.run("pk", mocks[0], ell, 0, ell, setup["n_mesh"], setup["boxsize"], b, assign="TSC")
                t += r.wall
        return {"mocks_per_s": cores / t, "per_mock_seconds": t, "cores": cores, "kind": "reference",
                "sample": "direct: P_0, P_2, P_4 of one mock, TSC without interlacing (the reference has neither PCS "
                          "nor interlacing), one single-core process per mock as in main.cpp:64-76"}
    if cfg == 5:
        # P_l directly; zeta from one timed row of (000) scaled by rows and (m1, m2) terms
        m = mocks[0]
        t = 0.0
        for ell in PK_ELLS:
            with ref_runner.RefRun() as r:
                r.run("pk", m, ell, 0, ell, setup["n_mesh"], setup["boxsize"], b, assign="TSC")
                t += r.wall
        with ref_runner.RefRun() as r:
            r.run("3PCF", m, 0, 0, 0, setup["n_mesh"], setup["boxsize"], b, assign="TSC", all_rows=False, ith=0)
            trow = r.wall
        terms = 1 + 3 + 1  # (m1, m2) terms of (000), (110), (202)
        tz = trow * b.n_rbin * terms
        return {"mocks_per_s": cores / (t + tz), "per_mock_seconds": t + tz, "cores": cores, "kind": "reference",
                "sample": f"P_0,2,4 direct ({t:.1f} s); zeta extrapolated from one ith_rbin row of (000) "
                          f"({trow:.1f} s) x {b.n_rbin} rows x {terms} (m1, m2) terms"}
    return {"unavailable": "survey P at 512^3 with 5e7 randoms takes many minutes per l in the reference; "
                           "not timed in the bench"}


def dtype_of(form: str) -> str:
    """The arithmetic a form computes in: FP64 stages named after the '+'."""
    parts = form.split("+")
    if parts[0] == "fp64":
        return "f64"
    if len(parts) == 1:
        return "f32"
    return "f64 (" + ", ".join(parts[1:]) + ") + f32 (the rest)"


def make_context(form: str, wl, device: int):
    """form: "fp64", "fp32", or "fp32+<stage>+..." with stages run in FP64 (density, bk_signal,
    bk_shot: hg_config.fp64_stages)."""
    from hitomi_b200.api import Context
    parts = form.split("+")
    return Context(wl["n_mesh"], wl["boxsize"], wl["binning"], "TSC", parts[0], device=device,
                   fp64_stages=parts[1:])


STAGE_VARIANTS = ("fp32", "fp32+density", "fp32+bk_signal", "fp32+bk_shot", "fp32+density+bk_shot",
                  "fp32+density+bk_signal", "fp32+bk_signal+bk_shot", "fp32+density+bk_signal+bk_shot")


def run_stage_table(args) -> int:
    """Per-stage error attribution of the FP32 form on the headline workload: each variant
    runs the named stages in FP64 (hg_config.fp64_stages); per statistic, the maximum over
    bins of |x - x_fp64| / max(|x_fp64|, 1e-12 max|x_fp64|), for the printed B (bk - sn) and
    for its signal (bk) and shot-noise (sn) parts separately; device time per mock."""
    import torch
    wl = workload(args.small, args.n_mesh, int(args.n_particles))
    pos = catalogue(wl, 2)
    n = pos.shape[0]
    d_pos = torch.from_numpy(pos).cuda()

    def mock(ctx):
        out = {}
        for ell in PK_ELLS:
            pk, _, norm = ctx.pk_box(ell)
            out[f"pk{ell}"] = norm * pk
        bk, sn, norm = ctx.bk_box_multi(MULTIPOLES)
        for q, mp in enumerate(MULTIPOLES):
            t = "".join(map(str, mp))
            out["bk" + t] = norm * (bk[q] - sn[q])
            out["signal" + t] = norm * bk[q]
            out["shot" + t] = norm * sn[q]
        return out

    res, ms = {}, {}
    for form in ("fp64",) + STAGE_VARIANTS:
        ctx = make_context(form, wl, 0)
        for _ in range(2):
            ctx.set_particles_device(0, d_pos.data_ptr(), n, 24, keep=d_pos)
            mock(ctx)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            ctx.set_particles_device(0, d_pos.data_ptr(), n, 24, keep=d_pos)
            res[form] = mock(ctx)
        e1.record()
        torch.cuda.synchronize()
        ms[form] = e0.elapsed_time(e1) / args.steps
        ctx.close()
    table = {}
    for form in STAGE_VARIANTS:
        table[form] = {"ms_per_mock": ms[form], "fp64_over_this": ms["fp64"] / ms[form],
                       "rel_err": {k: max_rel_err(res[form][k], res["fp64"][k]) for k in res["fp64"]}}
    line = {"stage_table": table, "fp64_ms_per_mock": ms["fp64"], "workload": wl["name"], "steps": args.steps,
            "metric": "max over bins of |x - x_fp64| / max(|x_fp64|, 1e-12 max |x_fp64|)"}
    if os.environ.get("HG_BENCH_DUMP"):
        np.savez_compressed(os.environ["HG_BENCH_DUMP"], **{f"{form}:{k}": v for form in res
                                                            for k, v in res[form].items()})
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="64^3 / 2e5-particle case for quick checks")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # the first form is the headline: the FP32 form with the stages that set its error floor
    # (density, bispectrum signal) in FP64 -- the fastest setting that meets 1e-5 per bin
    ap.add_argument("--forms", default=f"{CHOSEN},fp32,fp64")
    ap.add_argument("--lean", action="store_true",
                    help="profiling runs: device-resident steps only (no e2e, per-kernel or CPU legs)")
    ap.add_argument("--n-mesh", type=int, default=0, help="profiling size (not the headline workload)")
    ap.add_argument("--n-particles", type=float, default=0, help="profiling size (not the headline workload)")
    ap.add_argument("--config", type=int, default=0, help="measure another workload: 1 box P_l 128^3, 2 box P_l 512^3, 3 survey P_l, 5 P_l + zeta batch")
    ap.add_argument("--n-mocks", type=int, default=8, help="mocks timed for --config 5")
    ap.add_argument("--cpu", action="store_true", help="with --config: also time the reference's CPU code")
    ap.add_argument("--stage-table", action="store_true",
                    help="FP32-form error and time with each set of stages run in FP64 (not a bench line)")
    args = ap.parse_args()
    if args.config:
        return run_config(args)
    if args.stage_table:
        return run_stage_table(args)
    if not args.lean:
        args.warmup = max(args.warmup, 3)
    wl = workload(args.small, args.n_mesh, int(args.n_particles))
    world, rank, local = dist_setup()
    if args.impl == "reference":
        rc = run_reference(args, wl, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rc

    import torch
    from hitomi_b200.api import Context
    torch.cuda.set_device(local)
    pos = catalogue(wl, 2 + rank)
    n = pos.shape[0]
    d_pos = torch.from_numpy(pos).to(f"cuda:{local}")
    h_pos = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
    h_pos.copy_(torch.from_numpy(pos))
    h_np = h_pos.numpy()
    forms = [f.strip() for f in args.forms.split(",") if f.strip()]
    results = {}
    timing = {}
    for form in forms:
        ctx = make_context(form, wl, local)
        clk = ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[0])
                           if os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0].isdigit() else local)
        clk.start()
        for _ in range(args.warmup):
            ctx.set_particles_device(0, d_pos.data_ptr(), n, 24, keep=d_pos)
            run_mock(ctx)
        # ---- device-resident value
        barrier(world)
        torch.cuda.synchronize()
        clk.mark_start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        launches = 0
        for _ in range(args.steps):
            ctx.set_particles_device(0, d_pos.data_ptr(), n, 24, keep=d_pos)
            res, nl = run_mock(ctx)
            launches += nl
        ev1.record()
        torch.cuda.synchronize()
        clk.mark_stop()
        clocks = clk.stop()
        barrier(world)
        ms = reduce_max(ev0.elapsed_time(ev1) / args.steps, world)
        results[form] = res
        if args.lean or form != forms[0]:  # the other forms: device-resident rate and results only
            timing[form] = dict(ms=ms, e2e_ms=ms, launches=launches // args.steps, clocks=clocks, stats={}, d2h=0)
            ctx.close()
            continue
        # ---- end to end through the public API with host buffers, one mock after another
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        d2h = 0
        for _ in range(args.steps):
            ctx.set_particles(0, h_np)
            r2, _ = run_mock(ctx)
            d2h = result_bytes(r2)
        e1.record()
        torch.cuda.synchronize()
        sms = reduce_max(e0.elapsed_time(e1) / args.steps, world)
        # ---- the same through the library's batch entry point (hg_batch_run): every step's
        # catalogue is copied from host memory, the next one's upload overlapping the current
        # one's statistics (a host thread stages it through pinned memory, a second stream
        # copies it), and every result comes back to host memory.  Wall clock around the whole
        # call, the device drained on both sides.
        ctx.batch_run([h_np], pk_ells=PK_ELLS, bk_multipoles=MULTIPOLES)  # buffers sized
        barrier(world)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        ctx.batch_run([h_np] * args.steps, pk_ells=PK_ELLS, bk_multipoles=MULTIPOLES)
        torch.cuda.synchronize()
        ems = reduce_max((time.perf_counter() - w0) * 1000.0 / args.steps, world)
        # ---- one profiled step: per-kernel CUDA-event timing
        ctx.set_profiling(True)
        ctx.set_particles_device(0, d_pos.data_ptr(), n, 24, keep=d_pos)
        run_mock(ctx)
        stats = ctx.kernel_stats()
        ctx.set_profiling(False)
        tuned = ctx.tuning()
        timing[form] = dict(ms=ms, e2e_ms=ems, e2e_seq_ms=sms, launches=launches // args.steps, clocks=clocks, tuned=tuned,
                            stats=stats, d2h=d2h)
        ctx.close()

    head = forms[0]
    t = timing[head]
    value = world * 1000.0 / t["ms"]
    evalue = world * 1000.0 / t["e2e_ms"]
    peak, peak_kind = measured_peaks()
    top = max(t["stats"].items(), key=lambda kv: kv[1]["ms"]) if t["stats"] else None
    roof = None
    if top:
        name, st = top
        per_launch_ms = st["ms"] / st["launches"]
        per_launch_bytes = st["bytes"] / st["launches"]
        achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9
        trf = ncu_traffic().get(f"{head}:{name}")
        roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": trf,
                "share_of_step": st["ms"] / sum(v["ms"] for v in t["stats"].values())}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": dtype_of(head), "data": "synthetic",
        "config": workload_config(wl, world), "form": head,
        "clocks": t["clocks"],
        "e2e": {"value": evalue, "unit": UNIT, "h2d_bytes_per_step": int(n * 24), "d2h_bytes_per_step": int(t["d2h"]),
                "how": "hg_batch_run through the C ABI with host buffers (the next mock's upload overlaps the "
                       "current one's statistics), wall clock around the call",
                "sequential_value": (world * 1000.0 / t["e2e_seq_ms"]) if t.get("e2e_seq_ms") else None},
        "gpu_launches": int(t["launches"] * args.steps),
        "roofline": roof,
        "autotuned": t.get("tuned", "").strip().splitlines(),
    }
    if "fp64" in timing and head != "fp64":
        def errs_of(form):
            return {f"{k[0]}{''.join(map(str, k[1:]))}": max_rel_err(results[form][k], results["fp64"][k])
                    for k in results[form]}
        errs = errs_of(head)
        line["fp64_form"] = {"value": world * 1000.0 / timing["fp64"]["ms"], "ms_per_step": timing["fp64"]["ms"]}
        line["fp32_over_fp64"] = timing["fp64"]["ms"] / t["ms"]
        line["max_rel_err_fp32_vs_fp64"] = max(errs.values())
        line["rel_err_by_statistic"] = errs
        line["rel_err_metric"] = "max over bins of |x - x_fp64| / max(|x_fp64|, 1e-12 max|x_fp64|)"
        for other in forms[1:]:
            if other in ("fp64", head):
                continue
            e = errs_of(other)
            line.setdefault("other_forms", {})[other] = {
                "value": world * 1000.0 / timing[other]["ms"], "ms_per_step": timing[other]["ms"],
                "max_rel_err_vs_fp64": max(e.values()), "rel_err_by_statistic": e}
    for form in (f for f in timing if timing[f]["stats"]):
        line.setdefault("kernel_ms", {})[form] = {k: round(v["ms"], 4) for k, v in
                                                  sorted(timing[form]["stats"].items(), key=lambda kv: -kv[1]["ms"])}
        # algorithmic bytes (the library's per-launch model) over the measured time
        line.setdefault("kernel_gbs", {})[form] = {k: round(v["bytes"] / v["ms"] / 1e6, 1) for k, v in
                                                   sorted(timing[form]["stats"].items(), key=lambda kv: -kv[1]["ms"])
                                                   if v["ms"] > 0 and v["bytes"] > 0}
    if rank == 0 and not args.lean:
        line["cufft_reference"] = cufft_reference(wl["n_mesh"], timing)
    if os.environ.get("HG_BENCH_DUMP"):
        np.savez_compressed(os.environ["HG_BENCH_DUMP"], **{f"{form}:{'_'.join(map(str, k))}": v
                                                            for form in results for k, v in results[form].items()})
    if args.lean:
        line["lean"] = "profiling run: e2e, per-kernel and CPU legs skipped"
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.lean:
        try:
            from oracle import cpu_baseline
            cb = cpu_baseline.baseline(pos, wl["n_mesh"], wl["boxsize"], wl["binning"], PK_ELLS, MULTIPOLES)
            line["cpu_baseline"] = {
                "value": cb["mocks_per_s"], "unit": UNIT, "cores": cb["cores"], "kind": "reference",
                "sample": f"reference box P/B building blocks timed once each at {wl['n_mesh']}^3 / {n} particles "
                          f"(single-core processes, concurrently, {cb['sample_wall_seconds']:.1f} s wall); "
                          f"per-mock {cb['per_mock_seconds']:.0f} s extrapolated by the drivers' call counts; "
                          f"FFT is the project shim, not FFTW",
                "unit_seconds": cb["unit_seconds"]}
        except Exception as e:  # reported, not fatal
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                    "sample": f"failed: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
