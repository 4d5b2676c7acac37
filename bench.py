#!/usr/bin/env python
"""Benchmark of the time step on the single large case (4096x2048 lattice,
NACA 0012 of chord 512 lu with 1024 markers, heave 0.5c + pitch 30 deg at
St 0.3, Re 1000, FP32 population storage).

One step = one pass of the hot path: the immersed-boundary kernels and the
fused stream/collide/boundary lattice kernel over the whole lattice. The
lattice (2 x 302 MB of FP32 populations) is larger than the 126 MB L2, so no
flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun as N independent replicas (the step does not shard:
every GPU owns whole cases); `value` is the lattice updates of all ranks over
the slowest rank's device time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS & %HBM roofline; batched cases/hr + p99 vs plain FP32 at 1% C_L/C_D"
UNIT = "MLUPS"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--nx", type=int, default=4096)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched and served measurements")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def replica_value(local_ms, nodes, steps, world, device="cuda"):
    """Whole-job MLUPS of `world` independent replicas: every rank updated
    nodes*steps lattice nodes; the job time is the slowest rank's device time
    (max over ranks). Returns (value, max_ms). The max is the only collective."""
    import torch
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    tmax = float(t.item())
    return nodes * steps * world / (tmax / 1e3) / 1e6, tmax


def large_case(args, n_steps, precision=None):
    from fortran_loadfile_mitiwing_b200 import cases
    if (args.nx, args.ny) == (4096, 2048):
        return cases.heave_pitch_case(n_steps=n_steps, precision=precision or args.precision)
    chord = args.ny // 4
    return cases.heave_pitch_case(nx=args.nx, ny=args.ny, chord=chord, pivot=(2 * chord + 1, args.ny // 2 + 1),
                                  markers=2 * chord, n_steps=n_steps, precision=precision or args.precision)


def workload(args):
    return {
        "workload": f"heave+pitch NACA 0012, {args.nx}x{args.ny} D2Q9 MRT lattice, chord {args.ny // 4} lu, "
                    f"{args.ny // 2} markers in the reference's boundary.dat layout (x uniform; cosine spacing "
                    f"makes the marker system singular), live boundary_condition1 outer boundary, Re 1000, "
                    f"St 0.3, U0 0.05, 4-point delta",
        "nx": args.nx, "ny": args.ny, "markers": args.ny // 2, "storage": args.precision,
        "l2": "inputs larger than L2 (two population buffers of 9*nx*ny elements)",
        "parallelism": "replicas",
    }


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.skip = 0

    def _lines(self):
        try:
            return [ln for ln in open(self.path) if ln.strip()]
        except OSError:
            return []

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # wait for the sampler's first line, then keep only later samples
        t0 = time.perf_counter()
        while not self._lines() and time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.02)
        self.skip = len(self._lines())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self._lines()
        lines = lines[self.skip:] or lines
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def kf_traffic():
    """DRAM bytes per lattice-kernel launch from the committed ncu summary
    (the `key: value` lines of profiles/kf_tma_traffic.txt), or None."""
    try:
        d = {}
        for line in open(os.path.join(ROOT, "profiles", "kf_tma_traffic.txt")):
            k, sep, v = line.partition(":")
            if sep and k.strip() in ("nx", "ny", "bytes_per_launch"):
                d[k.strip()] = float(v.split()[0])
        return d or None
    except Exception:
        return None


def cpu_oracle_rate(case, max_seconds=20.0, threads=None):
    """Oracle (the CPU restatement, FP64) on the same case: MLUPS over a bounded
    number of steps; returns (mlups, steps, cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    cores = threads or os.cpu_count()
    pyoracle.set_threads(cores)
    o = pyoracle.Oracle.from_case(case)
    o.evolution()                       # first step outside the sample (impulsive start)
    steps, t0 = 0, time.perf_counter()
    while True:
        o.evolution()
        steps += 1
        el = time.perf_counter() - t0
        if el > max_seconds or steps >= 1000:
            break
    o.close()
    nn = case.params.nx * case.params.ny
    return nn * steps / el / 1e6, steps, cores, el


def run_reference(args, world, rank):
    if rank != 0:
        return
    case = large_case(args, n_steps=args.steps + args.warmup + 10)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    cores = os.cpu_count()
    pyoracle.set_threads(cores)
    o = pyoracle.Oracle.from_case(case)
    warm = max(1, args.warmup)   # untimed; each is one full time step of the case
    t_first = time.perf_counter()
    for _ in range(warm):
        o.evolution()
    per = (time.perf_counter() - t_first) / warm
    k = max(1, min(args.steps, int(150.0 / max(per, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(k):
        o.evolution()
    el = time.perf_counter() - t0
    nn = args.nx * args.ny
    v = nn * k / el / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": k,
        "warmup": warm, "ms_per_step": el / k * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload(args),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{k} full time steps of the {args.nx}x{args.ny} case (reference Fortran "
                                   f"has no compiler here; CPU FP64 restatement, OpenMP on {cores} threads)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import ctypes as C
    import numpy as np
    import torch
    from fortran_loadfile_mitiwing_b200 import Lbm, build, cases
    from fortran_loadfile_mitiwing_b200 import _abi
    build.build()
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    lib = _abi.load_library()
    k, w = args.steps, args.warmup
    kk = min(k, 2000)   # steps of the second pass, which times each kernel
    case = large_case(args, n_steps=k + w + kk + 8)
    s = Lbm.from_case(case, lib)
    s.run(w, keep_rows=False)
    # the timed steps: device events at the start and the end of each chunk of
    # steps only, so that no per-step event sits in the streams
    lib.lbm_set_timing(s.h, _abi.LBM_TIMING_SPAN)
    n0 = C.c_longlong()
    lib.lbm_get_launch_count(s.h, C.byref(n0))
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    rows = s.run(k)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    n1 = C.c_longlong()
    lib.lbm_get_launch_count(s.h, C.byref(n1))
    step_ms, ib_ms, kf_ms, nt = C.c_double(), C.c_double(), C.c_double(), C.c_int()
    lib.lbm_get_timing(s.h, C.byref(step_ms), None, None, C.byref(nt))
    assert nt.value == k and rows.shape[0] == k, (nt.value, rows.shape)
    assert np.all(np.isfinite(rows))
    # second pass: events around the lattice kernel and the IB chain of every
    # step, for the roofline (the per-step events cost the step itself a
    # little, so the step time above is taken without them)
    lib.lbm_set_timing(s.h, _abi.LBM_TIMING_KERNELS)
    rows2 = s.run(kk)
    torch.cuda.synchronize()
    k2_ms, nt2 = C.c_double(), C.c_int()
    lib.lbm_get_timing(s.h, C.byref(k2_ms), C.byref(ib_ms), C.byref(kf_ms), C.byref(nt2))
    assert nt2.value == kk and np.all(np.isfinite(rows2)), nt2.value
    nn = args.nx * args.ny
    value, tmax_ms = replica_value(step_ms.value, nn, k, world)
    elem = {"fp32": 4, "fp64": 8, "fp16": 2, "bf16": 2}[args.precision]
    bpl = 18 * elem
    kf_avg_s = kf_ms.value / kk / 1e3
    achieved = bpl * nn / kf_avg_s / 1e9
    peak, peak_kind = measured_peak()
    tr = kf_traffic()
    traffic = None
    if tr and tr.get("nx") and tr.get("bytes_per_launch"):
        traffic = tr["bytes_per_launch"] * nn / (tr["nx"] * tr["ny"])
    s.close()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": k, "warmup": w,
        "ms_per_step": tmax_ms / k, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp32": "f32", "fp64": "f64", "fp16": "f16-storage/f32", "bf16": "bf16-storage/f32"}[args.precision],
        "data": "synthetic (generated NACA 0012 contour and motion table, seeded 1e-4 initial perturbation)",
        "config": workload(args),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind, "bytes_per_update": bpl,
                     "kernel": "kf_tma (fused stream/collide/boundary; every node but the IB correction tiles)",
                     "kernel_ms": kf_ms.value / kk, "ib_ms": ib_ms.value / kk,
                     "kernel_timing": f"CUDA events around every step's kernels over {kk} further steps "
                                      f"(step time with those events: {k2_ms.value / kk:.4f} ms)"},
        "gpu_launches": int(n1.value - n0.value),
        "clocks": clocks,
    }
    if world > 1:
        torch.distributed.barrier()
    if rank == 0 and world == 1 and not args.no_e2e:
        line["e2e"] = run_e2e(args, lib)
    if rank == 0 and world == 1 and not args.no_batch:
        line["storage_variants"] = run_storage_variants(args, lib, exclude=args.precision)
        line["batched"] = run_batched(lib)
        line["served"] = run_served(lib)
    if rank == 0 and world == 1 and not args.no_cpu:
        mlups, steps, cores, el = cpu_oracle_rate(large_case(args, n_steps=200, precision="fp64"))
        line["cpu_baseline"] = {"value": mlups, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"{steps} time steps of the same {args.nx}x{args.ny} case "
                                          f"({el:.1f} s, CPU FP64 restatement, OpenMP)"}
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_e2e(args, lib):
    """The same metric through the public API with host buffers: set-up from
    host arrays (boundary, motion table, initial perturbation), one lbm_run
    call for the K steps that returns every step's force row into a host
    array, and the final fields."""
    import numpy as np
    from fortran_loadfile_mitiwing_b200 import Lbm
    k = args.steps
    case = large_case(args, n_steps=k + 8)
    nn = args.nx * args.ny
    marks = []
    t0 = time.perf_counter()
    s = Lbm(case.params, lib)
    marks.append(("create", time.perf_counter()))
    for wi, (x, y) in enumerate(case.contours, start=1):
        s.set_boundary(wi, x, y)
    s.set_motion_table(case.table)
    marks.append(("boundary_motion", time.perf_counter()))
    s.init(case.du, case.dv)
    marks.append(("init", time.perf_counter()))
    rows = s.run(k)
    marks.append(("run", time.perf_counter()))
    rho, u, v = s.fields()
    marks.append(("fields", time.perf_counter()))
    el = time.perf_counter() - t0
    assert rows.shape[0] == k and np.all(np.isfinite(rows))
    s.close()
    stages, prev = {}, t0
    for name, t in marks:
        stages[name] = (t - prev) * 1e3
        prev = t
    # host -> device: motion table, contours and the perturbation du, dv (the
    # initial populations and fields are built on the device from them)
    h2d = (case.table.nbytes + 2 * nn * 8 + sum(x.nbytes + y.nbytes for x, y in case.contours)) / k
    d2h = s.row_len * 8 + 3 * nn * 8 / k
    return {"value": nn * k / el / 1e6, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "stages_ms": stages,
            "note": "wall clock around the C-ABI calls (create, boundary, motion table, init, run, fields); "
                    "set-up upload and final fields amortised over the steps; device memory from the library's "
                    "stream-ordered pool, which the bench's earlier handles in this process have filled"}


def run_storage_variants(args, lib, exclude, steps=1000, kernel_steps=300):
    """The same case in the other storage precisions: step time over `steps`
    steps (events at the ends of the call only) and the lattice kernel's time
    with per-step events over `kernel_steps` more, each after 5 warm-up
    steps; bytes per update 18 x the storage size."""
    import ctypes as C
    from fortran_loadfile_mitiwing_b200 import Lbm
    from fortran_loadfile_mitiwing_b200 import _abi
    out = {}
    nn = args.nx * args.ny
    peak, peak_kind = measured_peak()
    for prec, elem in (("fp32", 4), ("fp16", 2), ("bf16", 2), ("fp64", 8)):
        if prec == exclude:
            continue
        s = Lbm.from_case(large_case(args, n_steps=steps + kernel_steps + 16, precision=prec), lib)
        s.run(5, keep_rows=False)
        lib.lbm_set_timing(s.h, _abi.LBM_TIMING_SPAN)
        s.run(steps, keep_rows=False)
        step_ms, n = C.c_double(), C.c_int()
        lib.lbm_get_timing(s.h, C.byref(step_ms), None, None, C.byref(n))
        lib.lbm_set_timing(s.h, _abi.LBM_TIMING_KERNELS)
        s.run(kernel_steps, keep_rows=False)
        kf_ms, n2 = C.c_double(), C.c_int()
        lib.lbm_get_timing(s.h, None, None, C.byref(kf_ms), C.byref(n2))
        s.close()
        ms = step_ms.value / n.value
        kms = kf_ms.value / n2.value
        achieved = 18 * elem * nn / (kms / 1e3) / 1e9
        out[prec] = {"ms_per_step": ms, "mlups": nn / (ms / 1e3) / 1e6, "kernel_ms": kms,
                     "kernel_gbs": achieved, "kernel_frac": achieved / peak, "peak_source": peak_kind,
                     "steps": n.value}
    return out


def run_batched(lib, n_cases=64, steps=100, warmup=12):
    """The metric's batched form: a seeded sweep of cases of different grids
    and kinematics (Nx in [512, 2048], Ny = Nx/2, chord = Ny/4; Re, heave,
    pitch, phase, St drawn per case), stepped one at a time in FP32
    (lbm_run per case) and together as one batch in FP16 storage
    (lbm_batch_run). Cases per hour extrapolate each form's measured lattice
    update rate to 5 flapping periods of every case."""
    from fortran_loadfile_mitiwing_b200 import sweep
    specs = sweep.sweep_specs(n_cases, 2026)
    t0 = time.perf_counter()
    r_alone, _ = sweep.run_alone(specs, steps, warmup, "fp32", lib)
    r16, _, _, choice = sweep.run_batch(specs, steps, warmup, "fp16", lib)
    base, b16 = sweep.cases_per_hour(specs, r_alone), sweep.cases_per_hour(specs, r16)
    return {"cases": n_cases, "steps_per_case": steps, "alone_fp32_mlups": r_alone / 1e6,
            "batch_fp16_mlups": r16 / 1e6, "alone_fp32_cases_per_hour": base, "batch_fp16_cases_per_hour": b16,
            "batch_fp16_vs_alone_fp32": b16 / base, "autotuned": choice,
            "floor_us_per_step": sweep.launch_floor(lib=lib),
            "wall_s": time.perf_counter() - t0}


def run_served(lib, n_req=64, rate=32.0, periods=3.0, check=8):
    """The metric's served form: the same case distribution arriving as a
    Poisson stream at `rate` requests/s in real time, each solved for
    `periods` flapping periods with continuous batching in FP16 storage under
    a 150 GB budget; p50/p99 time from arrival to result and cases per hour,
    against FP32 one-at-a-time service of the same arrivals (first come, first
    served, each case's service time measured alone), and the first `check`
    results' per-period mean C_D and C_L against the same cases in FP64."""
    from fortran_loadfile_mitiwing_b200 import serve, sweep
    specs = sweep.sweep_specs(n_req, 2026)
    t0 = time.perf_counter()
    service = serve.alone_service_times(specs, periods, lib=lib)
    res, summ = serve.serve_stream(specs, rate, periods, 150e9, "fp16", 100, seed=2026, lib=lib,
                                   keep_rows=set(range(check)))
    ref = serve.fp64_reference_rows(specs[:check], periods, lib)
    errs = [serve.period_errors(res[i].rows, ref[i], specs[i]["period_steps"], periods) for i in range(check)]
    arr = serve.poisson_arrivals(rate, n_req, 2026)
    fin = serve.fifo_one_at_a_time(arr, service)
    lat = [f - a for f, a in zip(fin, arr)]
    alone_cph = n_req * 3600.0 / float(max(fin))
    return {"requests": n_req, "rate_per_s": rate, "periods": periods, "storage": "fp16",
            "p50_s": summ["p50_s"], "p99_s": summ["p99_s"], "cases_per_hour": summ["cases_per_hour"],
            "fp32_one_at_a_time_p50_s": serve.percentile(lat, 50), "fp32_one_at_a_time_p99_s": serve.percentile(lat, 99),
            "fp32_one_at_a_time_cases_per_hour": alone_cph, "vs_fp32_one_at_a_time": summ["cases_per_hour"] / alone_cph,
            "max_period_mean_err_cd_vs_fp64": max(e["cd"] for e in errs),
            "max_period_mean_err_cl_vs_fp64": max(e["cl"] for e in errs),
            "peak_cases": summ["peak_cases"], "wall_s": time.perf_counter() - t0}


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
