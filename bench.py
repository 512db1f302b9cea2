"""Benchmark: FLIF_GL reservoir stepping on a B200 (neuron-steps/s).

Workload (one GPU; replicas for --gpus N, no collective on the data path):
  FLIF_GL N=20000, alpha=0.6, T_mem=1024 at dt=1 (L=1024), Barabasi-Albert
  m=5, spectral radius 0.9, 13 input channels (seeded bursty-sinusoid stream),
  10 readouts, FP64 dynamics; measured in steady state (the history ring is
  full, so every neuron-step sums 1023 lags).

A bench "step" is one launch of the persistent step kernel advancing the
reservoir --chunk macro steps (default 256). `value` times those launches with
CUDA events on the library's stream, inputs already in HBM; `e2e` times
spires_run (the public C API) with the inputs in pinned host memory and the
readouts copied back every call. The history ring (164 MB) is larger than the
126 MB L2, so no flush is needed between launches.

--impl reference times the reference spires C sources compiled from source
(oracle/_ref, OpenBLAS build, all host cores) on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_NEURONS = 20000
L_HIST = 1024
DIN = 13
DOUT = 10
ALPHA = 0.6
GL_PARAMS = (1.0, 0.0, 0.0, 20.0, ALPHA, float(L_HIST), 0.1, 2.0)
SEED = 1234


def workload_config(sp, n=N_NEURONS):
    return sp.make_config(n, DIN, DOUT, rho=0.9, ei=0.5, gamma=0.5, conn=5.0 / (n - 1),
                          dt=1.0, topo=sp.CONN_SCALE_FREE, neuron=sp.FLIF_GL,
                          nparams=GL_PARAMS)


def input_stream(T, seed=7):
    """Continuous 13-channel stream: bursty-sinusoid sequences laid end to end."""
    import numpy as np

    from spires_b200 import datasets

    seqs, _ = datasets.bursty_sinusoids(num_seq=max(8, T // 40 + 2), seed=seed)
    x = np.concatenate(seqs, axis=0)
    while x.shape[0] < T:
        x = np.concatenate([x, x], axis=0)
    return np.ascontiguousarray(x[:T])


def bytes_per_launch(n, L, din, nnz, steps, g0, rate):
    """Algorithmic HBM bytes of one launch: per neuron-step 8*min(g, L-1)
    history lags + 8 ring write + 8*din input weights + 16 state, plus the CSR
    walk (4 B per column index, 8 B per weight of a spiking presynaptic
    neuron) per step."""
    tot = 0.0
    for s in range(steps):
        g = g0 + s
        tot += n * (8 * min(g, L - 1) + 8 + 8 * din + 16)
        tot += 4 * nnz + 8 * nnz * rate
    return tot


class ClockSampler:
    def __init__(self, index=0):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(index)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        import statistics

        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(shape=None):
    """Per-launch DRAM bytes of the step kernel from the committed ncu summary,
    when it was captured with the launch shape `shape` (a
    ctas:warps:variant:stages:rows:l2_pin_rows string); None otherwise."""
    path = os.path.join(ROOT, "profiles", "flif_gl_step_n20000_l1024.md")
    traffic, captured = None, None
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    traffic = float(line.split(":", 1)[1])
                elif line.startswith("traffic_launch_shape:"):
                    captured = line.split(":", 1)[1].strip()
    except Exception:
        return None
    if shape is not None and captured != shape:
        return None
    return traffic


# --------------------------------------------------------------- CPU arms --

def cpu_reference_sample(n_fill, n_timed, n=N_NEURONS):
    """Time the reference (compiled from source, OpenBLAS build) on this host.
    Returns (neuron_steps_per_s, sample description, threads)."""
    import numpy as np

    import spires_b200 as sp

    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    from tests import _oracle as O

    lib = O.ref_lib("openblas")
    cfg = workload_config(sp, n)
    u = input_stream(n_fill + n_timed)
    r = sp.Reservoir(cfg, lib=lib, seed=SEED)
    for t in range(n_fill):
        r.step(u[t])
    t0 = time.perf_counter()
    for t in range(n_fill, n_fill + n_timed):
        r.step(u[t])
    dt = time.perf_counter() - t0
    r.close()
    return n * n_timed / dt, f"reference spires_step x{n_timed} at N={n}, L={L_HIST} after {n_fill} fill steps", threads


def run_reference_arm(args):
    import numpy as np

    import spires_b200 as sp
    from tests import _oracle as O

    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    lib = O.ref_lib("openblas")
    cfg = workload_config(sp)
    per_step = args.ref_chunk
    fill = L_HIST + 8
    u = input_stream(fill + (args.warmup + args.steps) * per_step)
    r = sp.Reservoir(cfg, lib=lib, seed=SEED)
    for t in range(fill):
        r.step(u[t])
    pos = fill
    for _ in range(args.warmup):
        for _ in range(per_step):
            r.step(u[pos])
            pos += 1
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for _ in range(per_step):
            r.step(u[pos])
            pos += 1
    el = time.perf_counter() - t0
    r.close()
    value = N_NEURONS * per_step * args.steps / el
    line = {
        "impl": "reference", "metric": "reservoir neuron-steps/s", "value": value,
        "unit": "neuron-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_dict(per_step),
        "cpu_baseline": {"value": value, "unit": "neuron-steps/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{per_step} reference spires_step calls per step after {fill} fill steps"},
        "e2e": {"value": value, "unit": "neuron-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def config_dict(chunk):
    return {"workload": f"FLIF_GL N={N_NEURONS} L={L_HIST} alpha={ALPHA} Barabasi-Albert m=5 "
                        f"rho=0.9 Din={DIN} Dout={DOUT}, steady state",
            "neurons": N_NEURONS, "history_len": L_HIST, "steps_per_launch": chunk,
            "l2_policy": "history ring 164 MB > 126 MB L2 (no flush)",
            "parallelism": "replicas"}


# ---------------------------------------------------------------- GPU arm --

def max_over_ranks(x, device):
    """Largest value of x over all ranks of the process group (every rank
    gets it): the job's elapsed time is that of its slowest replica."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, seconds):
    """Whole-job throughput: every replica processes units_per_rank."""
    return world * units_per_rank / seconds


def run_gpu_arm(args, rank, world):
    import numpy as np
    import torch

    import spires_b200 as sp

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    lib = sp.load()
    cfg = workload_config(sp)
    r = sp.Reservoir(cfg, seed=SEED + rank)
    if args.variant >= 0:
        assert r.set_launch(variant=args.variant) == sp.SPIRES_OK
    if args.l2_pin >= 0:
        assert r.set_launch(l2_pin=args.l2_pin) == sp.SPIRES_OK
    lau = r.launch()
    pin_rows = int(lib.spires_ext_l2_pin_rows(r.h))
    S = args.chunk
    fill = L_HIST + 8
    total = fill + (args.warmup + args.steps) * S
    u_host = input_stream(total)
    u_dev = torch.from_numpy(u_host).to(dev)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(lib.spires_ext_stream(r.h))
    nw = (N_NEURONS + 31) // 32
    ras = torch.empty((S, nw), dtype=torch.int32, device=dev)

    def launch(pos, steps, raster=None):
        st = lib.spires_ext_run_device(r.h, C.c_void_p(u_dev.data_ptr() + pos * DIN * 8), steps,
                                       None, None if raster is None else C.c_void_p(raster.data_ptr()),
                                       None)
        assert st == sp.SPIRES_OK, st

    # fill the ring (steady state), measure the spike rate on the last chunk
    launch(0, fill - S)
    launch(fill - S, S, ras)
    assert lib.spires_ext_sync(r.h) == sp.SPIRES_OK
    rate = float(np.unpackbits(ras.cpu().numpy().view(np.uint8)).sum()) / (S * N_NEURONS)
    info = sp.HostModel(cfg, seed=SEED + rank).info
    nnz = int(info.nnz)
    pos = fill
    for _ in range(args.warmup):
        launch(pos, S)
        pos += S
    assert lib.spires_ext_sync(r.h) == sp.SPIRES_OK

    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(int(os.environ.get("SPIRES_PHYS_GPU", "0")))
    time.sleep(0.3)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    l0 = lib.spires_ext_kernel_launches(r.h)
    ev[0].record(stream)
    for k in range(args.steps):
        launch(pos, S)
        pos += S
        ev[k + 1].record(stream)
    assert lib.spires_ext_sync(r.h) == sp.SPIRES_OK
    torch.cuda.synchronize()
    launches = lib.spires_ext_kernel_launches(r.h) - l0
    clocks = clk.stop()
    per = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    if world > 1:
        total_ms = max_over_ranks(total_ms, dev)
    value = job_rate(N_NEURONS * S * args.steps, world, total_ms * 1e-3)

    # roofline of the step kernel
    g0 = fill + args.warmup * S
    bpl = bytes_per_launch(N_NEURONS, L_HIST, DIN, nnz, S, g0, rate)
    avg_ms = sum(per) / len(per)
    achieved = bpl / (avg_ms * 1e-3) / 1e9
    peak, kind = peaks()
    traffic = profile_traffic(f"{lau.ctas}:{lau.warps_max}:{lau.variant}:{lau.stages}:"
                              f"{lau.rows}:{pin_rows}")

    # end to end through spires_run with host buffers
    e2e = None
    if not args.no_e2e:
        hu = torch.from_numpy(input_stream(args.e2e_steps * S, seed=11)).pin_memory()
        hp = hu.numpy()
        fn = lib.spires_run
        t0 = time.perf_counter()
        for k in range(args.e2e_steps):
            p = fn(r.h, hp[k * S:(k + 1) * S].ctypes.data_as(sp._dp), S)
            assert p
            sp.libc.free(C.cast(p, C.c_void_p))
        el = time.perf_counter() - t0
        if world > 1:
            el = max_over_ranks(el, dev)
        e2e = {"value": job_rate(N_NEURONS * S * args.e2e_steps, world, el),
               "unit": "neuron-steps/s",
               "h2d_bytes_per_step": S * DIN * 8, "d2h_bytes_per_step": S * DOUT * 8,
               "api": "spires_run", "steps": args.e2e_steps}
    r.close()

    line = {
        "metric": "reservoir neuron-steps/s", "value": value, "unit": "neuron-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_dict(S),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": kind,
                     "algorithmic_bytes_per_launch": bpl, "avg_launch_ms": avg_ms,
                     "spike_rate": rate,
                     # the ring lags kept L2-resident are algorithmic bytes
                     # served by the L2: the DRAM side of the same launch
                     "l2_resident_ring_lags": pin_rows,
                     "dram_achieved": (traffic / (avg_ms * 1e-3) / 1e9
                                       if traffic and pin_rows > 0 else None),
                     "dram_frac": (traffic / (avg_ms * 1e-3) / 1e9 / peak
                                   if traffic and pin_rows > 0 else None)},
        "clocks": clocks, "gpu_launches": int(launches), "e2e": e2e,
        "launch": {"ctas": lau.ctas, "warps": lau.warps_max, "variant": lau.variant,
                   "stages": lau.stages, "rows": lau.rows,
                   "l2_pin_rows": pin_rows},
    }
    return line


def run_profile_case(args):
    """The bench reservoir, 1032 fill steps in one launch, then exactly one
    launch of args.chunk steps: the launch an ncu capture with -s 1 -c 1 sees."""
    import torch

    import spires_b200 as sp

    lib = sp.load()
    r = sp.Reservoir(workload_config(sp), seed=SEED)
    if args.variant >= 0:
        assert r.set_launch(variant=args.variant) == sp.SPIRES_OK
    if args.l2_pin >= 0:
        assert r.set_launch(l2_pin=args.l2_pin) == sp.SPIRES_OK
    fill = L_HIST + 8
    u = torch.from_numpy(input_stream(fill + args.chunk)).cuda()
    torch.cuda.synchronize()
    assert lib.spires_ext_run_device(r.h, C.c_void_p(u.data_ptr()), fill, None, None, None) == 0
    assert lib.spires_ext_run_device(r.h, C.c_void_p(u.data_ptr() + fill * DIN * 8), args.chunk,
                                     None, None, None) == 0
    assert lib.spires_ext_sync(r.h) == 0
    r.close()
    print("profile case done")


def run_profile_gram(args):
    """The ridge workload's states (FLIF_GL N=4000 L=512 WS, T=20000), then
    exactly one tensor-core Gram of rows [1000, 20000) in the INT8 mode with
    7 slices: the launch an ncu capture with -k regex:k_gram_tc -c 1 sees."""
    import numpy as np
    import torch

    import spires_b200 as sp
    from spires_b200.datasets import mackey_glass

    lib = sp.load()
    n, T, w = 4000, 20000, 1000
    cfg = sp.make_config(n, 1, 1, rho=0.95, ei=0.5, gamma=0.5, conn=10.0 / (n - 1),
                         topo=sp.CONN_SMALL_WORLD, neuron=sp.FLIF_GL,
                         nparams=(1.0, 0.0, 0.0, 20.0, 0.7, 512.0, 0.1, 2.0))
    x = mackey_glass(T + 1, seed=0)
    r = sp.Reservoir(cfg, seed=42)
    phi, _, _ = r.run_record(np.ascontiguousarray(x[:-1, None]), phi=True, raster=False)
    r.close()
    dX = torch.from_numpy(phi).cuda()
    dC = torch.empty((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = lib.spires_ext_gram_device(C.c_void_p(dX.data_ptr()), T, n, w, args.gram_mode,
                                    args.gram_slices, C.c_void_p(dC.data_ptr()), None)
    assert st == sp.SPIRES_OK, st
    print("profile gram done")


# ------------------------------------------------- additional workloads --
# Printed only when asked for with --workload; the default line above is the
# headline measurement.

def bf16_peak(sustained=False):
    key = "bf16_tflops_sustained" if sustained else "bf16_tflops"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)[key]), "measured"
    except Exception:
        return (1400.0 if sustained else 1590.0), "fallback"


def run_sweep_workload(args):
    """256 uneven reservoirs (LIF_DISCRETE / FLIF_GL, N log-uniform in
    [500, 8000], own Mackey-Glass series of 2000..10000 steps) in one batched
    launch; all ridge readouts from one batched simulation."""
    import numpy as np

    import spires_b200 as sp
    from spires_b200 import sweep

    insts = sweep.sweep_space(args.sweep_count, seed=2024,
                              t_range=(min(2000, args.sweep_tmax), args.sweep_tmax))
    t0 = time.perf_counter()
    b = sp.Batch([i.cfg for i in insts], [i.seed for i in insts])
    build_s = time.perf_counter() - t0
    us, ys = sweep.series_for(insts)
    ns = float(sum(i.n * i.T for i in insts))
    # the autotuner picks the schedule on the first 400 steps of every series
    tuned = b.autotune([u[:400] for u in us])
    b.run(us, rasters=False, states=False)  # warm-up (plans, captures the graph)
    times = [b.run(us, rasters=False, states=False)[2] for _ in range(max(1, args.steps // 10))]
    ms = float(np.median(times))
    res = sweep.run_sweep(insts, batch=b, washout=min(500, args.sweep_tmax // 5))
    # the same instances one at a time through the single-reservoir path
    k = min(8, len(insts))
    solo_ms, solo_ns = 0.0, 0.0
    for inst, u in list(zip(insts, us))[:k]:
        r = sp.Reservoir(inst.cfg, seed=inst.seed)
        t = time.perf_counter()
        r.run_record(u, phi=False)
        solo_ms += (time.perf_counter() - t) * 1e3
        solo_ns += inst.n * inst.T
        r.close()
    # algorithmic bytes of one run: per FLIF_GL neuron-step 8 min(g, L-1)
    # history + 8 ring write, per neuron-step of either model 8 din input
    # weights + 16 state (recurrent CSR walks not counted: a lower bound)
    byt = 0.0
    for i in insts:
        per = 8 * 1 + 16
        byt += float(i.n) * i.T * per
        if i.neuron == sp.FLIF_GL:
            L1 = i.L - 1
            hist = L1 * (L1 + 1) / 2 + max(0, i.T - i.L) * L1 if i.T >= i.L else i.T * (i.T - 1) / 2
            byt += 8.0 * i.n * (hist + i.T)
    peak, kind = peaks()
    gbs = byt / (ms * 1e-3) / 1e9
    line = {"metric": "batched sweep neuron-steps/s", "value": ns / (ms * 1e-3),
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                         "frac": gbs / peak, "peak_kind": kind,
                         "algorithmic_bytes_per_run": byt,
                         "note": "history, ring writes, input weights and state; CSR walks not counted"},
            "autotune": tuned,
            "unit": "neuron-steps/s", "n_gpus": 1, "ms_per_run": ms, "instances": len(insts),
            "neuron_steps_per_run": ns, "build_s": build_s, "fit_score_all_s": res["fit_score_s"], "nrmse_median": float(np.median(res["nrmse"])),
            "nrmse_min": float(np.min(res["nrmse"])), "schedule": b.info(),
            "single_path_sample": {"instances": k, "value": solo_ns / (solo_ms * 1e-3)},
            "dtype": "f64", "data": "synthetic (seeded Mackey-Glass per instance)",
            "config": {"workload": "sweep of uneven reservoirs", "count": len(insts),
                       "t_max": args.sweep_tmax}}
    print(json.dumps(line))


def run_search_workload(args):
    """Surrogate-guided multi-fidelity AGILE against plain AGILE (lockstep
    chains, every point at full fidelity), same start points and seeds."""
    import math

    from spires_b200 import search as S

    if args.search_scale == "full":
        space, task = S.Space(), S.Task(length=16000, val=1000, washout=200)
        rungs, points, chains = (1000, 4000, 16000), 4096, 64
    else:
        space, task = S.Space(), S.Task(length=8000, val=1000, washout=200)
        rungs, points, chains = (500, 2000, 8000), 1024, 32
    out = {}
    # surrogate: the headline arm (with --search-prescreen); surrogate_full:
    # the same without the pre-screen; no_surrogate: the schedule without
    # the networks (ranked by the low-fidelity loss)
    names = ("plain", "surrogate", "surrogate_full", "no_surrogate")
    arms = [a for a in names if a in args.search_arms.split(",")]
    assert "plain" in arms and "surrogate" in arms, "plain and surrogate arms are required"
    for name in arms:
        ev = S.Evaluator(space, task, seed=1)
        if name == "plain":
            r = S.plain_agile(ev, chains=chains, T=rungs[-1], seed=0, max_points=points)
        else:
            r = S.surrogate_agile(ev, chains=chains, rungs=rungs, max_points=points, waves=8,
                                  prescreen=args.search_prescreen if name == "surrogate" else 0.0,
                                  keep=args.search_keep,
                                  tell_optimistic=args.search_tell_optimistic,
                                  seed=0, use_surrogate=(name != "no_surrogate"))
        out[name] = (r, ev.stats)
    plain = out["plain"][0]
    target = plain.best_loss + math.log(1.02)
    tt = out["surrogate"][0].time_to(target)
    line = {"metric": "AGILE wall-clock to plain AGILE's best NRMSE (within 2%)",
            "unit": "s", "higher_is_better": False, "value": tt,
            "ratio_to_plain_wall": (tt / plain.wall_s) if tt is not None else None,
            "plain_wall_s": plain.wall_s, "plain_best_nrmse": plain.best_nrmse,
            "plain_time_to_best_s": plain.time_to(plain.best_loss)}
    for name in [a for a in names[1:] if a in out]:
        r, st = out[name]
        line[name] = {"best_nrmse": r.best_nrmse, "wall_s": r.wall_s,
                      "time_to_target_s": r.time_to(target), "evals": r.evals,
                      "neuron_steps": st.neuron_steps, "build_s": st.build_s,
                      "build_wait_s": st.build_wait_s,
                      "construct_s": st.construct_s, "setup_s": st.setup_s,
                      "screened_out": r.extra.get("screened_out"),
                      "surrogate_rmse_logNRMSE": r.extra.get("surrogate_rmse"),
                      "low_fidelity_rmse_logNRMSE": r.extra.get("low_fidelity_rmse")}
    line["plain_neuron_steps"] = out["plain"][1].neuron_steps
    line["plain_build_s"] = out["plain"][1].build_s
    line["plain_build_wait_s"] = out["plain"][1].build_wait_s
    line["plain_construct_s"] = out["plain"][1].construct_s
    line["config"] = {"workload": "surrogate-guided AGILE", "scale": args.search_scale,
                      "rungs": list(rungs), "points": points, "chains": chains, "waves": 8,
                      "prescreen": args.search_prescreen, "keep": args.search_keep,
                      "tell_optimistic": args.search_tell_optimistic}
    line["data"] = "synthetic (seeded Mackey-Glass)"
    print(json.dumps(line))


def run_classify_workload(args):
    """FLIF_GL N=20000 L=1024 BA m=5 reservoir, 500 bursty-sinusoid sequences
    of 20..100 frames, reset between sequences, 10-way ridge classifier on
    the time-averaged states."""
    from spires_b200 import classify

    out = classify.run_classification(n=N_NEURONS, num_seq=500, seed=0)
    out.update({"metric": "classification accuracy", "value": out["accuracy"], "unit": "fraction",
                "states_neuron_steps_per_s": out["neuron_steps"] / out["states_s"],
                "data": "synthetic (seeded bursty sinusoids)",
                "config": {"workload": "FLIF_GL N=20000 L=1024 sequence classification"}})
    print(json.dumps(out))


def run_construct_workload(args):
    """Host construction over the search space: --construct-count
    configurations (N log-uniform in [500, 8000], connectivity U[0.02, 0.2],
    the three topologies, sign ratios cycling through six values), each built
    with its own seed by the private-generator host build on one thread, with
    the graph drawing and the spectral-radius rescale timed apart. No GPU."""
    import numpy as np

    import spires_b200 as sp
    from spires_b200 import search as S

    space = S.Space()
    rng = np.random.default_rng(0)
    eis = (0.5, 0.3, 0.8, 0.0, 1.0, 0.123456789)
    names = {sp.CONN_RANDOM: "erdos_renyi", sp.CONN_SMALL_WORLD: "small_world",
             sp.CONN_SCALE_FREE: "scale_free"}
    per = {v: {"count": 0, "topology_s": 0.0, "spectral_s": 0.0, "edges": 0} for v in names.values()}
    t0 = time.perf_counter()
    for k in range(args.construct_count):
        th = rng.uniform(0, 1, S.DIM)
        d = space.decode(th)
        cfg = sp.make_config(d["n"], 1, 1, rho=d["rho"], ei=eis[k % len(eis)], conn=d["conn"],
                             topo=d["topo"], neuron=sp.LIF_DISCRETE, nparams=(0.0, 1.0, 0.9, 0.0))
        m = sp.HostModel(cfg, seed=k + 1, private=True)
        e = per[names[d["topo"]]]
        e["count"] += 1
        e["topology_s"] += m.info.topology_ms / 1e3
        e["spectral_s"] += m.info.spectral_ms / 1e3
        e["edges"] += int(m.info.nnz)
        del m
    wall = time.perf_counter() - t0
    topo_s = sum(v["topology_s"] for v in per.values())
    vs_ref = None
    if args.construct_reference:
        # the baseline leg: whole builds (graph, power iteration, W_in, W_out)
        # by the reference's spires_reservoir_create and by this library's host
        # build, N = 4000, connectivity 0.1, each topology
        from tests import _oracle as O

        ref = O.ref_lib()
        vs_ref = {}
        for topo in (sp.CONN_RANDOM, sp.CONN_SMALL_WORLD, sp.CONN_SCALE_FREE):
            cfg = sp.make_config(4000, 1, 1, rho=0.9, ei=0.5, conn=0.1, topo=topo,
                                 neuron=sp.LIF_DISCRETE, nparams=(0.0, 1.0, 0.9, 0.0))
            ta = time.perf_counter()
            r = sp.Reservoir(cfg, lib=ref, seed=3)
            tb = time.perf_counter()
            r.close()
            sp.HostModel(cfg, seed=3, private=True)
            tc = time.perf_counter()
            vs_ref[names[topo]] = {"reference_create_s": tb - ta, "host_build_s": tc - tb}
    print(json.dumps({
        "metric": "host graph construction time", "value": topo_s, "unit": "s",
        "higher_is_better": False, "workload": "construct", "graph_threads": 1,
        "spectral_threads": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
        "data": "synthetic", "count": args.construct_count,
        "spectral_s": sum(v["spectral_s"] for v in per.values()), "wall_s": wall,
        "per_topology": per,
        "cpu_baseline": None if vs_ref is None else {
            "kind": "reference", "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
            "sample": "whole builds, N=4000, connectivity 0.1, one per topology", "builds": vs_ref},
        "note": "graph drawing (value, one thread) and host power iteration (OpenMP "
                "threads above 65536 edges) timed by the library; the batch and reservoir "
                "builds run the power iteration of large graphs on the GPU"}))


def run_small_lif_workload(args):
    """LIF_DISCRETE N=1000 [V_0=0, V_th=1, leak=0.9, bias=0], Erdos-Renyi 0.1
    with N(0,1) weights on the present edges rescaled to spectral radius 0.9
    (injected with spires_ext_set_weights), W_in U[-1, 1], gain 0.5,
    Mackey-Glass T=5000, washout 500, ridge lambda 1e-6 (FP64)."""
    import numpy as np

    import spires_b200 as sp
    from spires_b200.datasets import mackey_glass

    n, T, w, lam = 1000, 5000, 500, 1e-6
    cfg = sp.make_config(n, 1, 1, rho=0.9, ei=0.5, gamma=0.5, conn=0.1, dt=1.0,
                         topo=sp.CONN_RANDOM, neuron=sp.LIF_DISCRETE,
                         nparams=(0.0, 1.0, 0.9, 0.0))
    rng = np.random.default_rng(SEED)
    mask = rng.random((n, n)) < 0.1
    np.fill_diagonal(mask, False)
    D = np.where(mask, rng.standard_normal((n, n)), 0.0)
    x = mackey_glass(T + 1, seed=0)
    u, y = np.ascontiguousarray(x[:-1, None]), np.ascontiguousarray(x[1:, None])
    r = sp.Reservoir(cfg, seed=SEED)
    r.set_weights(D, rescale=True)
    r.run_record(u[:500], phi=False, raster=False)  # warm-up
    r.reset()
    t0 = time.perf_counter()
    _, R, _ = r.run_record(u, phi=False, raster=True)
    step_s = time.perf_counter() - t0
    o = sp.RidgeOpts(0, 30, 1e-13, w)
    rep = sp.RidgeReport()
    t0 = time.perf_counter()
    assert r.lib.spires_ext_train_ridge(r.h, sp.dptr(u), sp.dptr(y), T, lam, C.byref(o),
                                        C.byref(rep)) == sp.SPIRES_OK
    ridge_s = time.perf_counter() - t0
    r.reset()
    yhat = r.run(u)
    r.close()
    e = yhat[w:, 0] - y[w:, 0]
    nr = float(np.sqrt(np.mean(e * e)) / y[w:, 0].std())
    spikes = int(np.unpackbits(R.view(np.uint8)).sum())
    line = {"metric": "reservoir neuron-steps/s", "value": n * T / step_s,
            "unit": "neuron-steps/s", "note": "latency bound at N=1000 (one launch, T steps)",
            "train_ridge_s": ridge_s, "nrmse": nr, "spikes": spikes,
            "ridge": {"dual": rep.dual, "rel_residual": rep.rel_residual},
            "dtype": "f64", "data": "synthetic (seeded Mackey-Glass, N(0,1) weights)",
            "config": {"workload": "LIF_DISCRETE N=1000 ER 0.1 N(0,1) rho 0.9, T=5000"}}
    print(json.dumps(line))


def run_models_workload(args):
    """Every neuron model (SIMPLE synapses) and every synapse model (FLIF_GL
    neurons) on the bench's graph (N=20000, Barabasi-Albert m=5, Din=13):
    neuron-steps/s of the step kernel in steady state (history full), and for
    the models that stream a history, its bytes per neuron-step and rate.
    History lengths: FLIF_GL 1024, FLIF_CAPUTO 512, fractional synapse 512."""
    import numpy as np
    import torch

    import spires_b200 as sp

    lib = sp.load()
    S, reps = 128, 3
    neuron_params = {
        sp.LIF_DISCRETE: (0.0, 1.0, 0.3, 0.05),
        sp.LIF_BIO: (0.0, 1.0, 5.0, 0.85),
        sp.FLIF_CAPUTO: (1.0, 0.2, 0.0, 1.0, 0.0, 1.5, 0.7, 2.0, 512.0),
        sp.FLIF_GL: GL_PARAMS,
        sp.FLIF_DIFFUSIVE: (1.0, 0.0, 0.0, 5.0, 1.0, 3.0, 0.85),
    }
    syn_params = {sp.SYN_SIMPLE: None, sp.SYN_PSC_HOM: (3.0,), sp.SYN_PSC_HET: (1.0, 10.0),
                  sp.SYN_FRAC: (0.6, 4.0, 512.0), sp.SYN_FRAC_MEXP: (0.5, 4.0, 1.0, 40.0, 5)}
    nnames = {sp.LIF_DISCRETE: "LIF_DISCRETE", sp.LIF_BIO: "LIF_BIO", sp.FLIF_CAPUTO: "FLIF_CAPUTO",
              sp.FLIF_GL: "FLIF_GL", sp.FLIF_DIFFUSIVE: "FLIF_DIFFUSIVE"}
    snames = {sp.SYN_SIMPLE: "SIMPLE", sp.SYN_PSC_HOM: "PSC_HOMOGENEOUS",
              sp.SYN_PSC_HET: "PSC_HETEROGENEOUS", sp.SYN_FRAC: "FRACTIONAL",
              sp.SYN_FRAC_MEXP: "FRACTIONAL_MULTIEXP"}
    # history bytes per neuron-step (steady state): ring lags read
    hist_bytes = {sp.FLIF_GL: 8 * 1023, sp.FLIF_CAPUTO: 8 * 510}
    combos = [(nt, sp.SYN_SIMPLE) for nt in neuron_params] + \
             [(sp.FLIF_GL, st) for st in (sp.SYN_PSC_HOM, sp.SYN_PSC_HET, sp.SYN_FRAC,
                                          sp.SYN_FRAC_MEXP)]
    rows = []
    for nt, st in combos:
        cfg = sp.make_config(N_NEURONS, DIN, DOUT, rho=0.9, ei=0.5, gamma=0.5,
                             conn=5.0 / (N_NEURONS - 1), dt=1.0, topo=sp.CONN_SCALE_FREE,
                             neuron=nt, nparams=neuron_params[nt], synapse=st,
                             sparams=syn_params[st])
        r = sp.Reservoir(cfg, seed=SEED)
        lau = r.launch()
        fill = L_HIST + 8
        u = torch.from_numpy(input_stream(fill + S * (reps + 1))).cuda()
        torch.cuda.synchronize()

        def launch(pos, steps):
            assert lib.spires_ext_run_device(r.h, C.c_void_p(u.data_ptr() + pos * DIN * 8),
                                             steps, None, None, None) == sp.SPIRES_OK

        launch(0, fill)
        stream = torch.cuda.ExternalStream(lib.spires_ext_stream(r.h))
        pos, times = fill, []
        for k in range(reps + 1):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            launch(pos, S)
            e1.record(stream)
            pos += S
            assert lib.spires_ext_sync(r.h) == sp.SPIRES_OK
            times.append(e0.elapsed_time(e1))
        r.close()
        ms = float(np.median(times[1:]))
        us_step = ms * 1e3 / S
        row = {"neuron": nnames[nt], "synapse": snames[st], "us_per_step": us_step,
               "neuron_steps_per_s": N_NEURONS * S / (ms * 1e-3),
               "launch": {"ctas": lau.ctas, "warps": lau.warps_max, "variant": lau.variant}}
        hb = hist_bytes.get(nt, 0) + (8 * 512 if st == sp.SYN_FRAC else 0)
        if hb:
            row["history_bytes_per_neuron_step"] = hb
            row["history_GBps"] = hb * N_NEURONS / (us_step * 1e-6) / 1e9
        rows.append(row)
    peak, kind = peaks()
    print(json.dumps({"metric": "step throughput per model", "unit": "neuron-steps/s",
                      "models": rows, "peak_GBps": peak, "peak_kind": kind, "dtype": "f64",
                      "data": "synthetic", "config": {"workload": "FLIF_GL bench graph, every model",
                                                      "neurons": N_NEURONS, "steps_per_launch": S}}))


def run_ridge_workload(args):
    """FLIF_GL N=4000 L=512 Watts-Strogatz k=10, Mackey-Glass T=20000,
    washout 1000, lambda 1e-6: the Gram X^T X of the 19000 fitted states in
    every mode (FP64 CUDA cores; INT8 integer slices, 7 and 8, on the tensor
    cores; BF16X3 / TF32X3 splits), timed with CUDA events through
    spires_ext_gram_device, its error against the FP64 Gram, then the ridge
    readout solved from the FP64 and INT8 Grams, with W_out and NRMSE errors
    against an FP64 numpy solve on the same states."""
    import numpy as np
    import torch

    import spires_b200 as sp
    from spires_b200.datasets import mackey_glass

    lib = sp.load()
    n, T, w, lam = 4000, 20000, 1000, 1e-6
    cfg = sp.make_config(n, 1, 1, rho=0.95, ei=0.5, gamma=0.5, conn=10.0 / (n - 1),
                         topo=sp.CONN_SMALL_WORLD, neuron=sp.FLIF_GL,
                         nparams=(1.0, 0.0, 0.0, 20.0, 0.7, 512.0, 0.1, 2.0))
    x = mackey_glass(T + 1, seed=0)
    u, y = np.ascontiguousarray(x[:-1, None]), np.ascontiguousarray(x[1:, None])
    r = sp.Reservoir(cfg, seed=42)
    phi, _, _ = r.run_record(u, phi=True, raster=False)
    r.close()
    tw = T - w
    dX = torch.from_numpy(phi).cuda()
    dC = torch.empty((n, n), dtype=torch.float64, device="cuda")
    peak, kind = bf16_peak()

    def gram(mode, slices=0, reps=3):
        times = []
        for _ in range(reps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            st = lib.spires_ext_gram_device(C.c_void_p(dX.data_ptr()), T, n, w, mode, slices,
                                            C.c_void_p(dC.data_ptr()), None)
            e1.record()
            torch.cuda.synchronize()
            assert st == sp.SPIRES_OK, st
            times.append(e0.elapsed_time(e1))
        return float(np.median(times)), dC.clone()

    ms64, G64 = gram(0)
    g64n = torch.linalg.norm(G64).item()
    fl64 = 2.0 * tw * n * n
    # the tensor-core kernel's geometry: lower-triangle 128 x 256 tiles of the
    # n padded to 256, rows padded to 128
    n_pad = (n + 255) // 256 * 256
    tiles = sum(i // 2 + 1 for i in range(n_pad // 128))
    t_pad = (tw + 127) // 128 * 128
    modes = [{"mode": "fp64", "gram_ms": ms64, "fp64_equiv_tflops": fl64 / ms64 / 1e9}]
    int8 = None
    for mode, slices, name in ((3, 7, "int8x7"), (3, 8, "int8x8"), (1, 0, "bf16x3"),
                               (2, 0, "tf32x3")):
        ms, G = gram(mode, slices)
        nprod = slices * (slices + 1) // 2 if mode == 3 else 3
        issued = 2.0 * 128 * 256 * t_pad * nprod * tiles
        row = {"mode": name, "gram_ms": ms, "fp64_equiv_tflops": fl64 / ms / 1e9,
               "issued_tops": issued / ms / 1e9,
               "gram_rel_err_vs_fp64": torch.linalg.norm(G - G64).item() / g64n}
        modes.append(row)
        if name == "int8x7":
            int8 = row
    del dC

    # ridge from the FP64 and the INT8 Gram, against an FP64 numpy solve
    Xw = phi[w:]
    A = Xw.T @ Xw
    A[np.diag_indices(n)] += lam
    Wnp = np.linalg.solve(A, Xw.T @ y[w:]).T

    def nrmse(W):
        yh = Xw @ W.T
        return float(np.sqrt(np.mean((yh[:, 0] - y[w:, 0]) ** 2)) / y[w:, 0].std())

    n_np = nrmse(Wnp)
    fits = {}
    for mode, name in ((0, "fp64"), (3, "int8x7")):
        for _ in range(2):  # the first call warms the allocator pool
            t0 = time.perf_counter()
            W, rep = sp.ridge_fit(phi, y, lam, washout=w, gram_mode=mode, max_refine=30)
            el = time.perf_counter() - t0
        nr = nrmse(W)
        dev_ms = rep.gram_ms + rep.factor_ms + rep.solve_ms + rep.refine_ms
        fits[name] = {"ridge_s": el, "device_ms": dev_ms, "collect_ms": rep.collect_ms,
                      "gram_ms": rep.gram_ms, "factor_ms": rep.factor_ms,
                      "solve_ms": rep.solve_ms,
                      "refine_ms": rep.refine_ms, "refine_iters": rep.refine_iters,
                      "rel_residual": rep.rel_residual,
                      "w_rel_err_vs_numpy_fp64": float(np.linalg.norm(W - Wnp) / np.linalg.norm(Wnp)),
                      "nrmse": nr, "nrmse_rel_err_vs_numpy_fp64": abs(nr - n_np) / n_np}
    # spires_train_ridge end to end (reset, T steps recording states, ridge),
    # the library on the GPU against the reference on all host cores
    r = sp.Reservoir(cfg, seed=42)
    t0 = time.perf_counter()
    r.train_ridge(u, y, lam)
    gpu_s = time.perf_counter() - t0
    Wg = r.readout()
    r.close()
    cpu = None
    if not args.no_cpu_baseline:
        try:
            from tests import _oracle as O

            threads = os.cpu_count() or 1
            os.environ.setdefault("OMP_NUM_THREADS", str(threads))
            rr = sp.Reservoir(cfg, lib=O.ref_lib("openblas"), seed=42)
            t0 = time.perf_counter()
            rr.train_ridge(u, y, lam)
            cpu_s = time.perf_counter() - t0
            Wr = rr.readout()
            rr.close()
            cpu = {"value": cpu_s, "unit": "s", "cores": threads, "kind": "reference",
                   "sample": "reference spires_train_ridge, N=4000 T=20000 (OpenBLAS build)",
                   "w_rel_diff_vs_library": float(np.linalg.norm(Wg - Wr) / np.linalg.norm(Wr))}
        except Exception as exc:  # the reference build is optional on a GPU host
            cpu = {"unavailable": str(exc)[:200]}
    int8_peak = 2.0 * peak
    sust, skind = bf16_peak(sustained=True)
    bf16 = [m for m in modes if m["mode"] == "bf16x3"][0]
    line = {"metric": "ridge Gram FP64-equivalent TFLOP/s (INT8 slices x7 on tensor cores)",
            "value": int8["fp64_equiv_tflops"], "unit": "TFLOP/s",
            "roofline": {"bound": "tensor", "achieved": int8["issued_tops"], "peak": int8_peak,
                         "unit": "TOP/s (int8 issued)", "frac": int8["issued_tops"] / int8_peak,
                         "peak_kind": f"2 x bf16 {kind} (dense int8 rate is twice bf16's)",
                         "int8_issued_over_bf16_sustained": int8["issued_tops"] / sust,
                         "bf16x3_issued_over_bf16_sustained": bf16["issued_tops"] / sust,
                         "bf16_sustained": sust, "bf16_sustained_kind": skind},
            "gram_modes": modes, "fits": fits, "numpy_fp64_nrmse": n_np, "lambda": lam,
            "dtype": "int8 slices / f64", "train_ridge_e2e": {"value": gpu_s, "unit": "s",
                                                              "api": "spires_train_ridge"},
            "cpu_baseline": cpu, "data": "synthetic (seeded Mackey-Glass)",
            "config": {"workload": "FLIF_GL N=4000 L=512 WS ridge, T=20000 washout 1000",
                       "fitted_rows": tw}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--chunk", type=int, default=256)
    ap.add_argument("--ref-chunk", type=int, default=20)
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variant", type=int, default=-1, help="force step-kernel variant")
    ap.add_argument("--l2-pin", type=int, default=-1,
                    help="oldest ring lags kept L2-resident (-1: the library's automatic choice)")
    ap.add_argument("--profile-case", action="store_true",
                    help="fill the ring, then one launch of --chunk steps (for ncu -s 1 -c 1)")
    ap.add_argument("--profile-gram", action="store_true",
                    help="the ridge workload's states, then one tensor-core Gram (for ncu)")
    ap.add_argument("--gram-mode", type=int, default=3)
    ap.add_argument("--gram-slices", type=int, default=7)
    ap.add_argument("--cpu-fill", type=int, default=L_HIST + 8)
    ap.add_argument("--cpu-timed", type=int, default=100)
    ap.add_argument("--workload", default="step",
                    choices=["step", "sweep", "search", "classify", "ridge", "small", "construct",
                             "models"],
                    help="step (default, the headline line) or an additional workload")
    ap.add_argument("--sweep-count", type=int, default=256)
    ap.add_argument("--construct-count", type=int, default=300)
    ap.add_argument("--construct-reference", action="store_true",
                    help="also time whole N=4000 builds against the reference's create")
    ap.add_argument("--sweep-tmax", type=int, default=10000,
                    help="longest series of the sweep (smaller for profiling)")
    ap.add_argument("--search-scale", default="medium", choices=["medium", "full"])
    ap.add_argument("--search-tell-optimistic", action="store_true",
                    help="surrogate arms: tell the chains mean - std instead of the mean")
    ap.add_argument("--search-keep", type=float, default=0.1,
                    help="surrogate arms: fraction surviving each rung (the configuration's 10 %%)")
    ap.add_argument("--search-prescreen", type=float, default=0.0,
                    help="surrogate arm: fraction of asked points simulated once trained")
    ap.add_argument("--search-arms", default="plain,surrogate,no_surrogate",
                    help="comma list of plain, surrogate, no_surrogate")
    args = ap.parse_args()
    if args.workload != "step":
        {"sweep": run_sweep_workload, "search": run_search_workload,
         "classify": run_classify_workload, "ridge": run_ridge_workload,
         "small": run_small_lif_workload, "construct": run_construct_workload,
         "models": run_models_workload}[args.workload](args)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            try:
                run_reference_arm(args)
            except Exception as exc:  # a missing build must not end the run with a traceback
                print(json.dumps({"impl": "reference",
                                  "unavailable": f"{type(exc).__name__}: {exc}"[:300]}))
        return
    if args.profile_case:
        run_profile_case(args)
        return
    if args.profile_gram:
        run_profile_gram(args)
        return

    if world > 1:
        # one GPU per process; the library and torch both see it as device 0
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        devs = vis.split(",") if vis else [str(i) for i in range(64)]
        os.environ["CUDA_VISIBLE_DEVICES"] = devs[local]
        os.environ["SPIRES_PHYS_GPU"] = devs[local]
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line = run_gpu_arm(args, rank, world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sample, cores = cpu_reference_sample(args.cpu_fill, args.cpu_timed)
        line["cpu_baseline"] = {"value": v, "unit": "neuron-steps/s", "cores": cores,
                                "kind": "reference", "sample": sample}
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
