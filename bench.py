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


def profile_traffic():
    """Per-launch DRAM bytes of the step kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "flif_gl_step_n20000_l1024.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":")[1])
    except Exception:
        pass
    return None


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
    lau = r.launch()
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
        import torch.distributed as dist

        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * N_NEURONS * S * args.steps / (total_ms * 1e-3)

    # roofline of the step kernel
    g0 = fill + args.warmup * S
    bpl = bytes_per_launch(N_NEURONS, L_HIST, DIN, nnz, S, g0, rate)
    avg_ms = sum(per) / len(per)
    achieved = bpl / (avg_ms * 1e-3) / 1e9
    peak, kind = peaks()
    traffic = profile_traffic()

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
            import torch.distributed as dist

            t = torch.tensor([el], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        e2e = {"value": world * N_NEURONS * S * args.e2e_steps / el, "unit": "neuron-steps/s",
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
                     "spike_rate": rate},
        "clocks": clocks, "gpu_launches": int(launches), "e2e": e2e,
        "launch": {"ctas": lau.ctas, "warps": lau.warps_max, "variant": lau.variant,
                   "stages": lau.stages, "rows": lau.rows},
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
    fill = L_HIST + 8
    u = torch.from_numpy(input_stream(fill + args.chunk)).cuda()
    torch.cuda.synchronize()
    assert lib.spires_ext_run_device(r.h, C.c_void_p(u.data_ptr()), fill, None, None, None) == 0
    assert lib.spires_ext_run_device(r.h, C.c_void_p(u.data_ptr() + fill * DIN * 8), args.chunk,
                                     None, None, None) == 0
    assert lib.spires_ext_sync(r.h) == 0
    r.close()
    print("profile case done")


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
    ap.add_argument("--profile-case", action="store_true",
                    help="fill the ring, then one launch of --chunk steps (for ncu -s 1 -c 1)")
    ap.add_argument("--cpu-fill", type=int, default=L_HIST + 8)
    ap.add_argument("--cpu-timed", type=int, default=100)
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference_arm(args)
        return
    if args.profile_case:
        run_profile_case(args)
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
