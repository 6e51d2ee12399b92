#!/usr/bin/env python
"""Benchmark: boards/s of tablebase generation + solve on B200.

Workload (default): the LL/4422 pruned configuration -- 64 seeded 4-tile
boards, prune stsl=58 ltc=5 smallest_large=6, generation from the initial tile
sum up to 600, then the plain FP64 solve from 600 back down, 256 goal in the
top-left.  One step = one complete generation + solve sweep with every layer
resident in HBM (layers total tens of GB, far above L2, so no flush is needed
between steps).  value = (boards generated + boards solved) / device time.

Also reported on the same line:
  fp32     -- the same sweep with FP32 tables and Kahan spawn sums, its
              throughput and its max-abs error against the FP64 tables
  e2e      -- the sweep through the C ABI with every layer and table copied
              to host buffers inside the timed region
  batch    -- 64 seeded formations in one batched sweep (FP32 solve) against
              the same formations run one sweep each
  roofline -- the dominant kernel's algorithmic bytes / its CUDA-event time
  cpu_baseline -- the reference's own CPU code on a bounded sample

`--impl reference` runs the reference's CPU implementation (oracle/_ref/cli,
built from the reference sources) on a bounded sample of the same workload.
Multi-GPU: every rank runs an independent replica (the generator has no
cross-GPU exchange); value is the sum over ranks / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Boards/s gen+solve, FP32 vs FP64 solve at <=1e-6 err; lookup/sort HBM GB/s"
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "cli")
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes (read + write) per unit of work from the ncu captures summarised in profiles/
# (smaller cases of the same kernels; their traffic grows in proportion to the units):
# a sort digit pass per key (onesweep_byte512_88M_ll_keys.md), the solve per board
# (solve_items_f64_ll_layer196.md).
NCU_DRAM_BYTES_PER_UNIT = {"onesweep": 1.379122e9 / 88333334, "solve": 1.915215e9 / 5404078}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ll_pruned")
    ap.add_argument("--end", type=int, default=None, help="override the workload's end tile sum")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-formation batched sweep block")
    ap.add_argument("--no-large", action="store_true", help="skip the large-table (config 5 prefix) block")
    ap.add_argument("--large-end", type=int, default=70, help="end tile sum of the large-table block")
    ap.add_argument("--cpu-end", type=int, default=None, help="end tile sum of the CPU sample")
    ap.add_argument("--case", default=None, choices=["sort", "expand", "solve"],
                    help="one small kernel case for a profiler capture instead of the benchmark")
    ap.add_argument("--case-end", type=int, default=260, help="end tile sum of the solve case")
    ap.add_argument("--set", action="append", default=[], metavar="NAME=VALUE",
                    help="engine option (cgb_set_option) applied before the runs; repeatable")
    return ap.parse_args()


# ---------------------------------------------------------------- helpers
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local



def aggregate_ranks(dist, boards, dev_ms, e2e=None, tensor_device="cuda"):
    """Whole-job figures of N independent replicas: boards summed over ranks, the slowest
    rank's device time, and (e2e = (boards, wall seconds) of this rank) the end-to-end rate
    as all ranks' boards over the slowest rank's wall time.  Every rank makes the same
    collective calls in the same order."""
    import torch
    b = torch.tensor([float(boards)], dtype=torch.float64, device=tensor_device)
    t = torch.tensor([float(dev_ms)], dtype=torch.float64, device=tensor_device)
    dist.all_reduce(b, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    rate = None
    eb = torch.tensor([float(e2e[0]) if e2e else 0.0], dtype=torch.float64, device=tensor_device)
    ew = torch.tensor([float(e2e[1]) if e2e else 0.0], dtype=torch.float64, device=tensor_device)
    dist.all_reduce(eb, op=dist.ReduceOp.SUM)
    dist.all_reduce(ew, op=dist.ReduceOp.MAX)
    if e2e and float(ew[0]) > 0:
        rate = float(eb[0]) / float(ew[0])
    return float(b[0]), float(t[0]), rate

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def wait_first(self, timeout=10.0):
        """Block until the first sample arrived, so that nvidia-smi's start-up (a burst of
        host work) lies before the timed region, not inside it."""
        t_end = time.time() + timeout
        while self.proc and not self.samples and time.time() < t_end and self.proc.poll() is None:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 10:
                self.samples.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        return self.summary()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        load = [s for s in self.samples if (num(s[9]) or 0) > 10] or self.samples
        sm = [num(s[1]) for s in load if num(s[1]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in load:
            for name, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": num(self.samples[0][2]),
                "power_w_max": max((num(s[3]) or 0) for s in self.samples),
                "samples": len(self.samples), "samples_under_load": len(load),
                "reasons": sorted(reasons)}


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- CPU baseline (reference build)
def reference_sample(workload, end, cores, workdir=None):
    """Run the reference CLI (generate then solve) on the workload's first layers.

    Returns (boards processed, seconds, description).  The reference refuses
    more than 127 worker threads (src/array.c:247-251).
    """
    from cablegen_b200 import configs
    import numpy as np
    wl = configs.get(workload)
    form = wl.formations[0]
    cores = max(1, min(cores, 127))
    work = workdir or tempfile.mkdtemp(prefix="cgref_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        bdir = os.path.join(work, "boards") + "/"
        tdir = os.path.join(work, "tables") + "/"
        os.makedirs(bdir, exist_ok=True)
        os.makedirs(tdir, exist_ok=True)
        np.array(form.initial, dtype="<u8").tofile(os.path.join(work, "initial"))
        np.array(form.winstates, dtype="<u8").tofile(os.path.join(work, "winstates"))
        conf = os.path.join(work, "cablegen.conf")
        configs.reference_conf(conf, wl, form, bdir, tdir, cores, end_gen=end, end_solve=form.start)
        env = dict(os.environ, XDG_CONFIG_HOME=work)
        t0 = time.perf_counter()
        subprocess.run([REF_CLI, f"-C={conf}", f"-c={cores}", "generate"], check=True, cwd=work,
                       stdout=subprocess.DEVNULL, env=env)
        gen_boards = sum(os.path.getsize(os.path.join(bdir, f)) // 8 for f in os.listdir(bdir))
        subprocess.run([REF_CLI, f"-C={conf}", f"-c={cores}", "solve"], check=True, cwd=work,
                       stdout=subprocess.DEVNULL, env=env)
        dt = time.perf_counter() - t0
    finally:
        shutil.rmtree(work, ignore_errors=True)
    desc = (f"reference CLI (oracle/_ref/cli) -c={cores}: generate {form.start}..{end} then solve {end}..{form.start} "
            f"of {workload} ({gen_boards} boards each way)")
    return 2 * gen_boards, dt, desc


def default_cpu_end(workload):
    return {"ll_pruned": 160, "plain_2x4": 300, "dpdf": 340, "ll_large": 100}.get(workload, 120)


def bench_config(workload, end=None):
    """The workload both arms name in their JSON line (identical dicts): what one step is.
    The reference arm times a bounded sample of it (its `sample` says which)."""
    from cablegen_b200 import configs
    wl = configs.get(workload) if end is None else configs.get(workload, end_gen=end)
    form = wl.formations[0]
    return {"workload": workload, "description": wl.description, "start": form.start, "end_gen": form.end_gen,
            "solve": "fp64", "step": "generate start..end_gen, then solve end_gen..start",
            "l2": "inputs larger than L2 (layers resident in HBM, tens of GB)"}


def quiet_stdout():
    """Context manager: the C API's log lines (stdout) go to /dev/null, so the bench prints
    one JSON line."""
    import contextlib

    @contextlib.contextmanager
    def cm():
        sys.stdout.flush()
        saved = os.dup(1)
        null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(null, 1)
        try:
            yield
        finally:
            os.dup2(saved, 1)
            os.close(saved)
            os.close(null)
    return cm()


def dropin_sample(workload, end, workdir=None):
    """The drop-in path on the reference arm's sample: the reference's public C API as this
    library implements it (include/cablegen.h: change_config, generate, solve), called the way
    the reference CLI calls it (frontends/cli/main.c:79-139), writing every .boards and .tables
    file to /dev/shm.  Returns (boards processed, seconds, bytes written)."""
    import ctypes as C
    import numpy as np
    from cablegen_b200 import _lib, configs
    lib = _lib.lib()

    class SArr(C.Structure):
        _fields_ = [("valid", C.c_bool), ("bp", C.POINTER(C.c_uint64)), ("size", C.c_size_t)]
    lib.generate.argtypes = [C.c_int, C.c_int, C.c_char_p, C.POINTER(SArr)]
    lib.generate.restype = None
    lib.solve.argtypes = [C.c_uint, C.c_uint, C.c_char_p, C.c_char_p, C.POINTER(SArr)]
    lib.solve.restype = None
    lib.change_config.argtypes = [C.c_char_p]
    lib.change_config.restype = None
    wl = configs.get(workload)
    form = wl.formations[0]
    work = workdir or tempfile.mkdtemp(prefix="cgdrop_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        bdir = os.path.join(work, "boards") + "/"
        tdir = os.path.join(work, "tables") + "/"
        os.makedirs(bdir, exist_ok=True)
        os.makedirs(tdir, exist_ok=True)
        init = np.array(form.initial, dtype=np.uint64)
        ws = np.array(form.winstates, dtype=np.uint64)
        init.tofile(os.path.join(work, "initial"))
        ws.tofile(os.path.join(work, "winstates"))
        conf = os.path.join(work, "cablegen.conf")
        configs.reference_conf(conf, wl, form, bdir, tdir, host_cores(), end_gen=end, end_solve=form.start)
        lib.change_config(conf.encode())
        si = SArr(True, init.ctypes.data_as(C.POINTER(C.c_uint64)), len(init))
        sw = SArr(True, ws.ctypes.data_as(C.POINTER(C.c_uint64)), len(ws))
        with quiet_stdout():
            t0 = time.perf_counter()
            lib.generate(form.start, end, (bdir + "%d.boards").encode(), C.byref(si))
            lib.solve(end, form.start, (bdir + "%d.boards").encode(), (tdir + "%d.tables").encode(), C.byref(sw))
            dt = time.perf_counter() - t0
        gen = sum(os.path.getsize(os.path.join(bdir, f)) // 8 for f in os.listdir(bdir) if f.endswith(".boards"))
        written = sum(os.path.getsize(os.path.join(d, f)) for d in (bdir, tdir) for f in os.listdir(d))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return 2 * gen, dt, written


def run_reference_arm(args):
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    cores = host_cores()
    end = args.cpu_end or default_cpu_end(args.workload)
    if not os.path.exists(REF_CLI):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cli was not built (make -C oracle ref)"}))
        return 0
    for _ in range(args.warmup):
        reference_sample(args.workload, end, cores)
    boards = 0
    secs = 0.0
    desc = ""
    for _ in range(args.steps):
        b, dt, desc = reference_sample(args.workload, end, cores)
        boards += b
        secs += dt
    value = boards / secs
    line = {"metric": METRIC, "value": value, "unit": "boards/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * secs / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded SplitMix64 boards)",
            "impl": "reference",
            "config": bench_config(args.workload, args.end),
            "sample": {"end_gen": end, "cores": min(cores, 127), "what": desc},
            "cpu_baseline": {"value": value, "unit": "boards/s", "cores": min(cores, 127), "kind": "reference",
                             "sample": desc},
            "e2e": {"value": value, "unit": "boards/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    world, rank, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    else:
        dist = None
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    from cablegen_b200 import configs, device
    wl = configs.get(args.workload) if args.end is None else configs.get(args.workload, end_gen=args.end)
    form = wl.formations[0]
    device.init(dev)
    device.set_rules(wl.settings)
    for kv in args.set:
        k, v = kv.split("=", 1)
        device.set_option(k, int(v))

    def step(precision=64, e2e=False):
        h = {"d2h": 0}
        if e2e:
            def on_layer(s, ptr, n):
                h["d2h"] += 8 * n

            def on_table(s, kp, vp, n, prec):
                h["d2h"] += (8 + prec // 8) * n
            _, _, st = device.tablebase(form.initial, form.start, form.end_gen, form.start, form.winstates,
                                        precision, layer_fn=on_layer, table_fn=on_table)
        else:
            _, _, st = device.tablebase(form.initial, form.start, form.end_gen, form.start, form.winstates,
                                        precision)
        return st

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step(64)

    # ---- timed region: K steps of the FP64 sweep (the clock sampler is running before it starts)
    clocks = ClockSampler(dev)
    clocks.start()
    clocks.wait_first()
    barrier()
    device.reset_kernel_stats()
    t0 = time.perf_counter()
    stats = [step(64) for _ in range(args.steps)]
    barrier()
    wall = time.perf_counter() - t0
    clock_summary = clocks.stop()
    kst = device.kernel_stats()
    dev_ms = sum(s["total_ms"] for s in stats)
    boards = sum(s["boards_generated"] + s["boards_solved"] for s in stats)
    gpu_launches = kst["launches"]
    # per phase, per step: the sweep's device time and the part its kernels take (the rest is
    # copies, memsets, allocation and the gaps of host round trips)
    k = max(args.steps, 1)
    gen_k = sum(kst[f"{f}_ms"] for f in ("expand", "spawn", "onesweep", "hist", "unique", "merge"))
    sol_k = kst["solve_ms"] + kst["index_ms"]
    phases = {"gen_ms": sum(s["gen_ms"] for s in stats) / k, "gen_kernel_ms": gen_k / k,
              "solve_ms": sum(s["solve_ms"] for s in stats) / k, "solve_kernel_ms": sol_k / k,
              "step_ms": [round(s["total_ms"], 1) for s in stats],
              # resident-layer chunks moved to pinned host memory and back (the store's spill policy)
              "spilled_chunks": sum(s.get("spilled_chunks", 0) for s in stats),
              "restored_chunks": sum(s.get("restored_chunks", 0) for s in stats),
              "pool_trims": kst.get("pool_trims", 0)}

    # ---- like for like with the reference arm: the same sample (generate + solve over
    # the reference arm's tile sums) through the drop-in C API, every file written.  It runs
    # right after the timed sweep, as in a CLI user's fresh process: placed after the FP32
    # block it measured 1.0e8 boards/s on a B200, right after the timed sweep 1.95e8 (same
    # code), its file writes slowed by the host memory the earlier blocks had touched
    like = None
    if not args.no_e2e and rank == 0:
        cend = args.cpu_end or default_cpu_end(args.workload)
        dropin_sample(args.workload, cend)  # warm-up
        db, dsec, dbytes = 0, 0.0, 0
        for _ in range(max(1, min(args.steps, 5))):
            b, dt, nb = dropin_sample(args.workload, cend)
            db += b
            dsec += dt
            dbytes = nb
        device.set_rules(wl.settings)
        like = {"value": db / dsec, "unit": "boards/s", "end_gen": cend,
                "sample": f"generate {form.start}..{cend} then solve {cend}..{form.start} of {args.workload}, "
                          "the reference arm's sample",
                "path": "include/cablegen.h generate() + solve() (the calls the reference CLI makes), "
                        ".boards and .tables files written to /dev/shm",
                "bytes_written_per_step": dbytes, "h2d_bytes_per_step": 8 * len(form.initial),
                "d2h_bytes_per_step": dbytes}

    # ---- FP32 sweep, its error against FP64, and the plain (bisection) FP64 solve
    fp32 = None
    if not args.no_fp32:
        device.reset_kernel_stats()
        s32 = step(32)
        k32 = device.kernel_stats()
        _, _, s0 = device.tablebase(form.initial, form.start, form.end_gen, form.start, form.winstates, 0)
        errs = s0["layer_errors"]
        tot_n = sum(n for n, _, _ in errs.values())
        old_index = device.get_option("index")
        device.set_option("index", 0)
        device.reset_kernel_stats()
        step(64)
        kplain = device.kernel_stats()
        device.set_option("index", old_index)

        def rate(k):
            return k["solve_boards"] / (k["solve_ms"] / 1000.0) if k["solve_ms"] else None
        fp32 = {"value": (s32["boards_generated"] + s32["boards_solved"]) / (s32["total_ms"] / 1000.0),
                "solve_boards_per_s": rate(k32), "fp64_solve_boards_per_s": rate(kst),
                "plain_fp64_solve_boards_per_s": rate(kplain),
                "max_abs_err": max((mx for _, mx, _ in errs.values()), default=0.0),
                "mean_abs_err": (sum(n * mean for n, _, mean in errs.values()) / tot_n) if tot_n else 0.0,
                "layers_checked": len(errs),
                "tolerance": 1e-6}
        if fp32["solve_boards_per_s"] and fp32["plain_fp64_solve_boards_per_s"]:
            fp32["solve_speedup_vs_plain_fp64"] = fp32["solve_boards_per_s"] / fp32["plain_fp64_solve_boards_per_s"]
        if fp32["solve_boards_per_s"] and fp32["fp64_solve_boards_per_s"]:
            fp32["solve_speedup_vs_fp64_hash"] = fp32["solve_boards_per_s"] / fp32["fp64_solve_boards_per_s"]

    # ---- end to end through the C ABI: every layer and every table copied to host buffers
    e2e = None
    if not args.no_e2e:
        step(64, e2e=True)  # untimed: pins the host memory the layer copies are kept in (once per process)
        barrier()
        t1 = time.perf_counter()
        se = [step(64, e2e=True) for _ in range(args.steps)]
        barrier()
        e2e_wall = time.perf_counter() - t1
        e2e_boards = sum(s["boards_generated"] + s["boards_solved"] for s in se)
        e2e = {"value": e2e_boards / e2e_wall, "unit": "boards/s",
               "h2d_bytes_per_step": int(se[0]["h2d_bytes"]), "d2h_bytes_per_step": int(se[0]["d2h_bytes"]),
               "path": "cgb_sweep_run with layer and table callbacks: layers copied once into kept pinned host "
                       "memory on the I/O stream, tables' values through pinned double buffers"}

    # ---- FP32 (Kahan) against FP64 per configuration: config 2 (this workload, above),
    # config 3 (DPDF, in full) and config 5 (LL free formation, nox 10, to the end the
    # reference's digests pin) -- both chains side by side, max/mean |fp32 - fp64| per layer
    precision = None
    if not args.no_fp32 and rank == 0:
        precision = {}
        if fp32 is not None:
            precision[args.workload] = {"layers": fp32["layers_checked"], "max_abs_err": fp32["max_abs_err"],
                                        "mean_abs_err": fp32["mean_abs_err"], "end_gen": form.end_gen}
        for name, end in (("dpdf", None), ("ll_large", 70)):
            if name == args.workload:
                continue
            pw = configs.get(name) if end is None else configs.get(name, end_gen=end)
            pf = pw.formations[0]
            device.set_rules(pw.settings)
            _, _, sp = device.tablebase(pf.initial, pf.start, pf.end_gen, pf.start, pf.winstates, 0)
            pe = sp["layer_errors"]
            pn = sum(n for n, _, _ in pe.values())
            worst = max(pe.items(), key=lambda kv: kv[1][1]) if pe else (None, (0, 0.0, 0.0))
            precision[name] = {"layers": len(pe), "boards": pn, "end_gen": pf.end_gen,
                               "max_abs_err": max((mx for _, mx, _ in pe.values()), default=0.0),
                               "mean_abs_err": (sum(n * m for n, _, m in pe.values()) / pn) if pn else 0.0,
                               "worst_layer": worst[0], "fp64_top_layers": device.get_option("fp64_top_layers")}
        device.set_rules(wl.settings)
        for v in precision.values():
            v["within_1e-6"] = v["max_abs_err"] <= 1e-6

    # ---- large single table (config 5: LL, free formation, nox 10, prune 64/6/6) up to the
    # end the reference's digests pin: FP64, layers sliced at max_sort_keys, resident-layer
    # store with its spill policy.  Kernel share = the kernels' CUDA-event time / the sweep's
    large = None
    if not args.no_large and rank == 0:
        lw = configs.get("ll_large", end_gen=args.large_end)
        lf = lw.formations[0]
        device.set_rules(lw.settings)
        _, _, sl = device.tablebase(lf.initial, lf.start, lf.end_gen, lf.start, lf.winstates, 64)
        kern = sl["expand_ms"] + sl["sort_ms"] + sl["unique_ms"] + sl["merge_ms"] + sl["solve_kernel_ms"] + \
            sl["index_ms"]
        bl = sl["boards_generated"] + sl["boards_solved"]
        large = {"workload": "ll_large", "end_gen": lf.end_gen, "solve": "fp64", "layers": sl["layers"],
                 "boards": bl, "total_ms": sl["total_ms"], "gen_ms": sl["gen_ms"], "solve_ms": sl["solve_ms"],
                 "kernel_ms": kern, "kernel_share": kern / sl["total_ms"] if sl["total_ms"] else None,
                 "boards_per_s": bl / (sl["total_ms"] / 1000.0) if sl["total_ms"] else None,
                 "layer_slices": sl["layer_slices"], "spilled_chunks": sl["spilled_chunks"],
                 "restored_chunks": sl["restored_chunks"]}
        device.set_rules(wl.settings)

    # ---- the 64-formation batch (FP32 solve): one sweep for all formations, and
    # the same formations run one sweep each
    batch = None
    if not args.no_batch:
        from cablegen_b200 import autotune
        bw = configs.get("batch64")
        saved = {k: device.get_option(k) for k in autotune.KNOBS}
        tuned = autotune.tune("batch64", end_cap=300, precision=32, cache=None)
        device.set_rules(bw.settings)
        device.batch(bw.formations, precision=32)  # warm-up
        _, _, sb = device.batch(bw.formations, precision=32)
        seq_ms, seq_boards = 0.0, 0
        for f in bw.formations:
            _, _, sf = device.tablebase(f.initial, f.start, f.end_gen, f.end_solve, f.winstates, 32)
            seq_ms += sf["total_ms"]
            seq_boards += sf["boards_generated"] + sf["boards_solved"]
        for k, v in saved.items():
            device.set_option(k, v)
        device.set_rules(wl.settings)
        bb = sb["boards_generated"] + sb["boards_solved"]
        batch = {"workload": "batch64", "description": bw.description, "formations": len(bw.formations),
                 "groups": sb["groups"], "solve": "fp32", "boards": bb, "device_ms": sb["total_ms"],
                 "boards_per_s": bb / (sb["total_ms"] / 1000.0), "graph_launches": sb["graph_launches"],
                 "gpu_launches": sb["gpu_launches"],
                 "autotuned": {"params": tuned["params"], "prefix_ms": round(tuned["ms"], 2),
                               "trials": len(tuned["trials"]), "prefix": "batch64, ends capped at 300"},
                 "sequential_boards_per_s": seq_boards / (seq_ms / 1000.0) if seq_ms else None}
        if batch["sequential_boards_per_s"]:
            batch["speedup_vs_sequential"] = batch["boards_per_s"] / batch["sequential_boards_per_s"]

    # ---- aggregate over ranks: sum of boards / slowest rank
    if dist is not None:
        e2e_in = (e2e_boards, e2e_wall) if e2e is not None else None
        boards_all, dev_ms_max, e2e_rate = aggregate_ranks(dist, boards, dev_ms, e2e_in, "cuda")
        if e2e is not None:
            e2e["value"] = e2e_rate
    else:
        boards_all, dev_ms_max = boards, dev_ms
    value = boards_all / (dev_ms_max / 1000.0)

    # ---- roofline of the dominant kernel
    peak, peak_kind = hbm_peak()
    fams = {"onesweep": "sort digit pass (onesweep)", "solve": "solve (expectimax + lookups)",
            "expand": "move expansion", "spawn": "spawn expansion", "unique": "unique", "merge": "merge",
            "hist": "sort histogram"}
    # the index builds have no algorithmic-byte figure of their own; their time is listed
    dom = max(fams, key=lambda k: kst[f"{k}_ms"])
    achieved = kst[f"{dom}_bytes"] / 1e9 / (kst[f"{dom}_ms"] / 1000.0) if kst[f"{dom}_ms"] else 0.0
    # traffic of the dominant kernel per launch: ncu bytes per unit x the mean units per launch
    traffic, traffic_note = None, None
    units = {"onesweep": (kst["onesweep_bytes"] / 16.0, kst["onesweep_launches"], "keys per pass"),
             "solve": (kst["solve_boards"], kst["solve_launches"], "boards")}
    if dom in units and dom in NCU_DRAM_BYTES_PER_UNIT and units[dom][1]:
        per_launch_units = units[dom][0] / units[dom][1]
        traffic = NCU_DRAM_BYTES_PER_UNIT[dom] * per_launch_units / 1e9
        traffic_note = (f"GB per launch: ncu DRAM bytes per unit ({NCU_DRAM_BYTES_PER_UNIT[dom]:.2f}) x mean "
                        f"{units[dom][2]} per launch ({per_launch_units:.0f}); algorithmic GB per launch "
                        f"{kst[dom + '_bytes'] / units[dom][1] / 1e9:.4f}")
    roofline = {"kernel": fams[dom], "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": ("measured hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured" else
                                "fallback: the profiling recipe's earlier measurement on this pool "
                                "(MEASURED_PEAKS.json absent)"),
                "traffic": traffic, "traffic_note": traffic_note,
                "kernels": {k: {"ms": round(kst[f"{k}_ms"], 3),
                                "GB/s": round(kst[f"{k}_bytes"] / 1e6 / kst[f"{k}_ms"], 1) if kst[f"{k}_ms"] else None,
                                "share": round(kst[f"{k}_ms"] / max(dev_ms, 1e-9), 4)}
                            for k in fams}}
    roofline["kernels"]["solve"]["lookups"] = kst["lookups"]
    # the move results the expansion found and the ones left after its per-block set
    roofline["kernels"]["expand"]["moves_raw"] = kst["moves_raw"]
    roofline["kernels"]["expand"]["moves_kept"] = kst["moves_kept"]
    roofline["kernels"]["index"] = {"ms": round(kst["index_ms"], 3), "GB/s": None,
                                    "share": round(kst["index_ms"] / max(dev_ms, 1e-9), 4),
                                    "builds": kst["index_builds"]}

    # ---- CPU baseline: the reference build on a bounded sample (rank 0, N=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and os.path.exists(REF_CLI):
        cores = host_cores()
        end = args.cpu_end or default_cpu_end(args.workload)
        b, dt, desc = reference_sample(args.workload, end, cores)
        cpu = {"value": b / dt, "unit": "boards/s", "cores": min(cores, 127), "kind": "reference", "sample": desc}
    if like is not None and cpu is not None:
        # the same sample on both sides: the like-for-like speed-up of the drop-in path
        like["ratio_vs_cpu_baseline"] = like["value"] / cpu["value"]

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "boards/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded SplitMix64 initial boards)",
                "config": bench_config(args.workload, args.end),
                "parallelism": f"replicas x{world}", "boards_per_step": boards // max(args.steps, 1),
                "phases": phases,
                "wall_s": wall, "gpu_launches": gpu_launches, "clocks": clock_summary, "roofline": roofline,
                "fp32": fp32, "precision": precision, "e2e": e2e, "like_for_like": like, "large": large,
                "batch": batch,
                "cpu_baseline": cpu}
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------- kernel cases for profiler captures
def random_ll_boards(rng, n, max_exp=9, p_empty=0.35):
    """Seeded random LL/4422 boards (cells 10,11,14,15 fixed), tiles up to 2^max_exp."""
    import numpy as np
    from cablegen_b200 import configs
    cells = configs.LL_CELLS
    free = np.array([c for c in range(16) if c not in cells])
    out = np.zeros(n, dtype=np.uint64)
    for c in cells:
        out |= np.uint64(0xF) << np.uint64(60 - 4 * c)
    exps = rng.integers(1, max_exp + 1, size=(n, len(free))).astype(np.uint64)
    exps[rng.random((n, len(free))) < p_empty] = 0
    for j, c in enumerate(free):
        out |= exps[:, j] << np.uint64(60 - 4 * int(c))
    return out


def run_case(args):
    """Small stand-alone kernel cases (a few GB on the device at most), sized for
    `ncu --set full` captures of one launch:
      sort    ~88M LL-like canonical keys: histogram, digit passes, unique
      expand  30M LL-like boards: moves (prune 58/5/6) and spawns
      solve   the LL pruned workload generated and solved (FP64) up to --case-end"""
    import numpy as np
    import torch
    from cablegen_b200 import configs, device
    device.init(0)
    w = configs.get("ll_pruned")
    device.set_rules(w.settings)
    for kv in args.set:
        k, v = kv.split("=", 1)
        device.set_option(k, int(v))
    rng = np.random.default_rng(5)
    if args.case == "sort":
        c = device.canonicalize(device.to_device(random_ll_boards(rng, 25_000_000)))
        x = torch.cat([c, c.flip(0), c[1::2], c[::2], c[::3], c[::5]])
        srt, p = device.sort(x)
        u = device.unique(srt)
        print("keys", x.numel(), "passes", p, "unique", u.numel())
    elif args.case == "expand":
        b = device.to_device(random_ll_boards(rng, 30_000_000))
        o = device.expand_moves(b)
        o2, _ = device.expand_spawns(b)
        print("moves", o.numel(), "spawns", o2.numel())
    else:
        f = w.formations[0]
        _, _, st = device.tablebase(f.initial, f.start, args.case_end, f.start, f.winstates, 64)
        print(st)
    print(device.kernel_stats())
    return 0


def main():
    args = parse()
    if args.case:
        return run_case(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
