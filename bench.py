"""Benchmark of the DSGD++ epoch on B200: SGD updates/s, HBM GB/s, roofline.

One step = one DSGD++ epoch (2d sub-epochs over all training entries) of the
100M-entry workload (2,000,000 x 500,000, Zipf(1.1) rows and columns, rank
32, FP32 factors, Nzsl_L2(1) update, L2(0.05) regularize, d x 2d blocking).

* value:   updates/s over K epochs, device time (CUDA events on the library's
           stream), inputs resident in HBM;
* e2e:     the same metric through the C ABI from pinned host buffers: the
           training/test entries and the factors are uploaded and blocked, K
           epochs each followed by the training and test loss read back to the
           host, then the factors read back -- all inside the timed region;
* roofline: the Hogwild sub-epoch kernel's algorithmic bytes per launch
           (12 B entry + 4 r 4 B of factor rows/columns + 8 B inverse counts per
           update) over its event-timed average launch duration;
* cpu_baseline: the CPU restatement of the reference (oracle, threaded mode,
           d = threads tasks, all host threads) timed on a 10M-entry sample;
           test_rmse_vs_fp64_oracle compares this implementation's test RMSE
           with the oracle's on that sample (same d, seed and steps);
* time_to_target: plain FP32 BoldDriver runs 50 epochs; its final test RMSE
           (+0.5%) is the target that BF16 + BoldDriver and the learned
           controller (FP32, BF16) race to, in wall time of every epoch, loss
           and step decision.

`--impl reference` times only the CPU restatement of the reference path on
the whole workload (every training entry, d = 64, all host threads), without
loading the CUDA library, and prints its own line with the same `config`.
Under torchrun every rank runs an independent replica of the job (the path is
one GPU per job); value is the sum over ranks / the max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: m, n, nnz, nnz_test, rank, zipf s (rows, cols), d, noise
    "c2": dict(m=2_000_000, n=500_000, nnz=100_000_000, nnz_test=1_000_000, rank=32,
               s=1.1, d=64, noise=0.2,
               text="2,000,000 x 500,000, 100M entries (+1M test), Zipf(1.1) rows and columns, "
                    "rank 32, Nzsl_L2(1) update, L2(0.05) regularize, BoldDriver(0.001) first step"),
    # a smaller case of the same shape for profiler captures (a few GB on the device)
    "c2s": dict(m=400_000, n=100_000, nnz=20_000_000, nnz_test=200_000, rank=32, s=1.1, d=64,
                noise=0.2,
                text="400,000 x 100,000, 20M entries (+200k test), Zipf(1.1) rows and columns, "
                     "rank 32, Nzsl_L2(1) update, L2(0.05) regularize"),
    # Netflix-shaped stand-in (lognormal rows, Zipf(0.9) columns, ratings 1..5)
    "c3": dict(m=480_189, n=17_770, nnz=99_000_000, nnz_test=1_400_000, rank=128, s=None, d=64,
               noise=0.0, kind="ratings",
               text="480,189 x 17,770, 99M entries (+1.4M test), lognormal(4.2, 1.3) row degrees, "
                    "Zipf(0.9) columns, integer ratings 1..5 from a rank-16 truth, rank 128, "
                    "Nzsl_L2(1) update"),
    # the controller's evaluation matrix: the 100M-entry workload's family at 300M entries
    "c5": dict(m=2_000_000, n=1_000_000, nnz=300_000_000, nnz_test=3_000_000, rank=64, s=1.1,
               d=64, noise=0.2,
               text="2,000,000 x 1,000,000, 300M entries (+3M test), Zipf(1.1) rows and columns, "
                    "rank 64, Nzsl_L2(1) update, L2(0.05) regularize, BoldDriver(0.001) first step"),
    "c1": dict(m=100_000, n=100_000, nnz=1_000_000, nnz_test=100_000, rank=10, s=None, d=4,
               noise=0.1,
               text="100,000 x 100,000, 1M uniform entries (+100k test), rank 10, "
                    "Nzsl_L2(1) update, no regularize"),
}
CPU_SAMPLE = 10_000_000
C5_SEED = 4242  # held out: the controller was trained on other matrices


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Reads SM clocks, power and clock-event (throttle) reasons through NVML
    every 10 ms while the timed region runs (read-only queries)."""

    def __init__(self, cuda_index=0):
        self.cuda_index = cuda_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None
        self._h = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.cuda_index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def start(self):
        try:
            self._h = self._handle()
        except Exception:
            self._h = None
            return
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        import pynvml
        get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                self.rows.append((pynvml.nvmlDeviceGetClockInfo(self._h, pynvml.NVML_CLOCK_SM),
                                  pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM),
                                  pynvml.nvmlDeviceGetPowerUsage(self._h) / 1000.0,
                                  get_reasons(self._h)))
            except Exception:
                pass
            self._stop.wait(0.01)

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        bits = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
                "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}
        reasons = sorted({k for r in self.rows for k, b in bits.items() if r[3] & b})
        sm = [r[0] for r in self.rows]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(r[1] for r in self.rows) if self.rows else None,
                "power_w_max": max(r[2] for r in self.rows) if self.rows else None,
                "reasons": reasons, "samples": len(self.rows), "source": "nvml"}


def algorithmic_bytes_per_update(r, precision, update):
    s_f = {"fp64": 8, "fp32": 4, "bf16": 2}[precision]
    return 12 + 4 * r * s_f + (8 if update == "Nzsl_L2" else 0)


def traffic_per_launch(name, shape):
    """DRAM bytes per launch of the Hogwild kernel from the committed ncu summary,
    or None unless the summary profiled the same kernel instance: the same d,
    lanes per entry, vectors per lane and grid (`shape`, a dict of those four)."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        text = open(path).read()
    except OSError:
        return None
    m = re.search(r"dram_bytes_per_launch_scaled:\s*([0-9.eE+]+)", text)
    if not m:
        return None
    for key in ("d", "lanes", "vecs", "grid"):
        mk = re.search(rf"profiled_{key}:\s*([0-9]+)", text)
        if not mk or int(mk.group(1)) != int(shape[key]):
            return None
    return float(m.group(1))


def cpu_sample(data, count, seed=1):
    nnz = len(data["vals"])
    k = min(count, nnz)
    # the training entries are in random order already: a prefix is a uniform sample
    return data["rows"][:k], data["cols"][:k], data["vals"][:k]


def time_cpu_reference(data, wl, steps, warmup, threads=None, with_test=False):
    """The oracle's threaded epoch (one thread per task, d = threads) on a sample;
    with_test also gives the sample run's final FP64 test RMSE."""
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    rows, cols, vals = cpu_sample(data, CPU_SAMPLE)
    if with_test:
        prob = O.Problem(wl["m"], wl["n"], wl["rank"], threads, rows, cols, vals,
                         data["trows"], data["tcols"], data["tvals"])
    else:
        prob = O.Problem(wl["m"], wl["n"], wl["rank"], threads, rows, cols, vals)
    prob.configure(update="Nzsl_L2", update_lambda=1.0,
                   regularize="L2" if wl["s"] is not None else "None",
                   regularize_lambda=0.05, loss="Nzsl_L2", loss_lambda=1.0)
    prob.set_factors(data["W0"], data["H0"])
    prob.seed(1)
    times = []
    for e in range(warmup + steps):
        ns = prob.epoch(0.001, threads=threads)
        if e >= warmup:
            times.append(ns * 1e-9)
    t = statistics.median(times)
    out = dict(value=len(vals) / t, unit="updates/s", cores=threads, kind="port",
               sample=f"{len(vals):,} training entries of the workload (prefix of the random-order "
                      f"entries), FP64, d={threads} tasks x {2 * threads} column blocks, "
                      f"median of {steps} epochs", epoch_s=t)
    if with_test:
        out["test_rmse"] = float(np.sqrt(prob.nzsl(1) / len(data["tvals"])))
        out["epochs"] = warmup + steps
        out["d"] = threads
    return out


def gpu_sample_rmse(P, data, wl, precision, d, epochs, write_mode, device, layout):
    """Test RMSE of this implementation on the CPU baseline's sample, same d,
    seed and constant step as the oracle run."""
    rows, cols, vals = cpu_sample(data, CPU_SAMPLE)
    l2 = wl["s"] is not None
    cfg = P.Config(m=wl["m"], n=wl["n"], rank=wl["rank"], d=d, precision=precision,
                   update="Nzsl_L2", update_lambda=1.0, regularize="L2" if l2 else "None",
                   regularize_lambda=0.05 if l2 else 0.0, loss="Nzsl_L2", loss_lambda=1.0,
                   write_mode=write_mode, device=device, layout=layout)
    with P.Context(cfg) as ctx:
        ctx.set_matrix(P.TRAIN, rows, cols, vals)
        ctx.set_matrix(P.TEST, data["trows"], data["tcols"], data["tvals"])
        ctx.set_factors(data["W0"], data["H0"])
        ctx.seed(1)
        for _ in range(epochs):
            ctx.epoch(0.001)
        return float(np.sqrt(ctx.nzsl(P.TEST) / len(data["tvals"])))


def _synth_gpu():
    """dsgdpp_b200/synth_gpu.py loaded as a module of its own: it needs only torch
    and numpy, and importing it through the package would load the CUDA
    library, which the reference arm must not do."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "dsgdpp_synth_gpu", os.path.join(ROOT, "dsgdpp_b200", "synth_gpu.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def arm_oracle_errors(P, data, wl, arms, epochs, device, layout, net=None, threads=None):
    """Test RMSE error against the FP64 oracle of every time-to-target arm, on
    the CPU baseline's sample: the arm runs its own step rule there for
    `epochs` decisions in its precision (BoldDriver(0.001), or the controller
    with its rollbacks), and the oracle (FP64, sequential per block) replays
    the steps the arm kept, with the same d and seed.  (Steps chosen on the
    full workload are not replayed on the sample: a step the controller kept
    there can be past the sample's stable range, where BF16 Hogwild and the
    sequential oracle part ways.)"""
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    rows, cols, vals = cpu_sample(data, CPU_SAMPLE)
    l2 = wl["s"] is not None and wl.get("kind") != "ratings"
    conf = dict(update="Nzsl_L2", update_lambda=1.0, regularize="L2" if l2 else "None",
                regularize_lambda=0.05 if l2 else 0.0, loss="Nzsl_L2", loss_lambda=1.0)
    prob = O.Problem(wl["m"], wl["n"], wl["rank"], threads, rows, cols, vals,
                     data["trows"], data["tcols"], data["tvals"])
    prob.configure(**conf)
    ntest = len(data["tvals"])
    out = {}
    for name, arm in arms.items():
        cfg = P.Config(m=wl["m"], n=wl["n"], rank=wl["rank"], d=threads,
                       precision=arm["precision"], device=device, layout=layout, **conf)
        with P.Context(cfg) as ctx:
            ctx.set_matrix(P.TRAIN, rows, cols, vals)
            ctx.set_matrix(P.TEST, data["trows"], data["tcols"], data["tvals"])
            ctx.set_factors(data["W0"], data["H0"])
            ctx.seed(1)
            if arm["controller"]:
                trace, fallbacks = ctx.run_controlled(net, epochs, 0.001)
            else:
                trace, fallbacks = ctx.run(epochs, "BoldDriver", 0.001), None
            got = float(np.sqrt(trace[-1]["test_loss"] / ntest))
        steps = [row["eps"] for row in trace[1:]]
        prob.set_factors(data["W0"], data["H0"])
        prob.seed(1)
        for eps in steps:
            prob.epoch(eps, threads=threads)
        want = float(np.sqrt(prob.nzsl(1) / ntest))
        out[name] = {"precision": arm["precision"], "epochs": len(steps), "steps": steps,
                     "fallbacks": fallbacks, "oracle_fp64_test_rmse": want, "test_rmse": got,
                     "rel_error": (got - want) / want}
    return {"sample": f"{len(vals):,} entries of the workload (the CPU baseline's sample), "
                      f"d={threads}; each arm's own step rule for {epochs} decisions, "
                      "the oracle replaying the steps it kept", "arms": out}


def time_to_target_leg(P, wl, data, d, args, local, seed_note):
    """BF16 + learned controller (and the other tuned arms) against plain FP32
    BoldDriver(0.001) on `data`, with each arm's test RMSE error against the
    FP64 oracle."""
    from dsgdpp_b200 import ttt as TT
    net = P.Mlp(device=local, seed=1)
    net.params = np.load(TT.PARAMS)
    r = TT.evaluate(P, wl, data, d, epochs=50, eps0=0.001, net=net, device=local,
                    layout=args.layout)
    leg = {"workload": wl["text"], "data_seed": seed_note,
           "target": "plain FP32 BoldDriver's test RMSE after 50 epochs, +0.5%",
           "target_test_rmse": r["target_test_rmse"], "plain_fp32_s": r["plain_fp32_s_traced"]}
    for k in ("bf16_bolddriver", "fp32_controller", "bf16_controller"):
        leg[k] = {q: r[k][q] for q in ("epochs_to_target", "seconds_to_target",
                                        "ratio_to_plain", "fallbacks", "final_test_rmse")}
    if not args.no_cpu_baseline:
        arms = {k: {"precision": r[k]["precision"], "controller": k.endswith("controller")}
                for k in ("plain_fp32", "bf16_bolddriver", "fp32_controller", "bf16_controller")}
        errs = arm_oracle_errors(P, data, wl, arms, 4, local, args.layout, net=net)
        leg["vs_fp64_oracle"] = errs
        for k, v in errs["arms"].items():
            leg.setdefault(k, {})["test_rmse_rel_error_vs_fp64_oracle"] = v["rel_error"]
    net.close()
    return leg


def generate(wl, seed):
    import torch
    synth_gpu = _synth_gpu()
    t0 = time.time()
    dev = f"cuda:{torch.cuda.current_device()}" if torch.cuda.is_available() else "cpu"
    if wl.get("kind") == "ratings":
        data = synth_gpu.make_ratings(wl["m"], wl["n"], wl["nnz"], wl["nnz_test"], wl["rank"], seed,
                                      device=dev)
        return data, time.time() - t0
    data = synth_gpu.make(wl["m"], wl["n"], wl["nnz"], wl["nnz_test"], rank_true=wl["rank"],
                          r=wl["rank"], noise=wl["noise"], seed=seed, s_row=wl["s"],
                          s_col=wl["s"], device=dev)
    return data, time.time() - t0


def workload_config(wl, precision):
    """The `config` of both arms' lines: what defines the workload, nothing
    that depends on the implementation (launch shapes go to `launch`)."""
    entries_gb = 12 * wl["nnz"] / 1e9
    factors_mb = 4 * (wl["m"] + wl["n"]) * wl["rank"] / 1e6
    tuned = wl in (WORKLOADS["c2"], WORKLOADS["c2s"])
    return {"workload": wl["text"], "m": wl["m"], "n": wl["n"], "nnz": wl["nnz"],
            "nnz_test": wl["nnz_test"], "rank": wl["rank"], "precision": precision,
            "blocking": ("d x 2d, d autotuned in 64..512" if tuned else f"d x 2d, d = {wl['d']}"),
            "l2_flush": (f"inputs larger than L2 ({entries_gb:.1f} GB entries + "
                         f"{factors_mb:.0f} MB factors)")}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def pinned(a):
    import torch
    t = torch.from_numpy(a).pin_memory()
    return t.numpy()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def _reduce(pg, v, op):
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=op)
    return float(t.item())


def allreduce_max(pg, v):
    """max over ranks (the job's time is its slowest rank's)"""
    return v if pg is None else _reduce(pg, v, pg.ReduceOp.MAX)


def allreduce_sum(pg, v):
    return v if pg is None else _reduce(pg, v, pg.ReduceOp.SUM)


def job_rate(pg, units, seconds):
    """units processed by all ranks / the slowest rank's time"""
    return allreduce_sum(pg, units) / allreduce_max(pg, seconds)


def barrier(pg):
    import torch
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()


def run_reference(args):
    """The reference's CPU path (the oracle restatement of the DSGD++ epoch; the
    reference binary cannot be built here) on the whole workload: every
    training entry, FP64, d = 64 tasks (64 x 128 blocks) run by all host
    threads with a barrier per sub-epoch; the epoch time excludes losses, as
    the reference reports it.  Rank 0 only; the CUDA library is never loaded."""
    import torch
    from oracle import oracle as O
    wl = WORKLOADS[args.workload]
    d = args.d or wl["d"]
    data, gen_s = generate(wl, args.seed)
    if torch.cuda.is_available():
        torch.cuda.empty_cache()
    threads = os.cpu_count() or 1
    t0 = time.time()
    prob = O.Problem(wl["m"], wl["n"], wl["rank"], d, data["rows"], data["cols"], data["vals"],
                     data["trows"], data["tcols"], data["tvals"])
    l2 = wl["s"] is not None and wl.get("kind") != "ratings"
    prob.configure(update="Nzsl_L2", update_lambda=1.0, regularize="L2" if l2 else "None",
                   regularize_lambda=0.05 if l2 else 0.0, loss="Nzsl_L2", loss_lambda=1.0)
    prob.set_factors(data["W0"], data["H0"])
    prob.seed(args.seed)
    setup_s = time.time() - t0
    nnz = len(data["vals"])
    for _ in range(args.warmup):
        prob.epoch(0.001, threads=threads)
    times = [prob.epoch(0.001, threads=threads) * 1e-9 for _ in range(args.steps)]
    t = sum(times)
    value = nnz * args.steps / t
    sample = (f"the whole workload: {nnz:,} training entries per epoch, FP64, d={d} tasks x "
              f"{2 * d} column blocks on {threads} threads, {args.steps} epochs after "
              f"{args.warmup} warm-up epochs")
    line = {"metric": "SGD updates/s (DSGD++ epoch)", "value": value, "unit": "updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp64", "data": "synthetic (seeded; no public dataset)",
            "config": workload_config(wl, args.precision),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "updates/s", "cores": threads,
                             "cpu_model": cpu_model(), "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "epoch_s": {"median": statistics.median(times), "min": min(times),
                        "max": max(times)},
            "final_test_rmse": float(np.sqrt(prob.nzsl(1) / len(data["tvals"]))),
            "generate_s": gen_s, "setup_s": setup_s}
    print(json.dumps(line), flush=True)
    return 0


def run_shard(args, world, rank, local, pg):
    """One job over the ranks (`--mode shard`): rank r runs tasks r d/N ..
    (r+1) d/N - 1 on its GPU and the H column blocks move between the ranks
    over NCCL, each transfer overlapping the next sub-epoch (dsgdpp_shard_*).
    A step is one epoch plus the broadcast of every block from its holder
    (what the per-epoch losses need).  value = the job's updates / the
    slowest rank's device time of the epochs; scaling is strong (the job is
    the same at every N)."""
    import torch
    import dsgdpp_b200 as P
    wl = WORKLOADS[args.workload]
    d = args.d or wl["d"]
    d = world * ((d + world - 1) // world)  # d a multiple of the ranks
    data, gen_s = generate(wl, args.seed)  # the same matrix on every rank
    m, n = wl["m"], wl["n"]
    off1 = list(P.block_offsets(m, d)) + [m]
    per = d // world
    lo, hi = int(off1[rank * per]), int(off1[(rank + 1) * per])
    l2 = wl["s"] is not None and wl.get("kind") != "ratings"
    cfg = P.Config(m=m, n=n, rank=wl["rank"], d=d, precision=args.precision, exec="hogwild",
                   launch="stream", update="Nzsl_L2", update_lambda=1.0,
                   regularize="L2" if l2 else "None", regularize_lambda=0.05 if l2 else 0.0,
                   loss="Nzsl_L2", loss_lambda=1.0, lanes_per_nnz=args.lanes,
                   vecs_per_lane=args.vecs, ctas_per_sm=args.ctas_per_sm, device=local,
                   write_mode=args.write_mode, layout=args.layout)
    keep = (data["rows"] >= lo) & (data["rows"] < hi)
    tkeep = (data["trows"] >= lo) & (data["trows"] < hi)
    n1 = np.bincount(data["rows"], minlength=m).astype(np.uint64)
    n2 = np.bincount(data["cols"], minlength=n).astype(np.uint64)
    W = np.zeros_like(data["W0"])
    W[lo:hi] = data["W0"][lo:hi]
    ctx = P.Context(cfg)
    ctx.set_tasks(rank * per, per)
    ctx.set_matrix(P.TRAIN, data["rows"][keep], data["cols"][keep], data["vals"][keep])
    ctx.set_matrix(P.TEST, data["trows"][tkeep], data["tcols"][tkeep], data["tvals"][tkeep])
    ctx.set_counts(n1, n2)
    ctx.set_factors(W, data["H0"])
    ctx.seed(args.seed)
    nnz_rank = int(keep.sum())
    del data
    uid = [P.shard_unique_id() if rank == 0 else None]
    if pg is not None:
        pg.broadcast_object_list(uid, src=0)
    sh = P.Shard.nccl(ctx, rank, world, uid[0])
    sh.set_wait_limit(120)
    eps = 0.001
    for _ in range(args.warmup):
        sh.epoch(eps)
        sh.share()
    barrier(pg)
    clocks = ClockSampler(local)
    clocks.start()
    ep_ms, moved = [], 0
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        sh.epoch(eps)
        ep_ms.append(ctx.last_epoch_ms())
        moved += sh.moved()[1]
        sh.share()
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clk = clocks.stop()
    barrier(pg)
    loss, test = sh.losses()
    t_dev = allreduce_max(pg, sum(ep_ms) / 1e3)
    value = job_rate(pg, nnz_rank * args.steps, sum(ep_ms) / 1e3)
    wall = allreduce_max(pg, wall)
    moved = allreduce_sum(pg, moved)
    sh.close()
    ctx.close()
    if rank == 0:
        line = {
            "metric": "SGD updates/s (DSGD++ epoch)", "value": value, "unit": "updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_dev / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": args.precision,
            "data": "synthetic (seeded; no public dataset)",
            "config": workload_config(wl, args.precision),
            "launch": {"d": d, "blocks": f"{d} x {2 * d}", "exec": "hogwild", "launch": "stream",
                       "parallelism": f"one job over {world} ranks (tasks {per} per rank), "
                                      "H blocks over NCCL"},
            "shard": {"h_bytes_moved_per_epoch": moved / args.steps,
                      "wall_s_with_share": wall, "final_loss": loss,
                      "final_test_rmse": float(np.sqrt(test / wl["nnz_test"]))},
            "e2e": None, "roofline": None, "cpu_baseline": None,
            "gpu_launches": args.steps * 2 * d, "clocks": clk, "generate_s": gen_s,
        }
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--d", type=int, default=0)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "bf16", "fp64"])
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--vecs", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--write-mode", default="auto", choices=["auto", "store", "atomic"])
    ap.add_argument("--launch", default="graph", choices=["graph", "persistent", "stream"],
                    help="epoch as a graph of 2d launches, or one persistent launch")
    ap.add_argument("--layout", default="runs",
                    choices=["runs", "shuffled", "col_runs", "row_runs"])
    ap.add_argument("--no-autotune", action="store_true",
                    help="use --d (default 64) instead of tuning d in 64..512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ttt", action="store_true",
                    help="skip the time-to-target comparison (tuned vs plain FP32)")
    ap.add_argument("--no-bf16", action="store_true",
                    help="skip timing the same epochs with BF16 factors")
    ap.add_argument("--no-ttt-c5", action="store_true",
                    help="skip the time-to-target comparison on the 300M-entry workload")
    ap.add_argument("--mode", default="replicas", choices=["replicas", "shard"],
                    help="under torchrun: independent replicas of the job, or one job whose "
                         "tasks are spread over the ranks (H blocks handed over with NCCL)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        # rank 0 alone times the CPU path; other ranks exit without work and
        # without joining a process group
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        import torch
        if torch.cuda.is_available():
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        return run_reference(args)

    world, rank, local, pg = dist_setup()
    if args.mode == "shard":
        rc = run_shard(args, world, rank, local, pg)
        if pg is not None:
            barrier(pg)
            pg.destroy_process_group()
        return rc

    import dsgdpp_b200 as P
    wl = WORKLOADS[args.workload]
    d = args.d or wl["d"]
    data, gen_s = generate(wl, args.seed + rank)
    l2 = wl["s"] is not None and wl.get("kind") != "ratings"
    cfg = P.Config(m=wl["m"], n=wl["n"], rank=wl["rank"], d=d, precision=args.precision,
                   exec="hogwild", launch=args.launch, update="Nzsl_L2", update_lambda=1.0,
                   regularize="L2" if l2 else "None", regularize_lambda=0.05 if l2 else 0.0,
                   loss="Nzsl_L2", loss_lambda=1.0, lanes_per_nnz=args.lanes,
                   vecs_per_lane=args.vecs, ctas_per_sm=args.ctas_per_sm, device=local,
                   write_mode=args.write_mode, layout=args.layout)
    host = {k: pinned(np.ascontiguousarray(v)) for k, v in data.items()}
    tune = None
    if not args.no_autotune and not args.d and args.workload in ("c2", "c2s"):
        t0 = time.time()
        cfg, tune_ms = P.autotune(cfg, host["rows"], host["cols"], host["vals"], host["W0"],
                                  host["H0"], d_candidates=(64, 128, 256, 512))
        d = cfg.d
        tune = {"seconds": time.time() - t0, "best_epoch_ms": tune_ms,
                "candidates_d": [64, 128, 256, 512]}
    ctx = P.Context(cfg)
    t0 = time.time()
    ctx.set_matrix(P.TRAIN, host["rows"], host["cols"], host["vals"])
    ctx.set_matrix(P.TEST, host["trows"], host["tcols"], host["tvals"])
    ctx.set_factors(host["W0"], host["H0"])
    setup_s = time.time() - t0
    nnz = int(ctx.block_nnz(P.TRAIN).sum())
    lanes, vecs, grid = ctx.launch_shape()
    ctx.seed(args.seed)
    eps = 0.001

    # ---- device-timed epochs (value) ----
    for _ in range(args.warmup):
        ctx.epoch(eps)
    ctx.sync()
    barrier(pg)
    clocks = ClockSampler(local)
    clocks.start()
    dev_ms = []
    import torch
    torch.cuda.nvtx.range_push("timed_epochs")  # lets a profiler select the timed launches
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.epoch(eps)
        dev_ms.append(ctx.last_epoch_ms())
    ctx.sync()
    wall = time.perf_counter() - wall0
    torch.cuda.nvtx.range_pop()
    clk = clocks.stop()
    barrier(pg)
    t_dev = allreduce_max(pg, sum(dev_ms) / 1e3)
    value = job_rate(pg, nnz * args.steps, sum(dev_ms) / 1e3)

    # ---- per-kernel timing of the sub-epoch kernel (roofline) ----
    ctx.set_kernel_timing(True)
    for _ in range(2):
        ctx.epoch(eps)
    k_ms, k_launches = ctx.kernel_timing()
    ctx.set_kernel_timing(False)
    bpu = algorithmic_bytes_per_update(wl["rank"], args.precision, "Nzsl_L2")
    # two epochs: 2 x 2d sub-epoch launches, or 2 persistent epoch launches
    bytes_per_launch = 2 * nnz * bpu / max(k_launches, 1)
    avg_launch_s = k_ms / 1e3 / max(k_launches, 1)
    hbm, peak_kind = peaks()
    achieved = bytes_per_launch / avg_launch_s / 1e9
    suffix = "" if args.precision == "fp32" else "_" + args.precision
    shape = {"d": d, "lanes": lanes, "vecs": vecs, "grid": grid}
    traffic = (traffic_per_launch(f"hogwild_subepoch_{args.workload}{suffix}.md", shape)
               if args.launch != "persistent" else None)

    # ---- end to end through the C ABI from pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        barrier(pg)
        # results land in pinned host buffers, as the inputs come from them
        W = pinned(np.zeros((wl["m"], wl["rank"]), np.float64))
        H = pinned(np.zeros((wl["n"], wl["rank"]), np.float64))
        t0 = time.perf_counter()
        ctx.set_matrix(P.TRAIN, host["rows"], host["cols"], host["vals"])
        ctx.set_matrix(P.TEST, host["trows"], host["tcols"], host["tvals"])
        ctx.set_factors(host["W0"], host["H0"])
        t1 = time.perf_counter()
        losses = []
        for _ in range(args.steps):
            ctx.epoch(eps)
            losses.append((ctx.loss(), ctx.nzsl(P.TEST)))
        t2 = time.perf_counter()
        ctx.get_factors_into(W, H)
        t_e2e = time.perf_counter() - t0
        parts = {"upload_s": t1 - t0, "steps_s": t2 - t1, "download_s": t_e2e - (t2 - t0)}
        e2e_rate = job_rate(pg, nnz * args.steps, t_e2e)
        t_e2e = allreduce_max(pg, t_e2e)
        h2d = (16 * (len(host["vals"]) + len(host["tvals"])) + 8 * (wl["m"] + wl["n"]) * wl["rank"]
               + args.steps * (2 * d * d * 4 + 24))
        d2h = 8 * (wl["m"] + wl["n"]) * wl["rank"] + args.steps * 16
        e2e = {"value": e2e_rate, "unit": "updates/s",
               "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
               "seconds": t_e2e, **parts,
               "final_test_rmse": float(np.sqrt(losses[-1][1] / len(host["tvals"])))}

    cpu = None
    vs_oracle = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref = time_cpu_reference(data, wl, steps=2, warmup=0, with_test=True)
        cpu = {k: ref[k] for k in ("value", "unit", "cores", "kind", "sample")}
        cpu["cpu_model"] = cpu_model()
        # the same sample, d, seed and steps on the GPU: test RMSE against the FP64 oracle
        got = gpu_sample_rmse(P, data, wl, args.precision, ref["d"], ref["epochs"],
                              args.write_mode, local, args.layout)
        vs_oracle = {"precision": args.precision, "epochs": ref["epochs"], "d": ref["d"],
                     "sample": "the CPU baseline's sample", "oracle_fp64_test_rmse": ref["test_rmse"],
                     "test_rmse": got, "rel_error": (got - ref["test_rmse"]) / ref["test_rmse"]}

    ctx.close()

    # ---- the precision form: the same epochs with BF16 factors (FP32 context closed) ----
    bf16 = None
    if args.precision == "fp32" and not args.no_bf16 and args.launch != "persistent":
        import dataclasses
        cfg16 = dataclasses.replace(cfg, precision="bf16", lanes_per_nnz=0, vecs_per_lane=0,
                                    ctas_per_sm=0)
        with P.Context(cfg16) as c16:
            c16.set_matrix(P.TRAIN, host["rows"], host["cols"], host["vals"])
            c16.set_factors(host["W0"], host["H0"])
            c16.seed(args.seed)
            for _ in range(args.warmup):
                c16.epoch(eps)
            ms16 = []
            for _ in range(args.steps):
                c16.epoch(eps)
                ms16.append(c16.last_epoch_ms())
            c16.set_kernel_timing(True)
            for _ in range(2):
                c16.epoch(eps)
            k16, kl16 = c16.kernel_timing()
            l16, v16, g16 = c16.launch_shape()
        bpu16 = algorithmic_bytes_per_update(wl["rank"], "bf16", "Nzsl_L2")
        ach16 = 2 * nnz * bpu16 / max(kl16, 1) / (k16 / 1e3 / max(kl16, 1)) / 1e9
        bf16 = {"epoch_ms": sum(ms16) / len(ms16), "updates_per_s": nnz / (sum(ms16) / len(ms16) / 1e3),
                "lanes_per_nnz": l16, "vecs_per_lane": v16, "grid": g16,
                "roofline": {"bound": "hbm", "achieved": ach16, "peak": hbm, "unit": "GB/s",
                             "frac": ach16 / hbm, "bytes_per_update": bpu16,
                             "avg_launch_us": k16 * 1e3 / max(kl16, 1),
                             "achieved_epoch": nnz * bpu16 / (sum(ms16) / len(ms16) / 1e3) / 1e9,
                             "frac_epoch": nnz * bpu16 / (sum(ms16) / len(ms16) / 1e3) / 1e9
                             / hbm}}

    # ---- time to target test RMSE: BF16 + learned controller vs plain FP32 ----
    ttt = None
    if rank == 0 and world == 1 and args.workload == "c2" and not args.no_ttt:
        ttt = time_to_target_leg(P, wl, data, d, args, local, args.seed)
        if not args.no_ttt_c5:
            # the controller's evaluation workload: 300M entries, rank 64, a data
            # seed the controller was not trained on
            del data, host
            wl5 = WORKLOADS["c5"]
            data5, _ = generate(wl5, C5_SEED)
            ttt["c5"] = time_to_target_leg(P, wl5, data5, wl5["d"], args, local, C5_SEED)
            del data5
    if rank == 0:
        line = {
            "metric": "SGD updates/s (DSGD++ epoch)", "value": value, "unit": "updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_dev / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.precision,
            "data": "synthetic (seeded; no public dataset)",
            "config": workload_config(wl, args.precision),
            "launch": {"d": d, "blocks": f"{d} x {2 * d}", "exec": "hogwild",
                       "launch": args.launch, "lanes_per_nnz": lanes, "vecs_per_lane": vecs,
                       "write_mode": args.write_mode, "layout": args.layout, "grid": grid,
                       "parallelism": f"replicas x{world}", "autotune": tune},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "peak_source": peak_kind,
                         "bytes_per_update": bpu,
                         "kernel": ("hogwild_epoch_kernel" if args.launch == "persistent"
                                    else "hogwild_subepoch_kernel"),
                         "avg_launch_us": avg_launch_s * 1e6,
                         "timing": ("CUDA events around each one-launch epoch of 2 epochs"
                                    if args.launch == "persistent" else
                                    "CUDA events around each sub-epoch launch of 2 epochs "
                                    "launched on the library stream (not from the graph; "
                                    "the events keep the launches from overlapping)"),
                         # the timed epochs themselves: the epoch's algorithmic bytes over
                         # its device time, every kernel of the epoch included
                         "achieved_epoch": nnz * bpu / (t_dev / args.steps) / 1e9,
                         "frac_epoch": nnz * bpu / (t_dev / args.steps) / 1e9 / hbm},
            "cpu_baseline": cpu,
            "test_rmse_vs_fp64_oracle": vs_oracle,
            "bf16_factors": bf16,
            "time_to_target": ttt,
            "e2e": e2e,
            "gpu_launches": args.steps * ((2 if args.launch == "persistent" else 2 * d + 1)
                                          + (1 if l2 else 0)),
            "clocks": clk,
            "wall_s_timed": wall, "setup_s": setup_s, "generate_s": gen_s,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        barrier(pg)
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
