"""Benchmark of the B200 OnionPIRv2 server path (PirServer::make_query).

Workload (default, --workload k1): k1_comp parameters (N = 2048,
q = q1 q2 ~ 2^58, t = 4099), a 2^18-plaintext database (872 MB of 13-bit
coefficients; 4 GiB in NTT form on the device), first dimension 512 x 9
further binary dimensions. --workload c4: CONFIG_N4096_K2_MP (N = 4096, two
60-bit RNS limbs, t = generate_prime(40)), 2^20 plaintexts (64 GiB in NTT
form), first dimension 1024 x 10 further binary dimensions. A step is one
batch of B independent queries (each with its own client keys) answered by
one pass of the path; the first-dimension scan reads the database once per
batch. The database is larger than L2 (126 MB), so every step streams it from
HBM; no L2 flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--workload c4]
    python bench.py --impl reference ...      # the reference's CPU server

N > 1 runs one rank per GPU (torchrun), each holding a replica of the
database and serving its own queries (queries are independent: replicas
only, no collective on the data path); timing is the max over ranks.

    python bench.py --rows-sharded [--gpus N] ...

instead splits ONE database by candidate rows over the N ranks (strong
scaling): every step, each rank answers its shard for the same batch, the
partial ciphertexts are gathered to rank 0 over NCCL and rank 0 finishes
the last log2 N MUX levels. On one GPU this is the whole database (one
shard), and the line adds the per-GPU time of one shard of a 2-, 4- and
8-way split measured on this GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "queries/s and DB GB/s at 1 GB DB, batched vs plain GPU (bit-exact); p50/p99 ms"
TARGET, HEIGHT = 262144, 10
C4_TARGET, C4_HEIGHT = 1 << 20, 11
C4_CONFIG = "CONFIG_N4096_K2_MP"
K2_CONFIG = "CONFIG_N2048_K2_MP"
# the parameter set of each workload (tree: its own scheme)
K1P_CONFIG = "CONFIG_N2048_K1"
CONFIGS = {"k1": "CONFIG_N2048_K1_COMP", "c4": C4_CONFIG, "k2mp": K2_CONFIG, "k1p": K1P_CONFIG}
# suffix of the reference binaries built with each workload's configuration
REF_SUFFIX = {"k1": "", "k2mp": "_k2mp", "k1p": "_k1"}
# two timed layouts of the reference under CONFIG_N4096_K2_MP with the full
# workload's first dimension (1024) and expansion height (11): 4 and 32
# candidate rows
C4_REF_LAYOUTS = (4096, 32768)
DB_SEED = 20261203


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-queries", type=int, default=3)
    ap.add_argument("--workload", choices=["k1", "c4", "k2mp", "k1p", "tree"], default="k1",
                    help="k1: CONFIG_N2048_K1_COMP at 2^18 plaintexts; c4: CONFIG_N4096_K2_MP at 2^20; "
                         "k2mp: CONFIG_N2048_K2_MP at 2^18; k1p: CONFIG_N2048_K1 at 2^18; "
                         "tree: tree PIR path selection (L = 16, a = 3)")
    ap.add_argument("--target", type=int, default=None,
                    help="plaintexts (smaller layouts are for profiling captures)")
    ap.add_argument("--height", type=int, default=None)
    ap.add_argument("--sweep", default=None,
                    help="batch sizes timed after the headline (default 1,8,32,128 for k1, "
                         "1,8,32,64 for c4; 'none' to skip)")
    ap.add_argument("--concurrent", action="store_true",
                    help="also time two batches in flight at once (two handles on the same "
                         "database layout, two streams): the served form's overlap")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default scan tiling (or OPIR_SCAN_TILE)")
    ap.add_argument("--tree-config", choices=["k1", "c4"], default="k1",
                    help="--workload tree: CONFIG_N2048_K1_COMP (L=16, a=3) or CONFIG_N4096_K2_MP "
                         "(L=17, a=3)")
    ap.add_argument("--rows-sharded", action="store_true",
                    help="one database split by candidate rows over the ranks (strong scaling)")
    ap.add_argument("--client", action="store_true",
                    help="client-side batch operations: response decryption and query packing")
    ap.add_argument("--client-config", choices=["k1", "c4"], default="k1")
    ap.add_argument("--client-batch", type=int, default=1024,
                    help="responses (and queries) per step (--client)")
    ap.add_argument("--serve", action="store_true",
                    help="serving loop: Poisson arrivals over three resident databases")
    ap.add_argument("--rates", default="50,500,2000", help="offered queries/s (--serve)")
    ap.add_argument("--duration", type=float, default=3.0, help="seconds per rate (--serve)")
    args = ap.parse_args()
    c4 = args.workload == "c4"
    if args.target is None:
        args.target = C4_TARGET if c4 else TARGET
    if args.height is None:
        args.height = C4_HEIGHT if c4 else HEIGHT
    if args.sweep is None:
        args.sweep = "1,8,32,64" if c4 else "1,8,32,128"
    args.sweep = [] if args.sweep == "none" else [int(x) for x in args.sweep.split(",")]
    return args


# ---------------------------------------------------------------- distributed
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Max of a per-rank float over all ranks (identity when world == 1)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int, device=None):
    if world > 1:
        import torch.distributed as dist
        dist.barrier(device_ids=[device.index] if device is not None and device.type == "cuda" else None)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d.get("bf16_tflops"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": None, "source": "fallback"}


def ncu_traffic() -> dict | None:
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


def ntt_butterflies(params) -> dict:
    """NTT butterflies per query of the two NTT-bound stages, over both RNS
    residues (limbs): expansion = one BV key switch per heap node
    (L_KS digit NTTs + 2 INTTs, bv_keyswitch.cpp:296-367 / 373-481; nodes of
    level d = ceil(useful / 2^(h-d)), server.cpp:786-792); other dimensions =
    other_dim_sz - 1 external products (2 L_EP digit NTTs + 2 INTTs,
    gsw.cpp:119-250, server.cpp:652-722). One butterfly = one Shoup product."""
    N = params.N
    per_ntt = (N // 2) * (N.bit_length() - 1)
    # NTTs run per residue (k1_comp) or RNS limb; CONFIG_N2048_K1 has one prime
    planes = 1 if (params._p.num_limbs == 1 and params._p.q1 == 0) else 2
    h = params.expansion_height
    useful = params.fst_dim_sz + params.l_ep * (params.num_dims - 1)
    nodes = sum(-(-useful // (1 << (h - d))) for d in range(h))
    return {"Expand": nodes * (params.l_ks + 2) * per_ntt * planes,
            "Other dim": (params.other_dim_sz - 1) * (2 * params.l_ep + 2) * per_ntt * planes}


def int_pipe_roofline(params, config: str, stages: dict, batch: int, device: int) -> dict:
    """Achieved NTT butterflies/s of the NTT-bound stages (live stage times)
    against the device's measured butterfly rate (register-resident probe)."""
    from onionpirv2_b200.server import measure_butterfly_rate
    peak = measure_butterfly_rate(config, device) / 1e9
    out = {"bound": "integer multiply pipe (NTT butterflies, one Shoup product each)",
           "unit": "Gbutterflies/s", "peak": peak,
           "peak_source": "measured (opir_measure_butterfly_rate: the kernels' radix-8 pass on "
                          "register operands, all SMs)", "stages": {}}
    for name, per_query in ntt_butterflies(params).items():
        ms = stages.get(name)
        if not ms:
            continue
        achieved = per_query * batch / (ms / 1e3) / 1e9
        out["stages"][name] = {"achieved": achieved, "frac": achieved / peak,
                               "butterflies_per_query": per_query}
    if config in ("CONFIG_N2048_K1_COMP", "CONFIG_N2048_K2_MP"):
        out["tc_ntt_bound"] = tc_ntt_bound(peak, params.N, device)
    return out


def tc_ntt_bound(bfly_peak_g: float, N: int, device: int) -> dict:
    """Coefficients per second of a digit NTT on the register butterflies
    (each coefficient takes part in log2 N butterflies, two per butterfly)
    against the most a byte-sliced int8 tensor-core four-step NTT could
    finish with a free MMA: one 5-class epilogue (2-plane digits x 4-plane
    twiddles) and one 7-class epilogue (4 x 4 planes) per coefficient, each
    at the measured register-resident recombination rate."""
    from onionpirv2_b200.server import measure_recombine_rate
    r5 = measure_recombine_rate(5, device) / 1e9
    r7 = measure_recombine_rate(7, device) / 1e9
    reg = bfly_peak_g * 2 / (N.bit_length() - 1)
    tc = 1.0 / (1.0 / r5 + 1.0 / r7)
    return {"unit": "G coefficients/s", "recombine_5": r5, "recombine_7": r7,
            "register_ntt": reg, "tc_ntt_epilogue_only": tc, "register_over_tc": reg / tc}


def synthetic_inputs(params, batch: int, seed: int):
    """Seeded uniform ciphertexts and key material mod q (per RNS limb under
    CONFIG_N4096_K2_MP). make_query's work is data-independent, so uniform
    inputs time the same arithmetic as genuine client queries (parity is
    proven by tests/)."""
    shape = params.ct_shape
    mods = np.array(params.get_rns_mods(), dtype=np.uint64)
    rng = np.random.default_rng(seed)

    def uniform(lead):
        if len(mods) == 1:
            return rng.integers(0, mods[0], tuple(lead) + shape, dtype=np.uint64)
        a = rng.integers(0, np.iinfo(np.uint64).max, tuple(lead) + shape, dtype=np.uint64,
                         endpoint=True)
        return a % mods[:, None]     # limb axis is the second to last

    queries = uniform((batch,))
    keys = []
    for b in range(batch):
        bv = uniform((params.expansion_height, params.l_ks))
        gsw = uniform((2 * params.l_key,))
        keys.append((bv, gsw))
    return queries, keys


def ref_binary(suffix: str = "") -> str | None:
    d = os.path.join(ROOT, "oracle", "_ref")
    fast, port = os.path.join(d, f"opir_ref{suffix}_avx512"), os.path.join(d, f"opir_ref{suffix}")
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
    except OSError:
        flags = ""
    if os.path.exists(fast) and "avx512f" in flags and "avx512dq" in flags and "avx512bw" in flags:
        return fast
    return port if os.path.exists(port) else None


def run_reference(queries: int, warmup: int, procs: int, seed: int, suffix: str = "") -> dict:
    exe = ref_binary(suffix)
    if exe is None:
        raise FileNotFoundError("oracle/_ref is not built")
    cmd = [exe, "--mode", "time", "--target", str(TARGET), "--height", str(HEIGHT),
           "--db-seed", str(DB_SEED), "--client-seed", str(seed), "--queries", str(queries),
           "--warmup", str(warmup), "--procs", str(procs)]
    out = subprocess.run(cmd, check=True, capture_output=True, text=True)
    res = json.loads(out.stdout.strip().splitlines()[-1])
    res["binary"] = os.path.basename(exe)
    return res


def run_reference_c4(queries: int, procs: int, seed: int) -> dict:
    """The reference built with CONFIG_N4096_K2_MP, timed at two layouts that
    share the full workload's first dimension (1024) and expansion height
    (11). Its make_query cost is affine in the candidate-row count (the scan
    and the MUX tree grow with it; expansion and selectors barely change), so
    the per-query time at 1024 rows (2^20 plaintexts, a 64 GiB database the
    CPU server cannot load within a benchmark) is extrapolated from the two."""
    exe = ref_binary("_c4")
    if exe is None:
        raise FileNotFoundError("oracle/_ref is not built")
    runs = []
    for tgt in C4_REF_LAYOUTS:
        cmd = [exe, "--mode", "time", "--target", str(tgt), "--height", str(C4_HEIGHT),
               "--db-seed", str(DB_SEED), "--client-seed", str(seed), "--queries", str(queries),
               "--warmup", "0", "--procs", str(procs)]
        out = subprocess.run(cmd, check=True, capture_output=True, text=True)
        runs.append(json.loads(out.stdout.strip().splitlines()[-1]))
    rows = [(t + 1023) // 1024 for t in C4_REF_LAYOUTS]
    slope = (runs[1]["mean_ms"] - runs[0]["mean_ms"]) / (rows[1] - rows[0])
    full_ms = runs[0]["mean_ms"] + slope * (C4_TARGET // 1024 - rows[0])
    return {"mean_ms": full_ms, "qps": procs * 1000.0 / full_ms, "runs": runs, "rows": rows,
            "binary": os.path.basename(exe), "queries": queries * procs}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor()


# ---------------------------------------------------------------- reference arm
def bench_reference(args, world, rank):
    if rank != 0:
        return
    procs = os.cpu_count() or 1
    if args.workload == "c4":
        bench_reference_c4(args, procs)
        return
    if args.workload == "tree":
        bench_reference_tree(args, procs)
        return
    # a bounded sample: at most 8 timed queries (and 1 warm-up) per process,
    # ~2 s each on one core, so the run ends within a few minutes
    n_q, n_w = min(args.steps, 8), min(args.warmup, 1)
    k2 = args.workload == "k2mp"
    try:
        res = run_reference(n_q, n_w, procs, 7, REF_SUFFIX[args.workload])
    except Exception as e:  # reference binary missing or failed
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU server: {e}"}))
        return
    qps = res["qps"]
    line = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["mean_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": (f"{CONFIGS[args.workload] if args.workload != 'k1' else 'k1_comp'} N=2048, {TARGET} "
                                f"plaintexts, first dim 512 x 9 binary dims"),
                   "batch": 1, "parallelism": f"{procs} host processes"},
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": procs, "kind": "reference",
                         "sample": (f"reference make_query (oracle/_ref/{res['binary']}, HEXL stand-in) "
                                    f"on {procs} forked processes x {n_q} queries ({n_w} warm-up) after one "
                                    f"load_data; "
                                    f"CPU {cpu_model()}; " + HEXL_CAVEAT)},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# the CPU baseline runs the reference's sources against this repository's
# HEXL stand-in (Intel HEXL cannot be installed here)
HEXL_CAVEAT = ("the HEXL stand-in is written from the mathematics, not Intel HEXL's AVX-512 "
               "kernels: the paper's single-thread HEXL figure (1031 MB/s over the 805 MB "
               "logical database at 12 bits per coefficient, docs/2025-1142.pdf Table 2) is "
               "about 1.28 queries/s per core at this layout, about 2.3x this stand-in's rate")


def c4_workload_name(params) -> str:
    return (f"CONFIG_N4096_K2_MP N=4096 two 60-bit limbs, {params.num_pt} plaintexts "
            f"({2 * params.N * params.num_pt * 8} B NTT form), first dim {params.fst_dim_sz} x "
            f"{params.num_dims - 1} binary dims")


def c4_sample(res: dict, cores: int) -> str:
    a, b = res["runs"]
    return (f"reference make_query (oracle/_ref/{res['binary']}, HEXL stand-in) under "
            f"CONFIG_N4096_K2_MP on {cores} host process(es): {a['mean_ms']:.0f} ms/query at "
            f"{C4_REF_LAYOUTS[0]} plaintexts ({res['rows'][0]} candidate rows) and "
            f"{b['mean_ms']:.0f} ms at {C4_REF_LAYOUTS[1]} ({res['rows'][1]} rows), first dim 1024, "
            f"h={C4_HEIGHT}, {res['queries']} queries per layout; per-query time at 1024 rows "
            f"(2^20 plaintexts) extrapolated along the affine row dependence = "
            f"{res['mean_ms']:.0f} ms; CPU {cpu_model()}")


def bench_reference_c4(args, procs):
    n_q = max(1, min(args.steps, 2))
    try:
        res = run_reference_c4(n_q, procs, 7)
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU server: {e}"}))
        return
    qps = res["qps"]
    line = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["mean_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"CONFIG_N4096_K2_MP N=4096, {C4_TARGET} plaintexts, first dim "
                               f"1024 x 10 binary dims", "batch": 1,
                   "parallelism": f"{procs} host processes"},
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": procs, "kind": "reference",
                         "sample": c4_sample(res, procs)},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------- our arm
def bench_ours(args, world, rank, local):
    import torch
    from onionpirv2_b200 import PirParams, PirServer
    from onionpirv2_b200.server import launch_count

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=device)
    c4 = args.workload == "c4"
    k2 = args.workload == "k2mp"
    config = CONFIGS[args.workload]
    params = PirParams(args.target, args.height, config=config)
    N = params.N
    B = args.batch
    ct_words = int(np.prod(params.ct_shape))
    srv = PirServer(params, device=local)
    t0 = time.perf_counter()
    srv.load_data_seeded(args.target, DB_SEED)
    load_s = time.perf_counter() - t0
    nq = max([B] + args.sweep)           # queries (and clients) the runs need
    queries, keys = synthetic_inputs(params, nq, 1000 + rank)
    for b, (bv, gsw) in enumerate(keys):
        srv.set_client_keys(b, bv, gsw)
    t0 = time.perf_counter()
    if not args.no_autotune:
        srv.autotune(nq)                 # scan tiling per batch bucket (setup, untimed)
    tune_s = time.perf_counter() - t0
    ids = list(range(nq))
    # a dedicated (non-default) stream: the library orders its own stream
    # after this one and this one after its work, so events recorded here
    # bracket the whole batch
    stream = torch.cuda.Stream(device)
    d_q = torch.from_numpy(queries.view(np.int64)).to(device)
    d_r = torch.empty((nq, 2, N), dtype=torch.int64, device=device)

    def step(n, qbuf, rbuf):
        srv.make_query_batch_device(ids[:n], qbuf.data_ptr(), rbuf.data_ptr(), stream.cuda_stream)

    def nvtx(name):
        """NVTX range around a timed loop (lets a profiler select it)."""
        import contextlib
        try:
            return torch.cuda.nvtx.range(name)
        except Exception:
            return contextlib.nullcontext()

    def timed(n, steps, warm):
        qb, rb = d_q[:n].contiguous(), d_r[:n].contiguous()
        for _ in range(warm):
            step(n, qb, rb)
        torch.cuda.synchronize(device)
        barrier(world, device)
        torch.cuda.synchronize(device)
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        srv.set_stage_timing(True)
        l0 = launch_count()
        with nvtx(f"timed_b{n}"):
            evs[0].record(stream)
            for i in range(steps):
                step(n, qb, rb)
                evs[i + 1].record(stream)
            torch.cuda.synchronize(device)
        launches = launch_count() - l0
        barrier(world, device)
        per = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
        total = evs[0].elapsed_time(evs[-1])
        stages = srv.stage_times()
        srv.set_stage_timing(False)
        return total, per, stages, launches

    # plain single-query path (B = 1)
    plain_total, plain_per, plain_stages, _ = timed(1, args.steps, args.warmup)
    plain_total = max_over_ranks(plain_total, world, device)
    # batched path (headline), clocks sampled during the timed region
    with ClockSampler(local) as clk:
        total, per, stages, launches = timed(B, args.steps, args.warmup)
    total_max = max_over_ranks(total, world, device)
    queries_done = world * B * args.steps
    qps = queries_done / (total_max / 1e3)

    # end to end through the host-buffer C ABI call (pinned host memory)
    hq = torch.from_numpy(queries[:B].view(np.int64)).pin_memory()
    hr = torch.empty((B, 2, N), dtype=torch.int64).pin_memory()
    hq_np, hr_np = hq.numpy().view(np.uint64), hr.numpy().view(np.uint64)
    for _ in range(args.warmup):
        srv.make_query_batch(ids[:B], hq_np, out=hr_np)
    barrier(world, device)
    te = time.perf_counter()
    for _ in range(args.steps):
        srv.make_query_batch(ids[:B], hq_np, out=hr_np)
    e2e_s = max_over_ranks(time.perf_counter() - te, world, device)
    e2e_qps = queries_done / e2e_s

    # batch-size sweep (BASELINE's batched configs), fewer steps each
    sweep = []
    for sb in args.sweep:
        k = max(3, min(args.steps, 20))
        s_total, s_per, s_stages, _ = timed(sb, k, args.warmup)
        s_total = max_over_ranks(s_total, world, device)
        sweep.append({"batch": sb, "steps": k,
                      "queries_per_s": world * sb * k / (s_total / 1e3),
                      "ms_per_batch": s_total / k,
                      "p50_ms": float(np.percentile(s_per, 50)),
                      "scan_ms": round(s_stages["Core"], 4)})

    # two batches in flight: a second handle on its own stream (the serving
    # loop's overlap of batches), device-timed around both streams
    conc = None
    if args.concurrent and world == 1:
        srv2 = PirServer(params, device=local)
        srv2.load_data_seeded(args.target, DB_SEED)
        for b, (bv, gsw) in enumerate(keys):
            srv2.set_client_keys(b, bv, gsw)
        if not args.no_autotune:
            srv2.autotune(nq)
        s2 = torch.cuda.Stream(device)
        qb, rb = d_q[:B].contiguous(), d_r[:B].contiguous()
        rb2 = torch.empty_like(rb)

        def both():
            srv.make_query_batch_device(ids[:B], qb.data_ptr(), rb.data_ptr(), stream.cuda_stream)
            srv2.make_query_batch_device(ids[:B], qb.data_ptr(), rb2.data_ptr(), s2.cuda_stream)
        for _ in range(args.warmup):
            both()
        torch.cuda.synchronize(device)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        s2.wait_event(e0)
        for _ in range(args.steps):
            both()
        e2.record(s2)
        stream.wait_event(e2)
        e1.record(stream)
        torch.cuda.synchronize(device)
        ms = e0.elapsed_time(e1)
        conc = {"batches_in_flight": 2, "batch": B, "steps": args.steps,
                "queries_per_s": 2 * B * args.steps / (ms / 1e3),
                "ms_per_pair": ms / args.steps,
                "same_responses": bool(torch.equal(rb, rb2))}
        srv2.close()

    if rank != 0:
        srv.close()
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    peaks = measured_peaks()
    word = 8 if c4 else 4            # bytes per stored residue (u64 limb / u32 half)
    db_phys = 2 * N * params.num_pt * word
    qmat_bytes = 2 * N * params.fst_dim_sz * 2 * B * word
    cmat_bytes = 2 * N * params.other_dim_sz * 2 * B * word
    alg_bytes = db_phys + qmat_bytes + cmat_bytes
    core_ms = stages["Core"]
    achieved = alg_bytes / (core_ms / 1e3) / 1e9
    traffic = ncu_traffic()
    # logical database bytes: BASELINE's sizing is 13 bits per coefficient
    # for every config; the parameter set's own t gives the second figure
    # (t = 4099: 13 bits; generate_prime(40): 40; generate_prime(10) = 521: 10)
    t_bits = int(params._p.plain_mod - 1).bit_length()
    logical_db = params.num_pt * N * 13 / 8
    logical_db_t = params.num_pt * N * t_bits / 8
    if c4:
        workload = c4_workload_name(params)
    else:
        set_name = {"k1": "k1_comp N=2048", "k2mp": "CONFIG_N2048_K2_MP N=2048 two 29-bit limbs",
                    "k1p": "CONFIG_N2048_K1 N=2048 one 60-bit prime"}[args.workload]
        workload = (f"{set_name}, "
                    f"{args.target} plaintexts ({logical_db / 1e6:.1f} MB at 13 bits, "
                    f"{db_phys} B NTT form), first dim {params.fst_dim_sz} x "
                    f"{params.num_dims - 1} binary dims")
    line = {
        "metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64" if (c4 or args.workload == "k1p") else "u32",
        "data": "synthetic (seeded DB coefficients < t generated on device; seeded uniform "
                "ciphertexts and keys mod q -- the path is data-independent)",
        "config": {"workload": workload,
                   "batch": B, "num_pt": params.num_pt, "fst_dim_sz": params.fst_dim_sz,
                   "num_dims": params.num_dims,
                   "l2": (f"inputs larger than L2: the {db_phys / 2**30:.0f} GiB database streams "
                          "from HBM every step"),
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "db_gbs": logical_db * queries_done / (total_max / 1e3) / 1e9,
        "db_gbs_at_log_t": {"bits": t_bits,
                            "value": logical_db_t * queries_done / (total_max / 1e3) / 1e9},
        "latency_ms": {"p50": float(np.percentile(per, 50)), "p99": float(np.percentile(per, 99))},
        "stages_ms": {k: round(v, 4) for k, v in stages.items() if k != "calls"},
        "plain": {"batch": 1, "value": world * args.steps / (plain_total / 1e3), "unit": "queries/s",
                  "latency_ms": {"p50": float(np.percentile(plain_per, 50)),
                                 "p99": float(np.percentile(plain_per, 99))},
                  "db_gbs": logical_db * world * args.steps / (plain_total / 1e3) / 1e9,
                  "stages_ms": {k: round(v, 4) for k, v in plain_stages.items() if k != "calls"}},
        "e2e": {"value": e2e_qps, "unit": "queries/s", "h2d_bytes_per_step": B * ct_words * 8,
                "d2h_bytes_per_step": B * 2 * N * 8},
        "roofline": {"bound": "hbm",
                     "kernel": ("k4_scan_tc (first-dimension scan, tcgen05)" if (c4 or args.workload == "k1p")
                                else "k_scan_tc (first-dimension scan, tcgen05)"),
                     "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                     "algorithmic_bytes": alg_bytes,
                     # k2mp runs the k1_comp scan kernel on the same byte counts;
                     # the one-prime set's scan has no capture of its own
                     "traffic": (traffic or {}).get(
                         {"k1": "", "k2mp": "", "c4": "c4_", "k1p": "k1p_"}[args.workload]
                         + f"batch_{B}")},
        "int_pipe": int_pipe_roofline(params, config, stages, B, local),
        "batch_sweep": sweep,
        "clocks": clk.summary(),
        **({"concurrent": conc} if conc else {}),
        "gpu_launches": launches,
        "setup": {"db_load_s": round(load_s, 3), "autotune_s": round(tune_s, 3),
                  "scan_tile": srv.scan_tile(B), "scan_tile_plain": srv.scan_tile(1),
                  # cluster width per expansion / MUX level (0: the fixed rule)
                  "level_splits": {str(n): {k: v[:h] for k, v, h in
                                            (("expand", ls["expand"], params.expansion_height),
                                             ("mux", ls["mux"], params.num_dims - 1))}
                                   for n, ls in ((1, srv.level_splits(1)), (B, srv.level_splits(B)))},
                  "gpu": torch.cuda.get_device_name(device)},
    }
    if world == 1 and not args.no_cpu_baseline and c4 and args.target == C4_TARGET:
        try:
            res = run_reference_c4(1, 1, 7)
            line["cpu_baseline"] = {"value": 1000.0 / res["mean_ms"], "unit": "queries/s",
                                    "cores": 1, "kind": "reference", "sample": c4_sample(res, 1)}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": "queries/s", "cores": 0,
                                    "kind": "reference", "sample": f"unavailable: {e}"}
    if world == 1 and not args.no_cpu_baseline and not c4 and args.target == TARGET:
        try:
            res = run_reference(args.cpu_queries, 0, 1, 7, REF_SUFFIX[args.workload])
            line["cpu_baseline"] = {
                "value": 1000.0 / res["mean_ms"], "unit": "queries/s", "cores": 1,
                "kind": "reference",
                "sample": (f"reference make_query (oracle/_ref/{res['binary']}, HEXL stand-in), "
                           f"{res['queries']} queries on the same layout after one untimed "
                           f"load_data ({res['load_s']:.1f} s); CPU {cpu_model()}; "
                           + HEXL_CAVEAT)}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": "queries/s", "cores": 0,
                                    "kind": "reference", "sample": f"unavailable: {e}"}
    print(json.dumps(line))
    srv.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------- serving loop
SERVE_DBS = [  # name, plaintexts, expansion height, share of arrivals, batch limit, parameter
    # set, CUDA stream priority (cheapest queries first: the two-limb batches hold the GPU for
    # tens of ms, so the k1_comp lanes overtake them)
    ("c1_54MB", 16384, 9, 0.6, 32, "CONFIG_N2048_K1_COMP", -2),
    ("c2_872MB", 262144, 10, 0.3, 32, "CONFIG_N2048_K1_COMP", -1),
    ("c4_n4096_1M", 1 << 20, 11, 0.1, 16, C4_CONFIG, 0),
]


def bench_serve(args, world, rank, local):
    """Seeded Poisson arrivals mixed 60/30/10 over three device-resident
    databases, answered by the continuous-batching loop; p50/p99 and queries/s
    per offered rate, and a sample of responses re-checked bit for bit against
    the same query answered alone."""
    import threading

    import torch
    from onionpirv2_b200 import PirParams
    from onionpirv2_b200.serving import ServingEngine

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    eng = ServingEngine(device=local, depth=2)
    n_clients = 16
    inputs = {}
    t0 = time.perf_counter()
    for k, (name, target, h, _share, mb, cfg, prio) in enumerate(SERVE_DBS):
        params = PirParams(target, h, config=cfg)
        eng.add_database(name, params, max_batch=mb, seed=DB_SEED + k, priority=prio)
        queries, keys = synthetic_inputs(params, n_clients, 3000 + 100 * k + rank)
        for j, (bv, gsw) in enumerate(keys):
            eng.register_client(name, j, bv, gsw)
        inputs[name] = queries
    setup_s = time.perf_counter() - t0
    names = [d[0] for d in SERVE_DBS]
    shares = np.array([d[3] for d in SERVE_DBS])
    eng.start()

    def run(rate, duration, seed):
        rng = np.random.default_rng(seed)
        n = max(1, int(rate * duration))
        gaps = rng.exponential(1.0 / rate, n)
        offs = np.cumsum(gaps) - gaps[0]
        which = rng.choice(len(names), n, p=shares)
        cl = rng.integers(0, n_clients, n)
        subs = []

        def submitter():
            ts = time.perf_counter()
            for i in range(n):
                while True:
                    d = offs[i] - (time.perf_counter() - ts)
                    if d <= 0:
                        break
                    time.sleep(d if d > 0.0005 else 0)
                nm = names[which[i]]
                subs.append((nm, int(cl[i]), eng.submit(nm, int(cl[i]), inputs[nm][cl[i]])))

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        eng.drain(timeout=600)
        return subs

    run(200, 0.5, 1)                                   # warm-up
    eng.reset_stats()
    results = []
    last = None
    for r, rate in enumerate(float(x) for x in args.rates.split(",")):
        last = run(rate, args.duration, 10 + r)
        st = eng.stats()
        st["offered_qps"] = rate
        results.append(st)
        eng.reset_stats()
    eng.stop()
    # re-check a sample of the last level's responses against lone queries
    verified = 0
    for nm, c, f in last[:: max(1, len(last) // 24)]:
        alone = eng.dbs[nm].lane.server.make_query(c, inputs[nm][c])
        if not np.array_equal(f.result(), alone):
            raise AssertionError(f"served response differs from the lone query ({nm})")
        verified += 1
    line = {
        "metric": "serving: queries/s and p50/p99 ms under Poisson arrivals", "impl": "ours",
        "unit": "queries/s", "n_gpus": 1, "dtype": "u32 (k1_comp) / u64 (two-limb)",
        "data": "synthetic (seeded DBs generated on device; seeded uniform ciphertexts and keys)",
        "config": {"workload": "three resident databases (k1_comp 2^14 and 2^18, "
                               "CONFIG_N4096_K2_MP 2^20), arrivals mixed "
                               + "/".join(f"{int(100 * x)}" for x in shares),
                   "databases": {nm: {"num_pt": PirParams(t, h, config=cfg).num_pt,
                                      "expansion_height": h, "max_batch": mb, "params": cfg,
                                      "stream_priority": prio}
                                 for nm, t, h, _s, mb, cfg, prio in SERVE_DBS},
                   "depth": eng.depth, "clients_per_db": n_clients,
                   "duration_s_per_rate": args.duration},
        "levels": results,
        "verified_bit_exact": verified,
        "hbm_reserved_bytes": eng.reserved,
        "setup_s": round(setup_s, 2),
    }
    print(json.dumps(line))
    eng.close()


# ---------------------------------------------------------------- tree PIR
TREE_L, TREE_A = 16, 3


def tree_shape(c4: bool):
    """(parameter set name, L, a) of the tree workload."""
    return (C4_CONFIG, 17, 3) if c4 else ("CONFIG_N2048_K1_COMP", TREE_L, TREE_A)


def run_reference_tree(runs: int, c4: bool = False) -> dict:
    """The reference's tree layer (driver mode "tree"): server-side time of
    one tree query (unpack_tree_query + select_level at every level), best of
    the portable and AVX-512 builds, `runs` queries each."""
    best = None
    _, L, a = tree_shape(c4)
    base = "opir_ref_c4" if c4 else "opir_ref"
    for exe in (os.path.join(ROOT, "oracle", "_ref", base),
                os.path.join(ROOT, "oracle", "_ref", base + "_avx512")):
        if not os.path.exists(exe):
            continue
        ms = []
        for k in range(runs):
            import tempfile
            with tempfile.TemporaryDirectory() as tmp:
                out = subprocess.run([exe, "--mode", "tree", "--tree-L", str(L), "--tree-a",
                                      str(a), "--leaf", str(37 + 1000 * k), "--client-seed",
                                      str(61 + k), "--out", tmp],
                                     check=True, capture_output=True, text=True)
            ms.append(json.loads(out.stdout.strip().splitlines()[-1])["server_ms"])
        mean = sum(ms) / len(ms)
        if best is None or mean < best["mean_ms"]:
            best = {"mean_ms": mean, "binary": os.path.basename(exe), "runs": len(ms)}
    if best is None:
        raise FileNotFoundError("oracle/_ref is not built")
    return best


def bench_reference_tree(args, procs):
    """The reference arm of --workload tree: `procs` concurrent driver
    processes, each timing min(steps, 3) tree queries server-side."""
    from concurrent.futures import ThreadPoolExecutor
    runs = max(1, min(args.steps, 3))
    c4 = args.tree_config == "c4"
    cfg_name, L, A = tree_shape(c4)
    try:
        best = run_reference_tree(1, c4)          # picks the faster build
        exe = os.path.join(ROOT, "oracle", "_ref", best["binary"])

        def one(k):
            import tempfile
            ms = []
            for j in range(runs):
                with tempfile.TemporaryDirectory() as tmp:
                    out = subprocess.run([exe, "--mode", "tree", "--tree-L", str(L),
                                          "--tree-a", str(A), "--leaf", str(37 + 97 * (k * runs + j)),
                                          "--client-seed", str(100 + k * runs + j), "--out", tmp],
                                         check=True, capture_output=True, text=True)
                ms.append(json.loads(out.stdout.strip().splitlines()[-1])["server_ms"])
            return ms

        t0 = time.perf_counter()
        with ThreadPoolExecutor(procs) as ex:
            all_ms = [m for ms in ex.map(one, range(procs)) for m in ms]
        wall = time.perf_counter() - t0
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference tree layer: {e}"}))
        return
    mean = sum(all_ms) / len(all_ms)
    qps = procs * 1000.0 / mean
    line = {
        "impl": "reference", "metric": "tree PIR paths/s (unpack + select_level at every level, bit-exact)",
        "value": qps, "unit": "tree queries/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mean, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"tree PIR L={L} a={A} on {cfg_name}", "batch": 1,
                   "parallelism": f"{procs} host processes"},
        "cpu_baseline": {"value": qps, "unit": "tree queries/s", "cores": procs, "kind": "reference",
                         "sample": (f"reference unpack_tree_query + select_level (oracle/_ref/"
                                    f"{best['binary']} --mode tree) in {procs} concurrent processes x "
                                    f"{runs} queries, server-side time per query (wall {wall:.1f} s); "
                                    f"CPU {cpu_model()}")},
        "e2e": {"value": qps, "unit": "tree queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def bench_tree(args, world, rank, local):
    """One tree query = unpack (expansion + selector completion) +
    select_level at all L + 1 levels through the device-resident tree handle
    (opir_tree_query: host query in, the L + 1 selected ciphertexts out, one
    synchronising call), on synthetic uniform ciphertexts and keys (the path
    is data-independent); replicas at N > 1."""
    import torch
    from onionpirv2_b200 import PirParams, PirServer
    from onionpirv2_b200 import tree as T
    from onionpirv2_b200.server import launch_count

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=device)
    c4 = args.tree_config == "c4"
    cfg_name, L, A = tree_shape(c4)
    scheme = PirParams(config=cfg_name)
    tree = T.make_tree_pir_params_for_scheme(L, A, scheme)
    src = lambda level, idx: T.synthetic_tree_node_value(level, idx, scheme.plain_mod)
    t0 = time.perf_counter()
    whole = T.Tree(scheme, tree, [T.pack_tree_level(lv, tree, src) for lv in range(tree.L + 1)],
                   device=local)
    setup_s = time.perf_counter() - t0
    qp = T.tree_query_expansion_params(tree, scheme)
    queries, keys = synthetic_inputs(qp, 1, 4000 + rank)
    whole.set_client_keys(0, *keys[0])
    out = np.zeros((tree.L + 1,) + scheme.ct_shape, dtype=np.uint64)

    def step():
        whole.query(0, queries[0])

    for _ in range(args.warmup):
        step()
    barrier(world, device)
    l0 = launch_count()
    te = time.perf_counter()
    per = []
    for _ in range(args.steps):
        ts = time.perf_counter()
        step()
        per.append((time.perf_counter() - ts) * 1e3)
    total = max_over_ranks(time.perf_counter() - te, world, device)
    launches = launch_count() - l0
    qps = world * args.steps / total
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    line = {
        "metric": "tree PIR paths/s (unpack + select_level at every level, bit-exact)",
        "value": qps, "unit": "tree queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64" if c4 else "u32",
        "data": "synthetic (seeded uniform query and keys mod q; synthetic_tree_node_value tree)",
        "config": {"workload": f"tree PIR L={L} a={A} on {cfg_name}: N0="
                               f"{tree.N0}, b={tree.b}, r={tree.r}, h_q={tree.h_q}, "
                               f"{tree.L + 1} levels", "batch": 1,
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "latency_ms": {"p50": float(np.percentile(per, 50)), "p99": float(np.percentile(per, 99))},
        "e2e": {"value": qps, "unit": "tree queries/s",
                "h2d_bytes_per_step": int(queries[0].nbytes), "d2h_bytes_per_step": int(out.nbytes)},
        "gpu_launches": launches, "setup": {"levels_s": round(setup_s, 3)},
    }
    if world == 1 and not args.no_cpu_baseline:
        try:
            res = run_reference_tree(3, c4)
            line["cpu_baseline"] = {
                "value": 1000.0 / res["mean_ms"], "unit": "tree queries/s", "cores": 1,
                "kind": "reference",
                "sample": (f"reference unpack_tree_query + select_level over all {tree.L + 1} levels "
                           f"(oracle/_ref/{res['binary']} --mode tree, HEXL stand-in), "
                           f"{res['runs']} seeded tree queries; CPU {cpu_model()}")}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": "tree queries/s", "cores": 0,
                                    "kind": "reference", "sample": f"unavailable: {e}"}
    print(json.dumps(line))
    whole.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------- client side
def bench_client(args, world, rank, local):
    """Client-side batch operations of one client (one ternary secret):
    decrypt_mod_q over --client-batch responses per step (the headline value)
    and fast_generate_query over as many queries (reported beside it), on
    seeded synthetic responses, uniform c1 and rounded-Gaussian errors; the
    work is data-independent. Replicas at N > 1."""
    import torch
    from onionpirv2_b200 import PirParams
    from onionpirv2_b200.client import PirClient
    from onionpirv2_b200.server import launch_count

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=device)
    c4 = args.client_config == "c4"
    gp = PirParams(config="CONFIG_N4096_K2_MP") if c4 else PirParams()
    N, n = gp.N, args.client_batch
    rng = np.random.default_rng(1234 + rank)
    secret = rng.integers(-1, 2, N).astype(np.int8)
    nz = int(np.count_nonzero(secret))
    gc = PirClient(gp, secret, device=local)
    sq = int(gp.small_q)
    resp = rng.integers(0, sq, (n, 2, N), dtype=np.uint64)
    mods = gp.get_rns_mods()
    a = np.stack([np.stack([rng.integers(0, int(q), N, dtype=np.uint64) for q in mods])
                  for _ in range(n)])
    e = np.rint(rng.normal(0.0, 3.2, (n, N))).astype(np.int64)
    idx = rng.integers(0, gp.num_pt, n)
    d_resp = torch.from_numpy(resp.view(np.int64)).to(device)
    d_pt = torch.empty((n, N), dtype=torch.int64, device=device)
    d_a = torch.from_numpy(a.view(np.int64)).to(device)
    d_e = torch.from_numpy(e).to(device)
    d_q = torch.empty((n, 2) + a.shape[1:], dtype=torch.int64, device=device)
    h_resp = torch.from_numpy(resp.view(np.int64)).pin_memory()
    h_pt = torch.empty((n, N), dtype=torch.int64).pin_memory()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream(device)
    sp = stream.cuda_stream

    def dec():
        gc.decrypt_device(n, d_resp.data_ptr(), d_pt.data_ptr(), 0, sp)

    def pack():
        gc.generate_queries_device(idx, d_a.data_ptr(), d_e.data_ptr(), d_q.data_ptr(), sp)

    # one client's session keys per keygen step
    h, lks, lkey = gp.expansion_height, gp.l_ks, gp.l_key
    kshape = a.shape[1:]
    d_bva = torch.from_numpy(np.stack([np.stack([rng.integers(0, int(q), N, dtype=np.uint64)
                                                 for q in mods]) for _ in range(h * lks)])
                             .view(np.int64)).to(device)
    d_bve = torch.from_numpy(np.rint(rng.normal(0.0, 3.2, (h * lks, N))).astype(np.int64)).to(device)
    d_ga = torch.from_numpy(np.stack([np.stack([rng.integers(0, int(q), N, dtype=np.uint64)
                                                for q in mods]) for _ in range(2 * lkey)])
                            .view(np.int64)).to(device)
    d_ge = torch.from_numpy(np.rint(rng.normal(0.0, 3.2, (2 * lkey, N))).astype(np.int64)).to(device)
    d_bvk = torch.empty((h * lks, 2) + kshape, dtype=torch.int64, device=device)
    d_gk = torch.empty((2 * lkey, 2) + kshape, dtype=torch.int64, device=device)

    def keygen():
        gc.keygen_device(d_bva.data_ptr(), d_bve.data_ptr(), d_ga.data_ptr(), d_ge.data_ptr(),
                         d_bvk.data_ptr(), d_gk.data_ptr(), sp)

    def timed(fn, steps):
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            fn()
            s1.record(stream)
            s1.synchronize()
            total += s0.elapsed_time(s1) / 1e3
        return total

    for _ in range(args.warmup):
        dec()
        pack()
        keygen()
    torch.cuda.synchronize(device)
    barrier(world, device)
    l0 = launch_count()
    with ClockSampler(local) as clk:
        t_dec = max_over_ranks(timed(dec, args.steps), world, device)
        t_pack = max_over_ranks(timed(pack, args.steps), world, device)
        t_key = max_over_ranks(timed(keygen, args.steps), world, device)

        def e2e_step():
            d_resp.copy_(h_resp, non_blocking=True)
            dec()
            h_pt.copy_(d_pt, non_blocking=True)

        t_e2e = max_over_ranks(timed(e2e_step, args.steps), world, device)
    launches = launch_count() - l0
    torch.cuda.synchronize(device)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    clocks = clk.summary()
    parts = 1 if sq < (1 << 25) else 2
    adds = n * N * nz * parts                  # int32 additions of the ternary product
    ms_dec = t_dec * 1e3 / args.steps
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = clocks.get("sm_mhz") or 1965.0
    tensor_path = (n >= 32 and os.environ.get("OPIR_CLIENT_TC", "1") != "0"
                   and os.environ.get("OPIR_CLIENT_WINDOW", "1") != "0")
    if tensor_path:
        # tcgen05 byte-plane scans: 4 A planes x 4 x planes of N x N per response
        # and scan (one scan mod small_q < 2^29; else two 25-bit halves of c1,
        # each mod two primes: four scans)
        scans = 1 if sq < (1 << 29) else 4
        ops = n * scans * 2 * N * N * 16
        peaks = measured_peaks()
        bf16 = peaks.get("bf16_tflops")
        peak = 2 * bf16 if bf16 else 2 * 1590.0   # int8 dense = 2 x bf16 dense
        achieved = ops / (ms_dec / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TOP/s (int8)",
                "frac": achieved / peak, "traffic": None,
                "work": f"{scans} scan(s) x 2 N^2 x 16 byte-plane products per response "
                        "(one secret plane is nonzero)",
                "peak_kind": ("2 x measured" if bf16 else "2 x fallback")
                             + " dense bf16 (int8 dense is twice bf16 on B200)"}
    else:
        peak = sms * 128 * mhz * 1e6 / 1e9     # G lane-ops/s: 4 x 32 lanes issued per clk per SM
        achieved = adds / (ms_dec / 1e3) / 1e9
        roof = {"bound": "issue", "achieved": achieved, "peak": peak,
                "unit": "G int32 ops/s", "frac": achieved / peak, "traffic": None,
                "work": "N x nonzero secret coefficients x parts additions per response",
                "peak_kind": f"nominal: {sms} SMs x 128 lanes x sampled {mhz:.0f} MHz"}
    line = {
        "metric": "client responses decrypted/s (decrypt_mod_q, bit-exact)",
        "value": world * n * args.steps / t_dec, "unit": "responses/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_dec,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded ternary secret, uniform responses mod small_q, uniform c1, "
                "rounded Gaussian errors)",
        "config": {"workload": f"client batch of {n} on {gp.config}: N={N}, small_q={sq}, "
                               f"{nz} nonzero secret coefficients",
                   "batch": n, "l2": "flushed (256 MiB write) between timed steps",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "pack": {"value": world * n * args.steps / t_pack, "unit": "queries/s",
                 "ms_per_step": t_pack * 1e3 / args.steps},
        "keygen": {"value": world * args.steps / t_key, "unit": "session key sets/s",
                   "ms_per_step": t_key * 1e3 / args.steps,
                   "rows": h * lks + 2 * lkey},
        "e2e": {"value": world * n * args.steps / t_e2e, "unit": "responses/s",
                "h2d_bytes_per_step": int(resp.nbytes), "d2h_bytes_per_step": int(n * N * 8)},
        "roofline": roof,
        "gpu_launches": launches, "clocks": clocks,
    }
    if world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, ROOT)
        from oracle import oracle as O
        op = O.c4_params(gp.target_num_pt, gp.expansion_height) if c4 else \
            O.params(gp.target_num_pt, gp.expansion_height)
        cl = (O.C4Client if c4 else O.Client)(op, 99)
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < 10.0 and done < n:
            cl.decrypt(resp[done])
            done += 1
        el = time.perf_counter() - t0
        line["cpu_baseline"] = {
            "value": done / el, "unit": "responses/s", "cores": 1, "kind": "port",
            "sample": f"oracle decrypt_mod_q (NTT mod small_q, one core) of {done} of the "
                      f"step's responses; CPU {cpu_model()}"}
        t0 = time.perf_counter()
        made = 0
        while time.perf_counter() - t0 < 5.0 and made < 20:
            (O.C4Client if c4 else O.Client)(op, 100 + made)
            made += 1
        line["keygen"]["cpu_port"] = {
            "value": made / (time.perf_counter() - t0), "unit": "session key sets/s", "cores": 1,
            "sample": f"oracle client construction (secret + BV keys + RGSW key), {made} clients"}
    print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------- row shards
def bench_rows(args, world, rank, local):
    """One database split by candidate rows over the job's ranks: per step,
    every rank answers its shard for the same batch (make_query_shard), the
    partials are gathered to rank 0 (NCCL) and rank 0 combines them. value =
    the batch's queries / max-over-ranks step time (strong scaling)."""
    import torch
    from onionpirv2_b200 import PirParams, RowShardServer
    from onionpirv2_b200.server import launch_count

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=device)
    c4 = args.workload == "c4"
    params = (PirParams(args.target, args.height, config=C4_CONFIG) if c4
              else PirParams(args.target, args.height))
    N, B = params.N, args.batch
    ids = list(range(B))
    queries, keys = synthetic_inputs(params, B, 1000)   # the same batch on every rank
    stream = torch.cuda.Stream(device)

    def make_shard(g, G):
        srv = RowShardServer(params, g, G, device=local)
        srv.load_data_seeded(args.target, DB_SEED)
        for b, (bv, gsw) in enumerate(keys):
            srv.set_client_keys(b, bv, gsw)
        if not args.no_autotune:
            srv.autotune(B)
        return srv

    d_q = torch.from_numpy(queries.view(np.int64)).to(device)
    d_part = torch.empty((B,) + params.ct_shape, dtype=torch.int64, device=device)
    d_resp = torch.empty((B, 2, N), dtype=torch.int64, device=device)

    def timed(srv, G, gather, steps, warm):
        parts = torch.empty((G, B) + params.ct_shape, dtype=torch.int64, device=device)

        def step():
            srv.make_query_shard_batch_device(ids, d_q.data_ptr(), d_part.data_ptr(),
                                              stream.cuda_stream)
            with torch.cuda.stream(stream):
                if gather:
                    import torch.distributed as dist
                    dist.gather(d_part, [parts[g] for g in range(G)] if rank == 0 else None, dst=0)
                else:
                    parts[0].copy_(d_part)
            if rank == 0:
                srv.combine_shards_device(ids, parts.data_ptr(), d_resp.data_ptr(),
                                          stream.cuda_stream)

        if not gather:   # one GPU standing in for shard 0: the other slots hold copies
            srv.make_query_shard_batch_device(ids, d_q.data_ptr(), d_part.data_ptr(),
                                              stream.cuda_stream)
            with torch.cuda.stream(stream):
                parts.copy_(d_part.expand((G,) + tuple(d_part.shape)))
        for _ in range(warm):
            step()
        torch.cuda.synchronize(device)
        barrier(world, device)
        torch.cuda.synchronize(device)
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        l0 = launch_count()
        evs[0].record(stream)
        for i in range(steps):
            step()
            evs[i + 1].record(stream)
        torch.cuda.synchronize(device)
        launches = launch_count() - l0
        barrier(world, device)
        per = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
        return evs[0].elapsed_time(evs[-1]), per, launches

    srv = make_shard(rank, world)
    with ClockSampler(local) as clk:
        total, per, launches = timed(srv, world, world > 1, args.steps, args.warmup)
    total_max = max_over_ranks(total, world, device)
    qps = B * args.steps / (total_max / 1e3)

    # end to end: host queries in, host responses out on rank 0
    hq = torch.from_numpy(queries.view(np.int64)).pin_memory()
    hr = torch.empty((B, 2, N), dtype=torch.int64).pin_memory()

    def e2e_step():
        with torch.cuda.stream(stream):
            d_q.copy_(hq, non_blocking=True)
        srv.make_query_shard_batch_device(ids, d_q.data_ptr(), d_part.data_ptr(), stream.cuda_stream)
        parts = e2e_parts
        with torch.cuda.stream(stream):
            if world > 1:
                import torch.distributed as dist
                dist.gather(d_part, [parts[g] for g in range(world)] if rank == 0 else None, dst=0)
            else:
                parts[0].copy_(d_part)
        if rank == 0:
            srv.combine_shards_device(ids, parts.data_ptr(), d_resp.data_ptr(), stream.cuda_stream)
            with torch.cuda.stream(stream):
                hr.copy_(d_resp, non_blocking=True)
        stream.synchronize()

    e2e_parts = torch.empty((world, B) + params.ct_shape, dtype=torch.int64, device=device)
    for _ in range(args.warmup):
        e2e_step()
    barrier(world, device)
    te = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = max_over_ranks(time.perf_counter() - te, world, device)

    projection = []
    if world == 1:   # the per-GPU work of a G-way split, measured on this GPU
        srv.close()
        for G in (2, 4, 8):
            if G > 1 << (params.num_dims - 2):
                break
            one = make_shard(0, G)
            k = max(3, min(args.steps, 20))
            t, _, _ = timed(one, G, False, k, args.warmup)
            projection.append({"shards": G, "rows_per_shard": len(one_rows(params, G)),
                               "per_gpu_ms": t / k,
                               "per_gpu_queries_per_s": B * k / (t / 1e3)})
            one.close()
    if rank != 0:
        srv.close()
        import torch.distributed as dist
        dist.destroy_process_group()
        return
    logical_db = params.num_pt * N * 13 / 8   # BASELINE's 13 bits per coefficient
    line = {
        "metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_max / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "u64" if c4 else "u32",
        "data": "synthetic (seeded DB coefficients < t generated on device; seeded uniform "
                "ciphertexts and keys mod q -- the path is data-independent)",
        "config": {"workload": (c4_workload_name(params) if c4 else
                                f"k1_comp N=2048, {args.target} plaintexts, first dim "
                                f"{params.fst_dim_sz} x {params.num_dims - 1} binary dims"),
                   "batch": B, "parallelism": f"row shards x{world} (gather to rank 0)",
                   "l2": "inputs larger than L2: every shard streams its rows from HBM every step"},
        "db_gbs": logical_db * B * args.steps / (total_max / 1e3) / 1e9,
        "latency_ms": {"p50": float(np.percentile(per, 50)), "p99": float(np.percentile(per, 99))},
        "e2e": {"value": B * args.steps / e2e_s, "unit": "queries/s",
                "h2d_bytes_per_step": B * int(np.prod(params.ct_shape)) * 8,
                "d2h_bytes_per_step": B * 2 * N * 8},
        "clocks": clk.summary(), "gpu_launches": launches,
    }
    if projection:
        line["shard_projection"] = {
            "note": "one shard of a G-way split on this GPU (expansion and selectors replicated, "
                    "1/G of the rows scanned and MUXed) plus the root's combine; the gather is "
                    "not included",
            "runs": projection}
    print(json.dumps(line))
    if world > 1:
        srv.close()
        import torch.distributed as dist
        dist.destroy_process_group()


def one_rows(params, G):
    from onionpirv2_b200 import row_shard_rows
    return row_shard_rows(params, 0, G)[0]


def main():
    args = parse()
    world, rank, local = dist_env()
    if args.rows_sharded and args.impl == "ours":
        bench_rows(args, world, rank, local)
        return
    if args.client and args.impl == "ours":
        bench_client(args, world, rank, local)
        return
    if args.workload == "tree" and args.impl == "ours" and not args.serve:
        bench_tree(args, world, rank, local)
        return
    if args.serve:
        bench_serve(args, world, rank, local)
        return
    if args.impl == "reference":
        bench_reference(args, world, rank)
        return
    bench_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
