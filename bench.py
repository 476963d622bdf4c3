"""Benchmark of ISSL off-target scoring on B200 (one JSON line on rank 0).

Workload (default): 300,000,000 distinct 20-nt sites (95% i.i.d. GC 41%, 5% copies of 10,000
repeat seeds with Poisson(2) substitutions), occurrences min(1+Geometric(0.9),255), indexed with
the 20 x 8-nt slice-8-20 layout; 100,000 guides (half sampled sites with 0-4 planted substitutions,
half random); MIT+CFD with the 'and' rule, threshold 75, max 4 mismatches. Synthetic, seeded,
generated on the device. One step = scoring the whole 100,000-guide set.

  value  guides/s with guides and outputs resident in HBM (issl_score_device), device time from
         CUDA events on the scoring stream, max over ranks
  e2e    guides/s through issl_score with pinned host buffers: ASCII guides copied in and scores,
         codes and counts copied out inside every step
  roofline  the scan kernel (k_scan): bytes it must move per launch / its event-timed duration,
         against the measured HBM copy bandwidth
  cpu_baseline  the CPU restatement of the reference algorithm (oracle/, OpenMP on all host
         cores) on a bounded guide sample of the same index

--impl reference runs the reference's own ISSLScoreOfftargets (compiled from the reference sources
into oracle/_ref) on the same index, written as a .issl file, on all host cores.

Multi-GPU (torchrun): every rank holds a replica of the index and scores its own 100,000 guides
(weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "guides/sec (MIT+CFD, <=4 mm, 300M-site index, 1 B200)"
WORKLOAD = {
    "workload": "issl-score plain: 300M-site slice-8-20 index, 100k guides, MIT+CFD 'and', threshold 75, "
                "max 4 mismatches",
    "n_sites": 300_000_000,
    "slice_config": "slice-8-20",
    "n_queries": 100_000,
    "method": "and",
    "threshold": 75.0,
    "max_dist": 4,
    "repeat_frac": 0.05,
    "repeat_seeds": 10_000,
    "repeat_lambda": 2.0,
    "seed": 1235,
    "l2": "inputs larger than L2 (the 24 GB residual array streamed per step)",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sites", type=int, default=None, help="override the site count (smaller runs)")
    ap.add_argument("--queries", type=int, default=None)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample time")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the default scan tuning (no autotune sweep)")
    ap.add_argument("--form", default="plain",
                    help="plain (default: the headline line), or any of batched, served (the slice-10-37 forms), "
                         "capacity (500M sites, slice-8-28), mapped (lists in host memory) and extract "
                         "(off-target extraction), comma-separated, one JSON line each")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="length of the served-load run")
    ap.add_argument("--no-forms", action="store_true",
                    help="plain line only (without the batched and served sub-objects on the slice-10-37 index)")
    ap.add_argument("--ref-cases", default=None, help="--impl reference --form gpu: cases to run (c0,c1)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="request arrivals per second (Poisson)")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic():
    """Per-launch DRAM bytes of the scan kernel from the committed ncu summary, if present."""
    p = os.path.join(REPO, "profiles", "k_scan_300M_slice-8-20.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_launch_full:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---- replicas (one process per GPU, torchrun): each rank scores its own share of the guides on
# its own copy of the index; the only collectives are the barriers around the timed region and
# the max over ranks of the timings (no collective on the data path)
def rank_share(allq, rank, nq):
    """The guides rank `rank` scores: its own nq-guide slice of the generated set."""
    return np.ascontiguousarray(allq[rank * nq:(rank + 1) * nq])


def max_over_ranks(x, device=None):
    """The largest of every rank's x (all ranks must call it, in the same order)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, nq, steps, seconds):
    """Guides per second over all ranks: every rank scored nq guides per step."""
    return world * nq * steps / seconds


def spec_for(args, world):
    import cracklingplusplus_gpu_b200 as pkg
    n_sites = args.sites or WORKLOAD["n_sites"]
    nq = args.queries or WORKLOAD["n_queries"]
    return pkg.SynthSpec(seed=WORKLOAD["seed"], n_sites=n_sites, slice_config=WORKLOAD["slice_config"],
                         n_queries=nq * world, repeat_frac=WORKLOAD["repeat_frac"],
                         n_repeat_seeds=WORKLOAD["repeat_seeds"], repeat_lambda=WORKLOAD["repeat_lambda"],
                         copied_frac=0.5), n_sites, nq


def cpu_baseline_port(ix, queries, method_id, threshold, target_s, gpu_res=None):
    """The oracle (C restatement of the reference loop, OpenMP on every host core) on a guide
    sample of the same index, exported to host memory in the reference layout."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)
    pen = json.load(open(os.path.join(REPO, "tests", "golden", "penalties.json")))
    pyoracle.set_cfd_tables([float.fromhex(x) for x in pen["cfd_pos"]], [float.fromhex(x) for x in pen["cfd_pam"]])
    sigs, masks, sizes, lists = ix.export()
    oix = pyoracle.Index.from_arrays(sigs, masks, sizes, lists)
    cores = os.cpu_count() or 1
    probe = queries[: max(64, cores * 8)]
    t0 = time.perf_counter()
    oix.score(probe, method_id, threshold, threads=cores)
    dt = time.perf_counter() - t0
    n = int(min(len(queries), max(len(probe), target_s / max(dt / len(probe), 1e-9))))
    sample = queries[:n]
    t0 = time.perf_counter()
    tm, tc, cnt, _ = oix.score(sample, method_id, threshold, threads=cores)
    dt = time.perf_counter() - t0
    parity = None
    if gpu_res is not None:
        ms, cs, codes = pyoracle.finalise(method_id, threshold, tm, tc)
        rel = lambda a, b: float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))) if len(a) else 0.0
        parity = {"sample": n, "codes_equal": bytes(gpu_res.code[:n]) == codes,
                  "counts_equal": bool(np.array_equal(gpu_res.count[:n], cnt)),
                  "max_rel_err_mit": rel(gpu_res.mit[:n], ms), "max_rel_err_cfd": rel(gpu_res.cfd[:n], cs)}
    one = queries[:max(16, n // cores)]  # the same oracle on one core, for about the same time
    t0 = time.perf_counter()
    oix.score(one, method_id, threshold, threads=1)
    dt1 = time.perf_counter() - t0
    del oix, sigs, masks, sizes, lists
    return dict({"value": n / dt, "unit": "guides/s", "cores": cores, "kind": "port",
                 "sample": f"first {n} of the {len(queries)} benchmark guides on the full index ({dt:.1f} s)",
                 "single_core": {"value": len(one) / dt1, "unit": "guides/s", "cores": 1,
                                 "sample": f"the first {len(one)} of those guides ({dt1:.1f} s)"}},
                **host_info()), parity


def run_ours(args):
    import torch
    import cracklingplusplus_gpu_b200 as pkg
    from cracklingplusplus_gpu_b200 import build
    world, rank, local = dist_env()
    build.build()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    spec, n_sites, nq = spec_for(args, world)
    t0 = time.time()
    ix, allq = pkg.Index.synth(spec, device=local)
    gen_s = time.time() - t0
    q = rank_share(allq, rank, nq)
    method_id = pkg.CLI_METHODS[WORKLOAD["method"]]
    thr, md = WORKLOAD["threshold"], WORKLOAD["max_dist"]

    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    d_q = torch.from_numpy(q.view(np.int64)).to(dev)
    d_mit = torch.empty(nq, dtype=torch.float64, device=dev)
    d_cfd = torch.empty(nq, dtype=torch.float64, device=dev)
    d_code = torch.empty(nq, dtype=torch.uint8, device=dev)
    d_cnt = torch.empty(nq, dtype=torch.int64, device=dev)
    d_dist = torch.empty(1, dtype=torch.int64, device=dev)

    def step_device():
        ix.score_device(d_q.data_ptr(), nq, method_id, thr, md, d_mit.data_ptr(), d_cfd.data_ptr(),
                        d_code.data_ptr(), d_cnt.data_ptr(), d_dist.data_ptr(), stream.cuda_stream)

    # ---- scan tuning: swept on this workload's own guides before any timing -----------------
    tuning = None
    if not args.no_tune:
        t, rep = ix.autotune(d_q.data_ptr(), nq, method_id, thr, md)
        tuning = {"chunk": list(t.chunk), "stages": t.stages, "blocks_per_sm": t.blocks_per_sm, "first_wave": t.first_wave,
                  "default_ms": rep.default_ms, "tuned_ms": rep.best_ms, "configs_timed": rep.configs_timed,
                  "class_probes": list(rep.class_probes)}

    # ---- device-resident throughput -------------------------------------------------------
    scan_ms, scan_bytes, launches = [], [], 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:  # sampling starts before the warm-up (also under load)
        for _ in range(args.warmup):
            step_device()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed_device")
        ev0.record(stream)
        for _ in range(args.steps):
            step_device()
            st = ix.last_stats()
            scan_ms.append(st.scan_ms)
            scan_bytes.append(st.scan_bytes)
            launches += st.launches
        ev1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        ms = max_over_ranks(ms, dev)
    ms_per_step = ms / args.steps
    value = whole_job_rate(world, nq, args.steps, ms / 1e3)

    # ---- end to end through the public API with pinned host buffers -------------------------
    from cracklingplusplus_gpu_b200.index import decode
    ascii_np = np.frombuffer(b"".join(decode(s).encode() + b"\n" for s in q), dtype=np.uint8)
    h_in = torch.from_numpy(ascii_np.copy()).pin_memory()
    h_mit = torch.empty(nq, dtype=torch.float64).pin_memory()
    h_cfd = torch.empty(nq, dtype=torch.float64).pin_memory()
    h_code = torch.empty(nq, dtype=torch.uint8).pin_memory()
    h_cnt = torch.empty(nq, dtype=torch.int64).pin_memory()
    import ctypes as C
    L = pkg.lib()
    u64p, f64p = C.POINTER(C.c_uint64), C.POINTER(C.c_double)
    dist_out = (C.c_uint64 * 1)()

    def step_e2e():
        rc = L.issl_score(ix.handle, C.c_char_p(h_in.data_ptr()), 21, nq, method_id, thr, md,
                          C.cast(h_mit.data_ptr(), f64p), C.cast(h_cfd.data_ptr(), f64p),
                          C.c_char_p(h_code.data_ptr()), C.cast(h_cnt.data_ptr(), u64p), dist_out)
        if rc != 0:
            raise RuntimeError(L.issl_last_error())

    for _ in range(args.warmup):
        step_e2e()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.nvtx.range_push("timed_e2e")
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_e2e()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    torch.cuda.nvtx.range_pop()
    if world > 1:
        e2e_s = max_over_ranks(e2e_s, dev)
    e2e_value = whole_job_rate(world, nq, args.steps, e2e_s)

    # results of the last e2e step, for the CPU parity sample
    gpu_res = pkg.ScoreResult(h_mit.numpy().copy(), h_cfd.numpy().copy(), bytes(h_code.numpy()), h_cnt.numpy().view(
        np.uint64).copy(), int(dist_out[0]))

    peak, peak_kind = measured_peaks()
    scan_avg_ms = sum(scan_ms) / len(scan_ms)
    bytes_per_launch = sum(scan_bytes) / len(scan_bytes)
    achieved = bytes_per_launch / (scan_avg_ms / 1e3) / 1e9
    traffic = committed_traffic()
    line = {
        "metric": METRIC, "value": value, "unit": "guides/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32/u64 integer scan, f64 sums", "data": "synthetic (seeded, generated on device)",
        "config": dict(WORKLOAD, n_sites=n_sites, n_queries=nq, parallelism=f"replicas{world}" if world > 1 else "1 GPU"),
        "e2e": {"value": e2e_value, "unit": "guides/s", "h2d_bytes_per_step": int(len(ascii_np)),
                "d2h_bytes_per_step": int(nq * (8 + 8 + 1 + 8) + 8)},
        "roofline": {"bound": "hbm", "kernel": "k_scan", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "bytes_per_launch": bytes_per_launch, "kernel_ms": scan_avg_ms},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "probes_per_s": value * len(__import__("cracklingplusplus_gpu_b200").slice_masks(WORKLOAD["slice_config"])),
        "owned_hits_per_step": int(ix.last_stats().hits),
        "dropped_hits_per_step": int(ix.last_stats().dropped_hits),
        "tuning": tuning,
        "generation_s": gen_s,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu, parity = cpu_baseline_port(ix, q, method_id, thr, args.cpu_seconds, gpu_res)
        line["cpu_baseline"] = cpu
        line["parity_sample"] = parity
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    ix.close()
    if rank == 0 and world == 1 and not args.no_forms:
        # the batched and served forms on their own index (300M sites, slice-10-37), after the
        # plain index is gone: sub-objects of the same line
        line.update(forms_on_slice10_index(args))
    if rank == 0:
        print(json.dumps(line), flush=True)


def host_info():
    """CPU model, host RAM and hardware threads of this machine (for the CPU baseline's record)."""
    model, ram = None, None
    try:
        model = next(ln.split(":", 1)[1].strip() for ln in open("/proc/cpuinfo") if ln.startswith("model name"))
    except (OSError, StopIteration):
        pass
    try:
        kb = next(int(ln.split()[1]) for ln in open("/proc/meminfo") if ln.startswith("MemTotal"))
        ram = round(kb / 1048576, 1)
    except (OSError, StopIteration):
        pass
    return {"cpu_model": model, "host_ram_gib": ram, "host_threads": os.cpu_count()}


def slice_masks_of(name):
    """Slice masks from the pure-data slice_configs module, loaded by path (the reference arm never
    imports the library's package, which would load libissl_b200.so)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "_slice_configs", os.path.join(REPO, "cracklingplusplus_gpu_b200", "slice_configs.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.slice_masks(name)


def seq_of(sig) -> str:
    """2-bit packed 20-mer (base j at bits 2j, A=0 C=1 G=2 T=3) -> text."""
    return "".join("ACGT"[(int(sig) >> (2 * j)) & 3] for j in range(20))


def run_reference_cli(binary, idx, guides, cores, workdir):
    """One run of the reference's ISSLScoreOfftargets on `guides`; returns its 'ISSL scoring time'."""
    qf = os.path.join(workdir, "queries.txt")
    with open(qf, "w") as f:
        f.write("".join(seq_of(s) + "\n" for s in guides))
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    r = subprocess.run([binary, idx, qf, "4", str(WORKLOAD["threshold"]), WORKLOAD["method"], "out.txt"],
                       cwd=workdir, env=env, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference exited {r.returncode}: {r.stderr.strip()[-200:]}")
    return float(re.search(r"ISSL scoring time: ([0-9.eE+-]+) seconds", r.stdout).group(1))


def run_reference(args):
    """The reference's own CPU scorer on the same workload: all host cores, plus one core.

    The index is generated and written by the oracle's host restatement of the library's seeded
    generator (oracle/synth_oracle.c) with the reference builder's layout: no code of the library
    runs in this arm."""
    world, rank, local = dist_env()
    if rank != 0:
        return
    binary = os.path.join(REPO, "oracle", "_ref", "ISSLScoreOfftargets")
    if not os.path.exists(binary):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ISSLScoreOfftargets was not built "
                          "(needs the reference sources at build time)"}))
        return
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)
    import pyoracle
    n_sites = args.sites or WORKLOAD["n_sites"]
    nq = args.queries or WORKLOAD["n_queries"]
    cores = int(os.environ.get("ISSL_REF_THREADS", "0")) or os.cpu_count() or 1  # default: every host core
    workdir = tempfile.mkdtemp(dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        t0 = time.time()
        sites, occ, q = pyoracle.synth(WORKLOAD["seed"], n_sites, nq, repeat_frac=WORKLOAD["repeat_frac"],
                                       n_repeat_seeds=WORKLOAD["repeat_seeds"], repeat_lambda=WORKLOAD["repeat_lambda"],
                                       copied_frac=0.5)
        idx = os.path.join(workdir, "index.issl")
        pyoracle.write_built(idx, sites, occ, np.array(slice_masks_of(WORKLOAD["slice_config"]), np.uint64))
        del sites, occ
        gen_s = time.time() - t0
        # bounded sample: K steps of `per_step` guides scored in one invocation of the reference
        per_step = max(64, int(os.environ.get("ISSL_REF_GUIDES_PER_STEP", "0")) or (200 if n_sites >= 10**8 else 1000))
        sample = q[:per_step * args.steps]
        t = run_reference_cli(binary, idx, sample, cores, workdir)
        # the same reference on one core, on a sample sized for about the same time
        one = q[:max(16, len(sample) // cores)]
        t1 = run_reference_cli(binary, idx, one, 1, workdir)
    except RuntimeError as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return
    finally:
        shutil.rmtree(workdir, ignore_errors=True)
    value = len(sample) / t
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "guides/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 integer scan, f64 sums", "data": "synthetic",
        "config": dict(WORKLOAD, n_sites=n_sites, n_queries=nq, parallelism="host cores"),
        "cpu_baseline": dict({"value": value, "unit": "guides/s", "cores": cores, "kind": "reference",
                              "sample": f"{len(sample)} guides ({per_step} per step) of the benchmark set on the full "
                                        f"index; the reference's own 'ISSL scoring time'",
                              "single_core": {"value": len(one) / t1, "unit": "guides/s", "cores": 1,
                                              "sample": f"the first {len(one)} of those guides, OMP_NUM_THREADS=1"},
                              "build": "g++ -O3 -march=x86-64-v3 -fopenmp (oracle/Makefile)",
                              "index_from": "oracle/synth_oracle.c (host restatement of the seeded generator), "
                                            f"{gen_s:.0f} s"}, **host_info()),
        "e2e": {"value": value, "unit": "guides/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# The reference's own GPU scorer (ISSLScoreOfftargets/main_cuda.cpp + issl_cuda.cu, built unchanged
# for sm_100a into oracle/_ref/issl_cuda_ref) on the small case and on the headline workload.
REF_GPU_CASES = {
    "c0": {"workload": "1M-site slice-4-5 index, 1,000 guides (500 copied with 0-4 substitutions and inserted "
                       "into the site set, 500 random), MIT+CFD 'and', threshold 75",
           "n_sites": 1_000_000, "slice_config": "slice-4-5", "n_queries": 1000, "seed": 1234, "planted": True},
    "c1": {"workload": WORKLOAD["workload"], "n_sites": WORKLOAD["n_sites"], "slice_config": WORKLOAD["slice_config"],
           "n_queries": WORKLOAD["n_queries"], "seed": WORKLOAD["seed"], "planted": False},
}
REF_GPU_STAGES = ["Encode (GPU)", "Distance scan (GPU)", "Dedup (GPU)", "MIT LUT (CPU)", "Score (GPU)"]


def run_reference_gpu(args):
    """One JSON line per case: the reference GPU scorer's own stage timings (its stderr summary;
    scoring time = encode + scan + dedup + MIT LUT + score, index load and output excluded), its
    results against this library's on the same index and guides, and this library's time."""
    world, rank, local = dist_env()
    if rank != 0:
        return
    binary = os.path.join(REPO, "oracle", "_ref", "issl_cuda_ref")
    if not os.path.exists(binary):
        print(json.dumps({"impl": "reference", "form": "gpu", "unavailable": "oracle/_ref/issl_cuda_ref was not "
                          "built (needs the reference sources at build time)"}))
        return
    import torch
    import cracklingplusplus_gpu_b200 as pkg
    from cracklingplusplus_gpu_b200 import build
    from cracklingplusplus_gpu_b200.index import decode
    build.build()
    torch.cuda.set_device(local)
    cases = [c for c in ("c0", "c1") if c in (args.ref_cases or "c0,c1").split(",")]
    for name in cases:
        c = REF_GPU_CASES[name]
        n_sites = args.sites or c["n_sites"]
        nq = args.queries or c["n_queries"]
        spec = pkg.SynthSpec(seed=c["seed"], n_sites=n_sites, slice_config=c["slice_config"], n_queries=nq,
                             planted_into_sites=c["planted"])
        ix, q = pkg.Index.synth(spec, device=local)
        ours = ix.score(q, "and", 75.0, distinct=False)  # warm-up, and the results compared below
        d_q = torch.from_numpy(np.ascontiguousarray(q).view(np.int64)).cuda()
        outs = [torch.empty(nq, dtype=torch.float64, device="cuda") for _ in range(2)] + [
            torch.empty(nq, dtype=torch.uint8, device="cuda"), torch.empty(nq, dtype=torch.int64, device="cuda")]
        ms = []
        for _ in range(5):
            ix.score_device(d_q.data_ptr(), nq, 2, 75.0, 4, *[t.data_ptr() for t in outs])
            ms.append(ix.last_stats().total_ms)
        ours_ms = statistics.median(ms)
        workdir = tempfile.mkdtemp(dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
        try:
            idx = os.path.join(workdir, "index.issl")
            ix.save(idx)
            ix.close()
            qf = os.path.join(workdir, "queries.txt")
            with open(qf, "w") as f:
                f.write("".join(decode(x) + "\n" for x in q))
            r = subprocess.run([binary, idx, qf, "4", "75", "and", "out.txt"], cwd=workdir, capture_output=True,
                               text=True)
            if r.returncode != 0:
                print(json.dumps({"impl": "reference", "form": "gpu", "case": name,
                                  "unavailable": f"reference GPU scorer exited {r.returncode}: "
                                                 f"{r.stderr.strip()[-200:]}"}), flush=True)
                continue
            stage = {k: float(re.search(re.escape(k) + r" time: ([0-9]+) ms", r.stderr).group(1))
                     for k in REF_GPU_STAGES + ["Loading", "Total execution"]}
            # it writes to ".\\results\\gpu_final\\" + name (main_cuda.cpp:352-353): on Linux one file
            # of that literal name in the working directory
            outs_found = [f for f in os.listdir(workdir) if f.endswith("out.txt")]
            rows = [ln.split("\t") for ln in open(os.path.join(workdir, outs_found[0])).read().splitlines()[1:] if ln]
        finally:
            shutil.rmtree(workdir, ignore_errors=True)
        ref_mit = np.array([float(x[1]) for x in rows])
        ref_cfd = np.array([float(x[2]) for x in rows])
        ref_cnt = np.array([int(x[3]) for x in rows], dtype=np.uint64)
        # the reference prints %f: agreement to its 6 decimals
        same = (np.abs(ref_mit - np.round(ours.mit, 6)) <= 1.5e-6) & (np.abs(ref_cfd - np.round(ours.cfd, 6)) <= 1.5e-6) \
            & (ref_cnt == ours.count)
        scoring_ms = sum(stage[k] for k in REF_GPU_STAGES)
        codes = np.frombuffer(ours.code, dtype=np.uint8) == ord("1")
        print(json.dumps({
            "impl": "reference", "form": "gpu", "case": name,
            "metric": "guides/sec, the reference's own GPU scorer (issl_cuda.cu) on 1 B200",
            "value": nq / (scoring_ms / 1e3) if scoring_ms > 0 else None, "unit": "guides/s",
            "higher_is_better": True, "n_gpus": 1, "data": "synthetic (seeded)",
            "config": dict(c, n_sites=n_sites, n_queries=nq),
            "stages_ms": stage, "scoring_ms": scoring_ms,
            # its encode stage also pays for CUDA context creation (its first CUDA call)
            "scoring_ms_without_encode": scoring_ms - stage["Encode (GPU)"],
            "ours": {"value": nq / (ours_ms / 1e3), "device_ms": ours_ms},
            "agreement": {"guides": int(nq), "equal_to_6_decimals": int(same.sum()),
                          "max_abs_mit": float(np.max(np.abs(ref_mit - ours.mit))),
                          "max_abs_cfd": float(np.max(np.abs(ref_cfd - ours.cfd))),
                          "counts_equal": int((ref_cnt == ours.count).sum()),
                          # a guide whose test never fires is visited completely, so its totals
                          # do not depend on the visiting order; differences there would be errors
                          "differ_among_accepted": int((~same & (codes == 1)).sum()),
                          "differ_among_rejected": int((~same & (codes == 0)).sum())},
        }), flush=True)


# ---- batched and served forms (300M-site slice-10-37 index) -----------------------------------
FORMS = {
    "n_sites": 300_000_000,
    "slice_config": "slice-10-37",
    "repeat_frac": 0.05,
    "repeat_seeds": 10_000,
    "repeat_lambda": 2.0,
    "repeat_query_frac": 0.2,
    "seed": 1236,
    "pool": 2_000_000,
}
BATCHED = {"workload": "issl-score batched: 300M-site slice-10-37 index, 256 guide sets of log-uniform size "
                       "10..50,000 (20% repeat-derived guides), MIT+CFD 'and', threshold 75, max 4 mismatches",
           "n_sets": 256, "set_min": 10, "set_max": 50_000, "method": "and", "threshold": 75.0, "max_dist": 4}
SERVED = {"workload": "issl-score served: 300M-site slice-10-37 index, Poisson arrivals, log-normal request sizes "
                      "(median 1,000, sigma 1.5, cap 100,000), methods MIT / CFD / MIT+CFD, thresholds 50/75/90, "
                      "max 4 mismatches, 16 GB device-memory headroom",
          "median": 1000, "sigma": 1.5, "cap": 100_000, "methods": ["mit", "cfd", "and"], "thresholds": [50.0, 75.0, 90.0],
          "headroom_gb": 16, "slots": 3, "max_batch_guides": 131072}


CAPACITY = {"workload": "issl-score capacity: 500M-site slice-8-28 index, 5M guides (90% random, 10% repeat-derived), "
                        "MIT+CFD 'and', threshold 75, max 4 mismatches",
            "n_sites": 500_000_000, "slice_config": "slice-8-28", "n_queries": 5_000_000, "copied_frac": 0.0,
            "repeat_query_frac": 0.1, "seed": 1237, "method": "and", "threshold": 75.0, "max_dist": 4,
            "parity_guides": 50_000}


def reference_parity_streamed(ix, q, res, method_word, thr, n):
    """The reference's own ISSLScoreOfftargets (the build without FMA contraction) scores the first n
    guides on the same index, which is streamed to it through a named pipe: at 500M sites x 28 slices
    the reference's in-memory copy alone takes 116 GB of host memory, so the index never exists as a
    file. Off-target counts must be equal; the reference prints scores with six decimals, so scores
    must agree to that and the accept codes are compared wherever the printed scores decide them."""
    binary = os.path.join(REPO, "oracle", "_ref", "ISSLScoreOfftargets_exact")
    if not os.path.exists(binary):
        return {"skipped": "oracle/_ref/ISSLScoreOfftargets_exact was not built (needs the reference sources)"}
    workdir = tempfile.mkdtemp(dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        fifo = os.path.join(workdir, "index.issl")
        os.mkfifo(fifo)
        sample = q[:n]
        qf = os.path.join(workdir, "queries.txt")
        with open(qf, "w") as f:
            f.write("".join(seq_of(x) + "\n" for x in sample))
        proc = subprocess.Popen([binary, fifo, qf, "4", repr(thr), method_word, "cap_out.txt"], cwd=workdir,
                                stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
        err = []

        def writer():
            try:
                ix.save(fifo)
            except Exception as e:  # the reader went away: reported below
                err.append(str(e))

        t0 = time.time()
        w = threading.Thread(target=writer, daemon=True)
        w.start()
        out, errtxt = proc.communicate()
        if w.is_alive():  # the reference exited without reading: release the writer
            with open(fifo, "rb") as f:
                while f.read(1 << 20):
                    pass
        w.join()
        wall = time.time() - t0
        if proc.returncode != 0 or err:
            return {"skipped": f"reference exited {proc.returncode}: {errtxt.strip()[-200:]} {err}"}
        t_score = float(re.search(r"ISSL scoring time: ([0-9.eE+-]+) seconds", out).group(1))
        rows = [ln.split("\t") for ln in out.splitlines() if ln.count("\t") == 2]
        files = [p for p in os.listdir(workdir) if p.endswith("cap_out.txt")]
        counts = [int(ln.rstrip("\n").split("\t")[3]) for ln in open(os.path.join(workdir, files[0]))
                  if not ln.startswith("#")]
    finally:
        shutil.rmtree(workdir, ignore_errors=True)
    rm = np.array([float(r[1]) for r in rows])
    rc = np.array([float(r[2]) for r in rows])
    ours_code = np.frombuffer(res.code[:n], np.uint8)
    # 'and': rejected when both scores are below the threshold; a printed score within its rounding
    # (5e-7) of the threshold does not decide
    decided = (np.abs(rm - thr) > 1e-6) & (np.abs(rc - thr) > 1e-6)
    ref_code = np.where((rm < thr) & (rc < thr), ord("0"), ord("1")).astype(np.uint8)
    return {
        "sample": len(rows), "reference": "oracle/_ref/ISSLScoreOfftargets_exact, index streamed through a named pipe",
        "counts_equal": bool(np.array_equal(np.array(counts, np.uint64), res.count[:n])),
        "codes_equal": bool(np.array_equal(ours_code[decided], ref_code[decided])),
        "codes_undecided_by_printed_scores": int((~decided).sum()),
        "max_abs_score_diff_vs_printed": float(max(np.max(np.abs(rm - res.mit[:n])), np.max(np.abs(rc - res.cfd[:n])))),
        "cpu_guides_per_s": len(rows) / t_score, "cpu_cores": os.cpu_count(), "wall_s": wall,
    }


def bench_capacity(args, pkg):
    """The largest index: 500M sites x 28 slices, 5M guides in one call (chunked by the library
    if the workspace does not fit), with a CPU parity sample when the host can hold the export."""
    import torch
    n_sites = args.sites or CAPACITY["n_sites"]
    nq = args.queries or CAPACITY["n_queries"]
    spec = pkg.SynthSpec(seed=CAPACITY["seed"], n_sites=n_sites, slice_config=CAPACITY["slice_config"],
                         n_queries=nq, copied_frac=CAPACITY["copied_frac"],
                         repeat_query_frac=CAPACITY["repeat_query_frac"])
    t0 = time.time()
    ix, q = pkg.Index.synth(spec)
    gen_s = time.time() - t0
    info = ix.info()
    log(f"capacity: {n_sites} sites, {info.n_slices} slices, {info.device_bytes / 1e9:.1f} GB resident, "
        f"{info.entry_bytes}-byte entries, generated in {gen_s:.1f} s")
    meth = pkg.CLI_METHODS[CAPACITY["method"]]
    thr, md = CAPACITY["threshold"], CAPACITY["max_dist"]
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.Stream(device=dev)
    d_q = torch.from_numpy(np.ascontiguousarray(q).view(np.int64)).to(dev)
    d_mit = torch.empty(nq, dtype=torch.float64, device=dev)
    d_cfd = torch.empty(nq, dtype=torch.float64, device=dev)
    d_code = torch.empty(nq, dtype=torch.uint8, device=dev)
    d_cnt = torch.empty(nq, dtype=torch.int64, device=dev)
    sample = min(nq, 200_000)
    tuning = None
    if not args.no_tune:
        t, rep = ix.autotune(d_q.data_ptr(), sample, meth, thr, md)
        tuning = {"chunk": list(t.chunk), "stages": t.stages, "blocks_per_sm": t.blocks_per_sm,
                  "first_wave": t.first_wave, "default_ms": rep.default_ms, "tuned_ms": rep.best_ms,
                  "sample_guides": sample}
        ix.trim()

    def step():
        ix.score_device(d_q.data_ptr(), nq, meth, thr, md, d_mit.data_ptr(), d_cfd.data_ptr(), d_code.data_ptr(),
                        d_cnt.data_ptr(), 0, stream.cuda_stream)

    step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(1, min(args.steps, 3))
    with ClockSampler(torch.cuda.current_device()) as clocks:
        torch.cuda.nvtx.range_push("timed_device")
        ev0.record(stream)
        for _ in range(steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = ev0.elapsed_time(ev1) / steps
    st = ix.last_stats()
    log(f"capacity: {ms:.1f} ms per 5M-guide call")
    res = pkg.ScoreResult(d_mit.cpu().numpy(), d_cfd.cpu().numpy(), bytes(d_code.cpu().numpy()),
                          d_cnt.cpu().numpy().view(np.uint64), None)
    parity = None
    if not args.no_cpu:
        ix.trim()  # the index file is written from device memory through staging buffers
        parity = reference_parity_streamed(ix, q, res, CAPACITY["method"], thr, CAPACITY["parity_guides"])
    ix.close()
    return {
        "metric": "guides/sec, capacity run (500M-site slice-8-28 index, 5M guides, 1 B200)",
        "value": nq / (ms / 1e3), "unit": "guides/s", "n_gpus": 1, "steps": steps, "ms_per_step": ms,
        "higher_is_better": True, "dtype": "u32/u64 integer scan, f64 sums",
        "data": "synthetic (seeded, generated on device)",
        "config": dict(CAPACITY, n_sites=n_sites, n_queries=nq, entry_bytes=info.entry_bytes,
                       resident_gb=info.device_bytes / 1e9, generation_s=gen_s),
        "stats": {"scan_ms": st.scan_ms, "scan_bytes": st.scan_bytes, "hits": st.hits, "candidates": st.candidates,
                  "probes": st.probes, "launches": st.launches, "dropped_hits": st.dropped_hits,
                  "pipeline_runs": st.runs},
        "tuning": tuning, "parity_sample": parity, "clocks": clocks.summary(),
    }


MAPPED = {"workload": "issl-score with host-resident lists: the 300M-site slice-8-20 index (plain workload's "
                      "composition) with its list entries and bit-sliced codes in page-locked host memory, "
                      "streamed to the device 4 slices at a time per call; 1M guides per call, MIT+CFD 'and', "
                      "threshold 75, max 4 mismatches",
          "n_sites": 300_000_000, "slice_config": "slice-8-20", "n_queries": 1_000_000, "window_slices": 4,
          "seed": 1239, "method": "and", "threshold": 75.0, "max_dist": 4}


def h2d_copy_gbs(torch, dev, gib=2, reps=5):
    """Pinned host -> device copy rate of this box (the bound of a streamed index)."""
    src = torch.empty(gib << 28, dtype=torch.int32, pin_memory=True)
    dst = torch.empty(gib << 28, dtype=torch.int32, device=dev)
    s = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(s):
        dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    with torch.cuda.stream(s):
        for _ in range(reps):
            dst.copy_(src, non_blocking=True)
    e1.record(s)
    torch.cuda.synchronize()
    return reps * (gib << 30) / (e0.elapsed_time(e1) / 1e3) / 1e9


def bench_mapped(args, pkg):
    """The host-list index (issl_open_mapped / set_list_placement): every call streams the lists
    from page-locked host memory, so the bound is the host link, not HBM. Results must equal the
    resident index's bit for bit."""
    import torch
    n_sites = args.sites or MAPPED["n_sites"]
    nq = args.queries or MAPPED["n_queries"]
    spec = pkg.SynthSpec(seed=MAPPED["seed"], n_sites=n_sites, slice_config=MAPPED["slice_config"], n_queries=nq)
    t0 = time.time()
    ix, q = pkg.Index.synth(spec)
    gen_s = time.time() - t0
    meth = pkg.CLI_METHODS[MAPPED["method"]]
    thr, md = MAPPED["threshold"], MAPPED["max_dist"]
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.Stream(device=dev)
    d_q = torch.from_numpy(np.ascontiguousarray(q).view(np.int64)).to(dev)

    def outputs():
        return (torch.empty(nq, dtype=torch.float64, device=dev), torch.empty(nq, dtype=torch.float64, device=dev),
                torch.empty(nq, dtype=torch.uint8, device=dev), torch.empty(nq, dtype=torch.int64, device=dev))

    def step(o):
        ix.score_device(d_q.data_ptr(), nq, meth, thr, md, o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr(),
                        o[3].data_ptr(), 0, stream.cuda_stream)

    def timed(o, steps):
        step(o)  # warm-up (workspace growth)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step(o)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    steps = max(1, min(args.steps, 3))
    res_out = outputs()
    resident_ms = timed(res_out, steps)
    ix.trim()
    t0 = time.time()
    ix.set_list_placement(MAPPED["window_slices"])
    move_s = time.time() - t0
    info = ix.info()
    log(f"mapped: {info.host_bytes / 1e9:.1f} GB of lists in host memory (moved in {move_s:.1f} s), "
        f"{info.device_bytes / 1e9:.1f} GB left on the device")
    map_out = outputs()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        torch.cuda.nvtx.range_push("timed_mapped")
        mapped_ms = timed(map_out, steps)
        torch.cuda.nvtx.range_pop()
    st = ix.last_stats()
    equal = all(torch.equal(a, b) for a, b in zip(res_out, map_out))
    ix.close()
    del res_out, map_out
    peak = h2d_copy_gbs(torch, dev)
    staged_gbs = st.staged_bytes / (mapped_ms / 1e3) / 1e9
    log(f"mapped: {mapped_ms:.1f} ms per call (resident {resident_ms:.1f} ms), {staged_gbs:.1f} GB/s staged, "
        f"host copy peak {peak:.1f} GB/s")
    return {
        "metric": "guides/sec, host-resident lists (300M-site slice-8-20 index streamed from host memory, 1 B200)",
        "value": nq / (mapped_ms / 1e3), "unit": "guides/s", "n_gpus": 1, "steps": steps, "ms_per_step": mapped_ms,
        "higher_is_better": True, "dtype": "u32/u64 integer scan, f64 sums",
        "data": "synthetic (seeded, generated on device)",
        "config": dict(MAPPED, n_sites=n_sites, n_queries=nq, host_gb=info.host_bytes / 1e9,
                       device_gb=info.device_bytes / 1e9, generation_s=gen_s, move_to_host_s=move_s),
        "resident": {"value": nq / (resident_ms / 1e3), "ms_per_step": resident_ms},
        "results_equal_resident": bool(equal),
        "roofline": {"bound": "host link", "achieved": staged_gbs, "peak": peak, "unit": "GB/s",
                     "frac": staged_gbs / peak, "peak_kind": "measured pinned host-to-device copy in this run",
                     "staged_bytes_per_call": st.staged_bytes},
        "stats": {"scan_ms": st.scan_ms, "hits": st.hits, "candidates": st.candidates, "launches": st.launches},
        "clocks": clocks.summary(),
    }


EXTRACT = {"workload": "extract: 1 Gbp synthetic genome (GC 41%, 5% copies of 2,000 repeat segments of 2 kbp, "
                       "N runs) as 16 FASTA records of 60-nt lines -> every off-target site of both strands, "
                       "sorted; then the same FASTA -> resident slice-8-20 index",
           "genome_bp": 1_000_000_000, "records": 16, "seed": 1238, "slice_config": "slice-8-20"}


def _write_genome(path, n_bp, records, seed):
    rng = np.random.default_rng(seed)
    lut = np.frombuffer(b"ACGT", np.uint8)
    with open(path, "wb") as f:
        per = n_bp // records
        reps = lut[rng.choice(4, (2000, 2000), p=[0.295, 0.205, 0.205, 0.295])]
        for r in range(records):
            g = lut[rng.choice(4, per, p=[0.295, 0.205, 0.205, 0.295])]
            for _ in range(per // 40000):  # 5% of the bases are repeat copies
                a = int(rng.integers(0, per - 2000))
                g[a:a + 2000] = reps[int(rng.integers(0, 2000))]
            for _ in range(per // 1000000):
                a = int(rng.integers(0, per - 5000))
                g[a:a + int(rng.integers(10, 5000))] = ord("N")
            f.write(f">chr{r}\n".encode())
            lines = np.full((per + 59) // 60 * 61, ord("\n"), np.uint8)
            idx = np.arange(per)
            lines[idx + idx // 60] = g
            f.write(lines[: per + (per + 59) // 60].tobytes())


def bench_extract(args, pkg):
    """ExtractOfftargets on the GPU (file to file) and FASTA to resident index, wall clock, with
    the CPU restatement timed on a bounded prefix of the same genome."""
    n_bp = args.sites or EXTRACT["genome_bp"]
    work = tempfile.mkdtemp(dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        fa = os.path.join(work, "genome.fa")
        t0 = time.time()
        _write_genome(fa, n_bp, EXTRACT["records"], EXTRACT["seed"])
        log(f"extract: {n_bp} bp written in {time.time() - t0:.1f} s")
        out = os.path.join(work, "offtargets.txt")
        pkg.extract_offtargets([fa], out)  # warm-up (context, allocations)
        times = []
        for _ in range(max(1, min(args.steps, 3))):
            t0 = time.perf_counter()
            n = pkg.extract_offtargets([fa], out)
            times.append(time.perf_counter() - t0)
        t_ext = min(times)
        masks = np.array(pkg.slice_masks(EXTRACT["slice_config"]), np.uint64)
        t0 = time.perf_counter()
        ix, n2 = pkg.Index.from_sequences([fa], masks)
        t_idx = time.perf_counter() - t0
        info = ix.info()
        ix.close()
        # CPU restatement on a bounded prefix: the first record's first lines
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import extract_oracle
        sample_bp = 4_000_000
        head = os.path.join(work, "head.fa")
        with open(fa, "rb") as f, open(head, "wb") as h:
            h.write(f.read(sample_bp + sample_bp // 60 + 16))
        t0 = time.perf_counter()
        cpu_sites = len(extract_oracle.extract([head]))
        t_cpu = time.perf_counter() - t0
        gpu_head = os.path.join(work, "head_ot.txt")
        pkg.extract_offtargets([head], gpu_head)
        same = open(gpu_head, "rb").read() == extract_oracle.extract_text([head])
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return {
        "metric": "off-target extraction, genome bases per second (FASTA file to sorted site file, 1 B200)",
        "value": n_bp / t_ext, "unit": "bp/s", "n_gpus": 1, "steps": len(times), "higher_is_better": True,
        "sites": n, "sites_per_s": n / t_ext, "seconds": t_ext,
        "fasta_to_index": {"seconds": t_idx, "sites": n2, "distinct_sites": info.n_sites,
                           "resident_gb": info.device_bytes / 1e9},
        "cpu_restatement": {"bp_per_s": sample_bp / t_cpu, "sample_bp": sample_bp, "sites": cpu_sites, "cores": 1,
                            "kind": "port (Python re, the reference's regexes)", "gpu_output_equal": same},
        "data": "synthetic (seeded)", "config": dict(EXTRACT, genome_bp=n_bp),
    }


def run_forms(args, forms):
    import torch
    import cracklingplusplus_gpu_b200 as pkg
    from cracklingplusplus_gpu_b200 import build
    world, rank, local = dist_env()
    if rank != 0:
        return
    build.build()
    torch.cuda.set_device(local)
    if "capacity" in forms:
        print(json.dumps(bench_capacity(args, pkg)), flush=True)
    if "extract" in forms:
        print(json.dumps(bench_extract(args, pkg)), flush=True)
    if "mapped" in forms:
        print(json.dumps(bench_mapped(args, pkg)), flush=True)
    forms = [f for f in forms if f not in ("capacity", "extract", "mapped")]
    if not forms:
        return
    ix, q, base = slice10_index(args, pkg, local)
    if "batched" in forms:
        print(json.dumps(bench_batched(args, pkg, ix, q, base)), flush=True)
        ix.trim()  # the plain calls' workspace is not needed by the server
    if "served" in forms:
        print(json.dumps(bench_served(args, pkg, ix, q, base)), flush=True)
    ix.close()


def slice10_index(args, pkg, local):
    n_sites = args.sites or FORMS["n_sites"]
    pool = args.queries or FORMS["pool"]
    spec = pkg.SynthSpec(seed=FORMS["seed"], n_sites=n_sites, slice_config=FORMS["slice_config"], n_queries=pool,
                         repeat_frac=FORMS["repeat_frac"], n_repeat_seeds=FORMS["repeat_seeds"],
                         repeat_lambda=FORMS["repeat_lambda"], repeat_query_frac=FORMS["repeat_query_frac"])
    t0 = time.time()
    ix, q = pkg.Index.synth(spec, device=local)
    gen_s = time.time() - t0
    base = {"n_sites": n_sites, "slice_config": FORMS["slice_config"], "seed": FORMS["seed"],
            "repeat_query_frac": FORMS["repeat_query_frac"], "generation_s": gen_s}
    log(f"index: {n_sites} sites, {FORMS['slice_config']}, {pool} pool guides, generated in {gen_s:.1f} s")
    return ix, q, base


def forms_on_slice10_index(args):
    """{"batched": ..., "served": ...} on the slice-10-37 index, for the headline line."""
    import torch
    import cracklingplusplus_gpu_b200 as pkg
    ix, q, base = slice10_index(args, pkg, torch.cuda.current_device())
    out = {"batched": bench_batched(args, pkg, ix, q, base)}
    ix.trim()  # the plain calls' workspace is not needed by the server
    out["served"] = bench_served(args, pkg, ix, q, base)
    ix.close()
    return out


def log(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def bench_batched(args, pkg, ix, q, base):
    """256 sets in one graph replay against the plain form (one pipeline per set) on the same guides."""
    import torch
    rng = np.random.default_rng(FORMS["seed"])
    sizes = np.exp(rng.uniform(np.log(BATCHED["set_min"]), np.log(BATCHED["set_max"]), BATCHED["n_sets"])).astype(int)
    while sizes.sum() > len(q):
        sizes = (sizes * 0.9).astype(int) + 1
    n = int(sizes.sum())
    meth = pkg.CLI_METHODS[BATCHED["method"]]
    thr, md = BATCHED["threshold"], BATCHED["max_dist"]
    sets = [(int(k), meth, thr, md) for k in sizes]
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.Stream(device=dev)
    d_q = torch.from_numpy(np.ascontiguousarray(q[:n]).view(np.int64)).to(dev)
    d_mit = torch.empty(n, dtype=torch.float64, device=dev)
    d_cfd = torch.empty(n, dtype=torch.float64, device=dev)
    d_code = torch.empty(n, dtype=torch.uint8, device=dev)
    d_cnt = torch.empty(n, dtype=torch.int64, device=dev)
    tuning = None
    if not args.no_tune:
        t, rep = ix.autotune(d_q.data_ptr(), n, meth, thr, md)
        tuning = {"chunk": list(t.chunk), "stages": t.stages, "blocks_per_sm": t.blocks_per_sm, "first_wave": t.first_wave,
                  "default_ms": rep.default_ms, "tuned_ms": rep.best_ms, "class_probes": list(rep.class_probes)}
    ix.trim()  # the sweep's workspace; the batch context holds its own
    bt = pkg.Batch(ix)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(step, steps, warmup):
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / steps

    def batched():
        bt.score_device(d_q.data_ptr(), n, sets, d_mit.data_ptr(), d_cfd.data_ptr(), d_code.data_ptr(),
                        d_cnt.data_ptr(), stream.cuda_stream)

    offs = np.concatenate([[0], np.cumsum(sizes)])

    def per_set():  # the plain form: one pipeline (one query file) per set
        for i in range(len(sizes)):
            a = int(offs[i])
            ix.score_device(d_q.data_ptr() + 8 * a, int(sizes[i]), meth, thr, md, d_mit.data_ptr() + 8 * a,
                            d_cfd.data_ptr() + 8 * a, d_code.data_ptr() + a, d_cnt.data_ptr() + 8 * a, 0,
                            stream.cuda_stream)

    def one_call():
        ix.score_device(d_q.data_ptr(), n, meth, thr, md, d_mit.data_ptr(), d_cfd.data_ptr(), d_code.data_ptr(),
                        d_cnt.data_ptr(), 0, stream.cuda_stream)

    log(f"batched: {n} guides in {len(sizes)} sets; tuning {tuning}")
    steps = max(3, args.steps // 10)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for _ in range(max(args.warmup, 3)):
            batched()
        torch.cuda.nvtx.range_push("timed_batched")
        ms_batched = timed(batched, steps, 0)
        torch.cuda.nvtx.range_pop()
    st = bt.stats()
    code_b = d_code.cpu().numpy().copy()
    mit_b = d_mit.cpu().numpy().copy()
    log(f"batched: {ms_batched:.2f} ms per replay")
    # end to end: host signatures in, host results out, through issl_batch_score_host
    hq = np.ascontiguousarray(q[:n])
    t0 = time.perf_counter()
    for _ in range(2):
        bt.score(hq, sets)
    e2e_s = (time.perf_counter() - t0) / 2
    bt.close()  # the plain calls below use the index's own workspace
    ms_sets = timed(per_set, max(2, steps // 3), 1)
    equal = bool(np.array_equal(code_b, d_code.cpu().numpy()) and np.array_equal(mit_b, d_mit.cpu().numpy()))
    ms_one = timed(one_call, steps, 2)
    one = ix.last_stats()
    peak, peak_kind = measured_peaks()
    return {
        "metric": "guides/sec, batched form (256 guide sets, one graph replay)", "value": n / (ms_batched / 1e3),
        "unit": "guides/s", "n_gpus": 1, "steps": steps, "ms_per_step": ms_batched, "higher_is_better": True,
        "dtype": "u32/u64 integer scan, f64 sums", "data": "synthetic (seeded, generated on device)",
        "config": dict(BATCHED, **base, n_guides=n),
        "plain_per_set": {"value": n / (ms_sets / 1e3), "ms_per_step": ms_sets,
                          "note": "one issl_score_device pipeline per set, same guides and stream"},
        "plain_one_call": {"value": n / (ms_one / 1e3), "ms_per_step": ms_one,
                           "note": "all guides in one plain call (one parameter set)"},
        "batched_equals_per_set": equal,
        "e2e": {"value": n / e2e_s, "unit": "guides/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 25 * n},
        "gpu_launches_per_step": int(st.launches), "graph_replays_per_step": 1,
        "scan": {"kernel_ms": one.scan_ms, "bytes_per_launch": one.scan_bytes,
                 "achieved_gbs": one.scan_bytes / (one.scan_ms / 1e3) / 1e9 if one.scan_ms else None,
                 "peak": peak, "peak_kind": peak_kind, "class_probes": list(one.class_probes)},
        "owned_hits_per_step": int(st.hits), "tuning": tuning, "clocks": clocks.summary(),
    }


def bench_served(args, pkg, ix, q, base):
    """Open-loop Poisson arrivals against the server; latency from submit to results ready."""
    import queue
    rng = np.random.default_rng(FORMS["seed"] + 1)
    rate, seconds = args.serve_rate, args.serve_seconds
    srv = pkg.Server(ix, n_slots=SERVED["slots"], max_batch_guides=SERVED["max_batch_guides"],
                     headroom_bytes=SERVED["headroom_gb"] << 30)

    def draw():
        k = int(min(SERVED["cap"], max(1, round(rng.lognormal(np.log(SERVED["median"]), SERVED["sigma"])))))
        a = int(rng.integers(0, len(q) - k))
        return (q[a:a + k], SERVED["methods"][rng.integers(3)], SERVED["thresholds"][rng.integers(3)], 4)

    # warm-up: every slot reaches its full capacity (buffers and captured graph) before timing
    w = min(SERVED["max_batch_guides"], len(q))
    warm = [srv.submit(q[:w], "and", 75.0, 4) for _ in range(2 * SERVED["slots"])]
    for t in warm:
        srv.wait(t)
    srv.stats(reset=True)
    log(f"served: warm, {seconds:.0f} s at {rate:.0f} requests/s")
    tickets: "queue.Queue" = queue.Queue()
    replies = []

    def collector():
        while True:
            item = tickets.get()
            if item is None:
                return
            t, k, req = item
            r = srv.wait(t)
            replies.append((k, r.info.latency_ms, r.info.queue_ms, r.info.batch_requests, req, r.result))

    # daemon collectors, stopped in any case: an error in the submission loop must not leave the
    # process waiting for them at exit
    cols = [threading.Thread(target=collector, daemon=True) for _ in range(4)]
    for c in cols:
        c.start()
    start = time.perf_counter()
    next_t = start
    n_req = offered = 0
    sample_reqs = []
    arrivals = []  # (arrival time, request): the same request set for the plain form below
    try:
        while True:
            next_t += rng.exponential(1.0 / rate)
            if next_t - start > seconds:
                break
            delay = next_t - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            req = draw()
            t = srv.submit(*req)
            n_req += 1
            offered += len(req[0])
            arrivals.append((time.perf_counter() - start, req))
            tickets.put((t, len(req[0]), req if len(sample_reqs) < 40 and n_req % 25 == 0 else None))
    finally:
        for _ in cols:
            tickets.put(None)
    for c in cols:
        c.join()
    wall = time.perf_counter() - start
    st = srv.stats()
    srv.close()
    lat = np.array([r[1] for r in replies])
    k = np.array([r[0] for r in replies])
    one_k = lat[(k >= 500) & (k <= 2000)]
    # alone-vs-mixed check on a sample of the served requests
    mixed_ok, checked = True, 0
    for _, _, _, nb, req, res in replies:
        if req is None:
            continue
        alone = ix.score(req[0], req[1], req[2], max_dist=req[3], distinct=False)
        mixed_ok &= alone.code == res.code and np.array_equal(alone.mit, res.mit) and np.array_equal(alone.cfd, res.cfd)
        checked += 1
    # the plain form on the same request set: one query file at a time through issl_score_sigs (host
    # buffers, no batching, no overlap); latency under the same arrivals follows from its service
    # times with a first-come-first-served queue
    service = []
    t_plain = time.perf_counter()
    for _, req in arrivals:
        t1 = time.perf_counter()
        ix.score(req[0], req[1], req[2], max_dist=req[3], distinct=False)
        service.append(time.perf_counter() - t1)
    plain_wall = time.perf_counter() - t_plain
    done, plain_lat = 0.0, []
    for (a, _), sv in zip(arrivals, service):
        done = max(done, a) + sv
        plain_lat.append((done - a) * 1e3)
    plain_lat = np.array(plain_lat)
    plain_k = np.array([len(r[0]) for _, r in arrivals])
    plain_one_k = plain_lat[(plain_k >= 500) & (plain_k <= 2000)]
    return {
        "metric": "served latency p99 (ms), MIT/CFD <=4 mm, 300M-site slice-10-37 index",
        "value": float(np.percentile(lat, 99)), "unit": "ms", "higher_is_better": False, "n_gpus": 1,
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "p99_ms_1k_guide_requests": float(np.percentile(one_k, 99)) if len(one_k) else None,
        "p50_ms_1k_guide_requests": float(np.percentile(one_k, 50)) if len(one_k) else None,
        "requests": int(len(lat)), "throughput_guides_per_s": float(k.sum() / wall),
        "offered_guides_per_s": offered / seconds, "rate_req_per_s": rate, "seconds": seconds,
        "batches": int(st.batches), "mean_batch_guides": st.mean_batch_guides, "peak_in_flight": int(st.peak_in_flight),
        "slots": int(st.slots), "slot_budget_bytes": int(st.slot_budget_bytes), "peak_batch_bytes": int(st.peak_batch_bytes),
        "mixed_equals_alone": {"checked": checked, "equal": bool(mixed_ok)},
        "plain_same_requests": {
            "guides_per_s": float(plain_k.sum() / plain_wall), "service_p50_ms": float(np.percentile(service, 50) * 1e3),
            "service_p99_ms": float(np.percentile(service, 99) * 1e3),
            "queued_p50_ms": float(np.percentile(plain_lat, 50)), "queued_p99_ms": float(np.percentile(plain_lat, 99)),
            "queued_p99_ms_1k_guide_requests": float(np.percentile(plain_one_k, 99)) if len(plain_one_k) else None,
            "note": "one issl_score_sigs call per request, back to back; queued latencies replay the served run's "
                    "arrival times through a single first-come-first-served queue of these service times"},
        "data": "synthetic (seeded, generated on device)", "config": dict(SERVED, **base),
    }


def main():
    args = parse()
    forms = [f.strip() for f in args.form.split(",") if f.strip()]
    if args.impl == "reference":
        if forms == ["gpu"]:
            run_reference_gpu(args)
        else:
            run_reference(args)
    elif forms == ["plain"]:
        run_ours(args)
    else:
        run_forms(args, forms)


if __name__ == "__main__":
    main()
