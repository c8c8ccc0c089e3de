"""Benchmark of the H*v hot path (HPhi's mltply) on B200.

Workload (N=1): the half-filled 4x4 periodic Hubbard sector (t=1, U=8, Nup=Ndown=8,
dim 165,636,900), real FP64 vectors.  One step = one H*v in HPhi's accumulate form
v0 += H v1.  value = algorithmic bytes / time with B_alg = 3 * dim * 8 (read v1, read
v0, write v0), inputs resident in HBM, CUDA events on the engine's stream.  The
vectors (1.3 GB each) are larger than L2, so no flush is needed between steps.

e2e: the same metric through the reference-facing C-ABI mltply (hphi_mltply) on
HPhi-layout complex128 host vectors in pinned memory, host<->device copies inside the
timed region (B_alg = 3 * dim * 16 for complex vectors).

--impl reference: the reference HPhi's own OpenMP mltply (oracle/_ref/HPhi_ref, built
from the reference sources) on the same sector, timed per call on the host cores.

Multi-GPU (--gpus N under torchrun): the path does not shard for this workload, so
N independent replicas run (one per GPU); value = total bytes / max-over-ranks time.
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
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "H·v GB/s vs HBM roof; solves/s + p99 latency vs plain FP64 GPU at |ΔE|<1e-8"


def workload_model(name: str):
    from hphi_b200 import expert
    if name == "hubbard4x4":
        m = expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 8, 8, lanczos_max=2000)
        return m, "Hubbard 4x4 periodic, t=1, U=8, Nup=Ndown=8 (dim 165,636,900)"
    if name == "chain16":
        return expert.heisenberg(16, expert.chain_bonds(16)), "Heisenberg chain L=16, Sz=0 (dim 12,870)"
    if name == "hubbard3x4":
        m = expert.hubbard(12, expert.square_bonds(3, 4), 1.0, 8.0, 6, 6)
        return m, "Hubbard 3x4 periodic, t=1, U=8, half filling (dim 853,776)"
    raise SystemExit(f"unknown workload {name}")


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return float(json.load(open(p))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profile_traffic(kernel: str, workload: str):
    """DRAM bytes per launch from the committed ncu summary, if one exists."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits", "-lms", "100"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def reference_mltply_times(model, calls: int, threads: int, timeout: float = 3000.0):
    """Per-call wall times of the reference's mltply on this host (oracle/_ref/HPhi_ref)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import run_ref
    if not run_ref.available():
        return None, "oracle/_ref/HPhi_ref not built"
    with tempfile.TemporaryDirectory() as tmp:
        model.lanczos_max = max(2, calls)
        model.write(tmp)
        t0 = time.time()
        run_ref.run(tmp, threads=threads, dump_call=-1, timeout=timeout, extra_env={"HPHI_DUMP_LISTS": "0"})
        wall = time.time() - t0
        p = os.path.join(tmp, "mltply_times.txt")
        if not os.path.exists(p):
            return None, "reference produced no timing"
        return run_ref.read_times(tmp), f"{wall:.1f} s wall"


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    model, desc = workload_model(args.workload)
    dim = {"hubbard4x4": 165636900, "chain16": 12870, "hubbard3x4": 853776}[args.workload]
    threads = os.cpu_count()
    times, note = reference_mltply_times(model, args.warmup + args.steps, threads)
    if times is None:
        print(json.dumps({"impl": "reference", "unavailable": note}))
        return
    t = times[-args.steps:] if len(times) >= args.steps else times
    balg = 3.0 * dim * 16
    value = len(t) * balg / float(np.sum(t)) / 1e9
    out = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus, "steps": len(t),
           "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(t)), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic", "impl": "reference",
           "config": {"workload": args.workload, "desc": desc, "dim": dim,
                      "vector": "complex128 (the reference always uses complex vectors)",
                      "b_alg": "3*dim*16 bytes per mltply"},
           "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "reference",
                            "sample": f"{len(t)} calls of the reference's mltply (OMP_NUM_THREADS={threads}), "
                                      f"whole run {note}"},
           "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hubbard4x4")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
        return

    import torch
    import hphi_b200

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    model, desc = workload_model(args.workload)
    tmp = tempfile.mkdtemp()
    try:
        model.initial_vec_type = 1
        path = model.write(tmp)
        H = hphi_b200.Hamiltonian(path, device=local)
    finally:
        pass
    dim = H.dim
    H_native = bool(H.info.get("native_order"))
    vt = hphi_b200.REAL64
    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    v1 = torch.rand(dim, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    v1 /= torch.linalg.vector_norm(v1)
    v0 = torch.rand(dim, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    coef = torch.tensor([1.0, 1.0], dtype=torch.float64, device="cuda")
    prdct = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(H.stream)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        H.mltply_device_async(v0.data_ptr(), v1.data_ptr(), vt, coef.data_ptr(), prdct.data_ptr())
    H.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        H.mltply_device_async(v0.data_ptr(), v1.data_ptr(), vt, coef.data_ptr(), prdct.data_ptr())
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    t_ms = e0.elapsed_time(e1)
    t_max = t_ms
    if dist:
        tt = torch.tensor([t_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    balg = 3.0 * dim * 8
    value = world * args.steps * balg / (t_max * 1e-3) / 1e9
    per_launch = t_ms / args.steps
    achieved = balg / (per_launch * 1e-3) / 1e9

    # ---- the same H*v on HPhi-ordered device vectors (permutations to / from the native order included)
    hphi_order_ms = None
    if H.info.get("native_order"):
        H.mltply_device(v0.data_ptr(), v1.data_ptr(), vt)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            H.mltply_device(v0.data_ptr(), v1.data_ptr(), vt)
        hphi_order_ms = (time.perf_counter() - t0) / 3 * 1e3

    # ---- e2e through the reference-facing host mltply (complex128, pinned host buffers)
    e2e = None
    hv0 = torch.zeros(2 * (dim + 1), dtype=torch.float64).pin_memory()
    hv1 = torch.zeros(2 * (dim + 1), dtype=torch.float64).pin_memory()
    hv1[2::2] = v1.cpu()
    H.mltply_raw(hv0.data_ptr(), hv1.data_ptr())  # warm-up (allocates the staging buffers)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        H.mltply_raw(hv0.data_ptr(), hv1.data_ptr())
    te = (time.perf_counter() - t0) / args.e2e_steps
    if dist:
        tt = torch.tensor([te], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        te = float(tt.item())
    e2e = {"value": world * 3.0 * dim * 16 / te / 1e9, "unit": "GB/s",
           "h2d_bytes_per_step": 2 * 16 * (dim + 1), "d2h_bytes_per_step": 16 * (dim + 1),
           "steps": args.e2e_steps, "vector": "complex128 HPhi layout (dim+1), pinned host memory",
           "ms_per_step": te * 1e3}
    H.close()
    shutil.rmtree(tmp, ignore_errors=True)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peak, peak_kind = peak_hbm()
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count()
        times, note = reference_mltply_times(workload_model(args.workload)[0], 2, threads)
        if times is not None:
            t = float(np.min(times))
            cpu = {"value": 3.0 * dim * 16 / t / 1e9, "unit": "GB/s", "cores": threads, "kind": "reference",
                   "sample": f"reference mltply on the same sector, complex128, best of {len(times)} calls "
                             f"({t:.2f} s per call), OMP_NUM_THREADS={threads}"}
        else:
            cpu = {"value": None, "unit": "GB/s", "cores": threads, "kind": "reference", "sample": note}
    out = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": args.workload, "desc": desc, "dim": dim, "vector": "real f64",
                      "step": "one v0 += H v1 (mltply)", "b_alg_bytes": balg,
                      "l2": "inputs larger than L2 (1.3 GB vectors), no flush",
                      "parallelism": "replicas" if world > 1 else "single",
                      "vector_order": "native (per-block up x down product order)" if H_native else "HPhi",
                      "hphi_order_ms_per_step": hphi_order_ms},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_kind": peak_kind,
                        "traffic": profile_traffic("hv_hub_pass" if H_native else "hv_general", args.workload),
                        "kernels": "hv_hub_pass<double,0> + hv_hub_pass<double,1> per step" if H_native
                        else "hv_general_kernel per step"},
           "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": 2 * args.steps, "clocks": clocks}
    print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
