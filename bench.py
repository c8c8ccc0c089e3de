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

--mode batch | precision | serve print one JSON line each for the other workloads of the
metric (solves/s and latency against the plain FP64 GPU path):
  batch      256 J1-J2 chains (L from {18,20,22,24}, J2 in [0,1], seeded), 300 Lanczos steps
             each through the batched engine, FP64 and FP32 storage (FP64 refinement),
             against the plain single-instance FP64 driver (hphi_lanczos_steps) on the same
             start vectors.
  precision  4x8 periodic Heisenberg, Sz=0 (dim 601,080,390): FP32-storage Lanczos with FP64
             refinement against the plain FP64 GPU driver, |dE| stated.
  serve      Poisson request stream (seeded, mean 50 req/s) of Heisenberg chains L=16..26,
             half-filled Hubbard chains L=10..14 (U in [2,10]) and 24-site Kitaev-Heisenberg
             honeycomb (SpinGC, complex) through the continuous-batching server: solves/s,
             p50/p99 latency, |dE| against each request solved alone by the plain driver.
  tpq        mTPQ on a 26-site J1-J2 chain (dim 10,400,600): NumAve = 8 samples in lockstep with
             one block H*V per step (blocks of at most 2, 4, 8) against the same samples one
             after another, complex and real vectors.
  green      expec_cisajs on the 4x4 Hubbard sector: the 512 spin-conserving one-body rows of a
             normalised random vector (rows x sector rows per second), the reference's
             expec_cisajs timed on 8 of the rows as the CPU baseline.
  tem        real-time evolution (CalcByTEM) on the 4x4 Hubbard sector under a TEOneBody
             Peierls pulse, ExpandCoef 10: time steps per second through the C-ABI, the
             reference's mltply inside its own CalcByTEM as the CPU baseline.

The default line also carries "modes": bounded runs of batch (64 of the 256 chains), serve
(40 requests) and precision (the full 4x8 sector), each in its own process after the timed
H*v (--no-modes skips them).

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
    if name == "hubbard4x4_6e":
        m = expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 6, 6, lanczos_max=2000)
        return m, "Hubbard 4x4 periodic, t=1, U=8, Nup=Ndown=6 (dim 64,128,064; profiling case)"
    if name == "hubbard3x4":
        m = expert.hubbard(12, expert.square_bonds(3, 4), 1.0, 8.0, 6, 6)
        return m, "Hubbard 3x4 periodic, t=1, U=8, half filling (dim 853,776)"
    if name == "heisenberg4x8":
        m = expert.heisenberg(32, expert.square_bonds(4, 8), 1.0)
        return m, "Heisenberg 4x8 periodic, J=1, Sz=0 (dim 601,080,390)"
    if name == "heisenberg4x7":
        m = expert.heisenberg(28, expert.square_bonds(4, 7), 1.0)
        return m, "Heisenberg 4x7 periodic, J=1, Sz=0 (dim 40,116,600; profiling case)"
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
    dim = {"hubbard4x4": 165636900, "chain16": 12870, "hubbard3x4": 853776,
           "hubbard4x4_6e": 64128064, "heisenberg4x8": 601080390, "heisenberg4x7": 40116600}[args.workload]
    threads = os.cpu_count()
    # a bounded sample: one untimed call, then at most 6 timed calls (~8 s each on 16 cores)
    timed = max(1, min(args.steps, 6))
    times, note = reference_mltply_times(model, 1 + timed, threads)
    if times is None:
        print(json.dumps({"impl": "reference", "unavailable": note}))
        return
    t = times[-timed:] if len(times) >= timed else times
    balg = 3.0 * dim * 16
    value = len(t) * balg / float(np.sum(t)) / 1e9
    out = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus, "steps": len(t),
           "warmup": 1, "ms_per_step": 1e3 * float(np.mean(t)), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic", "impl": "reference",
           "config": {"workload": args.workload, "desc": desc, "dim": dim,
                      "vector": "complex128 (the reference always uses complex vectors)",
                      "b_alg": "3*dim*16 bytes per mltply"},
           "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "reference",
                            "sample": f"{len(t)} timed calls of the reference's mltply after 1 untimed call "
                                      f"(OMP_NUM_THREADS={threads}; --steps {args.steps} capped at 6 to bound "
                                      f"the run), whole run {note}"},
           "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def _clock_start():
    try:
        import torch
        idx = torch.cuda.current_device()
    except Exception:
        idx = 0
    c = ClockSampler(idx)
    c.start()
    return c


def j1j2_batch_models(n: int, seed: int = 2024):
    from hphi_b200 import expert
    rng = np.random.default_rng(seed)
    Ls = rng.choice([18, 20, 22, 24], size=n)
    J2 = rng.uniform(0.0, 1.0, size=n)
    return [(int(L), float(j2), expert.j1j2_chain(int(L), 1.0, float(j2))) for L, j2 in zip(Ls, J2)]


def _dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world == 1:
        return None, 0, 1
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return dist, dist.get_rank(), world


def run_batch_mode(args):
    """Batched Lanczos (256 J1-J2 chains, 300 steps) vs the plain FP64 driver.  Under
    torchrun the instances are split across ranks (hphi_b200.shard: no exchange during the
    solves), the time is the max over ranks and the energies are gathered."""
    import hphi_b200
    from hphi_b200 import expert, shard
    dist, rank, world = _dist_init()
    n, steps, seed = args.batch_size, args.batch_steps, 7
    models = j1j2_batch_models(n)
    dims_all = [expert.sector_dim_estimate(m) for _, _, m in models]
    mine = shard.partition(dims_all, world)[rank]
    tmp = tempfile.mkdtemp()
    hams = []
    for i in mine:
        m = models[i][2]
        d = os.path.join(tmp, f"i{i}")
        os.makedirs(d)
        m.initial_vec_type = 1
        hams.append(hphi_b200.Hamiltonian(m.write(d)))
    dims = dims_all
    res = {}
    clocks = _clock_start()
    for prec, name in ((hphi_b200.FP64, "fp64"), (hphi_b200.FP32, "fp32")):
        with hphi_b200.Batch(hams, prec) as b:
            tune = b.tuning()
            b.lanczos(steps, seed=seed, refine=(prec == hphi_b200.FP32))   # warm-up (graphs, allocations)
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            r = b.lanczos(steps, seed=seed, refine=(prec == hphi_b200.FP32))
            wall = shard.max_over_ranks(time.perf_counter() - t0, dist)
        cols = np.stack([r["e_lanczos"], r["e_refined"]], axis=1)
        full = shard.gather(cols, mine, n, dist)
        r = dict(r, e_lanczos=full[:, 0], e_refined=full[:, 1])
        res[name] = dict(r=r, wall=wall, tune=tune)
    # plain FP64 GPU path: each instance alone through the Lanczos driver, same start vector
    # (rank 0's instances; instance j of a batch starts from seed + 1000003 * j)
    nplain = min(len(hams), args.plain_sample)
    e_plain = []
    if rank == 0:
        hams[0].lanczos_steps(steps, seed=seed, nev=1)  # warm-up
        t0 = time.perf_counter()
        for j in range(nplain):
            e_plain.append(hams[j].lanczos_steps(steps, seed=seed + 1000003 * j, nev=1)[0])
        t_plain = time.perf_counter() - t0
    cl = clocks.stop()
    for h in hams:
        h.close()
    shutil.rmtree(tmp, ignore_errors=True)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    e64 = res["fp64"]["r"]["e_lanczos"]
    e32 = res["fp32"]["r"]["e_refined"]
    plain_idx = mine[:nplain]
    plain_rate = nplain / t_plain
    rate64 = n / res["fp64"]["wall"]
    rate32 = n / res["fp32"]["wall"]
    out = {"metric": METRIC, "mode": "batch", "value": rate32, "unit": "solves/s", "n_gpus": world,
           "scaling": "strong" if world > 1 else None,
           "higher_is_better": True, "dtype": "f32 storage, f64 sums/scalars/refinement", "data": "synthetic",
           "config": {"workload": f"{n} J1-J2 chains, L in {{18,20,22,24}}, J2 in [0,1], {steps} Lanczos steps",
                      "sum_dim": int(sum(dims)), "min_dim": int(min(dims)), "max_dim": int(max(dims)),
                      "graph": True, "launch_shape_fp64": res["fp64"]["tune"], "launch_shape_fp32": res["fp32"]["tune"]},
           "fp64_batched_solves_per_s": rate64, "fp32_batched_refined_solves_per_s": rate32,
           "plain_fp64_solves_per_s": plain_rate, "plain_sample": nplain,
           "speedup_fp32_vs_plain": rate32 / plain_rate, "speedup_fp64_batched_vs_plain": rate64 / plain_rate,
           "max_abs_dE_fp32_refined_vs_fp64": float(np.max(np.abs(e32 - e64))),
           "max_abs_dE_fp32_unrefined_vs_fp64": float(np.max(np.abs(res["fp32"]["r"]["e_lanczos"] - e64))),
           "max_abs_dE_batched_fp64_vs_plain": float(np.max(np.abs(np.array(e_plain) - e64[plain_idx]))),
           "fp32_phase_ms": {"forward": res["fp32"]["r"]["forward_ms"], "replay": res["fp32"]["r"]["replay_ms"],
                             "refine": res["fp32"]["r"]["refine_ms"]},
           "fp64_forward_ms": res["fp64"]["r"]["forward_ms"], "clocks": cl}
    print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


def run_precision_mode(args):
    """FP32-storage Lanczos on the 4x8 Heisenberg sector vs the plain FP64 GPU driver."""
    import hphi_b200
    from hphi_b200 import expert
    steps, seed = args.precision_steps, 11
    tmp = tempfile.mkdtemp()
    m = expert.heisenberg(32, expert.square_bonds(4, 8), 1.0)
    m.initial_vec_type = 1
    H = hphi_b200.Hamiltonian(m.write(tmp))
    clocks = _clock_start()
    t0 = time.perf_counter()
    e64 = H.lanczos_steps(steps, seed=seed, nev=1)[0]
    t64 = time.perf_counter() - t0
    with hphi_b200.Batch([H], hphi_b200.FP32) as b:
        t0 = time.perf_counter()
        r = b.lanczos(steps, seed=seed, refine=True)
        t32 = time.perf_counter() - t0
    cl = clocks.stop()
    dim = H.dim
    H.close()
    shutil.rmtree(tmp, ignore_errors=True)
    out = {"metric": METRIC, "mode": "precision", "value": 1.0 / t32, "unit": "solves/s", "n_gpus": 1,
           "higher_is_better": True, "dtype": "f32 storage, f64 sums/scalars/refinement", "data": "synthetic",
           "config": {"workload": "Heisenberg 4x8 periodic, J=1, Sz=0", "dim": dim, "steps": steps},
           "e_fp64_plain": e64, "e_fp32_refined": float(r["e_refined"][0]), "e_fp32_unrefined": float(r["e_lanczos"][0]),
           "abs_dE_refined": abs(float(r["e_refined"][0]) - e64),
           "abs_dE_unrefined": abs(float(r["e_lanczos"][0]) - e64),
           "residual_refined": float(r["residual"][0]), "replay_steps": int(r["replay_steps"][0]),
           "plain_fp64_s": t64, "fp32_s": t32, "speedup_vs_plain": t64 / t32,
           "fp32_phase_ms": {"forward": r["forward_ms"], "replay": r["replay_ms"], "refine": r["refine_ms"]},
           "clocks": cl}
    print(json.dumps(out))


def reference_green_times(model, vec_c128: np.ndarray, threads: int, timeout: float = 3000.0):
    """Wall time of the reference's expec_cisajs (oracle/_ref/HPhi_ref, link-time hook) on
    the vector vec_c128 (HPhi layout), read through CalcByLanczos with InputEigenVec 1."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import run_ref
    if not run_ref.available():
        return None, "oracle/_ref/HPhi_ref not built"
    with tempfile.TemporaryDirectory() as tmp:
        model.calc_eigenvec, model.output_eigenvec = 0, 0
        model.write(tmp)
        txt = open(os.path.join(tmp, "calcmod.def")).read() + "InputEigenVec 1\n"
        open(os.path.join(tmp, "calcmod.def"), "w").write(txt)
        os.makedirs(os.path.join(tmp, "output"))
        with open(os.path.join(tmp, "output", "zvo_eigenvec_0_rank_0.dat"), "wb") as f:
            f.write(np.array([0], dtype=np.int32).tobytes())
            f.write(np.array([vec_c128.size - 1], dtype=np.int64).tobytes())
            f.write(vec_c128.tobytes())
        t0 = time.time()
        run_ref.run(tmp, threads=threads, dump_call=-1, timeout=timeout, extra_env={"HPHI_DUMP_LISTS": "0"})
        wall = time.time() - t0
        p = os.path.join(tmp, "green_times.txt")
        if not os.path.exists(p):
            return None, "reference produced no timing"
        vals = open(p).read().split()
        return float(vals[1]), f"{wall:.1f} s wall"


def run_green_mode(args):
    """One-body Green's functions (expec_cisajs) on the half-filled 4x4 Hubbard sector: all 512
    spin-conserving rows <c+_{i s} c_{j s}> of a normalised random real vector."""
    import torch
    import hphi_b200
    from hphi_b200 import expert
    model, desc = workload_model(args.workload)
    n_elec = model.ncond
    rows = np.array([(i, s_, j, s_) for s_ in (0, 1) for i in range(16) for j in range(16)], dtype=np.int32)
    model.greenone = [tuple(int(x) for x in r) for r in rows]
    tmp = tempfile.mkdtemp()
    H = hphi_b200.Hamiltonian(model.write(tmp))
    dim = H.dim
    gen = torch.Generator(device="cuda").manual_seed(77)
    v = torch.rand(dim, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    v /= torch.linalg.vector_norm(v)
    stream = torch.cuda.ExternalStream(H.stream)
    for _ in range(args.warmup):
        g = H.expec_green_device(v.data_ptr(), hphi_b200.REAL64, rows, 1)
    clocks = _clock_start()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        g = H.expec_green_device(v.data_ptr(), hphi_b200.REAL64, rows, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    cl = clocks.stop()
    t = e0.elapsed_time(e1) / 1e3 / args.steps
    n_rows = len(rows)
    per_pass = 16                                   # real rows evaluated per pass over the sector
    passes = (n_rows + per_pass - 1) // per_pass
    stream_bytes = passes * dim * 16.0              # list_1 + the vector, once per pass
    value = n_rows * dim / t / 1e9
    # checks: densities sum to the electron number, every <n_i s> in [0, 1]
    dens = np.array([g[k] for k in range(n_rows) if rows[k, 0] == rows[k, 2]]).real
    ok = abs(dens.sum() - n_elec) < 1e-9 and dens.min() > -1e-12 and dens.max() < 1 + 1e-12
    # end to end: the reference-facing call on a pinned HPhi-layout complex128 host vector
    vh = torch.zeros(dim + 1, dtype=torch.complex128).pin_memory()
    vh[1:].real.copy_(v.cpu())
    vnp = vh.numpy()
    e2e = None
    if args.e2e_steps > 0:
        H.expec_green(vnp, rows, 1)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            ge = H.expec_green(vnp, rows, 1)
        te = (time.perf_counter() - t0) / args.e2e_steps
        e2e = {"value": n_rows * dim / te / 1e9, "unit": "G row-elements/s", "h2d_bytes_per_step": 16 * (dim + 1),
               "d2h_bytes_per_step": 16 * n_rows, "ms_per_step": 1e3 * te,
               "max_abs_diff_vs_device": float(np.max(np.abs(ge - g)))}
    peak, peak_src = peak_hbm()
    traffic = profile_traffic("green_kernel", args.workload)
    roof = {"bound": "hbm", "achieved": stream_bytes / t / 1e9, "peak": peak, "unit": "GB/s",
            "frac": stream_bytes / t / 1e9 / peak, "traffic": traffic, "peak_source": peak_src,
            "kernel": "green_kernel<double,false> + finalize_partials_kernel<16>, one pass per 16 rows; "
                      "achieved counts 16 bytes per sector row per pass (list_1 and the vector), traffic is "
                      "DRAM bytes per green_kernel launch"}
    cpu = None
    if not args.no_cpu_baseline:
        sample = 8
        mref, _ = workload_model(args.workload)
        mref.greenone = [tuple(int(x) for x in r) for r in rows[:sample]]
        threads = os.cpu_count()
        tr, note = reference_green_times(mref, vnp, threads)
        if tr is not None:
            cpu = {"value": sample * dim / tr / 1e9, "unit": "G row-elements/s", "cores": threads,
                   "kind": "reference", "sample": f"the reference's expec_cisajs on the first {sample} rows "
                                                 f"(OMP_NUM_THREADS={threads}), {tr:.2f} s; whole run {note}"}
        else:
            cpu = {"unavailable": note}
    H.close()
    shutil.rmtree(tmp, ignore_errors=True)
    out = {"metric": METRIC, "mode": "green", "value": value, "unit": "G row-elements/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"{args.workload} expec_cisajs", "desc": desc, "dim": dim, "rows": n_rows,
                      "rows_desc": "c+_{i s} c_{j s}, i, j = 0..15, s = 0, 1",
                      "l2": "vectors and list_1 (1.3 GB each) exceed L2; no flush"},
           "checks_ok": bool(ok), "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
           "gpu_launches": 2 * passes * args.steps, "clocks": cl}
    print(json.dumps(out))


def tem_model(workload: str, nsteps: int, expand: int):
    """The workload's static H plus a Peierls phase pulse on its hoppings as TEOneBody rows:
    t -> t e^{i A(t)} with A(t) = 0.5 sin(4 t), dt = 0.01."""
    import math
    m, desc = workload_model(workload)
    m.calc_type, m.lanczos_max, m.input_eigenvec, m.spectrum_vec = "TimeEvolution", nsteps, 1, "zvo_eigenvec_0"
    m.expand_coef, m.expec_interval = expand, 100000
    hops = [r for r in m.trans if (r[0], r[1]) != (r[2], r[3])]
    m.trans = []
    m.te_onebody = []
    for k in range(nsteps):
        t = 0.01 * k
        a = 0.5 * math.sin(4.0 * t)
        rows = []
        for (i, s1, j, s2, tr, ti) in hops:
            sign = 1.0 if i < j else -1.0
            rows.append((i, s1, j, s2, tr * math.cos(a), sign * tr * math.sin(a)))
        m.te_onebody.append((t, rows))
    return m, desc + "; TEOneBody Peierls pulse A(t) = 0.5 sin(4t), dt = 0.01"


def reference_tem_times(model, vec_c128: np.ndarray, threads: int, timeout: float = 3000.0):
    """Wall times of the reference's mltply calls (oracle/_ref/HPhi_ref, link-time hook) inside
    its CalcByTEM on the same input, started from vec_c128 (HPhi layout)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import run_ref
    if not run_ref.available():
        return None, "oracle/_ref/HPhi_ref not built"
    with tempfile.TemporaryDirectory() as tmp:
        model.write(tmp)
        os.makedirs(os.path.join(tmp, "output"))
        with open(os.path.join(tmp, "output", "zvo_eigenvec_0_rank_0.dat"), "wb") as f:
            f.write(np.array([0], dtype=np.int32).tobytes())
            f.write(np.array([vec_c128.size - 1], dtype=np.int64).tobytes())
            f.write(vec_c128.tobytes())
        t0 = time.time()
        run_ref.run(tmp, threads=threads, dump_call=-1, timeout=timeout, extra_env={"HPHI_DUMP_LISTS": "0"})
        wall = time.time() - t0
        if not os.path.exists(os.path.join(tmp, "mltply_times.txt")):
            return None, "reference produced no timing"
        return run_ref.read_times(tmp), f"{wall:.1f} s wall"


def run_tem_mode(args):
    """Real-time evolution (CalcByTEM) on the workload's sector: K timed steps of the Taylor
    propagator (ExpandCoef 10) under a time-dependent Peierls pulse, through the C-ABI."""
    import hphi_b200
    expand = 10
    W, K = max(args.warmup, 1), args.steps
    tmp = tempfile.mkdtemp()
    times = {}
    e_last = None
    for n in (W, W + K):
        m, desc = tem_model(args.workload, n, expand)
        d = os.path.join(tmp, f"run{n}")
        H = hphi_b200.Hamiltonian(m.write(d))
        dim = H.dim
        if n == W:
            rng = np.random.default_rng(21)
            v = np.zeros(dim + 1, dtype=np.complex128)
            v[1:] = rng.standard_normal(dim)
            v[1:] /= np.linalg.norm(v[1:])
            H.calc_by_tem(v_init=v, output_dir=os.path.join(d, "output"))    # first-call setup
            clocks = _clock_start()
        t0 = time.perf_counter()
        e = H.calc_by_tem(v_init=v, output_dir=os.path.join(d, "output"))
        times[n] = time.perf_counter() - t0
        e_last = e
        H.close()
    cl = clocks.stop()
    t_step = (times[W + K] - times[W]) / K
    hv_bytes = 3.0 * dim * 16
    peak, peak_src = peak_hbm()
    achieved = expand * hv_bytes / t_step / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": None, "peak_source": peak_src,
            "kernel": "one time step = ExpandCoef applications of H(t) (hv_general_kernel<cplx> + te_terms_kernel) "
                      "and the vector updates; achieved counts 3 * dim * 16 bytes per application (the complex "
                      "H*v's algorithmic bytes), not the axpy / norm passes"}
    norm = np.loadtxt(os.path.join(tmp, f"run{W + K}", "output", "Norm.dat"), comments="#")
    cpu = None
    if not args.no_cpu_baseline:
        mref, _ = tem_model(args.workload, 10, 1)    # its progress log divides by Lanczos_max / 10
        threads = os.cpu_count()
        tr, note = reference_tem_times(mref, v, threads)
        if tr is not None:
            tm = float(np.median(tr))
            cpu = {"value": hv_bytes / tm / 1e9, "unit": "GB/s", "cores": threads, "kind": "reference",
                   "sample": f"the reference's CalcByTEM, 10 first-order steps (OMP_NUM_THREADS={threads}): "
                             f"median of its {len(tr)} mltply calls {tm:.2f} s, counted with the same 3*dim*16 "
                             f"bytes; whole run {note}"}
        else:
            cpu = {"unavailable": note}
    shutil.rmtree(tmp, ignore_errors=True)
    out = {"metric": METRIC, "mode": "tem", "value": 1.0 / t_step, "unit": "time steps/s", "n_gpus": 1,
           "steps": K, "warmup": W, "ms_per_step": 1e3 * t_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "c128", "data": "synthetic",
           "config": {"workload": f"{args.workload} time evolution", "desc": desc, "dim": dim,
                      "expand_coef": expand, "timing": "host clock around calc_by_tem with W and W+K steps "
                                                      "(difference / K; each step reads its norm to the host)",
                      "l2": "vectors (2.65 GB each) exceed L2; no flush"},
           "hv_equivalent_gbs": achieved, "norm_before_normalisation_max_dev": float(np.max(np.abs(norm[:, 1] - 1.0))),
           "energy_last": float(e_last[-1]), "roofline": roof, "cpu_baseline": cpu,
           "gpu_launches_per_step": 4 * expand + 8, "clocks": cl}
    print(json.dumps(out))


def run_tpq_mode(args):
    """mTPQ with its NumAve = 8 samples in lockstep (one block H*V over the samples per step,
    hv_block_native; blocks of at most 2, 4 and 8 samples) against the same samples one after
    another, on a 26-site J1-J2 chain (2Sz = 0, dim 10,400,600, the general kernel), with complex
    vectors (the reference's default InitialVecType) and real ones: K timed steps each, host clock
    around calc_by_tpq with W and W + K steps from the same seeded start vectors (difference of the
    medians of three runs / K).
    Every run writes the same files; the last sample's first lines are compared."""
    import hphi_b200
    from hphi_b200 import expert
    W, K = max(args.warmup, 3), max(args.steps // 3, 60)
    L, nave = args.tpq_sites, 8
    bonds = expert.chain_bonds(L) + expert.chain_bonds(L, 2)
    tmp = tempfile.mkdtemp()
    clocks = None
    results = {}
    dim = 0
    for ivt, tname in ((0, "c128"), (1, "f64")):
        per, lines = {}, {}
        starts = None
        for cap in ("0", "2", "4", "8"):
            os.environ["HPHI_B200_TPQ_BLOCK"] = cap
            times = {W: [], W + K: []}
            for n in (W, W + K):
                m = expert.heisenberg(L, bonds, J=[1.0] * L + [0.35] * L, calc_type="TPQ", lanczos_max=n,
                                      num_ave=nave, large_value=2.0, expec_interval=100000, initial_vec_type=ivt)
                d = os.path.join(tmp, f"{tname}_{cap}_{n}")
                with hphi_b200.Hamiltonian(m.write(d)) as H:
                    dim = H.dim
                    if starts is None or starts.shape[1] != dim + 1:
                        # seeded start vectors made once, so the timed calls hold no host RNG
                        rng = np.random.default_rng(26)
                        starts = np.zeros((nave, dim + 1), dtype=np.complex128)
                        starts[:, 1:] = rng.standard_normal((nave, dim))
                        if ivt == 0:
                            starts[:, 1:] += 1j * rng.standard_normal((nave, dim))
                    if clocks is None:
                        H.calc_by_tpq(v_init=list(starts), output_dir=os.path.join(d, "warm"))   # first-call setup
                        clocks = _clock_start()
                    for _ in range(3):  # median of three runs: the step reads scalars to the host
                        t0 = time.perf_counter()
                        H.calc_by_tpq(v_init=list(starts), output_dir=os.path.join(d, "output"))
                        times[n].append(time.perf_counter() - t0)
            per[cap] = (float(np.median(times[W + K])) - float(np.median(times[W]))) / K
            with open(os.path.join(tmp, f"{tname}_{cap}_{W + K}", "output", f"SS_rand{nave - 1}.dat")) as f:
                lines[cap] = f.read().split("\n")[:6]
            for n in (W, W + K):
                shutil.rmtree(os.path.join(tmp, f"{tname}_{cap}_{n}"), ignore_errors=True)
        esz = 16 if ivt == 0 else 8
        results[tname] = {"serial_ms_per_step": 1e3 * per["0"],
                          "block_ms_per_step": {c: 1e3 * per[c] for c in ("2", "4", "8")},
                          "speedup_vs_serial": {c: per["0"] / per[c] for c in ("2", "4", "8")},
                          "hv_equivalent_gbs": {c: nave * 3.0 * dim * esz / per[c] / 1e9 for c in ("0", "2", "4", "8")},
                          "files_equal": all(lines[c] == lines["0"] for c in ("2", "4", "8"))}
    os.environ.pop("HPHI_B200_TPQ_BLOCK", None)
    cl = clocks.stop()
    shutil.rmtree(tmp, ignore_errors=True)
    best = min(results["c128"]["block_ms_per_step"].values())
    out = {"metric": METRIC, "mode": "tpq", "value": nave / (best / 1e3), "unit": "sample-steps/s", "n_gpus": 1,
           "steps": K, "warmup": W, "ms_per_step": best, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "c128", "data": "synthetic",
           "config": {"workload": f"J1-J2 chain L={L} (J2=0.35), 2Sz=0, mTPQ, {nave} samples", "dim": dim,
                      "timing": "host clock around calc_by_tpq with W and W+K steps from the same seeded start "
                                "vectors (difference of the medians of 3 runs / K); each step reads its norms and "
                                "energies to the host and appends the files",
                      "default_block": "8 samples",
                      "l2": f"the {nave} samples' vectors exceed L2; no flush"},
           "complex": results["c128"], "real": results["f64"], "clocks": cl}
    print(json.dumps(out))


def serve_requests(n: int, seed: int = 50):
    from hphi_b200 import expert
    rng = np.random.default_rng(seed)
    kw = dict(lanczos_max=1000, lanczos_eps=12, lanczos_target=1)
    out = []
    for i in range(n):
        kind = int(rng.integers(0, 3))
        if kind == 0:
            L = int(rng.choice([16, 18, 20, 22, 24, 26]))
            out.append((f"heis{L}", expert.heisenberg(L, expert.chain_bonds(L), 1.0, **kw)))
        elif kind == 1:
            L = int(rng.choice([10, 12, 14]))
            U = float(rng.uniform(2.0, 10.0))
            out.append((f"hub{L}", expert.hubbard(L, expert.chain_bonds(L), 1.0, U, L // 2, L // 2, **kw)))
        else:
            J = float(rng.uniform(0.0, 0.3))
            out.append(("kh24", expert.kitaev_heisenberg(3, 4, -1.0, J, initial_vec_type=0, **kw)))
    arrivals = np.cumsum(rng.exponential(1.0 / 50.0, size=n))
    return out, arrivals


def run_serve_mode(args):
    """Continuous-batching server on a Poisson stream vs the plain FP64 driver per request."""
    import hphi_b200
    n = args.serve_requests
    reqs, arr = serve_requests(n)
    tmp = tempfile.mkdtemp()
    paths = []
    for i, (name, m) in enumerate(reqs):
        d = os.path.join(tmp, f"r{i}")
        os.makedirs(d)
        paths.append(m.write(d))
    result = {}
    clocks = _clock_start()
    for prec, pname in ((hphi_b200.FP64, "fp64"), (hphi_b200.FP32, "fp32")):
        srv = hphi_b200.Server(precision=prec, max_active=args.serve_slots, steps_per_iteration=16)
        t0 = srv.clock()
        ids, res, nxt = {}, {}, 0
        while len(res) < n:
            now = srv.clock() - t0
            while nxt < n and arr[nxt] <= now:
                ids[srv.submit(paths[nxt], seed=nxt + 1, arrival=t0 + arr[nxt])] = nxt
                nxt += 1
            c = srv.step()
            for rid, d in srv.poll():
                res[ids[rid]] = d
            if c["active"] == 0 and c["queued"] == 0 and nxt < n:
                time.sleep(max(0.0, arr[nxt] - (srv.clock() - t0)))
        wall = srv.clock() - t0
        srv.close()
        lat = np.array([res[i]["latency_s"] for i in range(n)])
        result[pname] = dict(res=res, wall=wall, lat=lat)
    # plain FP64 GPU path: a sample of the same requests, one at a time, open + Lanczos each
    nplain = min(n, args.plain_sample)
    e_plain, t_plain = [], 0.0
    for i in range(nplain):
        t0 = time.perf_counter()
        with hphi_b200.Hamiltonian(paths[i]) as H:
            r = H.calc_by_lanczos()
        t_plain += time.perf_counter() - t0
        e_plain.append(r["e1"])
    cl = clocks.stop()
    shutil.rmtree(tmp, ignore_errors=True)
    plain_rate = nplain / t_plain
    out = {"metric": METRIC, "mode": "serve", "unit": "solves/s", "n_gpus": 1, "higher_is_better": True,
           "data": "synthetic", "dtype": "f64 (fp64 server) / f32 storage + f64 refinement (fp32 server)",
           "config": {"workload": f"{n} Poisson requests at mean 50/s: Heisenberg chains L=16..26, half-filled "
                                  "Hubbard chains L=10..14 (U in [2,10]), Kitaev-Heisenberg 24-site honeycomb "
                                  "(SpinGC dim 2^24, complex)", "max_active": args.serve_slots,
                      "steps_per_iteration": 16, "convergence": "LanczosEps=12 on E[LanczosTarget=1]"},
           "plain_fp64_solves_per_s": plain_rate, "plain_sample": nplain, "clocks": cl}
    for pname in ("fp64", "fp32"):
        r = result[pname]
        e = np.array([r["res"][i]["energy"] for i in range(nplain)])
        out[pname] = {"solves_per_s": n / r["wall"], "p50_latency_s": float(np.percentile(r["lat"], 50)),
                      "p99_latency_s": float(np.percentile(r["lat"], 99)), "wall_s": r["wall"],
                      "status_codes": sorted({int(r["res"][i]["status"]) for i in range(n)}),
                      "max_abs_dE_vs_plain": float(np.max(np.abs(e - np.array(e_plain)))),
                      "speedup_vs_plain": (n / r["wall"]) / plain_rate}
    out["value"] = out["fp32"]["solves_per_s"]
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", default="hv", choices=["hv", "batch", "precision", "serve", "green", "tem", "tpq"])
    ap.add_argument("--batch-size", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=300)
    ap.add_argument("--precision-steps", type=int, default=300)
    ap.add_argument("--serve-requests", type=int, default=100)
    ap.add_argument("--serve-slots", type=int, default=64)
    ap.add_argument("--plain-sample", type=int, default=256)
    ap.add_argument("--tpq-sites", type=int, default=26, help="--mode tpq: sites of the J1-J2 chain")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=250)  # ~1 s timed: several clock samples
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hubbard4x4")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3, help="0 skips the end-to-end leg")
    ap.add_argument("--no-hphi-order", action="store_true", help="skip the HPhi-order device leg")
    ap.add_argument("--no-modes", action="store_true",
                    help="skip the bounded batch / serve / precision runs reported under 'modes'")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.mode != "hv":
        if args.mode != "batch" and int(os.environ.get("RANK", "0")) != 0:
            return
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        {"batch": run_batch_mode, "precision": run_precision_mode, "serve": run_serve_mode,
         "green": run_green_mode, "tem": run_tem_mode, "tpq": run_tpq_mode}[args.mode](args)
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
    kind = H.info.get("kernel", 0)
    kname, kdesc = {3: ("prod_two_pass", "prod_down_kernel (row pass) + prod_up_warp_kernel (column pass) + "
                                         "finalize_partials_kernel<2> per step; achieved = B_alg / time of all three"),
                    2: ("prod_hv_kernel", "prod_hv_kernel<double> + finalize_partials_kernel<2> per step"),
                    1: ("hv_hub_pass", "hv_hub_pass<double,0> + hv_hub_pass<double,1> + finalize per step"),
                    4: ("spin_rowblock", "spin_row_kernel (row pass) + rb_col_kernel<double,0,4> (column pass) + "
                                         "finalize_partials_kernel<2> per step; achieved = B_alg / time of all three")}.get(
        kind, ("hv_general", "hv_general_kernel + finalize per step"))
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
    if H.info.get("native_order") and not args.no_hphi_order:
        H.mltply_device(v0.data_ptr(), v1.data_ptr(), vt)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            H.mltply_device(v0.data_ptr(), v1.data_ptr(), vt)
        hphi_order_ms = (time.perf_counter() - t0) / 3 * 1e3

    # ---- e2e through the reference-facing host mltply (complex128, pinned host buffers)
    e2e = None
    if args.e2e_steps > 0:
        e2e = run_e2e(H, v1, dim, world, dist, args)
    H.close()
    shutil.rmtree(tmp, ignore_errors=True)
    finish(args, H_native, kind, kname, kdesc, desc, dim, balg, value, t_max, achieved, hphi_order_ms, e2e, clocks,
           world, rank, dist)


def _mode_line(argv, timeout):
    """Runs `bench.py --mode ...` in a fresh process (its own device memory); its JSON line."""
    cmd = [sys.executable, os.path.abspath(__file__)] + argv
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"error": f"timed out after {timeout} s"}
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    if p.returncode != 0 or not lines:
        return {"error": (p.stderr or p.stdout)[-300:]}
    return json.loads(lines[-1])


def run_modes():
    """Bounded runs of the batching, serving, TPQ-block and precision workloads after the timed
    H*v, so the default line carries their solves/s, latency and accuracy: batch with 64 of the
    256 J1-J2 chains (300 steps), serve with 40 Poisson requests, 8 TPQ samples in lockstep
    against one after another, precision on the full 4x8 Heisenberg sector (300 steps).  The
    full-size runs are --mode batch / serve."""
    modes = {}
    b = _mode_line(["--mode", "batch", "--batch-size", "64", "--plain-sample", "16"], 600)
    if "error" in b:
        modes["batch"] = b
    else:
        modes["batch"] = {k: b[k] for k in ("config", "fp64_batched_solves_per_s", "fp32_batched_refined_solves_per_s",
                                            "plain_fp64_solves_per_s", "plain_sample", "speedup_fp32_vs_plain",
                                            "speedup_fp64_batched_vs_plain", "max_abs_dE_fp32_refined_vs_fp64",
                                            "max_abs_dE_batched_fp64_vs_plain", "clocks")}
    sv = _mode_line(["--mode", "serve", "--serve-requests", "40", "--plain-sample", "8"], 900)
    if "error" in sv:
        modes["serve"] = sv
    else:
        modes["serve"] = {k: sv[k] for k in ("config", "fp64", "fp32", "plain_fp64_solves_per_s", "plain_sample",
                                             "clocks")}
    tq = _mode_line(["--mode", "tpq"], 600)
    if "error" in tq:
        modes["tpq"] = tq
    else:
        modes["tpq"] = {k: tq[k] for k in ("config", "value", "unit", "complex", "real", "clocks")}
    pr = _mode_line(["--mode", "precision"], 900)
    if "error" in pr:
        modes["precision"] = pr
    else:
        modes["precision"] = {k: pr[k] for k in ("config", "plain_fp64_s", "fp32_s", "speedup_vs_plain",
                                                 "abs_dE_refined", "abs_dE_unrefined", "e_fp64_plain",
                                                 "fp32_phase_ms", "clocks")}
    return modes


def run_e2e(H, v1, dim, world, dist, args):
    import torch
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
    return {"value": world * 3.0 * dim * 16 / te / 1e9, "unit": "GB/s",
            "h2d_bytes_per_step": 2 * 16 * (dim + 1), "d2h_bytes_per_step": 16 * (dim + 1),
            "steps": args.e2e_steps, "vector": "complex128 HPhi layout (dim+1), pinned host memory",
            "ms_per_step": te * 1e3}


def finish(args, H_native, kind, kname, kdesc, desc, dim, balg, value, t_max, achieved, hphi_order_ms, e2e, clocks,
           world, rank, dist):
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
                      "vector_order": {3: "native (up-rank x down-rank product matrix)",
                                       2: "native (up-rank x down-rank product matrix)",
                                       1: "native (per-block up x down product order)"}.get(kind, "HPhi"),
                      "hphi_order_ms_per_step": hphi_order_ms},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_kind": peak_kind,
                        "traffic": profile_traffic(kname, args.workload),
                        "kernels": kdesc},
           "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": (2 if kind == 2 else 3) * args.steps, "clocks": clocks}
    if world == 1 and not args.no_modes:
        out["modes"] = run_modes()
    print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
