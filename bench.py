"""Benchmark: HS site-slice updates/s of the finite-temperature DQMC sweep.

Workload (the single-chain GPU drop-in configuration): SU(2) Hubbard on the
16 x 16 square lattice (N = 256 sites), U/t = 4, mu = 0, beta = 10,
dtau = 0.05 (ltrot = 200), FFT kinetic propagator, delayed update with
nublock = 32, general 4-component HS field, nwrap = 10 (nst = 20).  A step is
one full sweep (b0 + 0b: 2 * ltrot * N = 102,400 proposals per chain) with
equal-time measurement of every slice, stabilisation and wrap checks.  Each GPU
advances --chains independent chains (the reference's one-chain-per-MPI-rank
parallelism, batched: one CTA per chain, 296 = two per SM by default); the HS fields are drawn from the
reference's -DTEST seeds, one per chain.  The working set (about 52 MiB per
chain) is far larger than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--chains C] [--impl reference]

--impl reference times the reference algorithm on the host CPU cores (the C
restatement in oracle/, with BLAS/LAPACK from scipy's OpenBLAS, one chain per
core) on the same configuration; each step is a bounded sample of 20 slices of
a b0 sweep per core.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIG = dict(lattice=1, l1=16, l2=16, beta=10.0, dtau=0.05, rhub=4.0, nflr=2, mu=0.0,
              kinetic=1, update=1, hs=1, nwrap=10, nublock=32)
WORKLOAD = "square L=16 (N=256) SU(2) Hubbard U=4 beta=10 dtau=0.05 (ltrot=200) FFT kinetic, delay nublock=32, general 4-comp HS, nwrap=10"
METRIC = "HS site-slice updates/s"
# finite-temperature spinless t-V on the honeycomb lattice (the bond field's
# delayed updates; not one of the reference's benchmark configurations):
# L = 12 (N = 288), V = 1, beta = 4, dtau = 0.1, checkerboard, nublock = 32, 64 chains
CONFIG_TV = dict(lattice=2, l1=12, l2=12, beta=4.0, dtau=0.1, rv=1.0, nflr=1, kinetic=0, update=1, nwrap=10,
                 nublock=32)
WORKLOAD_TV = "honeycomb L=12 (N=288) spinless t-V V=1 beta=4 dtau=0.1 (ltrot=40), finite temperature, delayed bond updates nublock=32"
# batched configuration: SU(4) Hubbard, honeycomb L = 6/9/12 (N = 72/162/288,
# 48/48/32 chains), U = 6, beta = 8, dtau = 0.1, exact 4-component HS,
# submatrix update with the flush depth autotuned over {16, 32, 64}
CONFIG3 = [(dict(lattice=2, l1=L, l2=L, beta=8.0, dtau=0.1, rhub=6.0, nflr=4, kinetic=0, update=2, hs=0,
                 nwrap=10, nublock=32), n) for L, n in ((6, 48), (9, 48), (12, 32))]
WORKLOAD3 = "honeycomb L=6/9/12 (N=72/162/288, 48/48/32 chains) SU(4) Hubbard U=6 beta=8 dtau=0.1 (ltrot=80), exact HS, submatrix, autotuned flush depth"
# projective t-V: spinless honeycomb L=12 (N=288, ne=144), V/t=1, projection
# length 20, dtau=0.1 (ltrot=200, nwrap=10, nst=20), submatrix-LR with
# nustock=32, trial state = H0 eigenvectors with the reference's rndness=1e-3
# random hopping perturbation lifting the Dirac-point degeneracy; 64 walkers
CONFIG4 = dict(lattice=2, l1=12, l2=12, beta=20.0, dtau=0.1, rv=1.0, rhub=0.0, nflr=1, kinetic=0, update=2,
               nwrap=10, nublock=32, proj=1, rndness=1e-3)
# learned proposal: SU(2) Hubbard square L=20 (N=400), U=6, mu=0, beta=12,
# dtau=0.1 (ltrot=120), delay update (the plain base), exact two-valued HS
# field (the block flip needs lcomp = 2), checkerboard kinetic term, 64 chains
CONFIG5 = dict(lattice=1, l1=20, l2=20, beta=12.0, dtau=0.1, rhub=6.0, nflr=2, mu=0.0, kinetic=0, update=1, hs=0,
               nwrap=10)
WORKLOAD5 = "square L=20 (N=400) SU(2) Hubbard U=6 beta=12 dtau=0.1 (ltrot=120), delay, exact 2-comp HS, 64 chains; learned 8x4x4 block proposals vs plain"
WORKLOAD4 = "projective spinless t-V, honeycomb L=12 (N=288, ne=144) V=1 theta=20 dtau=0.1 (ltrot=200), submatrix-LR nustock=32, rndness=1e-3 trial, 64 walkers"


def test_seed(irank: int) -> int:
    v = ((irank * 1981 + 2008) * 951049) & 0xFFFFFFFF
    if v >= 1 << 31:
        v -= 1 << 32
    return abs(v)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[3 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------ CPU arm
def cpu_sample(nslices: int, threads: int, steps: int = 1, warmup: int = 0):
    """Time the oracle (reference restatement, OpenBLAS) on `threads` cores:
    each core runs its own chain of the benchmark configuration for `nslices`
    slices of a b0 sweep (updates, measurement, stabilisation) per step."""
    from threadpoolctl import threadpool_limits

    from oracle import pyoracle
    pyoracle.build()
    pyoracle.use_scipy_lapack(True)
    model = pyoracle.Model(**CONFIG)
    chains = [pyoracle.Chain(model, test_seed(c)) for c in range(threads)]

    def run(fn):
        ts = [threading.Thread(target=fn, args=(c,)) for c in chains]
        t0 = time.perf_counter()
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        return time.perf_counter() - t0

    with threadpool_limits(1):
        run(lambda c: c.sweep_start())
        for _ in range(warmup):
            run(lambda c: c.sweep_b0_slices(nslices))
        times = [run(lambda c: c.sweep_b0_slices(nslices)) for _ in range(steps)]
    per_step = threads * nslices * model.ndim
    return per_step, times, model


def cpu_sample_proj(nslices: int, threads: int, steps: int = 1, warmup: int = 0):
    """The projective workload on the oracle (submatrix-LR bond update, as the
    reference's -DSUBMATRIX build): one walker per core, nslices slices of a
    b0 projective sweep per step."""
    from threadpoolctl import threadpool_limits

    from oracle import pyoracle
    pyoracle.build()
    pyoracle.use_scipy_lapack(True)
    model = pyoracle.Model(**CONFIG4)
    chains = [pyoracle.Chain(model, test_seed(c)) for c in range(threads)]

    def run(fn):
        ts = [threading.Thread(target=fn, args=(c,)) for c in chains]
        t0 = time.perf_counter()
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        return time.perf_counter() - t0

    with threadpool_limits(1):
        run(lambda c: c.proj_sweep_start())
        for _ in range(warmup):
            run(lambda c: c.proj_sweep_b0_slices(nslices))
        times = [run(lambda c: c.proj_sweep_b0_slices(nslices)) for _ in range(steps)]
    per_step = threads * nslices * model.nn_nf * model.nn_lf
    return per_step, times, model


def reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if args.workload == "config4":
        nsl = 4
        per_step, times, model = cpu_sample_proj(nsl, threads, steps=args.steps, warmup=min(args.warmup, 1))
        workload = WORKLOAD4
        sample = f"{nsl} slices of a b0 projective sweep per walker per step, {threads} walkers on {threads} cores"
    else:
        nsl = 20
        per_step, times, model = cpu_sample(nsl, threads, steps=args.steps, warmup=args.warmup)
        workload = WORKLOAD
        sample = f"{nsl} slices of a b0 sweep per chain per step, {threads} chains on {threads} cores (one per core)"
    tot = sum(times)
    value = per_step * len(times) / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (HS field drawn from the reference's -DTEST seeds)",
        "config": {"workload": workload, "chains": threads, "threads": threads,
                   "implementation": "C restatement of the Fortran reference (oracle/), OpenBLAS single-threaded per chain"},
        "cpu_baseline": {"value": value, "unit": "updates/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm
def fp64_peak_tflops() -> float:
    """Measured FP64 tensor throughput: cuBLAS DGEMM 8192^3 via torch (best of 5)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(); torch.matmul(a, b); e1.record(); e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def sweep_roofline(prof: dict, work: dict, names: dict, fp64: float) -> dict:
    """Roofline of the kernel with the largest share of an event-timed sweep
    (dqmc_gpu_sweep_profile: an event after every launch group), with every
    kind's per-launch time, share and fraction of its peak."""
    hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs", 6650.0) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 6650.0
    total = sum(v[0] for v in prof.values())
    kinds = {}
    for k, (ms, n) in prof.items():
        if n == 0:
            continue
        per = ms / n
        ent = {"kernel": names.get(k, k), "ms_per_launch": per, "launches": n, "sweep_share": ms / total}
        fl, by = work.get(k, (None, None))
        if fl is not None:
            ach = fl / (per * 1e-3) / 1e12
            # FFT passes run on the FP64 FMA pipe; DMMA and DFMA share one FP64
            # datapath on B200, so both are set against the same measured peak
            ent.update({"bound": "fp64" if k == "bprod" else "tensor", "achieved": ach, "peak": fp64,
                        "unit": "TFLOP/s", "frac": ach / fp64, "algorithmic_flops_per_launch": fl})
        elif by is not None:
            ach = by / (per * 1e-3) / 1e9
            ent.update({"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                        "algorithmic_bytes_per_launch": by})
        kinds[k] = ent
    dom = max((k for k in kinds if "frac" in kinds[k]), key=lambda k: kinds[k]["sweep_share"])
    d = kinds[dom]
    roof = {"kernel": d["kernel"], "bound": d["bound"], "achieved": d["achieved"], "peak": d["peak"],
            "unit": d["unit"], "frac": d["frac"], "traffic": None,
            "peak_source": ("measured in this run: cuBLAS DGEMM 8192^3 (FP64 tensor)" if d["bound"] == "tensor"
                            else "MEASURED_PEAKS.json hbm_gbs"),
            "timing": "one extra sweep launched kernel by kernel with a CUDA event after each launch group",
            "kinds": kinds}
    if "update" in kinds and "frac" in kinds["update"]:
        roof["update_gemm"] = {k: kinds["update"][k] for k in ("kernel", "achieved", "peak", "unit", "frac")}
        roof["update_gemm"]["note"] = ("flush GEMM flops (8 N^2 per accepted site) over the whole update "
                                       "kernel time, sequential accept walk included")
    return roof


def make_handle(args, rank: int):
    """The DQMC handle of the selected workload, chains seeded from the
    reference's -DTEST seeds offset by rank; returns (handle, workload, tuning).
    With --streams S > 1 the chains are split over S handles whose sweeps run
    concurrently on their own streams."""
    import sunhubbardmy_b200 as sb
    from sunhubbardmy_b200.autotune import ChainGroup
    if args.workload == "config4":
        p4 = sb.DqmcParams.make(**CONFIG4)
        nw = args.chains if args.chains_set else 64
        S = args.streams if args.streams else 8
        if S > 1 and nw % S == 0:
            k = nw // S
            seeds = [test_seed(rank * nw + c) for c in range(nw)]
            hs = [sb.Dqmc(p4, n_chains=k, seeds=seeds[j * k:(j + 1) * k]) for j in range(S)]
            return ChainGroup(hs, [p4] * nw, seeds), WORKLOAD4 + f", {S} concurrent handles of {k} walkers", None
        return sb.Dqmc(p4, n_chains=nw, seeds=[test_seed(rank * nw + c) for c in range(nw)]), WORKLOAD4, None
    if args.workload == "tvft":
        ptv = sb.DqmcParams.make(**CONFIG_TV)
        nw = args.chains if args.chains_set else 64
        return sb.Dqmc(ptv, n_chains=nw, seeds=[test_seed(rank * nw + c) for c in range(nw)]), WORKLOAD_TV, None
    if args.workload == "config3":
        from sunhubbardmy_b200.autotune import batched, size_classes
        groups = [(sb.DqmcParams.make(**kw), n) for kw, n in CONFIG3]
        seed0 = rank * sum(n for _, n in CONFIG3)
        if args.streams == 1:
            g, tune_report = batched(groups, tune=True, seed0=seed0)
            return g, WORKLOAD3 + ", one handle", tune_report
        g, tune_report = size_classes(groups, tune=True, seed0=seed0, split=args.streams)
        return g, WORKLOAD3 + f", size classes on {len(g.handles)} concurrent streams", tune_report
    p0 = sb.DqmcParams.make(**CONFIG)
    g = sb.Dqmc(p0, n_chains=args.chains, seeds=[test_seed(rank * args.chains + c) for c in range(args.chains)])
    return g, WORKLOAD, None


def profile_arm(args) -> None:
    """Single-kernel runs for profiling on one GPU, after sweep_start.

    --profile 2,1,0 launches each named operation of dqmc_gpu_time_op once
    untimed and --reps times timed, in the given order (finite T: 0 delayed
    update of one slice, 1 stabilisation step, 2 Green's function, 3 / 5 one
    slice of propagation of G from the left / right, 4 measurement;
    projective: 0 one bond family of updates, 1 tall QR, 2 (UL UR)^-1 and G,
    3 / 5 one slice of propagation of UR / UL^T, 4 measurement) and prints the
    per-launch milliseconds.  --profile sweep runs one full sweep with
    measurement.  --profile nn (effective action of the learned workload) runs
    one forward and one training step of 8 random fields."""
    import numpy as np
    import torch
    torch.cuda.set_device(0)
    if args.profile == "nn":
        from sunhubbardmy_b200.learned import EffectiveAction
        import sunhubbardmy_b200 as sb
        p = sb.DqmcParams.make(**CONFIG5)
        nn = EffectiveAction(p.ltrot, p.l1, max_batch=8)
        rng = np.random.default_rng(0)
        f = rng.choice(np.array([-1, 1], np.int8), size=(8, p.ltrot, p.l1, p.l1))
        S = nn.forward(f)
        loss = nn.train_step(f, rng.standard_normal(8), 1e-3)
        print(json.dumps({"profile": "nn", "S0": float(S[0]), "loss": float(loss)}), flush=True)
        return
    g, workload, _ = make_handle(args, 0)
    g.sweep_start()
    if args.profile == "sweep":
        g.obser_init()
        ms = g.sweeps(1, True)
        print(json.dumps({"profile": "sweep", "workload": workload, "chains": g.n_chains, "ms": ms}), flush=True)
    else:
        ops = [int(x) for x in args.profile.split(",")]
        out = {str(op): g.time_op(op, args.reps) for op in ops}
        print(json.dumps({"profile": "ops", "workload": workload, "chains": g.n_chains, "reps": args.reps,
                          "ms_per_launch": out}), flush=True)
    g.close()


def single_chain_block(args, result: dict, Ns, lt: int) -> dict:
    """The single-chain drop-in (one Markov chain on the GPU, the reference's
    one-chain-per-rank case): device sweep time and updates/s, the same through
    the C ABI with host buffers, and the batched/plain ESS/s ratio of double
    occupancy (the batched run's tau_int stands for both: same model and
    update)."""
    import numpy as np
    import torch
    import sunhubbardmy_b200 as sb
    p0 = sb.DqmcParams.make(**CONFIG)
    g1 = sb.Dqmc(p0, n_chains=1, seeds=[test_seed(0)])
    g1.sweep_start()
    g1.obser_init()
    g1.sweeps(2, True)
    torch.cuda.synchronize()
    n = 3
    ms = g1.sweeps(n, True)          # device ms per sweep
    per = 2 * lt * int(Ns[0])
    conf = torch.empty(lt * int(Ns[0]), dtype=torch.int32, pin_memory=True).numpy()
    g1.conf_all(conf)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(n):
        g1.set_conf_all(conf)
        g1.sweep_start()
        g1.sweeps(1, True)
        g1.bins_raw(0)
        g1.conf_all(conf)
    e2e_s = (time.perf_counter() - t0) / n
    g1.close()
    out = {"chains": 1, "ms_per_sweep": ms, "value": per / (ms * 1e-3), "unit": "updates/s",
           "e2e": {"value": per / e2e_s, "unit": "updates/s", "note": "set_conf_all + sweep_start + 1 sweep + "
                   "get_bins + get_conf_all, pinned host buffers"}}
    cb = result.get("cpu_baseline")
    if cb:
        out["cpu_one_core"] = cb["value"] / cb["cores"]
        out["vs_one_core"] = out["value"] / out["cpu_one_core"]
    es = result.get("ess")
    if es:
        tau = max(es["tau_int_sweeps"], 0.5)
        single = (1.0 / (2.0 * tau)) / (ms * 1e-3)
        out["ess_per_s"] = single
        out["batched_vs_single_ess_per_s"] = es["ess_per_s"] / single
    return out


def gpu_arm(args, rank: int, world: int, local_rank: int) -> None:
    import numpy as np
    import torch
    import sunhubbardmy_b200 as sb

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    g, workload, tune_report = make_handle(args, rank)
    C = g.n_chains
    p = g.params[0]
    lt = p.ltrot
    Ns = np.array([g.ndim(c) for c in range(C)], dtype=np.float64)
    N = int(Ns.max())
    g.sweep_start()
    g.obser_init()
    g.sweeps(max(args.warmup, 1), True)
    g.reset_diag()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    with ClockSampler(local_rank) as clk:
        ms = g.sweeps(args.steps, True)          # CUDA events on the library stream
    barrier()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    proj = bool(p.proj)
    bond = p.rv != 0 and (proj or p.rhub == 0)     # the bond field's proposals are the unit
    if proj or p.rv != 0:
        nnf = 3 if p.lattice == 2 else 4
        units = np.array([(nnf * (Nc // 2 if p.lattice == 2 else Nc // 2) if p.rv != 0 else 0) +
                          (Nc if p.rhub != 0 else 0) for Nc in Ns])
        per_step = world * int(2 * lt * units.sum())
    else:
        per_step = world * int(2 * lt * Ns.sum())
    value = per_step / (ms * 1e-3)
    kernels_per_sweep = g.sweep_kernels()
    d0 = g.diag(0)
    wrap = max(g.diag(c)["max_wrap_error"] for c in range(C))
    if bond:
        acc = d0["accepted_v"] / max(1.0, d0["proposed_v"])
    else:
        acc = d0["accepted"] / max(1.0, d0["proposed"])

    # end to end through the public API with host buffers: h2d of every chain's
    # HS field, sweep_start + one sweep, d2h of every chain's bins and field
    nbins = sum(len(g.bins_raw(c)) for c in range(C)) / C
    e2e_steps = max(1, min(args.steps, 5))
    if bond:
        # the bond field of every walker (vconf%conf), walker by walker
        vhost = [torch.empty(g.vconf(c).shape, dtype=torch.int32, pin_memory=True).numpy() for c in range(C)]
        for c in range(C):
            vhost[c][...] = g.vconf(c)
        nconf = sum(v.size for v in vhost)
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            for c in range(C):
                g.set_vconf(vhost[c], c)
            g.sweep_start()
            g.sweeps(1, True)
            bins = [g.bins_raw(c) for c in range(C)]
            for c in range(C):
                vhost[c][...] = g.vconf(c)
        barrier()
    else:
        nconf = int(lt * Ns.sum())
        conf_host = torch.empty(nconf, dtype=torch.int32, pin_memory=True).numpy()
        g.conf_all(conf_host)
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            g.set_conf_all(conf_host)
            g.sweep_start()
            g.sweeps(1, True)
            bins = [g.bins_raw(c) for c in range(C)]
            g.conf_all(conf_host)
        barrier()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_s = float(t.item())
    del bins

    result = None
    if rank == 0 and proj:
        result = proj_roofline_and_line(args, g, p, Ns, ms, value, per_step, world, workload, acc, wrap,
                                        kernels_per_sweep, clk, e2e_s, nconf, nbins)
    elif rank == 0:
        ka, kp = ("accepted_v", "proposed_v") if bond else ("accepted", "proposed")
        acc_c = np.array([g.diag(c)[ka] / max(1.0, g.diag(c)[kp]) for c in range(C)])
        fp64 = fp64_peak_tflops()
        N2, N3 = float((Ns ** 2).sum()), float((Ns ** 3).sum())     # sums over chains
        work = {   # algorithmic work of one launch group over all chains: (flops, bytes)
            # flush GEMMs: 8 N^2 per accepted site, or 16 N^2 per accepted bond of a
            # family of N / 2 bonds (the honeycomb t-V launch covers one family)
            "update": (8.0 * float((acc_c * Ns ** 3).sum()), None),
            "stab": ((14.0 + 2.0 / 3.0) * N3, None),   # QR 16/3, Q 16/3, triangular (D^-1 R) V 4
            "green": ((41.0 + 1.0 / 3.0) * N3, None),
            "prop_left": (None, 32.0 * N2), "prop_right": (None, 32.0 * N2), "bprod": (None, 32.0 * N2),
            "measure": (None, 16.0 * N2),
        }
        if p.kinetic == 1:
            # The B product of a stabilisation applies nwrap slices (FFT, diagonal,
            # FFT) to every column in registers: one read and one write of the
            # matrix, so it is bound by the FP64 pipe, not by HBM.  A 2D radix-2
            # FFT of l x l points is l^2 log2(l) butterflies of 10 flops; an FFT
            # operator is a forward and an inverse FFT and l^2 complex products.
            l = float(p.l1)
            fft_op = 20.0 * l * l * np.log2(l) + 6.0 * l * l
            per_vec = p.nwrap * (2.0 * fft_op + 6.0 * l * l)
            work["bprod"] = (per_vec * float(Ns.sum()), None)
        names = {"update": "k_vbond_delay (one bond family)" if bond else "k_update_delay", "stab": "k_stab", "green": "k_green",
                 "prop_left": "k_prop_fft (columns)" if p.kinetic == 1 else "k_prop_cols",
                 "prop_right": "k_prop_fft (rows)" if p.kinetic == 1 else "k_prop_rows",
                 "bprod": "B product of the stabilisation (k_prop_fft over nwrap slices)", "measure": "k_transpose_g + k_measure",
                 "other": "copies, wrap checks, SFMT"}
        roof = sweep_roofline(g.sweep_profile(1, True), work, names, fp64)
        trf = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(trf):
            tr = json.load(open(trf)).get(roof["kernel"])
            if tr:
                roof["traffic"] = tr["bytes_per_chain"] * C
                roof["traffic_note"] = tr.get("note", "")
        result = {
            "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (HS field drawn from the reference's -DTEST seeds, one per chain)",
            "config": {"workload": workload, "chains_per_gpu": C, "parallelism": f"replicas x{world}",
                       "l2": "working set ~52 MiB/chain >> L2 (no flush needed)",
                       "acceptance": acc, "max_wrap_error": wrap},
            "e2e": {"value": per_step / e2e_s, "unit": "updates/s",
                    "h2d_bytes_per_step": nconf * 4,
                    "d2h_bytes_per_step": int(C * nbins * 16 + nconf * 4),
                    "note": ("per step: set_vconf of every chain (pinned host) + sweep_start + 1 sweep + get_bins + get_vconf"
                             if bond else
                             "per step: set_conf_all (pinned host) + sweep_start + 1 sweep + get_bins + get_conf_all")},
            "gpu_launches": kernels_per_sweep * args.steps,
            "roofline": roof,
            "clocks": clk.summary(),
        }
        if tune_report is not None:
            result["config"]["autotune"] = {str(k): v for k, v in tune_report.items()}
        ku = roof.get("kinds", {}).get("update")
        if ku and ku.get("ms_per_launch") and ku.get("launches"):
            # the same proposals over the update kernel's own device time in one
            # sweep (in-sweep CUDA events), without propagation, stabilisation,
            # Green's functions and measurement
            upd_s = ku["ms_per_launch"] * ku["launches"] * 1e-3
            result["update_only"] = {"value": per_step / world / upd_s, "unit": "updates/s",
                                     "kernel": ku.get("kernel"), "s_per_step": upd_s}
        ess_sweeps = args.ess if args.ess > 0 else (10 if args.workload == "config2" else 0)
        if ess_sweeps > 0:
            from sunhubbardmy_b200.stats import double_occupancy, ess
            series = []
            g.sweeps(args.ess_warmup if args.ess > 0 else 0, False)     # equilibrate before the series
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(ess_sweeps):
                g.obser_init()
                g.sweeps(1, True)
                series.append(double_occupancy(g.energy_all(), Ns))
            wall = time.perf_counter() - t0
            x = np.array(series).T            # [chain, sweep]
            n_ess, tau = ess(x)
            result["ess"] = {"observable": "double occupancy (per-sweep, per chain)", "sweeps": ess_sweeps,
                             "warmup_sweeps": (args.ess_warmup if args.ess > 0 else 0) + args.warmup + args.steps,
                             "chains": C, "tau_int_sweeps": tau, "ess": n_ess, "ess_per_s": n_ess / wall,
                             "mean": float(x.mean()), "stderr": float(x.std(ddof=1) / np.sqrt(n_ess)),
                             "wall_s": wall}
        if args.workload == "config2" and hasattr(g, "time_op"):
            # the delayed-update GEMM alone (dqmc_gpu_time_op 6: G += A B^T over
            # nublock columns, one CTA per chain); it modifies G, so it runs last
            fms = g.time_op(6, 5)
            fl = 8.0 * float((Ns ** 2).sum()) * p.nublock
            ach = fl / (fms * 1e-3) / 1e12
            roof["update_gemm_isolated"] = {
                "kernel": "k_update_flush (the flush_addto of k_update_delay)", "ms_per_launch": fms,
                "achieved": ach, "peak": fp64, "unit": "TFLOP/s", "frac": ach / fp64,
                "note": f"G += A B^T with N = {int(Ns.max())}, K = nublock = {p.nublock}, one CTA per chain "
                        f"({C} chains) as inside the update kernel"}
        if world == 1 and not args.no_cpu and args.workload == "config2":
            per, times, _ = cpu_sample(20, os.cpu_count() or 1, steps=1)
            cv = per / times[0]
            result["cpu_baseline"] = {"value": cv, "unit": "updates/s", "cores": os.cpu_count() or 1, "kind": "port",
                                      "sample": f"20 slices of a b0 sweep per chain, one chain per core ({os.cpu_count()} cores), OpenBLAS"}
        if args.workload == "config2" and C > 1 and world == 1:
            result["single_chain"] = single_chain_block(args, result, Ns, lt)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result), flush=True)


def proj_roofline_and_line(args, g, p, Ns, ms, value, per_step, world, workload, acc, wrap,
                           kernels_per_sweep, clk, e2e_s, nconf, nbins):
    """JSON line of the projective workload.  Dominant-kernel roofline from
    per-kernel CUDA-event times; algorithmic flops of the submatrix-LR update
    per bond family and walker: 8 [N ne^2 + N R ne + a (2 N ne^2 + N R ne)]
    (Rrows and Felms GEMMs of every window, the flush GEMMs of accepted rows;
    R = nustock window rows, a = acceptance)."""
    import numpy as np
    C = g.n_chains
    lt, nst, ne = p.ltrot, p.nst, p.ne
    R = min(32, p.nublock)
    fp64 = fp64_peak_tflops()
    N = Ns
    upd = 8.0 * (N * ne ** 2 + N * R * ne + acc * (2 * N * ne ** 2 + N * R * ne))
    qr = 16.0 * (N * ne ** 2 - ne ** 3 / 3.0)
    ulrg = 8.0 * (ne ** 2 * N + (2.0 / 3.0 + 1.0 + 0.5) * ne ** 3 + N * ne ** 2 + N * N * ne)
    work = {"update": (float(upd.sum()), None), "stab": (float(qr.sum()), None), "green": (float(ulrg.sum()), None),
            "prop_left": (None, 32.0 * float((N * ne).sum())), "prop_right": (None, 32.0 * float((N * ne).sum())),
            "measure": (None, 16.0 * float((N * N).sum()))}
    names = {"update": "k_pwin_rg + k_pwin_seq + k_pwin_flush (one bond family)", "stab": "k_proj_qr",
             "green": "k_proj_ulr + k_proj_t1 + k_proj_gmat", "prop_left": "k_prop_cols (UR)",
             "prop_right": "k_prop_cols (UL^T)", "measure": "k_transpose_g + k_measure",
             "other": "copies, wrap checks, SFMT"}
    roof = sweep_roofline(g.sweep_profile(1, True), work, names, fp64)
    from sunhubbardmy_b200.autotune import ChainGroup
    if isinstance(g, ChainGroup):
        roof["timing"] += f" (one handle of all {len(Ns)} walkers, after one warm-up sweep)"
    trf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(trf):
        tr = json.load(open(trf)).get(roof["kernel"])
        if tr:
            roof["traffic"] = tr["bytes_per_chain"] * C
            roof["traffic_note"] = tr.get("note", "")
    result = {
        "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (bond field drawn from the reference's -DTEST seeds, one per walker)",
        "config": {"workload": workload, "chains_per_gpu": C, "parallelism": f"replicas x{world}",
                   "l2": "working set ~30 MiB/walker x 64 >> L2 (no flush needed)",
                   "acceptance": acc, "max_wrap_error": wrap},
        "e2e": {"value": per_step / e2e_s, "unit": "updates/s",
                "h2d_bytes_per_step": nconf * 4,
                "d2h_bytes_per_step": int(C * nbins * 16 + nconf * 4),
                "note": "per step: set_vconf of every walker (pinned host) + sweep_start + 1 sweep + get_bins + get_vconf"},
        "gpu_launches": kernels_per_sweep * args.steps,
        "roofline": roof,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu:
        per, times, _ = cpu_sample_proj(4, os.cpu_count() or 1, steps=1)
        cv = per / times[0]
        result["cpu_baseline"] = {"value": cv, "unit": "updates/s", "cores": os.cpu_count() or 1, "kind": "port",
                                  "sample": f"4 slices of a b0 projective sweep per walker, one walker per core "
                                            f"({os.cpu_count()} cores), submatrix-LR, OpenBLAS"}
    return result


def learned_arm(args, rank: int, local_rank: int) -> None:
    """ESS/s of the per-sweep double occupancy: plain sweeps (which also record
    the training pairs at every stabilisation), then the effective action is
    trained on the recorded pairs, then learned sweeps (plain local updates +
    global block proposals) continue the same chains."""
    import numpy as np
    import torch
    import sunhubbardmy_b200 as sb
    from sunhubbardmy_b200.learned import EffectiveAction, train
    from sunhubbardmy_b200.stats import double_occupancy, ess

    torch.cuda.set_device(local_rank)
    p = sb.DqmcParams.make(**CONFIG5)
    nch = args.chains if args.chains_set else 64
    g = sb.Dqmc(p, n_chains=nch, seeds=[test_seed(rank * nch + c) for c in range(nch)])
    Ns = np.full(nch, float(p.ndim))
    g.sweep_start()
    g.sweeps(max(args.ess_warmup, 1), False)

    def run(step, n):
        xs, dev = [], 0.0
        t0 = time.perf_counter()
        for _ in range(n):
            g.obser_init()
            dev += step()
            xs.append(double_occupancy(g.energy_all(), Ns))
        return np.array(xs).T, time.perf_counter() - t0, dev * 1e-3

    cap = max(args.pairs, 1)
    g.record(cap)
    with ClockSampler(local_rank) as clk_p:
        xp, wall_p, dev_p = run(lambda: g.sweeps(1, True), args.ess)
    npairs = g.record_count()
    targets = -g.record_values(cap)[:npairs]
    g.record(0)
    ess_p, tau_p = ess(xp)

    nn = EffectiveAction(p.ltrot, p.l1, max_batch=32, seed=1)
    rng = np.random.default_rng(0)
    perm = rng.permutation(npairs)
    nval = min(256, npairs // 10)
    val, tr = perm[:nval], perm[nval:]
    vf = np.stack([g.record_get(int(i))[0] for i in val])

    def val_loss():
        S = np.concatenate([nn.forward(vf[k:k + 32]) for k in range(0, len(vf), 32)])
        d = S - targets[val]
        return float(np.var(d)), float(np.var(targets[val]))

    l0, var_y = val_loss()
    t0 = time.perf_counter()
    losses = train(nn, g, targets[tr], args.train_steps, batch=32, lr=args.lr, seed=1, slots=tr,
                   pair_lag=nch, diff_every=args.diff_every)
    train_s = time.perf_counter() - t0
    l1, _ = val_loss()

    g.reset_diag()
    with ClockSampler(local_rank) as clk_l:
        xl, wall_l, dev_l = run(lambda: g.sweeps_learned(nn, 1, True), args.ess)
    ess_l, tau_l = ess(xl)
    ds = [g.diag(c) for c in range(nch)]
    tot = {k: sum(d[k] for d in ds) for k in ("blk_proposed", "blk_stage1", "blk_accepted", "blk_err_learned", "blk_err_zero")}
    line = {
        "metric": "ESS/s of double occupancy (learned + batched vs plain)", "value": ess_l / wall_l, "unit": "1/s",
        "n_gpus": 1, "steps": args.ess, "warmup": args.ess_warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128 (DQMC), bf16/fp32 (effective action)",
        "data": "synthetic (HS fields drawn from the reference's -DTEST seeds; training pairs recorded from the plain chains)",
        "config": {"workload": WORKLOAD5, "chains": nch},
        "plain": {"ess": ess_p, "tau_int_sweeps": tau_p, "wall_s": wall_p, "device_s": dev_p,
                  "ess_per_s": ess_p / wall_p, "mean": float(xp.mean()),
                  "stderr": float(xp.std(ddof=1) / np.sqrt(ess_p)), "clocks": clk_p.summary()},
        "learned": {"ess": ess_l, "tau_int_sweeps": tau_l, "wall_s": wall_l, "device_s": dev_l,
                    "ess_per_s": ess_l / wall_l, "mean": float(xl.mean()),
                    "stderr": float(xl.std(ddof=1) / np.sqrt(ess_l)), "clocks": clk_l.summary(),
                    "blocks_proposed": tot["blk_proposed"],
                    "stage1_pass": tot["blk_stage1"] / max(1.0, tot["blk_proposed"]),
                    "accepted": tot["blk_accepted"] / max(1.0, tot["blk_proposed"]),
                    "ratio_prediction_mse_learned": tot["blk_err_learned"] / max(1.0, tot["blk_stage1"]),
                    "ratio_prediction_mse_zero": tot["blk_err_zero"] / max(1.0, tot["blk_stage1"])},
        "ess_per_s_ratio_learned_vs_plain": (ess_l / wall_l) / (ess_p / wall_p),
        "training": {"pairs": int(npairs), "steps": args.train_steps, "batch": 32, "lr": args.lr, "wall_s": train_s,
                     "diff_every": args.diff_every,
                     "heldout_var_residual_before": l0, "heldout_var_residual_after": l1,
                     "heldout_var_target": var_y, "loss_first": float(np.mean(losses[:20])),
                     "loss_last": float(np.mean(losses[-20:]))},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--chains", type=int, default=None)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--workload", default="config2", choices=["config2", "config3", "config4", "config5", "tvft"])
    ap.add_argument("--pairs", type=int, default=200000, help="config5: training-pair ring capacity")
    ap.add_argument("--train-steps", type=int, default=3000, help="config5: Adam steps of 32 pairs")
    ap.add_argument("--lr", type=float, default=3e-4, help="config5: Adam learning rate")
    ap.add_argument("--diff-every", type=int, default=1,
                    help="config5: every n-th Adam step fits the change of -log|W| between a chain's consecutive records (0: off)")
    ap.add_argument("--ess", type=int, default=0, help="extra sweeps for the ESS/s of double occupancy")
    ap.add_argument("--ess-warmup", type=int, default=20, help="equilibration sweeps before the ESS series")
    ap.add_argument("--streams", type=int, default=0,
                    help="config4: handles of walkers swept concurrently (default 8); config3: handles per size "
                         "class (default: up to 4 per class, 16 in all; 1: one handle of all chains)")
    ap.add_argument("--profile", default=None,
                    help="single-kernel runs for profiling: comma-separated time_op ids, 'sweep' or 'nn'")
    ap.add_argument("--reps", type=int, default=1, help="--profile: timed launches per operation")
    args = ap.parse_args()
    args.chains_set = args.chains is not None
    if args.chains is None:
        args.chains = 296
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    if args.profile:
        profile_arm(args)
        return
    if args.workload == "config5":
        if rank == 0:
            learned_arm(args, rank, local_rank)
        return
    gpu_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
