#!/usr/bin/env python3
"""bench.py -- chain-sweeps/s of STRUCTURE's per-sweep MCMC on B200.

Workload (the large SNP panel): N=2000 diploid individuals, L=50,000 biallelic
SNPs packed 2 bits/genotype, 3% missing genotypes, K=5 correlated-frequency (F)
model with Fst_k = {0.05..0.25}, Q_i ~ Dirichlet(0.3), alpha and F inferred,
METROFREQ=10, FPRIORMEAN/SD = 0.01/0.05; 20 chains (seeds 2000+r) batched on
one GPU.  A step is one batched sweep (20 chain-sweeps: P, Q, Z, alpha, eps, F,
DataCollection).  Warm-up steps are the burn-in; timed steps collect.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own 20-chain batch (weak scaling, no
collective on the data path); rank 0 prints one JSON line.
"""
import argparse
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WL = dict(N=2000, L=50000, K=5, chains=20, F=[0.05, 0.10, 0.15, 0.20, 0.25], qalpha=0.3,
          missing=0.03, metrofreq=10, fpriormean=0.01, fpriorsd=0.05, alphapropsd=0.025)
WORKLOAD_NAME = "snp-fmodel N=2000 L=50000 K=5, 20 chains batched"
SLICE_L = 10000          # CPU legs time a 10,000-locus slice and scale by L
METRIC = "chain-sweeps/s"


def model_kwargs(burnin, numreps):
    return dict(maxpops=WL["K"], burnin=burnin, numreps=numreps, freqscorr=1, onefst=0,
                inferalpha=1, popalphas=0, unifprioralpha=1, alpha=1.0, alphamax=10.0,
                alphapropsd=WL["alphapropsd"], fpriormean=WL["fpriormean"],
                fpriorsd=WL["fpriorsd"], metrofreq=WL["metrofreq"], computeprob=1, store_z=0)


def make_data():
    from structure_b200 import synth
    return synth.config2(N=WL["N"], L=WL["L"], want_int32=False)


# ---------------------------------------------------------------------------
# CPU legs: the reference's own CPU update functions (oracle/_ref) in
# structure.c order, timed over consecutive sweeps of a locus slice (one
# METROFREQ cycle = 9 Gibbs + 1 Metropolis sweep per ten); time scales
# linearly in L.
# ---------------------------------------------------------------------------
def _ref_worker(q, path, N, L_slice, seed, core, warmup, steps):
    try:
        # the reference prints progress on stdout; keep the bench's stdout to one line
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        if core is not None:
            os.sched_setaffinity(0, {core})
        from oracle.oracle import RefLib, ref_model
        geno = np.load(path)
        r = RefLib()
        m = ref_model(N=N, L=L_slice, K=WL["K"], maxalleles=2, freqscorr=1,
                      fpriormean=WL["fpriormean"], fpriorsd=WL["fpriorsd"],
                      metrofreq=WL["metrofreq"], burnin=0, numreps=100,
                      alphapropsd=WL["alphapropsd"])
        ch = r.chain_new(m, geno, seed=seed)
        r.lib.stref_chain_sweeps(ch, warmup)              # reps 0..warmup-1, untimed
        t0 = time.perf_counter()
        r.lib.stref_chain_sweeps(ch, steps)               # the timed sweeps
        dt = time.perf_counter() - t0
        r.lib.stref_chain_free(ch)
        q.put(dt)
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put(repr(e))


def cpu_reference(packed, workers, pin=False, warmup=1, steps=10, slice_l=SLICE_L):
    """chain-sweeps/s of `workers` concurrent reference chains at full L, from
    `steps` timed sweeps (after `warmup` untimed ones) of a `slice_l`-locus slice."""
    from structure_b200 import synth
    geno = synth.unpack_int32(packed, WL["N"], 0, slice_l)
    tmp = tempfile.NamedTemporaryFile(suffix=".npy", delete=False)
    np.save(tmp.name, geno)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_ref_worker,
                         args=(q, tmp.name, WL["N"], slice_l, 1000 + w, (w if pin else None),
                               warmup, steps))
             for w in range(workers)]
    for p in procs:
        p.start()
    res = []
    while len(res) < len(procs):
        try:
            res.append(q.get(timeout=5))
        except Exception:
            dead = [p for p in procs if not p.is_alive() and p.exitcode not in (0, None)]
            if dead:
                for p in procs:
                    p.kill()
                raise RuntimeError(f"reference worker exited with code {dead[0].exitcode}")
    for p in procs:
        p.join()
    os.unlink(tmp.name)
    bad = [x for x in res if not isinstance(x, float)]
    if bad:
        raise RuntimeError(f"reference worker failed: {bad[0]}")
    scale = slice_l / WL["L"]
    rate = sum(steps / dt for dt in res) * scale
    sample = (f"{workers} concurrent reference chain(s), each timed over sweeps "
              f"{warmup}-{warmup + steps - 1} (one Metropolis sweep in {WL['metrofreq']}) of a "
              f"{slice_l}-locus slice (N={WL['N']}, K={WL['K']}, F model), scaled by "
              f"{slice_l}/{WL['L']} loci; uniforms for the array-fed updates from xorshift128+")
    return rate, sample, max(res)


def cpu_model():
    """The host CPU's model name (as lscpu reports it, from /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def usable_workers():
    n = os.cpu_count() or 1
    try:
        import psutil
        mem = psutil.virtual_memory().available
        n = min(n, max(1, int(mem // (2 << 30))))
    except Exception:
        pass
    return max(1, min(n, WL["chains"]))


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.p is None:
            return out
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
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows for j in range(4) if r[5 + j] == "Active"})
        out.update(sm_mhz=float(np.median(sm)) if sm else None,
                   sm_max_mhz=max(mx) if mx else None, reasons=reasons, samples=len(rows))
        return out


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_profile_figure(key):
    """A figure of the committed ncu summary of the Z pass (a line "key: value"),
    if any."""
    path = os.path.join(ROOT, "profiles", "zpass_b2g_snp2000x50000_k5_batch20.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(key + ":"):
                    return float(line.split(":")[1])
    except Exception:
        pass
    return None


def read_traffic():
    """DRAM bytes per Z-pass launch from the committed ncu summary, if any."""
    return read_profile_figure("dram_bytes_per_launch")


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    from structure_b200 import api

    d = make_data()
    packed, na = d["packed"], d["numalleles"]
    N, L, K, B = WL["N"], WL["L"], WL["K"], WL["chains"]
    W, S = args.warmup, args.steps
    codes = (packed[:, :, None] >> (2 * np.arange(16, dtype=np.uint32))[None, None, :]) & 3
    copies = int(2 * (codes.reshape(L, -1)[:, :N] != 3).sum())

    ctx = api.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    data = api.Data(ctx, na, packed=packed, num_inds=N, num_loci=L, layout=api.LAYOUT_B2G)
    mk = model_kwargs(burnin=W, numreps=S + 10)
    chains = [api.Chain(ctx, data, api.model_defaults(**mk), 2000 + 1000 * rank + r)
              for r in range(B)]
    batch = api.Batch(ctx, chains)
    # Z-pass tiles timed on these chains (st_batch_autotune); batches of the
    # same shapes made later in the process (the e2e leg) start from them
    batch.autotune()
    tdims = chains[0].get(api.F_DIMS)

    # warm-up = burn-in
    batch.sweep(W)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    # the timed sweeps replay the batch's CUDA graphs (one per sweep kind)
    clocks = ClockSampler(local)
    l0 = ctx.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    batch.sweep(S)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = ctx.launches() - l0
    clk = clocks.stop()
    for c in chains:
        assert c.sync() == 0, "device error word set"
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * B * S / (ms / 1e3)

    # per-kernel times: graph replay cannot bracket single launches, so the
    # same batch runs PS more sweeps (one Metropolis sweep in METROFREQ, as in
    # the timed ones) launch by launch with CUDA events around every launch
    PS = max(WL["metrofreq"], min(S, 2 * WL["metrofreq"]))
    ctx.profile(True)
    ctx.profile_read()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    batch.sweep(PS)
    q1.record(stream)
    torch.cuda.synchronize()
    eager_ms = q0.elapsed_time(q1) / PS
    prof = ctx.profile_read()
    ctx.profile(False)

    # plain path: the same chains one at a time (one chain per launch), each
    # replaying its own CUDA graphs, captured by untimed sweeps first
    plain_sweeps = WL["metrofreq"]
    singles = [api.Batch(ctx, [c]) for c in chains]
    for sb in singles:
        sb.sweep(WL["metrofreq"])
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for sb in singles:
        sb.sweep(plain_sweeps)
    p1.record(stream)
    torch.cuda.synchronize()
    plain = B * plain_sweeps / (p0.elapsed_time(p1) / 1e3)
    for sb in singles:
        sb.close()
    like = [c.get(api.F_STATS)[api.ST_SUMLIKES] / max(1, c.get(api.F_STATS)[api.ST_NLIKE])
            for c in chains]
    # page-locked result arrays for the end-to-end leg's reads (fields of the same shapes)
    out_fields = (api.F_QSUM, api.F_PSUM, api.F_STATS, api.F_ALPHA, api.F_F)
    out_spec = [(f, chains[0].get(f).dtype, api.lib().st_field_bytes(chains[0].h, f))
                for f in out_fields]
    outs = [{f: torch.empty(n, dtype=torch.uint8, pin_memory=True).numpy().view(dt)
             for f, dt, n in out_spec} for _ in range(B)]
    batch.close()
    for c in chains:
        c.close()
    data.close()

    # end to end through the C ABI from pinned host memory
    pinned = torch.from_numpy(packed).pin_memory()
    ppk = pinned.numpy()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    data2 = api.Data(ctx, na, packed=ppk, num_inds=N, num_loci=L, layout=api.LAYOUT_B2G)
    t1 = time.perf_counter()
    mk2 = model_kwargs(burnin=0, numreps=S)
    ch2 = [api.Chain(ctx, data2, api.model_defaults(**mk2), 9000 + r) for r in range(B)]
    b2 = api.Batch(ctx, ch2)
    t2 = time.perf_counter()
    b2.sweep(S)
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    d2h = 0
    for c, o in zip(ch2, outs):
        for f in out_fields:
            d2h += c.get(f, out=o[f]).nbytes
    t_e2e = time.perf_counter() - t0
    e2e_parts = {"upload_ms": round((t1 - t0) * 1e3, 2), "create_ms": round((t2 - t1) * 1e3, 2),
                 "sweeps_ms": round((t3 - t2) * 1e3, 2),
                 "d2h_ms": round((t0 + t_e2e - t3) * 1e3, 2)}
    e2e = B * S / t_e2e
    b2.close()
    for c in ch2:
        c.close()
    data2.close()

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    # roofline of the dominant kernel (the Z pass)
    zms, zn = prof["zpass"]
    zavg = zms / max(1, zn)
    G = packed.nbytes
    per_chain = N * K * 4 + L * K * 2 * 4 + (L * K * 2 + N * K) * 4
    alg_bytes = G + B * per_chain
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (zavg / 1e3) / 1e9
    ops_per_copy = 2 * K + 2 + 10 + 0.5
    alu_achieved = B * copies * ops_per_copy / (zavg / 1e3) / 1e12
    sm_mhz = clk["sm_mhz"] or 1965.0
    alu_peak = 148 * 128 * sm_mhz * 1e6 / 1e12
    # issue roofline of the same kernel, the limit it actually meets: warp
    # instructions per 32 genotypes from the ncu capture of a collecting launch
    # (profiles/zpass_b2g_snp2000x50000_k5_batch20.txt), as the timed launches are
    inst_per_32 = read_profile_figure("inst_per_32_genotypes")
    issue_achieved = (B * N * L / 32 * inst_per_32 / (zavg / 1e3) / 1e12) if inst_per_32 else None
    issue_peak = 148 * 4 * sm_mhz * 1e6 / 1e12
    traffic = read_traffic()
    total_ms = sum(v[0] for v in prof.values())

    cpu_rate, cpu_sample, _ = (None, None, None)
    if not args.no_cpu_baseline and world == 1:
        cpu_rate, cpu_sample, _ = cpu_reference(packed, 1, pin=True)

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": METRIC, "n_gpus": world,
        "steps": S, "warmup": W, "ms_per_step": round(ms / S, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (Z/P/Q) + f64 (MH ratios, lnP(D))",
        "data": "synthetic, seeded (STRUCTURE's generative model; no public dataset is named)",
        "config": {"workload": WORKLOAD_NAME, "N": N, "L": L, "K": K, "chains_per_gpu": B,
                   "model": "admixture + F model, alpha and F inferred, METROFREQ=10",
                   "genotypes": "2 bits/genotype, locus-major", "store_z": False,
                   "l2": f"no flush: per-sweep working set {(G + B * (per_chain + L * K * 2 * 12)) / 1e9:.2f} GB > 126 MB L2",
                   "parallelism": f"{world} GPU x {B} chains (replicas)",
                   "z_tile": {"chunks_of_individuals": int(tdims[6]),
                              "locus_groups": int(tdims[7]), "chosen_by": "st_batch_autotune"}},
        "z_updates_per_s": round(value * copies, 1),
        "plain": {"value": round(plain, 3), "unit": METRIC,
                  "path": "one chain per launch, same kernels, each chain's sweep replayed "
                          "from its own CUDA graphs"},
        "batched_over_plain": round(value / world / plain, 3),
        "mean_lnpd_over_chains": round(float(np.mean(like)), 2),
        "e2e": {"value": round(e2e, 3), "unit": METRIC,
                "h2d_bytes_per_step": int(math.ceil(packed.nbytes / S)),
                "d2h_bytes_per_step": int(math.ceil(d2h / S)), "parts": e2e_parts,
                "includes": "st_data_upload from pinned host words, 20 x st_chain_create "
                            "(initial Z pass), st_batch_sweep, st_get_state of QSum/PSum/"
                            "stats/alpha/F into page-locked host arrays allocated beforehand"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 5), "traffic": traffic,
                     "peak_source": peak_kind,
                     "kernel": f"zpass_b2g_kernel<K class {api.fast_class(K)}, Normal, 8 warps> "
                               f"(batched, {B} chains)",
                     "avg_launch_ms": round(zavg, 4),
                     "algorithmic_bytes_per_launch": int(alg_bytes)},
        "roofline_alu": {"bound": "alu", "achieved": round(alu_achieved, 3),
                         "peak": round(alu_peak, 2), "unit": "Top/s",
                         "frac": round(alu_achieved / alu_peak, 4),
                         "ops_per_copy": ops_per_copy,
                         "note": "2K+2 FP32 + ~10 int (Philox/4) + 0.5 log per allele copy; "
                                 "peak = 148 SM x 128 lanes x median SM clock"},
        "roofline_issue": {"bound": "issue",
                           "achieved": round(issue_achieved, 4) if issue_achieved else None,
                           "peak": round(issue_peak, 4), "unit": "T warp-inst/s",
                           "frac": round(issue_achieved / issue_peak, 4) if issue_achieved else None,
                           "inst_per_32_genotypes": inst_per_32,
                           "note": "instructions from an ncu capture of a collecting "
                                   "launch (ln P(D) terms on, as in the timed sweeps); peak "
                                   "= 148 SM x 4 schedulers x median SM clock"},
        "timed_path": "CUDA-graph replay of the batched sweep (st_batch_sweep, graphs on)",
        "profiled_pass": {"sweeps": PS, "ms_per_step": round(eager_ms, 4),
                          "note": "kernels_ms_per_step, kernel_share and the Z-pass launch "
                                  "time come from these sweeps, run launch by launch with "
                                  "CUDA events around every launch right after the timed ones"},
        "kernels_ms_per_step": {k: round(v[0] / PS, 4) for k, v in prof.items()},
        "kernel_share": {k: round(v[0] / total_ms, 4) for k, v in prof.items()} if total_ms else {},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if world == 1 and not args.headline_only:
        ctx.close()
        out["other_configs"] = other_configs(not args.no_cpu_baseline)
    if cpu_rate is not None:
        out["cpu_baseline"] = {"value": round(cpu_rate, 5), "unit": METRIC, "cores": 1,
                               "kind": "reference", "sample": cpu_sample,
                               "cpu_model": cpu_model(), "host_cpus": os.cpu_count()}
    print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    d = make_data()
    workers = usable_workers()
    # each step is one sweep of a locus slice sized so that warm-up + steps take
    # about two minutes (~0.26 ms per locus and sweep for one reference chain)
    steps, warmup = max(1, args.steps), max(1, args.warmup)
    slice_l = int(min(SLICE_L, max(1000, 120.0 / ((steps + warmup) * 0.26e-3) // 1000 * 1000)))
    rate, sample, tmax = cpu_reference(d["packed"], workers, pin=False, warmup=warmup,
                                       steps=steps, slice_l=slice_l)
    out = {"metric": METRIC, "value": round(rate, 5), "unit": METRIC, "n_gpus": world,
           "steps": steps, "warmup": warmup, "ms_per_step": round(tmax * 1e3 / steps, 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic, seeded (same generator and seed as the GPU arm)",
           "config": {"workload": WORKLOAD_NAME, "N": WL["N"], "L": WL["L"], "K": WL["K"],
                      "slice_loci": slice_l, "workers": workers},
           "impl": "reference",
           "cpu_baseline": {"value": round(rate, 5), "unit": METRIC, "cores": workers,
                            "kind": "reference", "sample": sample, "cpu_model": cpu_model(),
                            "host_cpus": os.cpu_count()},
           "e2e": {"value": round(rate, 5), "unit": METRIC, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# Opt-in workloads (--workload): the other configurations' measurements.
# ---------------------------------------------------------------------------
def _ess(x):
    """Effective sample size, Geyer's initial monotone sequence estimator."""
    x = np.asarray(x, np.float64)
    n = len(x)
    x = x - x.mean()
    if n < 4 or not np.any(x):
        return float(n)
    f = np.fft.rfft(x, 2 * n)
    ac = np.fft.irfft(f * np.conj(f))[:n]
    ac = ac / ac[0]
    s, prev = 0.0, np.inf
    for t in range(0, n - 1, 2):
        g = ac[t] + ac[t + 1]
        if g <= 0:
            break
        g = min(g, prev)
        prev = g
        s += g
    return n / max(-1.0 + 2.0 * s, 1e-12)


def _ref_jobs_worker(q, jobs, core):
    """Runs reference chains one after another on one pinned core; each job is
    (npy path, ref_model kwargs, seed, untimed sweeps, timed sweeps)."""
    try:
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        if core is not None:
            os.sched_setaffinity(0, {core})
        from oracle.oracle import RefLib, ref_model
        r = RefLib()
        out = []
        for path, mkw, seed, warm, steps in jobs:
            geno = np.load(path)
            ch = r.chain_new(ref_model(**mkw), geno, seed=seed)
            if warm:
                r.lib.stref_chain_sweeps(ch, warm)
            t0 = time.perf_counter()
            r.lib.stref_chain_sweeps(ch, steps)
            out.append(time.perf_counter() - t0)
            r.lib.stref_chain_free(ch)
        q.put(out)
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put(repr(e))


def cpu_reference_jobs(jobs):
    """Times reference chains (genotype arrays, model kwargs, seed, untimed and
    timed sweeps) one after another in one process on one core; returns the
    timed seconds of each job."""
    tmp, spec = [], []
    for geno, mkw, seed, warm, steps in jobs:
        f = tempfile.NamedTemporaryFile(suffix=".npy", delete=False)
        np.save(f.name, np.ascontiguousarray(geno, np.int32))
        tmp.append(f.name)
        spec.append((f.name, mkw, seed, warm, steps))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_ref_jobs_worker, args=(q, spec, 0))
    p.start()
    res = None
    while res is None:
        try:
            res = q.get(timeout=5)
        except Exception:
            if not p.is_alive() and p.exitcode not in (0, None):
                raise RuntimeError(f"reference worker exited with code {p.exitcode}")
    p.join()
    for f in tmp:
        os.unlink(f)
    if not isinstance(res, list):
        raise RuntimeError(f"reference worker failed: {res}")
    return res


def _timed(stream, fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def _observed_copies(packed, N):
    L = packed.shape[0]
    codes = (packed[:, :, None] >> (2 * np.arange(16, dtype=np.uint32))[None, None, :]) & 3
    return int(2 * (codes.reshape(L, -1)[:, :N] != 3).sum())


def _alu_roofline(copies_by_kclass, zpass_ms, sm_mhz):
    """ALU roofline of the Z pass: (2K+2) FP32 + ~10 integer (Philox/4) + 1/2 log
    per allele copy at each chain's K class, against 148 SM x 128 lanes."""
    ops = sum(c * (2 * kc + 2 + 10 + 0.5) for kc, c in copies_by_kclass)
    ach = ops / (zpass_ms / 1e3) / 1e12
    peak = 148 * 128 * sm_mhz * 1e6 / 1e12
    return {"bound": "alu", "achieved": round(ach, 3), "peak": round(peak, 2), "unit": "Top/s",
            "frac": round(ach / peak, 4), "kernel": "zpass_b2g_kernel (per K class)",
            "avg_zpass_ms_per_sweep": round(zpass_ms, 4),
            "note": "(2K+2) FP32 + ~10 int (Philox/4) + 0.5 log per allele copy at the K "
                    "class; peak = 148 SM x 128 lanes x median SM clock; Z-pass time from "
                    "a profiled pass of the same sweeps (CUDA events per launch)"}


def _kernel_share(prof):
    tot = max(1e-9, sum(v[0] for v in prof.values()))
    return {k: round(v[0] / tot, 4) for k, v in prof.items()}


def measure_config1(with_cpu=True):
    """Config 1: N=200, L=100 microsatellite-like loci (2-10 alleles, 5% of
    copies missing), K=3 admixture model, independent frequencies (lambda=1),
    alpha inferred; the whole run of 1,000 burn-in + 10,000 sweeps of one
    chain, on the device and on the reference's CPU code."""
    import torch
    from structure_b200 import api, synth
    d = synth.microsat()
    geno, na = d["geno"], d["numalleles"]
    N, _, L = geno.shape
    K, burn, reps = 3, 1000, 10000
    mk = dict(maxpops=K, burnin=burn, numreps=reps, freqscorr=0, inferalpha=1, alpha=1.0,
              unifprioralpha=1, alphamax=10.0, alphapropsd=0.025, metrofreq=10, computeprob=1)
    ctx = api.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    data = api.Data(ctx, na, geno=geno)
    c = api.Chain(ctx, data, api.model_defaults(**mk), 1001)
    b = api.Batch(ctx, [c])
    l0 = ctx.launches()
    ms = _timed(stream, lambda: b.sweep(burn + reps))
    launches = ctx.launches() - l0
    c.get(api.F_QSUM)
    st = c.get(api.F_STATS)
    e2e_s = time.perf_counter() - t0
    assert c.sync() == 0
    # per-kernel times from 200 more sweeps launch by launch (CUDA events)
    ctx.profile(True)
    ctx.profile_read()
    b.sweep(200)
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    copies = int((geno >= 0).sum())
    sweeps = burn + reps
    out = {"workload": "config 1: N=200 L=100 microsatellites (2-10 alleles), K=3, "
                       "1,000 + 10,000 sweeps, one chain",
           "value": round(sweeps / (ms / 1e3), 1), "unit": "sweeps/s",
           "run_s": round(ms / 1e3, 4), "z_updates_per_s": round(sweeps * copies / (ms / 1e3), 1),
           "e2e": {"value": round(sweeps / e2e_s, 1), "unit": "sweeps/s",
                   "includes": "st_data_upload, st_chain_create, the whole run, QSum and "
                               "stats read back"},
           "gpu_launches": int(launches),
           "kernel_us_per_sweep": {k: round(v[0] * 1e3 / 200, 2) for k, v in prof.items()},
           "mean_lnpd": round(st[api.ST_SUMLIKES] / max(1, st[api.ST_NLIKE]), 3),
           "roofline": {"bound": "launch", "achieved_us_per_sweep": round(ms * 1e3 / sweeps, 2),
                        "kernels_per_sweep": round(launches / sweeps, 2),
                        "note": "4e4 allele copies per sweep: each sweep is a few "
                                "microsecond-scale kernels replayed from a CUDA graph, so "
                                "launch latency bounds it, not HBM or the ALUs"}}
    b.close(); c.close(); data.close(); ctx.close()
    if with_cpu:
        A = int(na.max())
        mkw = dict(N=N, L=L, K=K, maxalleles=A, freqscorr=0, inferalpha=1, alpha=1.0,
                   unifprioralpha=1, alphamax=10.0, alphapropsd=0.025, metrofreq=10,
                   burnin=burn, numreps=reps, lambda_=1.0)
        (dt,) = cpu_reference_jobs([(geno, mkw, 1001, 0, sweeps)])
        out["cpu_baseline"] = {"value": round(sweeps / dt, 2), "unit": "sweeps/s",
                               "cores": 1, "kind": "reference",
                               "sample": "the whole run (1,000 + 10,000 sweeps) of one "
                                         "reference chain", "cpu_model": cpu_model()}
    return out


def measure_config3(steps, warmup, with_cpu=True):
    """Config 3: 40 chains = K in 1..10 x 4 seeds, seed s on data set s of
    (N, L) = (300, 5000), (1000, 10000), (2500, 20000), (4000, 8000) (true
    K=4, F_k ~ U[0.02, 0.2]), batched (one launch per update step and K class,
    CUDA graphs, autotuned tiles) against the same chains one at a time."""
    import torch
    from structure_b200 import api, synth
    sets = synth.config3_datasets(want_int32=False)
    ctx = api.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    datas = [api.Data(ctx, d["numalleles"], packed=d["packed"], num_inds=d["N"], num_loci=d["L"],
                      layout=api.LAYOUT_B2G) for d in sets]
    mk = lambda K: api.model_defaults(maxpops=K, burnin=warmup, numreps=steps + 40,
                                      freqscorr=1, inferalpha=1, alpha=1.0, metrofreq=10,
                                      fpriormean=0.01, fpriorsd=0.05, computeprob=1)
    spec = [(K, s) for K in range(1, 11) for s in range(4)]
    chains = [api.Chain(ctx, datas[s], mk(K), 3000 + 10 * K + s) for K, s in spec]
    b = api.Batch(ctx, chains)
    b.autotune()
    b.sweep(warmup)
    clocks = ClockSampler(0)
    l0 = ctx.launches()
    ms = _timed(stream, lambda: b.sweep(steps))
    launches = ctx.launches() - l0
    clk = clocks.stop()
    n = len(chains)
    # Z-pass time per sweep from a profiled pass (CUDA events around each launch)
    ctx.profile(True)
    ctx.profile_read()
    ps = 10
    b.sweep(ps)
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    # plain: each chain alone, replaying its own graphs
    singles = [api.Batch(ctx, [c]) for c in chains]
    for sb in singles:
        sb.sweep(10)
    pms = _timed(stream, lambda: [sb.sweep(10) for sb in singles])
    for c in chains:
        assert c.sync() == 0
    value = n * steps / (ms / 1e3)
    plain = n * 10 / (pms / 1e3)
    cp = [_observed_copies(d["packed"], d["N"]) for d in sets]
    copies = sum(cp[s] for _, s in spec)
    kcl = [(api.fast_class(K), cp[s]) for K, s in spec]
    out = {"workload": "config 3: 40 chains, K=1..10 x 4 seeds over 4 SNP data sets "
                       "(300x5000, 1000x10000, 2500x20000, 4000x8000), F model, batched",
           "value": round(value, 3), "unit": METRIC, "steps": steps, "warmup": warmup,
           "ms_per_step": round(ms / steps, 4),
           "z_updates_per_s": round(value / n * copies, 1),
           "plain": {"value": round(plain, 3), "unit": METRIC,
                     "path": "each chain alone, replaying its own CUDA graphs"},
           "batched_over_plain": round(value / plain, 3),
           "gpu_launches": int(launches),
           "kernel_share": _kernel_share(prof),
           "roofline": _alu_roofline(kcl, prof["zpass"][0] / ps, clk["sm_mhz"] or 1965.0),
           "clocks": clk}
    for sb in singles:
        sb.close()
    b.close()
    for c in chains:
        c.close()
    for d in datas:
        d.close()
    ctx.close()
    if with_cpu:
        # sweep 1 of each of the 40 reference chains (after one untimed sweep)
        # on a slice of at most 1,000 loci, scaled to the chain's L
        jobs, scale = [], []
        for K, s in spec:
            d = sets[s]
            sl = min(d["L"], 1000)
            g = synth.unpack_int32(d["packed"], d["N"], 0, sl)
            jobs.append((g, dict(N=d["N"], L=sl, K=K, maxalleles=2, freqscorr=1,
                                 fpriormean=0.01, fpriorsd=0.05, metrofreq=10, burnin=0,
                                 numreps=100), 3000 + 10 * K + s, 1, 1))
            scale.append(d["L"] / sl)
        dts = cpu_reference_jobs(jobs)
        total = sum(dt * sc for dt, sc in zip(dts, scale))
        out["cpu_baseline"] = {"value": round(n / total, 5), "unit": METRIC, "cores": 1,
                               "kind": "reference",
                               "sample": "sweep 1 of each of the 40 reference chains on a slice "
                                         "of min(L, 1000) loci, scaled to its L; the 40 chains "
                                         "run one after another on one core",
                               "cpu_model": cpu_model()}
    return out


def measure_config4(steps, warmup, with_cpu=True, data=None):
    """Config 4: forward + backward of ln P(D|Q,P) w.r.t. softmax logits,
    N=5000, L=100,000, K=8, FP32, one evaluation per step."""
    import torch
    from structure_b200 import api, synth
    from structure_b200.grad import LogLikGrad
    d = data or synth.snp_fmodel_device(5000, 100000, 8, np.full(8, 0.5), 0.2, 0.0,
                                        synth.DATA_SEED_BASE + 4, indep_beta=(0.5, 0.5))
    N, L, K = d["N"], d["L"], 8
    ctx = api.Context(0)
    dd = api.Data(ctx, d["numalleles"], packed=d["packed"], num_inds=N, num_loci=L,
                  layout=api.LAYOUT_B2G)
    ev = LogLikGrad(ctx, dd, K, precision=32)
    g = torch.Generator(device="cuda").manual_seed(4)
    ql = torch.randn(N, K, device="cuda", generator=g)
    pl = torch.randn(L, K, 2, device="cuda", generator=g)
    for _ in range(warmup):
        ev(ql, pl)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    stream = torch.cuda.current_stream()
    ms = _timed(stream, lambda: [ev(ql, pl) for _ in range(steps)]) / steps
    clk = clocks.stop()
    geno_obs = _observed_copies(d["packed"], N) // 2
    flops = geno_obs * 2 * (4 * K) * 2         # two passes x (2K + 2K FMA) x 2 FLOP
    sm_mhz = clk["sm_mhz"] or 1965.0
    peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    ach = flops / (ms / 1e3) / 1e12
    qh, ph = ql.cpu().pin_memory(), pl.cpu().pin_memory()
    t0 = time.perf_counter()
    for _ in range(steps):
        ll, dq, dp = ev(qh.to("cuda", non_blocking=True), ph.to("cuda", non_blocking=True))
        ll.cpu(); dq.cpu(); dp.cpu()
    e2e = steps / (time.perf_counter() - t0)
    out = {"workload": "config 4: differentiation N=5000 L=100000 K=8 (forward + backward, "
                       "softmax logits, FP32)",
           "metric": "loglik+gradient evaluations/s", "value": round(1e3 / ms, 3),
           "unit": "evals/s", "steps": steps, "warmup": warmup, "ms_per_step": round(ms, 4),
           "genotypes_per_s": round(geno_obs * 1e3 / ms, 1),
           "roofline": {"bound": "fp32-fma", "achieved": round(ach, 3), "peak": round(peak, 2),
                        "unit": "TFLOP/s", "frac": round(ach / peak, 4),
                        "note": "4K FMA per genotype per pass, two passes; peak = 148 SM x "
                                "128 lanes x 2 x median SM clock (no tensor cores: the "
                                "contraction is K=8 wide)"},
           "e2e": {"value": round(e2e, 3), "unit": "evals/s",
                   "h2d_bytes_per_step": int(qh.nbytes + ph.nbytes),
                   "d2h_bytes_per_step": int(8 + qh.nbytes + ph.nbytes)},
           "gpu_launches": 6 * steps, "clocks": clk,
           "data": "synthetic, seeded: config 4's generative model drawn on the GPU "
                   "(synth.snp_fmodel_device)"}
    del ev
    dd.close()
    ctx.close()
    if with_cpu:
        # the FP64 CPU restatement of the same forward + backward (the oracle;
        # the reference has no gradient) on a 1,000-locus slice, scaled by L
        from oracle.oracle import Oracle
        sl = 1000
        gs = synth.unpack_int32(d["packed"], N, 0, sl)
        rng = np.random.default_rng(4)
        qn, pn = rng.standard_normal((N, K)), rng.standard_normal((sl, K, 2))
        orc = Oracle()
        t0 = time.perf_counter()
        orc.loglik_grad(gs, qn, pn)
        dt = (time.perf_counter() - t0) * L / sl
        out["cpu_baseline"] = {"value": round(1.0 / dt, 5), "unit": "evals/s", "cores": 1,
                               "kind": "port",
                               "sample": "one FP64 forward + backward of the oracle's "
                                         "restatement on a 1,000-locus slice, scaled by L",
                               "cpu_model": cpu_model()}
    return out


def measure_config5(steps, warmup, with_cpu=True, loci=500000):
    """Config 5: N=10,000, L=500,000 (2-bit packed, 1.25 GB), 2% missing, K=10 F
    model with F_k ~ U[0.01, 0.3], POPALPHAS=1, Q ~ Dir(0.1); 8 replicate chains
    batched on one GPU under the context's HBM admission budget.  `loci` < 500,000
    runs the same model on fewer loci (a shape small enough for a profiler capture)."""
    import torch
    from structure_b200 import api, synth
    N, L, K, B = 10000, int(loci), 10, 8
    rng = np.random.default_rng(synth.DATA_SEED_BASE + 5)
    F = rng.uniform(0.01, 0.3, K)
    d = synth.snp_fmodel_device(N, L, K, F, 0.1, 0.02, synth.DATA_SEED_BASE + 5)
    ctx = api.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    data = api.Data(ctx, d["numalleles"], packed=d["packed"], num_inds=N, num_loci=L,
                    layout=api.LAYOUT_B2G)
    mk = dict(maxpops=K, burnin=warmup, numreps=steps + 40, freqscorr=1, inferalpha=1,
              popalphas=1, alpha=1.0, metrofreq=10, fpriormean=0.01, fpriorsd=0.05,
              computeprob=1)
    chains = [api.Chain(ctx, data, api.model_defaults(**mk), 5000 + r) for r in range(B)]
    used, budget = ctx.memory()
    b = api.Batch(ctx, chains)
    b.sweep(warmup)
    clocks = ClockSampler(0)
    l0 = ctx.launches()
    ms = _timed(stream, lambda: b.sweep(steps))
    launches = ctx.launches() - l0
    clk = clocks.stop()
    ctx.profile(True)
    ctx.profile_read()
    ps = 10
    b.sweep(ps)
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    # plain: each chain alone, replaying its own graphs (captured by untimed
    # sweeps first), ten sweeps each with one Metropolis sweep among them
    singles = [api.Batch(ctx, [c]) for c in chains]
    for sb in singles:
        sb.sweep(10)
    pms = _timed(stream, lambda: [sb.sweep(10) for sb in singles])
    for sb in singles:
        sb.close()
    for c in chains:
        assert c.sync() == 0
    copies = _observed_copies(d["packed"], N)
    value = B * steps / (ms / 1e3)
    plain = B * 10 / (pms / 1e3)
    out = {"workload": f"config 5: N=10000 L={L} K=10 F model, POPALPHAS=1, 8 chains batched",
           "value": round(value, 3), "unit": METRIC, "steps": steps, "warmup": warmup,
           "ms_per_step": round(ms / steps, 3), "z_updates_per_s": round(value * copies, 1),
           "plain": {"value": round(plain, 3), "unit": METRIC,
                     "path": "each chain alone, replaying its own CUDA graphs"},
           "batched_over_plain": round(value / plain, 3),
           "hbm_in_use_gb": round(used / 1e9, 2), "hbm_budget_gb": round(budget / 1e9, 2),
           "gpu_launches": int(launches),
           "kernel_share": _kernel_share(prof),
           "roofline": _alu_roofline([(api.fast_class(K), B * copies)], prof["zpass"][0] / ps,
                                     clk["sm_mhz"] or 1965.0),
           "data": "synthetic, seeded: config 5's generative model drawn on the GPU "
                   "(synth.snp_fmodel_device)",
           "clocks": clk}
    b.close()
    for c in chains:
        c.close()
    data.close()
    ctx.close()
    if with_cpu:
        sl = 1000
        g = synth.unpack_int32(d["packed"], N, 0, sl)
        mkw = dict(N=N, L=sl, K=K, maxalleles=2, freqscorr=1, popalphas=1, fpriormean=0.01,
                   fpriorsd=0.05, metrofreq=10, burnin=0, numreps=100)
        (dt,) = cpu_reference_jobs([(g, mkw, 5000, 1, 1)])
        out["cpu_baseline"] = {"value": round(1.0 / (dt * L / sl), 6), "unit": METRIC,
                               "cores": 1, "kind": "reference",
                               "sample": "sweep 1 of one reference chain on a 1,000-locus slice "
                                         f"(N=10,000, K=10), scaled by {L:,}/1,000 loci",
                               "cpu_model": cpu_model()}
    return out


def _print_workload(name, res, steps, warmup):
    out = {"metric": res.get("metric", METRIC), "value": res["value"], "unit": res["unit"],
           "n_gpus": 1, "steps": steps, "warmup": warmup, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None,
           "dtype": "f32" if name == "grad" else "f32 (Z/P/Q) + f64 (MH ratios, lnP(D))",
           "data": res.get("data", "synthetic, seeded"), "config": {"workload": res["workload"]}}
    out.update({k: v for k, v in res.items() if k not in out and k != "workload"})
    print(json.dumps(out), flush=True)


def run_grad(args):
    _print_workload("grad", measure_config4(args.steps, args.warmup, not args.no_cpu_baseline),
                    args.steps, args.warmup)


def run_scale(args):
    _print_workload("scale", measure_config5(args.steps, args.warmup, not args.no_cpu_baseline,
                                             args.scale_loci),
                    args.steps, args.warmup)


def run_uneven(args):
    _print_workload("uneven", measure_config3(args.steps, args.warmup, not args.no_cpu_baseline),
                    args.steps, args.warmup)


def run_small(args):
    _print_workload("small", measure_config1(not args.no_cpu_baseline), 1, 0)


def other_configs(with_cpu):
    """The other configurations, measured briefly for the default bench line."""
    out = {}
    for key, fn in (("config1", lambda: measure_config1(with_cpu)),
                    ("config3", lambda: measure_config3(20, 3, with_cpu)),
                    ("config4", lambda: measure_config4(10, 3, with_cpu)),
                    ("config5", lambda: measure_config5(10, 3, with_cpu))):
        try:
            out[key] = fn()
        except Exception as e:  # reported in the line, never hides the headline
            out[key] = {"error": repr(e)[:300]}
    return out


def run_mala(args):
    """Config 4 mixing: Gibbs chain vs Gibbs + Langevin-on-Q chain, ESS per
    second of device time for ln P(D) and for Q (median over entries)."""
    from structure_b200 import api, synth
    d = synth.snp_fmodel_device(5000, 100000, 8, np.full(8, 0.5), 0.2, 0.0,
                                synth.DATA_SEED_BASE + 4, indep_beta=(0.5, 0.5))
    N, L, K = d["N"], d["L"], 8
    ctx = api.Context(0)
    data = api.Data(ctx, d["numalleles"], packed=d["packed"], num_inds=N, num_loci=L,
                    layout=api.LAYOUT_B2G)
    burn, reps = max(args.warmup, 100), max(args.steps, 200)
    sel = np.random.default_rng(0).choice(N, 64, replace=False)
    res = {}
    for name, mala in (("gibbs", 0), ("gibbs+mala", 1)):
        m = api.model_defaults(maxpops=K, burnin=burn, numreps=reps, freqscorr=0, inferalpha=1,
                               alpha=1.0, metrofreq=10, mala=mala)
        c = api.Chain(ctx, data, m, 4000)
        c.sweep(burn)
        c.sync()
        lnl, qs, t = [], [], 0.0
        for _ in range(reps):
            c.sweep(1)
            c.sync()
            t += c.timing_ms()
            lnl.append(c.get(api.F_STATS)[api.ST_LIKE])
            qs.append(c.get(api.F_Q)[sel])
        qs = np.array(qs).reshape(reps, -1)
        ess_l = _ess(lnl)
        ess_q = float(np.median([_ess(qs[:, j]) for j in range(qs.shape[1])]))
        st = c.get(api.F_STATS)
        res[name] = {"sweeps": reps, "device_s": round(t / 1e3, 4),
                     "ms_per_sweep": round(t / reps, 4),
                     "ess_lnpd": round(ess_l, 1), "ess_lnpd_per_s": round(ess_l / (t / 1e3), 2),
                     "ess_q_median": round(ess_q, 1),
                     "ess_q_per_s": round(ess_q / (t / 1e3), 2),
                     "mean_lnpd": round(float(np.mean(lnl)), 2)}
        if mala:
            res[name]["mala_acceptance"] = round(st[api.ST_MALA_ACC] / st[api.ST_MALA_TRIES], 4)
        c.close()
    out = {"metric": "ESS/s of ln P(D) and Q (Gibbs vs Gibbs + Langevin on Q)",
           "value": res["gibbs+mala"]["ess_q_per_s"], "unit": "ESS/s (Q, median)",
           "n_gpus": 1, "steps": reps, "warmup": burn, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32 (Z/P/Q) + f64 (MH)",
           "data": "synthetic, seeded (config 4 generator)",
           "config": {"workload": "mixing N=5000 L=100000 K=8, independent frequencies",
                      "selected_q": "64 individuals x 8"},
           "chains": res}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the brief measurements of configs 1, 3, 4 and 5 that the "
                         "default line carries under other_configs")
    ap.add_argument("--scale-loci", type=int, default=500000,
                    help="loci of the scale workload (config 5 has 500,000; fewer for a "
                         "profiler capture of the same model)")
    ap.add_argument("--workload", default="snp",
                    choices=["snp", "small", "grad", "mala", "scale", "uneven"],
                    help="snp: the headline (default); small: config 1 whole run; grad: "
                         "config 4 forward+backward; mala: config 4 ESS/s, Gibbs vs "
                         "Gibbs+Langevin; scale: config 5; uneven: config 3 batched vs one "
                         "chain at a time")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload != "snp" and args.impl == "ours":
        {"grad": run_grad, "mala": run_mala, "scale": run_scale, "small": run_small,
         "uneven": run_uneven}[args.workload](args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
