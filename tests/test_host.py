"""Host-side checks that need no GPU: the C ABI library exports everything
include/stgpu.h declares, the multi-rank timing plumbing over gloo, and the
reference CPU chain driver."""
import os
import re
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "stgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(st_[a-z0-9_]+)\s*\(", src)))


def test_cabi_library_exports_every_declared_symbol():
    import ctypes
    from structure_b200 import api
    lib = ctypes.CDLL(api.LIB_PATH)
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.st_version() == 10000


def test_cabi_reports_no_device_without_gpu():
    import torch
    from structure_b200 import api
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.StError) as e:
        api.Context(0)
    assert e.value.code == api.ST_ERR_NODEVICE


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from structure_b200 import dist as sd
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    r, w, lr = sd.rank_env()
    seeds = sd.chain_seeds(r, 20)
    ms = 10.0 + 5.0 * r                       # per-rank device time
    mx = sd.max_over_ranks(ms)
    tot = sd.sum_over_ranks(len(seeds))
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, w, seeds, mx, tot))


def test_multirank_timing_and_seeds_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(30)
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    assert all(r[3] == 15.0 for r in res)           # max over ranks
    assert all(r[4] == 40.0 for r in res)           # chains over ranks
    assert not set(res[0][2]) & set(res[1][2])      # disjoint chain seeds


def test_reference_chain_driver_runs(ref):
    """The reference's CPU sweep (structure.c order) on a small data set."""
    from structure_b200 import synth
    from oracle.oracle import ref_model
    d = synth.microsat(N=30, L=12, K=2, seed=3)
    m = ref_model(N=30, L=12, K=2, maxalleles=int(d["numalleles"].max()), metrofreq=5,
                  burnin=3, numreps=6, freqscorr=1, fpriormean=0.05, fpriorsd=0.05)
    ch = ref.chain_new(m, d["geno_raw"], seed=11)
    ref.lib.stref_chain_sweeps(ch, 9)
    v = ref.chain_view(ch, 30, 12, 2)
    ref.lib.stref_chain_free(ch)
    assert v["rep"] == 9 and np.isfinite(v["sumlikes"]) and v["sumlikes"] < 0
    np.testing.assert_allclose(v["QSum"].sum(1), 6.0, rtol=1e-9)
    assert (v["Geno"] == d["geno"]).all()      # the reference's recoding == synth.recode


def test_get_into_caller_array_checks_type_and_size(monkeypatch):
    """Chain.get(f, out=...) hands the caller's array to st_get_state and
    refuses, before any library call, one of the wrong type, size or layout."""
    from structure_b200 import api

    calls = []

    class FakeLib:
        def st_field_bytes(self, h, f):
            return 6 * 8

        def st_get_state(self, h, f, ptr, n):
            calls.append((ptr, n))
            return 0

    class FakeCtx:
        def check(self, rc):
            assert rc == 0

    monkeypatch.setattr(api, "lib", lambda: FakeLib())
    c = api.Chain.__new__(api.Chain)
    c.h, c.ctx = 1, FakeCtx()
    monkeypatch.setattr(c, "_shape", lambda f: (2, 3), raising=False)
    buf = np.empty(6, np.float64)
    got = c.get(api.F_QSUM, out=buf)
    assert got.shape == (2, 3) and np.shares_memory(got, buf)
    assert calls == [(buf.ctypes.data, 48)]
    for bad in (np.empty(7), np.empty(6, np.float32), np.empty(12)[::2]):
        with pytest.raises(api.StError) as e:
            c.get(api.F_QSUM, out=bad)
        assert e.value.code == api.ST_ERR_ARG
    assert len(calls) == 1


def test_bench_reference_arm_line(ref):
    """`bench.py --impl reference` runs the reference's CPU functions for the
    requested warm-up and timed sweeps and prints one JSON line in the bench
    contract (same metric and workload as the GPU arm, no host-device bytes)."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, WORLD_SIZE="1", RANK="0")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2",
                        "--warmup", "3"], cwd=root, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "chain-sweeps/s"
    assert d["steps"] == 2 and d["warmup"] == 3 and d["value"] > 0
    assert d["higher_is_better"] is True
    assert d["config"]["workload"].startswith("snp-fmodel N=2000 L=50000 K=5")
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_bench_reads_the_committed_z_pass_profile():
    """The bench's roofline keys take the Z pass's DRAM bytes per launch and its
    warp instructions per 32 genotypes from the committed ncu summary; both
    lines must be there and plausible (traffic at least the 25 MB genotype
    array, fewer than 200 instructions per 32 genotypes)."""
    import importlib.util
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    traffic = bench.read_traffic()
    inst = bench.read_profile_figure("inst_per_32_genotypes")
    assert traffic is not None and traffic >= 25e6
    assert inst is not None and 32 < inst < 200
    assert bench.read_profile_figure("no_such_figure") is None
