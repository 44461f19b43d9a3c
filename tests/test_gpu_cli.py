"""stgpu_structure end to end: mainparams / extraparams and a data file in, a
run of the GPU chain, OUTFILE_f out, for multi-allelic data (one byte per
allele copy) and for biallelic data (2 bits per genotype).  The file format
itself is checked byte for byte against the reference's writer in
tests/test_frontend.py; here the run's numbers are checked for sense."""
import os
import re
import subprocess

import numpy as np
import pytest

from test_frontend import _scenario

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "structure_b200", "stgpu_structure")


def _snp_data(d, p):
    s = __import__("structure_b200.synth", fromlist=["synth"])
    g = s.snp_fmodel(p["N"], p["L"], 3, np.array([0.1, 0.2, 0.3]), 0.4, 0.02, 5)["geno"]
    rows = []
    for i in range(p["N"]):
        for line in range(2):
            rows.append(" ".join([f"s{i}", str(1 + i % 3)] + [str(v) for v in g[i, line]]))
    with open(os.path.join(d, p["infile"]), "w") as f:
        f.write("\n".join(rows) + "\n")


@pytest.mark.parametrize("kind", ["microsat", "snp", "usepopinfo", "locprior", "locprior-noadmix",
                                  "intermedsave"])
def test_cli_run_writes_results(tmp_path, kind):
    d = str(tmp_path)
    if kind == "usepopinfo":
        return _usepopinfo_run(d)
    if kind.startswith("locprior"):
        return _locprior_run(d, kind.endswith("noadmix"))
    if kind == "intermedsave":
        return _intermedsave_run(d)
    if kind == "microsat":
        p = _scenario(d, N=60, L=30, burnin=200, numreps=600, updatefreq=200, echodata=1,
                      printnet=1)
    else:
        p = _scenario(d, N=80, L=300, burnin=200, numreps=600, updatefreq=200, markernames=0)
        _snp_data(d, p)
    r = subprocess.run([CLI, "-D", "99"], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Final results printed to file results_f" in r.stdout
    # the screen trace: a line after every UPDATEFREQ-th sweep, Ln Like once
    # collecting (the line format itself is pinned in tests/test_frontend.py)
    lines = re.findall(r"^\s*(\d+):    (.*)$", r.stdout, re.M)
    assert [int(x) for x, _ in lines] == [200, 400, 600, 800]
    assert "BURNIN completed" in r.stdout and " Rep#:   " in r.stdout
    like = [float(t.split()[-2]) for x, t in lines if int(x) > 202]
    assert len(like) == 3 and all(np.isfinite(v) and v < 0 for v in like)
    if kind == "microsat":
        assert 'Data file "data file.str" (truncated) --' in r.stdout
        assert lines[0][1].count(".") == 1 + 3 + 3    # alpha, F1..F3, D1,2 D1,3 D2,3
    text = open(os.path.join(d, "results_f")).read()
    for section in ("Run parameters:", "Proportion of membership", "Net nucleotide distance",
                    "Estimated Ln Prob of Data", "Inferred ancestry of individuals:",
                    "Estimated Allele Frequencies in each cluster",
                    "Values of parameters used in structure:"):
        assert section in text, section
    lnp = float(re.search(r"Estimated Ln Prob of Data   = (\S+)", text).group(1))
    mean = float(re.search(r"Mean value of ln likelihood = (\S+)", text).group(1))
    assert np.isfinite(lnp) and lnp <= mean < 0
    assert "   600 Reps" in text
    rows = re.findall(r"^\s*\d+\s+\S+\s+\(\s*\d+\)\s+\d+ :\s+((?:[0-9.]+ ){3})", text, re.M)
    assert len(rows) == p["N"]
    q = np.array([[float(x) for x in row.split()] for row in rows])
    np.testing.assert_allclose(q.sum(1), 1.0, atol=0.003)
    fst = [float(x) for x in re.findall(r"Mean value of Fst_\d+\s+= (\S+)", text)]
    assert len(fst) == 3 and all(0 < f < 1 for f in fst)
    assert "SEED=99" in text
    assert open(os.path.join(d, "seed.txt")).read().strip() == "99"


def _usepopinfo_run(d):
    """USEPOPINFO=1 with a POPFLAG column: individuals i % 2 == 1 carry prior
    information; population 4 is outside 1..3, so those lose it with a
    warning.  Flagged rows print the migrant-model posterior, the others Q."""
    p = _scenario(d, N=60, L=30, burnin=200, numreps=600, updatefreq=200, usepopinfo=1,
                  popflag=1)
    r = subprocess.run([CLI, "-D", "7"], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    pops = [1 + i % 4 for i in range(p["N"])]
    flagged = [i % 2 == 1 and pops[i] <= 3 for i in range(p["N"])]
    assert r.stdout.count("Warning: population prior for individual") == \
        sum(i % 2 == 1 and pops[i] == 4 for i in range(p["N"]))
    text = open(os.path.join(d, "results_f")).read()
    assert "USEPOPINFO turned on" in text and "MIGRPRIOR = 0.0500" in text
    assert "Probability of being from assumed population | prob of other pops" in text
    rows = re.findall(r"^\s*(\d+)\s+\S+\s+\(\s*\d+\)\s+\d+ :  (.*)$", text, re.M)
    assert len(rows) == p["N"]
    for idx, body in rows:
        i = int(idx) - 1
        if flagged[i]:
            ph = float(body.split("|")[0])
            groups = re.findall(r"Pop \d+: ((?:[0-9.]+ ){3})", body)
            others = [float(v) for g in groups for v in g.split()]
            assert len(others) == 2 * 3
            assert ph + sum(others) == pytest.approx(1.0, abs=0.01)
        else:
            q = [float(x) for x in body.split()[:3]]
            assert sum(q) == pytest.approx(1.0, abs=0.003)


def _locprior_run(d, noadmix):
    """LOCPRIOR=1 with a LOCDATA column (location ids 5, 8, 11)."""
    p = _scenario(d, N=60, L=30, burnin=200, numreps=600, updatefreq=200, locprior=1,
                  locdata=1, noadmix=int(noadmix))
    r = subprocess.run([CLI, "-D", "11"], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    text = open(os.path.join(d, "results_f")).read()
    assert "LOCPRIOR model used" in text
    rv = float(re.search(r"Mean value of r = (\S+)", text).group(1))
    assert 0 < rv < 20                                   # MAXLOCPRIOR
    if noadmix:
        assert "NO ADMIXTURE model assumed" in text
        nu = [float(x) for x in re.search(r"Mean value of nu = (.*)$", text, re.M).group(1).split()]
        assert len(nu) == 3 and sum(nu) == pytest.approx(1.0, abs=1e-3)
        rows = re.findall(r"^\tlocation\s+(\d+):((?:\s+[0-9.]+){3})$", text, re.M)
        assert [int(x) for x, _ in rows] == [5, 8, 11]
        for _, g in rows:
            assert sum(float(v) for v in g.split()) == pytest.approx(1.0, abs=1e-3)
    else:
        assert "Mean value of alpha_local for each location:" in text
        rows = re.findall(r"^\tlocation\s+(\d+):((?:\s+[0-9.]+){3})$", text, re.M)
        assert [int(x) for x, _ in rows] == [5, 8, 11]


def _intermedsave_run(d):
    """INTERMEDSAVE=2 writes results_1 and results_2 after 200 and 400 of the
    600 collected sweeps (src/structure.c:640-660); PRINTLIKES=1 prints one ln
    likelihood per sweep (src/output.c:187-200)."""
    p = _scenario(d, N=40, L=20, burnin=100, numreps=600, updatefreq=100, intermedsave=2,
                  printlikes=1)
    r = subprocess.run([CLI, "-D", "5"], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    for k, reps in ((1, 200), (2, 400)):
        text = open(os.path.join(d, f"results_{k}")).read()
        assert f"   {reps} Reps" in text
        assert "Estimated Ln Prob of Data" in text
    assert not os.path.exists(os.path.join(d, "results_3"))
    assert "   600 Reps" in open(os.path.join(d, "results_f")).read()
    likes = re.findall(r"^\s*(-\d+)$", r.stdout, re.M)
    assert len(likes) == p["burnin"] + p["numreps"]
    assert all(float(x) < 0 for x in likes)
