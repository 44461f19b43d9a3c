"""Whole runs against the reference: posterior summaries agree within Monte
Carlo standard error.

The device chains and the reference's own CPU chains (tests/golden/mcse_*.npz,
made by tests/golden/make_mcse.py with the reference functions compiled from
its sources) use different random streams and different Dirichlet samplers,
so single draws cannot be compared; whole runs are compared through their
summaries instead: mean and variance of ln P(D), mean alpha, mean F (F model),
mean lambda (INFERLAMBDA) and the posterior-mean Q.  Eight chains per side; each summary's standard
error comes from the spread over chains.  Population labels are arbitrary in
every chain, so each chain's labels are first matched to the generating Q.

Bounds: |difference| <= 5 pooled standard errors for the scalar summaries;
for Q, every entry within 6 pooled standard errors (floor 0.002) and a mean
absolute difference under 0.01.
"""
import itertools
import os

import numpy as np
import pytest

from structure_b200 import api

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    z = np.load(os.path.join(GOLDEN, f"mcse_{name}.npz"))
    model = {k[len("model_"):]: z[k].item() for k in z.files if k.startswith("model_")}
    return z, model


def _align(Qm, Qtrue):
    K = Qm.shape[1]
    return np.array(max(itertools.permutations(range(K)),
                        key=lambda p: float((Qm[:, list(p)] * Qtrue).sum())))


def _summaries(sumlikes, sumsqlikes, QSum, sumAlpha, FstSum, n, Qtrue):
    out = {"lnL_mean": [], "lnL_var": [], "alpha": [], "F": [], "Q": []}
    K = QSum.shape[2]
    for c in range(len(sumlikes)):
        m = sumlikes[c] / n
        out["lnL_mean"].append(m)
        out["lnL_var"].append(sumsqlikes[c] / n - m * m)
        # one alpha, or (LOCPRIOR) the mean of the global row over populations,
        # which does not depend on the chain's labels
        out["alpha"].append(sumAlpha[c][:K].mean() / n)
        perm = _align(QSum[c] / n, Qtrue)
        out["Q"].append(QSum[c][:, perm] / n)
        out["F"].append(FstSum[c][perm] / n)
    return {k: np.array(v) for k, v in out.items()}


def _z(a, b, floor=0.0):
    se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b) + floor * floor)
    return np.abs(a.mean(0) - b.mean(0)) / np.maximum(se, 1e-300)


def _run_device(ctx, z, model, mala=0):
    geno = z["geno"].astype(np.int32)
    K = int(z["K"])
    R = len(z["sumlikes"])
    data = api.Data(ctx, z["numalleles"], geno=geno,
                    popflags=z["popflags"] if "popflags" in z.files else None,
                    population=z["population"] if "population" in z.files else None,
                    location=z["location"] if "location" in z.files else None)
    mk = dict(maxpops=K, burnin=model["burnin"], numreps=model["numreps"],
              freqscorr=model["freqscorr"], inferalpha=model["inferalpha"], alpha=model["alpha"],
              alphapropsd=model["alphapropsd"], metrofreq=model["metrofreq"],
              lambda_=model["lambda_"], mala=mala)
    for k in ("fpriormean", "fpriorsd", "inferlambda", "noadmix", "admburnin", "usepopinfo",
              "gensback", "migrprior", "locprior"):
        if k in model:
            mk[k] = model[k]
    if "popflag" in model:
        mk["popflag_given"] = model["popflag"]
    chains = [api.Chain(ctx, data, api.model_defaults(**mk), 77000 + r) for r in range(R)]
    b = api.Batch(ctx, chains)
    b.sweep(model["burnin"] + model["numreps"])
    res = dict(sumlikes=[], sumsqlikes=[], QSum=[], sumAlpha=[], FstSum=[], sumlambda=[],
               usepop=[], sumLocPrior=[])
    for c in chains:
        assert c.sync() == 0
        if mala:
            st = c.get(api.F_STATS)
            assert 0.2 < st[api.ST_MALA_ACC] / st[api.ST_MALA_TRIES] < 0.95
        st = c.get(api.F_STATS)
        assert st[api.ST_NLIKE] == model["numreps"]
        res["sumlikes"].append(st[api.ST_SUMLIKES])
        res["sumsqlikes"].append(st[api.ST_SUMSQ])
        res["QSum"].append(c.get(api.F_QSUM))
        res["sumAlpha"].append(c.get(api.F_SUMALPHA))
        res["FstSum"].append(c.get(api.F_FSTSUM))
        res["sumlambda"].append(c.get(api.F_SUMLAMBDA))
        if model.get("usepopinfo"):
            res["usepop"].append(c.get(api.F_USEPOPPROBS))
        if model.get("locprior"):
            res["sumLocPrior"].append(c.get(api.F_SUMLOCPRIOR))
    b.close()
    for c in chains:
        c.close()
    data.close()
    return {k: np.array(v) for k, v in res.items()}


@pytest.mark.parametrize("name,mala", [("c1", 0), ("c1l", 0), ("c1n", 0), ("c1p", 0),
                                       ("c1lp", 0), ("c1nlp", 0), ("c2s", 0), ("c2s", 1)])
def test_whole_runs_agree_with_reference_within_mcse(ctx, name, mala):
    """mala=1: the same chains with the Langevin move on Q added to every
    sweep still sample the reference's posterior."""
    z, model = _load(name)
    n = model["numreps"]
    Qtrue = z["Qtrue"]
    dev = _run_device(ctx, z, model, mala)
    sd = _summaries(dev["sumlikes"], dev["sumsqlikes"], dev["QSum"], dev["sumAlpha"],
                    dev["FstSum"], n, Qtrue)
    sr = _summaries(z["sumlikes"], z["sumsqlikes"], z["QSum"], z["sumAlpha"], z["FstSum"], n,
                    Qtrue)
    report = {k: (sd[k].mean(0), sr[k].mean(0)) for k in ("lnL_mean", "lnL_var", "alpha")}
    print(f"\n{name}: device vs reference (mean over chains; z = |diff| / pooled SE)")
    for k in ("lnL_mean", "lnL_var", "alpha"):
        print(f"  {k:9s} {sd[k].mean():14.4f} {sr[k].mean():14.4f}  z={float(_z(sd[k], sr[k])):.2f}")
    if model["freqscorr"]:
        print("  F        ", sd["F"].mean(0), sr["F"].mean(0), "z", _z(sd["F"], sr["F"]))
    for k in ("lnL_mean", "lnL_var", "alpha"):
        assert _z(sd[k], sr[k]) <= 5.0, (k, report)
    if model["freqscorr"]:
        assert (_z(sd["F"], sr["F"]) <= 5.0).all(), (sd["F"].mean(0), sr["F"].mean(0))
    if model.get("inferlambda"):
        ld, lr = dev["sumlambda"][:, 0] / n, z["sumlambda"][:, 0] / n
        print("  lambda   ", ld.mean(), lr.mean(), "z", float(_z(ld, lr)))
        assert _z(ld, lr) <= 5.0, (ld.mean(), lr.mean())
    if model.get("usepopinfo"):
        # posterior probability of the given population (UsePopProbs, gen 0)
        # of the flagged individuals, summed over the collecting sweeps
        f = z["popflags"].astype(bool)
        hp = z["population"][f] - 1
        ud = dev["usepop"][..., 0][:, f][:, np.arange(f.sum()), hp] / n
        ur = z["usepop"][..., 0][:, f][:, np.arange(f.sum()), hp] / n
        zu = _z(ud, ur, floor=0.002)
        print("  P(home)  ", ud.mean(), ur.mean(), "max z", zu.max())
        assert zu.max() <= 6.0
    if model.get("locprior"):
        # r, the concentration of the location priors (LocPrior[0])
        rd, rr = dev["sumLocPrior"][:, 0] / n, z["sumLocPrior"][:, 0] / n
        print("  r        ", rd.mean(), rr.mean(), "z", float(_z(rd, rr)))
        assert _z(rd, rr) <= 5.0, (rd.mean(), rr.mean())
    zq = _z(sd["Q"], sr["Q"], floor=0.002)
    assert zq.max() <= 6.0, zq.max()
    assert np.abs(sd["Q"].mean(0) - sr["Q"].mean(0)).mean() <= 0.01
