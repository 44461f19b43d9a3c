"""Regenerate tests/golden/mcse_*.npz: full reference runs for the Monte Carlo
standard-error comparison of whole chains.

    python tests/golden/make_mcse.py

Needs oracle/_ref/libstref.so (oracle/Makefile builds it from the reference
sources).  Each reference chain runs the reference's own CPU updates in the
order of src/structure.c:497-685 (oracle/ref_driver.c), with the reference's
rand()/RNormal() fed by a seeded xorshift stream, one chain per process (the
reference keeps its model in process globals).  Per chain the fixture keeps
the run's summaries: sumlikes, sumsqlikes, QSum, sumAlpha, FstSum and the
number of collected sweeps, together with the recoded genotypes the GPU chains
are run on.

Runs:
  c1  -- N=200, L=100 multi-allelic loci (2..10 alleles), K=3, 5% copies
         missing; admixture, alpha inferred, independent frequencies, lambda=1;
         1,000 burn-in + 10,000 sweeps; 8 chains.
  c1l -- the same data and run with lambda inferred (INFERLAMBDA=1).
  c1n -- the same data under the no-admixture model (NOADMIX=1, ADMBURNIN=500);
         24 chains (the variance of ln P(D) varies more between chains here).
  c1p -- the same data with prior population information for half of the
         individuals (USEPOPINFO=1, populations = the generating Q's largest
         component, GENSBACK=2, MIGRPRIOR=0.05).
  c1lp -- the same data with sampling locations (LOCPRIOR=1, admixture: an
         alpha vector per location); locations = 3 x the generating Q's
         largest component + a coin flip (six location ids with gaps).
  c1nlp -- the same locations under the no-admixture model with LOCPRIOR (r,
         nu and per-location gamma); 24 chains.
  c2s -- N=200, L=1,000 biallelic SNPs, K=3 F model (F = .10, .20, .30), 3%
         genotypes missing; alpha and F inferred; 2,000 burn-in + 4,000 sweeps;
         8 chains.
"""
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from structure_b200 import synth  # noqa: E402

CHAINS = 8


def runs():
    c1 = synth.microsat(N=200, L=100, K=3, seed=synth.DATA_SEED_BASE + 1)
    c2 = synth.snp_fmodel(200, 1000, 3, np.array([0.10, 0.20, 0.30]), 0.5, 0.03,
                          synth.DATA_SEED_BASE + 2)
    loc = (3 * c1["Q"].argmax(1) + (np.random.default_rng(6).random(200) < 0.5)).astype(np.int32)
    return {
        "c1": dict(geno=c1["geno"], raw=c1["geno_raw"], numalleles=c1["numalleles"], Q=c1["Q"],
                   K=3, model=dict(burnin=1000, numreps=10000, freqscorr=0, inferalpha=1,
                                   alpha=1.0, alphapropsd=0.025, metrofreq=10, lambda_=1.0)),
        "c1l": dict(geno=c1["geno"], raw=c1["geno_raw"], numalleles=c1["numalleles"], Q=c1["Q"],
                    K=3, model=dict(burnin=1000, numreps=10000, freqscorr=0, inferalpha=1,
                                    alpha=1.0, alphapropsd=0.025, metrofreq=10, lambda_=1.0,
                                    inferlambda=1)),
        "c1n": dict(geno=c1["geno"], raw=c1["geno_raw"], numalleles=c1["numalleles"], Q=c1["Q"],
                    K=3, model=dict(burnin=1000, numreps=10000, freqscorr=0, inferalpha=1,
                                    alpha=1.0, alphapropsd=0.025, metrofreq=10, lambda_=1.0,
                                    noadmix=1, admburnin=500), chains=24),
        "c1p": dict(geno=c1["geno"], raw=c1["geno_raw"], numalleles=c1["numalleles"], Q=c1["Q"],
                    K=3, model=dict(burnin=1000, numreps=10000, freqscorr=0, inferalpha=1,
                                    alpha=1.0, alphapropsd=0.025, metrofreq=10, lambda_=1.0,
                                    usepopinfo=1, popflag=1, gensback=2, migrprior=0.05),
                    population=(c1["Q"].argmax(1) + 1).astype(np.int32),
                    popflags=(np.random.default_rng(5).random(200) < 0.5).astype(np.int32)),
        "c1lp": dict(geno=c1["geno"], raw=c1["geno_raw"], numalleles=c1["numalleles"], Q=c1["Q"],
                     K=3, model=dict(burnin=1000, numreps=10000, freqscorr=0, inferalpha=1,
                                     alpha=1.0, alphapropsd=0.025, metrofreq=10, lambda_=1.0,
                                     locprior=1), location=loc),
        "c1nlp": dict(geno=c1["geno"], raw=c1["geno_raw"], numalleles=c1["numalleles"],
                      Q=c1["Q"], K=3,
                      model=dict(burnin=1000, numreps=10000, freqscorr=0, inferalpha=1,
                                 alpha=1.0, alphapropsd=0.025, metrofreq=10, lambda_=1.0,
                                 noadmix=1, admburnin=500, locprior=1),
                      location=loc, chains=24),
        "c2s": dict(geno=c2["geno"], raw=c2["geno"], numalleles=c2["numalleles"], Q=c2["Q"],
                    K=3, model=dict(burnin=2000, numreps=4000, freqscorr=1, inferalpha=1,
                                    alpha=1.0, alphapropsd=0.025, metrofreq=10, lambda_=1.0,
                                    fpriormean=0.01, fpriorsd=0.05)),
    }


def _chain(job):
    name, r, raw, K, model, pf, pp, lc = job
    from oracle.oracle import RefLib, ref_model
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)                     # the reference prints to stdout
    ref = RefLib()
    N, _, L = raw.shape
    m = ref_model(N=N, L=L, K=K, maxalleles=2, **model)
    ch = ref.chain_new(m, raw, popflags=pf, population=pp, location=lc,
                       seed=1000 * (2 if name == "c2s" else 1) + r)
    ref.lib.stref_chain_sweeps(ch, model["burnin"] + model["numreps"])
    v = ref.chain_view(ch, N, L, K, model.get("gensback", 2))
    out = dict(sumlikes=v["sumlikes"], sumsqlikes=v["sumsqlikes"], QSum=v["QSum"],
               sumAlpha=v["sumAlpha"], FstSum=v["FstSum"], Alpha=v["Alpha"], Fst=v["Fst"],
               sumlambda=v["sumlambda"])
    if v["usepop"] is not None:
        out["usepop"] = v["usepop"]
    if v["sumLocPrior"] is not None:
        out["sumLocPrior"] = v["sumLocPrior"]
    return out


def main():
    ctx = mp.get_context("spawn")
    only = sys.argv[1:]
    for name, run in runs().items():
        if only and name not in only:
            continue
        nch = run.get("chains", CHAINS)
        jobs = [(name, r, run["raw"], run["K"], run["model"], run.get("popflags"),
                 run.get("population"), run.get("location")) for r in range(nch)]
        with ctx.Pool(min(nch, os.cpu_count() or 1)) as pool:
            res = pool.map(_chain, jobs)
        out = {k: np.array([x[k] for x in res]) for k in res[0]}
        np.savez_compressed(os.path.join(HERE, f"mcse_{name}.npz"),
                            geno=run["geno"].astype(np.int8), numalleles=run["numalleles"],
                            Qtrue=run["Q"], K=run["K"], nlike=run["model"]["numreps"],
                            **({"popflags": run["popflags"], "population": run["population"]}
                               if "population" in run else {}),
                            **({"location": run["location"]} if "location" in run else {}),
                            **{f"model_{k}": v for k, v in run["model"].items()}, **out)
        print(name, "lnL means", out["sumlikes"] / run["model"]["numreps"])


if __name__ == "__main__":
    main()
