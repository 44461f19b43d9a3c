"""Parity at the benchmarked shapes.

The other parity tests run at N <= 1,024 individuals, where one Z-pass tile
covers every individual of a locus block.  These build chains the way
bench.py does (N=2000, L=50,000 biallelic SNPs, K=5 F model, 20 chains in one
batch, Z-pass tiles chosen by st_batch_autotune, warm-up sweeps as burn-in)
and check collecting sweeps of that batch against the oracle and the
reference's own CalcLike (src/CalcLike.c:387-426) for the first and the last
chain; then the multi-chunk tiles of K classes 9-12 (K=10, N=2600) and 24
(two-warp CTAs).

Checked per sweep and chain: the allele and ancestry counts of the Z pass
bit-exact against GetNumFromPops/GetNumLociPop of the oracle's Z on the same
Q, P and stream; ln P(D) within 1e-5 relative of the reference's CalcLike;
on the Metropolis sweep the log ratios within the derived FP32 bound of the
oracle's FP64 sums, and the accept decisions equal outside that band; on the
Gibbs sweep P and Q against the oracle's draws from the counts the device
held before the sweep.  The measured errors are printed (pytest -s or -rP).
"""
import numpy as np
import pytest

import bench
from conftest import check_metro_decisions, metro_terms_and_bound, metro_uniforms
from structure_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def config2():
    return synth.config2(N=bench.WL["N"], L=bench.WL["L"], want_int32=True)


def _bench_batch(ctx, d, nchains, mk, seed0):
    data = api.Data(ctx, d["numalleles"], packed=d["packed"], num_inds=d["N"], num_loci=d["L"],
                    layout=api.LAYOUT_B2G)
    chains = [api.Chain(ctx, data, api.model_defaults(**mk), seed0 + r) for r in range(nchains)]
    b = api.Batch(ctx, chains)
    b.autotune()
    return data, chains, b


def _check_counts_and_like(orc, ref, geno, c, seed, rep, tag):
    """Counts of the Z pass at sweep `rep` on the chain's final Q and P, and its
    ln P(D), against the oracle and the reference.  Returns the relative
    ln P(D) error."""
    Q, P = c.get(api.F_Q), c.get(api.F_P)
    zo = orc.zupdate_f32(geno, Q, P, seed, rep)
    n_o, m_o = orc.counts(geno, zo, c.K, c.A)
    n_d, m_d = c.get(api.F_N), c.get(api.F_M)
    assert (n_d == n_o).all(), f"{tag}: {(n_d != n_o).sum()} allele counts differ"
    assert (m_d == m_o).all(), f"{tag}: {(m_d != m_o).sum()} ancestry counts differ"
    N, _, L = geno.shape
    ref.set_globals(N=N, L=L, K=c.K, maxalleles=c.A)
    lr = ref.lib.CalcLike(geno, None, Q.astype(np.float64), P.astype(np.float64), None, None,
                          None)
    like = c.get(api.F_STATS)[api.ST_LIKE]
    rel = abs(like - lr) / abs(lr)
    assert rel <= 1e-5, (tag, like, lr)
    return rel


def test_config2_batch_sweeps_match_oracle(ctx, orc, ref, config2):
    d = config2
    geno, na = d["geno"], d["numalleles"]
    N, B = d["N"], bench.WL["chains"]
    burn = 10
    mk = bench.model_kwargs(burnin=burn, numreps=20)
    data, chains, b = _bench_batch(ctx, d, B, mk, 2000)
    dims = chains[0].get(api.F_DIMS)
    assert dims[6] > 1, "the tile must split the individuals into several chunks"
    b.sweep(burn)                       # reps 0..9; rep 10 is a Metropolis sweep
    check = (0, B - 1)
    keep = (api.F_Q, api.F_N, api.F_EPS, api.F_F, api.F_LAMBDA)
    before = {j: {f: chains[j].get(f) for f in keep} for j in check}
    b.sweep(1)                          # rep 10: P, Metropolis Q, Z (+ ln P(D)), alpha, eps, F
    for c in chains:
        assert c.sync() == 0
    report = {}
    for j in check:
        c, seed = chains[j], 2000 + j
        assert c.get(api.F_REP) == burn + 1
        rel = _check_counts_and_like(orc, ref, geno, c, seed, burn, f"chain {j} rep {burn}")
        # P drawn from the counts before the sweep
        s0 = before[j]
        Po, _, err = orc.update_p(na, s0[api.F_N], 1, s0[api.F_EPS], s0[api.F_F],
                                  s0[api.F_LAMBDA], seed, burn)
        assert err == 0
        P = c.get(api.F_P)
        np.testing.assert_allclose(P, Po, rtol=1e-5, atol=1e-30)
        # the FP32 gamma draws (counts up to 2N = 4,000: the series form of the
        # acceptance test) are the oracle's bits; P agrees to an ulp or two
        ulps = np.abs(P.view(np.int32).astype(np.int64) - Po.view(np.int32).astype(np.int64))
        assert ulps.max() <= 2, int(ulps.max())
        # the Metropolis step: log ratios of TestQ against the Q before the sweep
        T = c.get(api.F_TESTQ)
        ld_dev = c.get(api.F_LOGDIFF)
        ld_o = orc.metro_logdiff(geno, s0[api.F_Q], T, P)
        _, mag, bound = metro_terms_and_bound(geno, s0[api.F_Q], T, P)
        err_ld = np.abs(ld_dev - ld_o)
        assert (err_ld <= bound).all(), (err_ld / bound).max()
        u = metro_uniforms(orc, N, seed, burn)
        inband, flips = check_metro_decisions(ld_dev, ld_o, bound, u)
        report[j] = dict(lnpd_rel=rel, ld_abs_max=float(err_ld.max()),
                         ld_rel_max=float((err_ld / np.maximum(np.abs(ld_o), 1e-300)).max()),
                         ld_err_over_bound=float((err_ld / bound).max()), inband=inband,
                         flips=flips, accepted=int((np.log(u) < ld_o).sum()),
                         p_ulps_max=int(ulps.max()))
    # rep 11: a Gibbs sweep, Q drawn from the counts of rep 10
    before = {j: {f: chains[j].get(f) for f in (api.F_M, api.F_ALPHA)} for j in check}
    b.sweep(1)
    for j in check:
        c, seed = chains[j], 2000 + j
        Qo, _, err = orc.update_q_gibbs(before[j][api.F_M], before[j][api.F_ALPHA], seed, burn + 1)
        np.testing.assert_allclose(c.get(api.F_Q), Qo, rtol=1e-5, atol=1e-35)
        report[j]["lnpd_rel_rep11"] = _check_counts_and_like(orc, ref, geno, c, seed, burn + 1,
                                                             f"chain {j} rep {burn + 1}")
    print("config 2 batch, measured errors:", report)
    b.close()
    for c in chains:
        c.close()
    data.close()


def test_config2_fp64_quantities_against_the_oracle(ctx, orc, config2):
    """The FP64 quantities of one config-2 chain against the oracle's FP64
    restatement on the same FP32 inputs: ln P(D) (reference-checked in the
    test above), the alpha sums of log Q, the per-population F log ratios and
    the lambda log ratio.  Prints the measured relative errors."""
    d = config2
    geno, na = d["geno"], d["numalleles"]
    N, L, K = d["N"], d["L"], 5
    mk = bench.model_kwargs(burnin=2, numreps=10)
    mk.update(inferlambda=1)
    data = api.Data(ctx, na, packed=d["packed"], num_inds=N, num_loci=L, layout=api.LAYOUT_B2G)
    c = api.Chain(ctx, data, api.model_defaults(**mk), 2000)
    c.sweep(3)
    assert c.sync() == 0
    rep = c.get(api.F_REP)
    errs = {}
    like = c.CalcLike()
    lo = orc.calc_like(geno, c.get(api.F_Q), c.get(api.F_P))
    errs["lnpd"] = abs(like - lo) / abs(lo)
    assert errs["lnpd"] <= 1e-5
    # alpha: S_k = sum_i log Q_ik and T = sum log max(Q, sqrt(1e-100))
    c.UpdateAlpha()
    st = c.get(api.F_STATS)
    S_o, T_o = orc.alpha_sums(c.get(api.F_LOGQ))
    errs["alpha_S"] = float(np.max(np.abs(st[api.ST_ALPHA_S:api.ST_ALPHA_S + K] - S_o) / np.abs(S_o)))
    errs["alpha_T"] = abs(st[api.ST_ALPHA_T] - T_o) / abs(T_o)
    assert errs["alpha_S"] <= 1e-11 and errs["alpha_T"] <= 1e-11
    # lambda: the log ratio of the proposal over loci and populations
    lam0 = c.get(api.F_LAMBDA)
    logP, eps = c.get(api.F_LOGP), c.get(api.F_EPS)
    c.UpdateLambda()
    lpd = c.get(api.F_STATS)[api.ST_LAMBDA_LPD]
    _, lpo = orc.update_lambda(na, logP, eps, 1, 0, lam0, 2000, rep)
    if np.isfinite(lpo[0]):
        errs["lambda_lpd"] = abs(lpd - lpo[0]) / max(abs(lpo[0]), 1e-300)
        assert errs["lambda_lpd"] <= 1e-9
    # F: per-population sum over loci of FlikeFreqs(F') - FlikeFreqs(F)
    F0 = c.get(api.F_F)
    c.UpdateFst()
    st = c.get(api.F_STATS)
    nf, diff = orc.fst_diffs(na, logP, c.get(api.F_EPS), F0, 0, bench.WL["fpriorsd"], 2000, rep)
    ok = (nf > 0) & (nf < 1)
    dd = st[api.ST_FST_DIFF:api.ST_FST_DIFF + K]
    if ok.any():
        errs["fst_diff"] = float(np.max(np.abs(dd[ok] - diff[ok]) /
                                        np.maximum(np.abs(diff[ok]), 1e-300)))
        assert errs["fst_diff"] <= 1e-9
    print("config 2 chain, FP64 quantities vs the oracle (relative error):", errs)
    c.close()
    data.close()


@pytest.mark.parametrize("N,L,K,B", [(2600, 20000, 10, 4), (1500, 10000, 24, 3)])
def test_multichunk_k_classes_match_oracle(ctx, orc, ref, N, L, K, B):
    """K=10 (class 9-12 tiles sized for 110 KB of shared memory, two CTAs per
    SM) and K=24 (two-warp CTAs) with several chunks of individuals per locus
    block, batched and autotuned: counts bit-exact, ln P(D) within 1e-5."""
    d = synth.snp_fmodel(N, L, K, np.linspace(0.02, 0.3, K), 0.2, 0.02, 77 + K)
    geno = d["geno"]
    mk = dict(maxpops=K, burnin=2, numreps=10, freqscorr=1, inferalpha=1, alpha=1.0,
              metrofreq=10, fpriormean=0.01, fpriorsd=0.05, computeprob=1)
    data, chains, b = _bench_batch(ctx, d, B, mk, 7000 + 10 * K)
    dims = chains[0].get(api.F_DIMS)
    assert dims[6] > 1, f"K={K}: one chunk of individuals only ({dims})"
    b.sweep(3)
    rels = []
    for j in (0, B - 1):
        c = chains[j]
        assert c.sync() == 0
        rels.append(_check_counts_and_like(orc, ref, geno, c, 7000 + 10 * K + j, 2,
                                           f"K={K} chain {j}"))
    print(f"K={K} N={N} L={L}: tile chunks x groups = {dims[6]} x {dims[7]}, "
          f"ln P(D) relative errors {rels}")
    b.close()
    for c in chains:
        c.close()
    data.close()
