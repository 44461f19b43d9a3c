"""Pins of the oracle restatement (oracle/st_oracle.c) against the reference's
own CPU functions (pmelsted/structure src/*.c, built into oracle/_ref by
oracle/Makefile and driven with controlled rand()/RNormal streams).

These run on the CPU.  Deterministic pieces must agree exactly (or to the last
few ulps where the summation order differs); Metropolis updates fed the same
normals and uniforms must make the same moves; the Dirichlet samplers differ in
algorithm (reference: Ripley/Cheng-Feast gamma; build: Marsaglia-Tsang) and are
compared in distribution.
"""
import math

import numpy as np
import pytest

from structure_b200 import synth
from oracle.oracle import S_ALPHA, S_EPS, S_FST, S_INITZ, rnd_words

KEY = 0x1234ABCD5678


def _microsat(N, L, K, seed):
    d = synth.microsat(N=N, L=L, K=K, seed=seed)
    return d["geno"], d["numalleles"]


def _snp(N, L, K, seed):
    d = synth.snp_fmodel(N, L, K, np.linspace(0.05, 0.25, K), 0.4, 0.03, seed)
    return d["geno"], d["numalleles"]


def _state(rng, N, L, K, na, qa=0.7):
    A = int(max(1, na.max()))
    Q = rng.dirichlet(np.full(K, qa), N)
    P = np.zeros((L, K, A))
    for l in range(L):
        if na[l] > 0:
            P[l, :, :na[l]] = rng.dirichlet(np.ones(na[l]), K)
    return Q.astype(np.float32).astype(np.float64), P.astype(np.float32).astype(np.float64)


def test_philox_known_answers(orc):
    # Random123 philox4x32_10 known-answer vectors
    assert [hex(x) for x in orc.philox([0, 0, 0, 0], 0)] == \
        ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(x) for x in orc.philox([0xffffffff] * 4, 0xffffffffffffffff)] == \
        ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(x) for x in orc.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                                       0x299f31d0a4093822)] == \
        ["0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def test_lgamma_matches_reference_mylgamma(orc, ref):
    zs = np.concatenate([np.linspace(1e-4, 8, 400), np.logspace(-4, 6, 400)])
    for z in zs:
        assert orc.lgamma(z) == ref.lib.mylgamma(z)


@pytest.mark.parametrize("K,seed", [(1, 1), (2, 2), (3, 3), (6, 4), (10, 5), (17, 6), (32, 7)])
def test_updatez_f64_matches_reference(orc, ref, K, seed):
    geno, na = _microsat(40, 30, 3, seed)
    N, _, L = geno.shape
    rng = np.random.default_rng(seed)
    Q, P = _state(rng, N, L, K, na)
    u = rng.random(N * L * 2)
    ref.set_globals(N=N, L=L, K=K, maxalleles=P.shape[2])
    zr = np.zeros_like(geno)
    ref.lib.UpdateZ(zr, Q, P, geno.copy(), u)
    zo, flags = orc.zupdate_f64_injected(geno, Q, P, u)
    assert (zo == zr).all() and flags == 0


@pytest.mark.parametrize("pfonly", [0, 1])
def test_counts_match_reference(orc, ref, pfonly):
    geno, na = _microsat(50, 25, 3, 9)
    N, _, L = geno.shape
    K, A = 4, int(na.max())
    rng = np.random.default_rng(9)
    Z = rng.integers(0, K, size=geno.shape).astype(np.int32)
    Z[geno < 0] = -9
    pf = (rng.random(N) < 0.5).astype(np.int32)
    ref.set_globals(N=N, L=L, K=K, maxalleles=A, pfrompopflagonly=pfonly)
    nr = np.zeros(L * K * A, np.int32)
    ref.lib.GetNumFromPops(nr, geno.copy(), Z, na.astype(np.int32), ref.individuals(N, pf))
    no, mo = orc.counts(geno, Z, K, A, popflags=pf, pfrompopflagonly=pfonly)
    assert (nr.reshape(L, K, A) == no).all()
    tmp = np.zeros(K, np.int32)
    for i in range(N):
        ref.lib.GetNumLociPop(tmp, Z, i)
        assert (tmp == mo[i]).all()


def test_initializez_matches_reference(orc, ref):
    geno, na = _microsat(30, 20, 3, 4)
    N, _, L = geno.shape
    K = 5
    zi = orc.init_z(geno, K, KEY)
    vals = []
    for i in range(N):
        for line in range(2):
            for l in range(L):
                if geno[i, line, l] >= 0:
                    w = orc.stream(l, i >> 1, 0, S_INITZ, KEY)
                    vals.append(int(w[2 * (i & 1) + line]) >> 1)
    ref.set_globals(N=N, L=L, K=K, maxalleles=int(na.max()))
    ref.rand_queue(vals)
    zr = np.zeros_like(geno)
    ref.lib.InitializeZ(geno.copy(), ref.individuals(N), zr)
    ref.rand_queue(None)
    assert (zr == zi).all()


@pytest.mark.parametrize("freqscorr", [0, 1])
def test_initfreqpriors_matches_reference(orc, ref, freqscorr):
    geno, na = _microsat(30, 20, 3, 5)
    N, _, L = geno.shape
    K, A = 3, int(na.max())
    ref.set_globals(N=N, L=L, K=K, maxalleles=A, freqscorr=freqscorr, fpriormean=0.02,
                    lambda_=1.0)
    er = np.zeros(L * A)
    fr = np.zeros(K)
    ref.lib.InitFreqPriors(er, fr, geno.copy(), na.astype(np.int32))
    eo, fo = orc.init_eps(geno, na, A, freqscorr, 1.0, 0.02, K)
    np.testing.assert_array_equal(eo.reshape(-1)[np.arange(L * A) % A < np.repeat(na, A)],
                                  er[np.arange(L * A) % A < np.repeat(na, A)])
    np.testing.assert_array_equal(fo, fr)


@pytest.mark.parametrize("K", [1, 4, 9, 20])
def test_calclike_and_metro_logdiff_match_reference(orc, ref, K):
    geno, na = _snp(60, 200, 3, 6)
    N, _, L = geno.shape
    rng = np.random.default_rng(6 + K)
    Q, P = _state(rng, N, L, K, na)
    T, _ = _state(rng, N, L, K, na)
    ref.set_globals(N=N, L=L, K=K, maxalleles=P.shape[2])
    lr = ref.lib.CalcLike(geno.copy(), None, Q, P, None, None, None)
    assert orc.calc_like(geno, Q, P) == lr
    ld = orc.metro_logdiff(geno, Q.astype(np.float32), T.astype(np.float32), P.astype(np.float32))
    for i in range(N):
        r = ref.lib.CalcLikeIndDiff(geno.copy(), None, T[i].copy(), Q[i].copy(), P, i, None)
        assert abs(r - ld[i]) <= 1e-9 * max(1.0, abs(r))


def test_estlogprob_matches_reference(orc, ref):
    for s, ss, n in [(-1000.0, 1e6 + 50.0, 1), (-5000.0, 2.5e6 + 900, 10), (-1.2e8, 7.2e15, 500)]:
        assert orc.est_logprob(s, ss, n) == ref.lib.EstLogProb(s, ss, n) or n == 1


@pytest.mark.parametrize("popalphas,unif", [(0, 1), (1, 1), (0, 0), (1, 0)])
def test_updatealpha_matches_reference(orc, ref, popalphas, unif):
    N, K = 150, 4
    rng = np.random.default_rng(popalphas * 2 + unif)
    Q = rng.dirichlet(np.full(K, 0.6), N).astype(np.float32)
    logQ = np.log(Q.astype(np.float64)).astype(np.float32)
    Qd = np.exp(logQ.astype(np.float64))          # so that log(Q) == logQ as the oracle sees it
    alpha = np.array([0.7, 0.9, 0.5, 1.3])[:K] if popalphas else np.full(K, 0.8)
    S, T = orc.alpha_sums(logQ)
    for rep in range(8):
        a_o, lpd = orc.update_alpha(N, S, T, alpha, KEY, rep, popalphas, unif, 10.0, 0.2,
                                    2.0, 0.5)
        nal = K if popalphas else 1
        normals = [orc.normal(p, rep, S_ALPHA, KEY) for p in range(nal)]
        rands = []
        for p in range(nal):
            newa = alpha[p] + 0.2 * normals[p]
            if newa > 0 and (newa < 10.0 or not unif):
                rands += rnd_words(orc.stream(p, 1, rep, S_ALPHA, KEY))
        ref.set_globals(N=N, L=1, K=K, maxalleles=2, popalphas=popalphas, unifprioralpha=unif,
                        alphapropsd=0.2, alphamax=10.0, alphapriora=2.0, alphapriorb=0.5)
        ar = alpha.copy()
        ref.normal_queue(normals)
        ref.rand_queue(rands)
        ref.lib.UpdateAlpha(Qd.copy(), ar, ref.individuals(N), rep)
        ref.rand_queue(None)
        ref.normal_queue(None)
        np.testing.assert_allclose(ar, a_o, rtol=1e-13)
        alpha = a_o


@pytest.mark.parametrize("lam", [1.0, 0.5])
def test_updateepsilon_matches_reference(orc, ref, lam):
    geno, na = _microsat(60, 40, 3, 12)
    N, _, L = geno.shape
    K, A = 3, int(na.max())
    rng = np.random.default_rng(12)
    _, P = _state(rng, N, L, K, na)
    logP = np.where(P > 0, np.log(np.maximum(P, 1e-300)), 0).astype(np.float32)
    Pd = np.where(P > 0, np.exp(logP.astype(np.float64)), 0)
    eps, F = orc.init_eps(geno, na, A, 1, 1.0, 0.1, K)
    F = np.array([0.05, 0.2, 0.4])
    inv = float(N) ** -0.5
    for rep in range(5):
        e_o, acc = orc.update_eps(na, logP, eps, F, lam, inv, KEY, rep)
        vals = []
        for l in range(L):
            if na[l] > 1:
                w = orc.stream(l, 0, rep, S_EPS, KEY)
                a1 = int(((int(w[0]) >> 1) / 2147483648.0) * na[l])
                a2 = int(((int(w[1]) >> 1) / 2147483648.0) * (na[l] - 1))
                a2 = a2 + 1 if a2 >= a1 else a2
                dl = ((int(w[2]) >> 1) / 2147483648.0) * inv
                vals += [int(w[0]) >> 1, int(w[1]) >> 1, int(w[2]) >> 1]
                if eps[l, a1] + dl < 1.0 and eps[l, a2] - dl > 0.0:
                    vals += rnd_words(orc.stream(l, 1, rep, S_EPS, KEY))
        ref.set_globals(N=N, L=L, K=K, maxalleles=A, freqscorr=1)
        er = eps.copy()
        ref.rand_queue(vals)
        ref.lib.UpdateEpsilon(Pd, er, F.copy(), na.astype(np.int32), lam)
        assert ref.lib.stref_rand_overrun() == 0
        ref.rand_queue(None)
        np.testing.assert_allclose(er, e_o, rtol=1e-12, atol=1e-15)
        assert acc.sum() > 0
        eps = e_o


@pytest.mark.parametrize("onefst", [0, 1])
def test_updatefst_matches_reference(orc, ref, onefst):
    geno, na = _snp(80, 150, 3, 13)
    N, _, L = geno.shape
    K, A = 3, 2
    rng = np.random.default_rng(13)
    _, P = _state(rng, N, L, K, na)
    logP = np.where(P > 0, np.log(np.maximum(P, 1e-300)), 0).astype(np.float32)
    Pd = np.where(P > 0, np.exp(logP.astype(np.float64)), 0)
    eps, _ = orc.init_eps(geno, na, A, 1, 1.0, 0.1, K)
    F = np.array([0.05, 0.2, 0.4]) if not onefst else np.full(K, 0.15)
    Leff = int((na > 0).sum())
    for rep in range(6):
        nf, diff = orc.fst_diffs(na, logP, eps, F, onefst, 0.05, KEY, rep)
        F_o, lpd = orc.update_fst(F, onefst, 0.1, 0.05, Leff, diff, nf, KEY, rep)
        # reference: FlikeFreqs differences agree; UpdateFst makes the same move
        ref.set_globals(N=N, L=L, K=K, maxalleles=A, freqscorr=1, onefst=onefst,
                        fpriormean=0.1, fpriorsd=0.05)
        numfst = 1 if onefst else K
        for j in range(numfst):
            if not (0 < nf[j] < 1):
                continue
            pops = range(K) if onefst else [j]
            dr = sum(ref.lib.FlikeFreqs(nf[j], eps.reshape(-1).copy(), Pd.reshape(-1).copy(),
                                        na.astype(np.int32), p) -
                     ref.lib.FlikeFreqs(F[j], eps.reshape(-1).copy(), Pd.reshape(-1).copy(),
                                        na.astype(np.int32), p) for p in pops)
            npops = K if onefst else 1
            do = diff[j] + Leff * npops * (orc.lgamma((1 - nf[j]) / nf[j]) - orc.lgamma((1 - F[j]) / F[j]))
            assert abs(dr - do) <= 1e-8 * max(1.0, abs(dr))
        normals = [orc.normal(j, rep, S_FST, KEY) for j in range(numfst)]
        rands = []
        for j in range(numfst):
            if 0 < nf[j] < 1 and lpd[j] < 0:
                rands += rnd_words(orc.stream(j, 1, rep, S_FST, KEY))
        Fr = F.copy()
        ref.normal_queue(normals)
        ref.rand_queue(rands)
        ref.lib.UpdateFst(eps.reshape(-1).copy(), Fr, Pd.reshape(-1).copy(), na.astype(np.int32))
        ref.rand_queue(None)
        ref.normal_queue(None)
        np.testing.assert_allclose(Fr, F_o, rtol=1e-14)
        F = F_o


def test_dirichlet_p_matches_reference_in_distribution(orc, ref):
    """Same posterior Dir(lambda + n) from the reference's array-fed UpdateP
    (Ripley / Cheng-Feast gamma) and the oracle's Marsaglia-Tsang draws."""
    L, K, A = 400, 2, 3
    rng = np.random.default_rng(21)
    n = rng.integers(0, 6, size=(L, K, A)).astype(np.int32)
    n[:, 0, :] = [0, 2, 7]
    na = np.full(L, A, np.int32)
    lam = np.full(K, 0.7)
    eps = np.zeros((L, A))
    F = np.full(K, 0.5)
    draws_o, draws_r = [], []
    # reference UpdateP counts from Z itself: a genotype table that reproduces n
    for rep in range(20):
        Po, _, err = orc.update_p(na, n, 0, eps, F, lam, KEY, rep)
        assert err == 0
        draws_o.append(Po.astype(np.float64))
    N = int(n.sum(axis=(1, 2)).max() // 2 + 2)
    geno = np.full((N, 2, L), -9, np.int32)
    Z = np.full((N, 2, L), -9, np.int32)
    for l in range(L):
        c = 0
        for k in range(K):
            for a in range(A):
                for _ in range(n[l, k, a]):
                    geno[c // 2, c % 2, l] = a
                    Z[c // 2, c % 2, l] = k
                    c += 1
    ref.set_globals(N=N, L=L, K=K, maxalleles=A, freqscorr=0, lambda_=0.7)
    ind = ref.individuals(N)
    for rep in range(20):
        u = rng.random(L * K * A * 64)
        P = np.zeros(L * K * A)
        ref.lib.UpdateP(P, eps.reshape(-1).copy(), F.copy(), na, geno, Z, lam.copy(), ind, u)
        draws_r.append(P.reshape(L, K, A))
    do = np.stack(draws_o)[:, :, 0, :].reshape(-1, A)
    dr = np.stack(draws_r)[:, :, 0, :].reshape(-1, A)
    alpha = 0.7 + np.array([0, 2, 7])
    mean = alpha / alpha.sum()
    var = mean * (1 - mean) / (alpha.sum() + 1)
    for x in (do, dr):
        np.testing.assert_allclose(x.mean(0), mean, atol=4 * np.sqrt(var / len(x)).max())
        np.testing.assert_allclose(x.var(0), var, rtol=0.15)


def test_loglik_grad_oracle_matches_finite_differences_and_calclike(orc, ref):
    """The FP64 gradient restatement: ln P(D) equals the reference's CalcLike
    (no clamp is reached here) and central differences match the gradient."""
    from structure_b200 import synth
    d = synth.snp_fmodel(30, 60, 3, np.array([.1, .2, .3]), .5, .05, 3)
    g = d["geno"]
    rng = np.random.default_rng(1)
    ql, pl = rng.normal(size=(30, 3)), rng.normal(size=(60, 3, 2))
    ll, dq, dp, lli = orc.loglik_grad(g, ql, pl)
    Q = np.exp(ql) / np.exp(ql).sum(1, keepdims=True)
    P = np.exp(pl) / np.exp(pl).sum(2, keepdims=True)
    ref.set_globals(N=30, L=60, K=3, maxalleles=2)
    lr = ref.lib.CalcLike(g.copy(), None, Q.copy(), P.copy(), None, None, None)
    assert abs(ll - lr) <= 1e-12 * abs(lr)
    assert abs(lli.sum() - ll) <= 1e-12 * abs(ll)
    h = 1e-6
    for i, k in [(0, 0), (5, 2), (29, 1)]:
        a, b = ql.copy(), ql.copy()
        a[i, k] += h
        b[i, k] -= h
        fd = (orc.loglik_grad(g, a, pl)[0] - orc.loglik_grad(g, b, pl)[0]) / (2 * h)
        assert abs(fd - dq[i, k]) <= 1e-6 * max(1.0, abs(fd))
    for l, k, a_ in [(0, 0, 0), (7, 2, 1), (59, 1, 0)]:
        a, b = pl.copy(), pl.copy()
        a[l, k, a_] += h
        b[l, k, a_] -= h
        fd = (orc.loglik_grad(g, ql, a)[0] - orc.loglik_grad(g, ql, b)[0]) / (2 * h)
        assert abs(fd - dp[l, k, a_]) <= 1e-6 * max(1.0, abs(fd))


@pytest.mark.parametrize("freqscorr,popspecific", [(0, 0), (1, 0), (0, 1)])
def test_update_lambda_matches_reference(orc, ref, freqscorr, popspecific):
    """UpdateLambda / UpdatePopLambda fed the oracle's normals and rand()
    words make the same moves; the oracle's log ratios are the reference's."""
    from structure_b200 import synth
    from oracle.oracle import S_LAMBDA
    d = synth.microsat(N=30, L=50, K=3, seed=12)
    na = d["numalleles"].astype(np.int32)
    L, K, A = len(na), 3, int(na.max())
    rng = np.random.default_rng(4 + freqscorr + 2 * popspecific)
    key, rep = 0x1A3B, 7
    for trial in range(6):
        P = np.zeros((L, K, A))
        for l in range(L):
            P[l, :, :na[l]] = rng.dirichlet(np.full(na[l], 0.8), K)
        logP = np.log(np.maximum(P, 1e-300)).astype(np.float32)
        Pd = np.where(P > 0, np.exp(logP.astype(np.float64)), 0.0)
        eps = np.zeros((L, A))
        for l in range(L):
            eps[l, :na[l]] = rng.dirichlet(np.ones(na[l]) * 3)
        lam = rng.uniform(0.3, 3.0, K) if popspecific else np.full(K, rng.uniform(0.3, 3.0))
        mine, lpd = orc.update_lambda(na, logP, eps, freqscorr, popspecific, lam, key, rep + trial)
        npop = K if popspecific else 1
        normals = [orc.normal(q, rep + trial, S_LAMBDA, key) for q in range(npop)]
        rands = []
        for q in range(npop):
            nw = lam[q] + 0.3 * normals[q]
            if 0 < nw < 10:
                rands += rnd_words(orc.stream(q, 1, rep + trial, S_LAMBDA, key))
        ref.set_globals(N=30, L=L, K=K, maxalleles=A, freqscorr=freqscorr)
        theirs = lam.copy()
        ref.normal_queue(normals)
        ref.rand_queue(rands)
        if popspecific:
            ref.lib.UpdatePopLambda(Pd.copy(), theirs, na)
        else:
            ref.lib.UpdateLambda(Pd.copy(), eps.copy(), theirs, na)
        ref.rand_queue(None)
        ref.normal_queue(None)
        np.testing.assert_array_equal(mine, theirs)


def test_update_q_noadmix_matches_reference(orc, ref):
    """UpdateQNoAdmix (running product of P rescaled below 1e-100, then
    PickAnOption on rand()) fed the oracle's rand() words picks the same
    population for every individual."""
    from structure_b200 import synth
    from oracle.oracle import S_NOADMIX
    d = synth.microsat(N=50, L=80, K=4, seed=21)
    geno, na = d["geno"], d["numalleles"].astype(np.int32)
    N, _, L = geno.shape
    K, A = 4, int(na.max())
    rng = np.random.default_rng(3)
    P = np.zeros((L, K, A))
    for l in range(L):
        P[l, :, :na[l]] = rng.dirichlet(np.full(na[l], 0.9), K)
    logP = np.log(np.maximum(P, 1e-300)).astype(np.float32)
    Pd = np.where(P > 0, np.exp(logP.astype(np.float64)), 0.0)
    key, rep = 0x9A9A, 11
    Qo, _, pick = orc.update_q_noadmix(geno, logP, key, rep)
    words = [int(orc.stream(i, 0, rep, S_NOADMIX, key)[0]) >> 1 for i in range(N)]
    ref.set_globals(N=N, L=L, K=K, maxalleles=A, noadmix=1)
    Qr = np.zeros((N, K))
    ref.rand_queue(words)
    ref.lib.UpdateQNoAdmix(geno.copy(), Qr, Pd.copy(), ref.individuals(N), None, None)
    ref.rand_queue(None)
    np.testing.assert_array_equal(Qr.argmax(1), pick)
    np.testing.assert_array_equal(Qo, Qr.astype(np.float32))
    assert len(set(pick)) > 1


@pytest.mark.parametrize("gensback,migr", [(2, 0.05), (0, 0.3), (3, 0.01)])
def test_update_q_withpops_matches_reference(orc, ref, gensback, migr):
    """UpdateQWithPops (USEPOPINFO migrant model) fed the oracle's rand()
    words: same Q for every flagged individual, same posterior sums."""
    from structure_b200 import synth
    from oracle.oracle import S_POPINFO
    d = synth.microsat(N=40, L=60, K=3, seed=33)
    geno, na = d["geno"], d["numalleles"].astype(np.int32)
    N, _, L = geno.shape
    K, A = 3, int(na.max())
    rng = np.random.default_rng(gensback)
    P = np.zeros((L, K, A), np.float32)
    for l in range(L):
        P[l, :, :na[l]] = rng.dirichlet(np.full(na[l], 0.6), K)
    pop = rng.integers(1, K + 1, N).astype(np.int32)
    flags = (rng.random(N) < 0.6).astype(np.int32)
    Q0 = rng.dirichlet(np.ones(K), N).astype(np.float32)
    key, rep, burnin = 0x7070, 12, 10
    Qo, _, upo = orc.update_q_withpops(geno, P, pop, flags, gensback, migr, key, rep, burnin,
                                       Q0, np.log(Q0))
    words = [int(orc.stream(i, 0, rep, S_POPINFO, key)[0]) >> 1 for i in range(N) if flags[i]]
    ref.set_globals(N=N, L=L, K=K, maxalleles=A, usepopinfo=1, gensback=gensback,
                    migrprior=migr, burnin=burnin, popflag=1)
    Qr = Q0.astype(np.float64).copy()
    up = np.zeros(N * K * (gensback + 1))
    ref.rand_queue(words)
    ref.lib.UpdateQWithPops(geno.copy(), Qr, P.astype(np.float64), None, np.ones(K), rep,
                            ref.individuals_pop(N, flags, pop), up, None)
    ref.rand_queue(None)
    f = flags.astype(bool)
    np.testing.assert_array_equal(Qo[f], Qr[f].astype(np.float32))
    np.testing.assert_array_equal(Qo[~f], Q0[~f])
    np.testing.assert_allclose(upo.reshape(-1), up, rtol=1e-9, atol=1e-12)
    assert (Qr[f] < 1).any() or gensback == 0


def _locations(rng, N, nloc_ids):
    """Raw location ids with gaps (GetNumLocations compacts them, in
    increasing order of id) and the expected myloc."""
    ids = np.sort(rng.choice(np.arange(0, 3 * nloc_ids), nloc_ids, replace=False))
    loc = ids[rng.integers(0, nloc_ids, N)].astype(np.int32)
    loc[:nloc_ids] = ids                      # every id used
    myloc = np.searchsorted(ids, loc).astype(np.int32)
    return loc, myloc


@pytest.mark.parametrize("noadmix", [0, 1])
def test_update_locprior_matches_reference(orc, ref, noadmix):
    """UpdateLocPrior (src/Updates/UpdateLocPrior.c: r, nu and gamma with no
    admixture, r alone with admixture) fed the rand() words the oracle used,
    in the reference's order: the same moves, bit for bit, over 30 sweeps of
    proposals that are accepted and rejected."""
    K, N = 4, 90
    rng = np.random.default_rng(40 + noadmix)
    loc, myloc = _locations(rng, N, 6)
    nloc = int(myloc.max()) + 1
    ref.set_globals(N=N, L=1, K=K, noadmix=noadmix, locprior=1, alphapropsd=0.05,
                    maxlocprior=20.0, locpriorstep=0.4)
    inds, n_ref = ref.individuals_loc(N, loc)      # GetNumLocations reads NUMINDS
    assert n_ref == nloc
    moves = 0
    for trial in range(30):
        if noadmix:
            Q = np.eye(K)[rng.integers(0, K, N)].astype(np.float32)
            locp = np.concatenate([[rng.uniform(0.3, 4.0)], rng.dirichlet(np.ones(K) * 3),
                                   rng.dirichlet(np.ones(K) * 2, nloc).reshape(-1)])
        else:
            Q = rng.dirichlet(np.ones(K), N).astype(np.float32)
            locp = np.array([rng.uniform(0.3, 4.0)])
        alpha = rng.uniform(0.2, 2.0, (nloc + 1) * K)
        mine, words, normals = orc.update_locprior(myloc, Q, alpha, locp, noadmix, 0.05, 0.4,
                                                   20.0, KEY, 100 + trial)
        assert len(normals) == 0
        theirs = locp.copy()
        ref.rand_queue(words)
        ref.lib.UpdateLocPrior(Q.astype(np.float64), theirs, alpha.copy(), inds)
        assert ref.lib.stref_rand_consumed() == len(words)
        assert ref.lib.stref_rand_overrun() == 0
        ref.rand_queue(None)
        np.testing.assert_array_equal(mine, theirs)
        moves += int(np.sum(mine != locp))
    assert moves > 10


def test_update_alpha_locprior_matches_reference(orc, ref):
    """UpdateAlphaLocPrior (src/Updates/UpdateAlpha.c:257-305): global
    alphas, then each location's alphas against the Q of its individuals,
    fed the oracle's normals and rand() words: the same alphas, bit for
    bit."""
    K, N = 3, 80
    rng = np.random.default_rng(77)
    loc, myloc = _locations(rng, N, 5)
    nloc = int(myloc.max()) + 1
    ref.set_globals(N=N, L=1, K=K, noadmix=0, locprior=1, alphapropsd=0.3, alphamax=10.0)
    inds, n_ref = ref.individuals_loc(N, loc)
    assert n_ref == nloc
    moved = 0
    for trial in range(25):
        Q = rng.dirichlet(np.full(K, 0.8), N)
        alpha = rng.uniform(0.2, 3.0, (nloc + 1) * K)
        r = rng.uniform(0.5, 5.0)
        mine, words, normals = orc.update_alpha_locprior(myloc, np.log(Q), alpha, r, 0.3, 10.0,
                                                         KEY, 300 + trial)
        theirs = alpha.copy()
        ref.normal_queue(normals)
        ref.rand_queue(words)
        ref.lib.UpdateAlphaLocPrior(Q.copy(), theirs, np.array([r]), inds)
        assert ref.lib.stref_rand_consumed() == len(words)
        assert ref.lib.stref_normal_consumed() == len(normals) == (nloc + 1) * K
        ref.rand_queue(None)
        ref.normal_queue(None)
        np.testing.assert_array_equal(mine, theirs)
        moved += int(np.sum(mine != alpha))
    assert moved > 20


def test_q_updates_with_location_priors_match_reference(orc, ref):
    """LOCPRIOR in the Q updates: UpdateQNoAdmix starts each individual's
    product at gamma of its location (src/Updates/UpdateQ.c:339-345)."""
    from oracle.oracle import S_NOADMIX
    d = synth.microsat(N=60, L=40, K=3, seed=8)
    geno, na = d["geno"], d["numalleles"].astype(np.int32)
    N, _, L = geno.shape
    K, A = 3, int(na.max())
    rng = np.random.default_rng(9)
    loc, myloc = _locations(rng, N, 4)
    nloc = int(myloc.max()) + 1
    P = np.zeros((L, K, A))
    for l in range(L):
        P[l, :, :na[l]] = rng.dirichlet(np.full(na[l], 0.4), K)
    logP = np.log(np.maximum(P, 1e-300)).astype(np.float32)
    Pd = np.where(P > 0, np.exp(logP.astype(np.float64)), 0.0)
    # strong location priors so that they change picks
    locp = np.concatenate([[1.0], np.ones(K) / K, rng.dirichlet(np.ones(K) * 0.3, nloc).reshape(-1)])
    key, rep = 0x5151, 4
    Qo, _, pick = orc.update_q_noadmix(geno, logP, key, rep, locp=locp, myloc=myloc)
    _, _, pick0 = orc.update_q_noadmix(geno, logP, key, rep)
    words = [int(orc.stream(i, 0, rep, S_NOADMIX, key)[0]) >> 1 for i in range(N)]
    ref.set_globals(N=N, L=L, K=K, maxalleles=A, noadmix=1, locprior=1)
    inds, n_ref = ref.individuals_loc(N, loc)
    assert n_ref == nloc
    Qr = np.zeros((N, K))
    ref.rand_queue(words)
    ref.lib.UpdateQNoAdmix(geno.copy(), Qr, Pd.copy(), inds, locp.ctypes.data, None)
    ref.rand_queue(None)
    np.testing.assert_array_equal(Qr.argmax(1), pick)
    assert (pick != pick0).any()


def test_fp32_ln_and_sincos_series(orc):
    """The FP32 logarithm and sine/cosine the P draws use (atanh and Taylor
    series after exact range reductions) against libm in double: within
    2 ulp (relative 2.4e-7) for ln away from 1, 1e-6 absolute near 1, and
    1.2e-7 absolute for sin and cos of 2 pi u."""
    xs = np.concatenate([np.geomspace(2.0 ** -24, 1.0, 4001), np.linspace(0.5, 2.0, 4001),
                         np.geomspace(1.0, 1e6, 401)]).astype(np.float32)
    for x in xs:
        ref_v = math.log(float(x))
        got = orc.ln_f32(float(x))
        assert abs(got - ref_v) <= max(2.4e-7 * abs(ref_v), 1e-6), (x, got, ref_v)
    for u in np.linspace(0.0, 1.0, 8001)[:-1].astype(np.float32):
        sn, cs = orc.sincos_2pi_f32(float(u))
        assert abs(sn - math.sin(2 * math.pi * float(u))) <= 1.2e-7
        assert abs(cs - math.cos(2 * math.pi * float(u))) <= 1.2e-7


@pytest.mark.parametrize("a", [0.05, 0.5, 1.0, 2.5, 10.0, 100.0, 4000.0])
def test_fp32_gamma_draws_in_distribution(orc, a):
    """The FP32 Marsaglia-Tsang draw of the P update against Gamma(a, 1):
    Kolmogorov-Smirnov on the draws, and the mean and variance of their
    logarithm (digamma and trigamma of a) with standard errors from the
    sample's own fourth moment; from small shapes (the U^(1/a) boost) to the
    counts of large samples (the series form of the acceptance test)."""
    from scipy import special, stats
    n = 20000
    lg = np.array([orc.loggamma_f32(a, e, 3, 7, KEY + int(a * 1000))[0] for e in range(n)],
                  np.float64)
    assert stats.kstest(np.exp(lg), stats.gamma(a).cdf).pvalue > 1e-4
    s2 = special.polygamma(1, a)
    zm = (lg.mean() - special.digamma(a)) / math.sqrt(s2 / n)
    d = lg - lg.mean()
    zv = (lg.var() - s2) / math.sqrt((d ** 4).mean() / n - lg.var() ** 2 / n)
    assert abs(zm) < 4.5 and abs(zv) < 4.5, (zm, zv)
