"""USEPOPINFO on the device against the oracle's restatement of
UpdateQWithPops (pinned to the reference in test_oracle_pins.py): the
migrant-model Q of flagged individuals and the posterior sums, on both
genotype layouts; flagged individuals kept by the Gibbs update and by the
Metropolis test, left out of the alpha sums; initial Z at the given
populations."""
import numpy as np
import pytest

from structure_b200 import api, synth

pytestmark = pytest.mark.gpu

SEED = 0x504F5049


def _setup(ctx, layout, K=3, burnin=5):
    if layout == api.LAYOUT_U8:
        d = synth.microsat(N=120, L=300, K=K, seed=41)
        geno, na = d["geno"], d["numalleles"]
        N, L = geno.shape[0], geno.shape[2]
        Qt = d["Q"]
    else:
        d = synth.snp_fmodel(160, 900, K, np.linspace(0.1, 0.3, K), 0.3, 0.03, 42)
        geno, na = d["geno"], d["numalleles"]
        N, L = 160, 900
        Qt = d["Q"]
    rng = np.random.default_rng(layout)
    pop = (Qt.argmax(1) + 1).astype(np.int32)
    pop[rng.random(N) < 0.05] = K + 1                 # out of range: unflagged by the engine
    flags = (rng.random(N) < 0.5).astype(np.int32)
    if layout == api.LAYOUT_U8:
        data = api.Data(ctx, na, geno=geno, layout=layout, popflags=flags, population=pop)
    else:
        data = api.Data(ctx, na, packed=d["packed"], layout=layout, num_inds=N, num_loci=L,
                        popflags=flags, population=pop)
    m = api.model_defaults(maxpops=K, burnin=burnin, numreps=20, usepopinfo=1, popflag_given=1,
                           gensback=2, migrprior=0.05, metrofreq=4)
    eff = flags * ((pop >= 1) & (pop <= K))
    return geno, na, pop, eff, data, m


@pytest.mark.parametrize("layout", [api.LAYOUT_U8, api.LAYOUT_B2G])
def test_popinfo_q_matches_oracle(ctx, orc, layout):
    geno, na, pop, eff, data, m = _setup(ctx, layout)
    K = 3
    c = api.Chain(ctx, data, m, SEED)
    # initial Z: every individual with a valid population starts there
    M = c.get(api.F_M)
    ok = (pop >= 1) & (pop <= K)
    home = np.clip(pop - 1, 0, K - 1)
    assert (M[ok, home[ok]] == M[ok].sum(1)).all()
    rng = np.random.default_rng(7)
    P = np.zeros((c.L, K, c.A), np.float32)
    for l in range(c.L):
        if na[l] > 0:
            P[l, :, :na[l]] = rng.dirichlet(np.full(na[l], 0.7), K)
    c.set(api.F_P, P)
    Q0 = rng.dirichlet(np.ones(K), c.N).astype(np.float32)
    c.set(api.F_Q, Q0)
    c.set(api.F_REP, np.array([6], np.int32))       # collecting (6 >= BURNIN), Gibbs sweep
    lQ0 = c.get(api.F_LOGQ)
    c.UpdateQ()
    assert c.sync() == 0
    Qd = c.get(api.F_Q)
    Qo, _, upo = orc.update_q_withpops(geno, c.get(api.F_P), pop, eff, 2, 0.05, SEED, 6, 5,
                                       Q0, lQ0)
    f = eff.astype(bool)
    np.testing.assert_array_equal(Qd[f], Qo[f])
    assert not np.array_equal(Qd[~f], Q0[~f])         # the others: Gibbs
    np.testing.assert_allclose(c.get(api.F_USEPOPPROBS), upo, rtol=1e-9, atol=1e-12)
    # alpha sums over individuals without prior information only
    c.UpdateAlpha()
    S, T = orc.alpha_sums(np.ascontiguousarray(c.get(api.F_LOGQ)[~f]))
    st = c.get(api.F_STATS)
    np.testing.assert_allclose(st[api.ST_ALPHA_S:api.ST_ALPHA_S + K], S, rtol=1e-11)
    assert st[api.ST_ALPHA_T] == pytest.approx(T, rel=1e-11)
    # a Metropolis sweep: the migrant-model draw again, the Metropolis test
    # leaves flagged individuals alone (src/Updates/UpdateQ.c:727-743,247)
    c.set(api.F_REP, np.array([8], np.int32))
    Q1, lQ1 = c.get(api.F_Q), c.get(api.F_LOGQ)
    c.UpdateQ()
    assert c.sync() == 0
    Qm = c.get(api.F_Q)
    Qo8, _, _ = orc.update_q_withpops(geno, c.get(api.F_P), pop, eff, 2, 0.05, SEED, 8, 5,
                                      Q1, lQ1)
    np.testing.assert_array_equal(Qm[f], Qo8[f])
    c.close(); data.close()


@pytest.mark.parametrize("layout", [api.LAYOUT_U8, api.LAYOUT_B2G])
def test_startatpopinfo_initial_z(ctx, layout):
    """STARTATPOPINFO without USEPOPINFO (src/Init.c:412-413 InitFromGeogPop):
    every copy of an individual whose population is in 1..K starts there,
    the others at random; without it the start is random for everyone."""
    geno, na, pop, eff, data, _ = _setup(ctx, layout)
    K = 3
    ok = (pop >= 1) & (pop <= K)
    home = np.clip(pop - 1, 0, K - 1)
    for start in (1, 0):
        m = api.model_defaults(maxpops=K, burnin=5, numreps=20, startatpopinfo=start)
        c = api.Chain(ctx, data, m, SEED)
        M = c.get(api.F_M)
        at_home = M[ok, home[ok]] == M[ok].sum(1)
        if start:
            assert at_home.all()
            assert not (M[~ok].max(1) == M[~ok].sum(1)).all()   # out of range: random
        else:
            assert not at_home.any()
        c.close()
    data.close()
