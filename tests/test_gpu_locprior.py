"""LOCPRIOR on the device against the oracle's restatements (pinned to the
reference's UpdateLocPrior / UpdateAlphaLocPrior / UpdateQNoAdmix in
test_oracle_pins.py): locations numbered as GetNumLocations does, the Q
updates drawing with the location's alpha row (admixture) or starting from
the location's gamma (no admixture), the r / nu / gamma moves, the global and
location alpha moves, and the sums a collecting sweep adds."""
import numpy as np
import pytest

from structure_b200 import api, synth

pytestmark = pytest.mark.gpu

SEED = 0x10C9A10


def _setup(ctx, noadmix, K=3, layout=api.LAYOUT_U8, metrofreq=4, burnin=5):
    d = synth.microsat(N=150, L=120, K=K, seed=61)
    geno, na = d["geno"], d["numalleles"]
    N = geno.shape[0]
    rng = np.random.default_rng(62)
    ids = np.array([2, 3, 7, 11, 12])                      # location ids with gaps
    loc = ids[rng.integers(0, len(ids), N)].astype(np.int32)
    loc[:len(ids)] = ids
    myloc = np.searchsorted(ids, loc).astype(np.int32)
    data = api.Data(ctx, na, geno=geno, layout=layout, location=loc)
    m = api.model_defaults(maxpops=K, burnin=burnin, numreps=20, locprior=1, noadmix=noadmix,
                           admburnin=0, metrofreq=metrofreq, alphapropsd=0.2,
                           locpriorstep=0.3, freqscorr=0)
    c = api.Chain(ctx, data, m, SEED)
    return geno, na, myloc, len(ids), data, c


def test_locations_and_initial_state(ctx):
    for noadmix in (0, 1):
        _, _, myloc, nloc, data, c = _setup(ctx, noadmix)
        K = c.K
        np.testing.assert_array_equal(c.get(api.F_MYLOC), myloc)
        lp = c.get(api.F_LOCPRIOR)
        if noadmix:
            assert lp.shape == (1 + K * (nloc + 1),)
            np.testing.assert_array_equal(lp[1:], 1.0 / K)
            assert c.get(api.F_ALPHA).shape == (K,)
        else:
            assert lp.shape == (1,)
            np.testing.assert_array_equal(c.get(api.F_ALPHA), np.ones(K * (nloc + 1)))
        assert lp[0] == 1.0                                 # LOCPRIORINIT
        c.close(); data.close()


def test_q_updates_use_location_alphas(ctx, orc):
    geno, na, myloc, nloc, data, c = _setup(ctx, 0)
    K, N = c.K, c.N
    rng = np.random.default_rng(5)
    alpha = rng.uniform(0.1, 3.0, K * (nloc + 1))
    c.set(api.F_ALPHA, alpha)
    # Gibbs sweep (5 % METROFREQ != 0)
    c.set(api.F_REP, np.array([5], np.int32))
    m = c.get(api.F_M)
    c.UpdateQ()
    assert c.sync() == 0
    Qo, lQo, _ = orc.update_q_gibbs(m, alpha, SEED, 5, arow=1 + myloc)
    np.testing.assert_allclose(c.get(api.F_Q), Qo, rtol=1e-5, atol=1e-35)
    np.testing.assert_allclose(c.get(api.F_LOGQ), lQo, rtol=1e-5, atol=1e-5)
    Qg, _, _ = orc.update_q_gibbs(m, alpha[:K], SEED, 5)
    assert not np.allclose(Qg, Qo)                          # the rows matter
    # Metropolis sweep: proposals from Dir(alpha of the location)
    c.set(api.F_REP, np.array([8], np.int32))
    c.UpdateQ()
    T, _, _ = orc.metro_propose(N, alpha.reshape(-1, K), SEED, 8, arow=1 + myloc)
    np.testing.assert_allclose(c.get(api.F_TESTQ), T, rtol=1e-5, atol=1e-35)
    c.close(); data.close()


def test_noadmix_q_uses_location_gamma(ctx, orc):
    geno, na, myloc, nloc, data, c = _setup(ctx, 1)
    K = c.K
    rng = np.random.default_rng(6)
    lp = np.concatenate([[1.5], rng.dirichlet(np.ones(K)),
                         rng.dirichlet(np.full(K, 0.2), nloc).reshape(-1)])
    c.set(api.F_LOCPRIOR, lp)
    c.set(api.F_REP, np.array([3], np.int32))
    c.UpdateQ()
    assert c.sync() == 0
    _, _, pick = orc.update_q_noadmix(geno, c.get(api.F_LOGP), SEED, 3, locp=lp, myloc=myloc)
    Q = c.get(api.F_Q)
    np.testing.assert_array_equal(Q.argmax(1), pick)
    np.testing.assert_array_equal(Q.max(1), 1.0)
    c.close(); data.close()


@pytest.mark.parametrize("noadmix", [0, 1])
def test_locprior_moves_match_oracle(ctx, orc, noadmix):
    geno, na, myloc, nloc, data, c = _setup(ctx, noadmix, burnin=50)
    K, N = c.K, c.N
    rng = np.random.default_rng(7 + noadmix)
    moves = 0
    for trial in range(12):
        rep = 2 + trial                                      # before BURNIN: no sums
        if noadmix:
            Q = np.eye(K, dtype=np.float32)[rng.integers(0, K, N)]
            lp = np.concatenate([[rng.uniform(0.5, 3.0)], rng.dirichlet(np.ones(K) * 3),
                                 rng.dirichlet(np.ones(K) * 2, nloc).reshape(-1)])
            alpha = c.get(api.F_ALPHA)
        else:
            Q = rng.dirichlet(np.ones(K), N).astype(np.float32)
            lp = np.array([rng.uniform(0.5, 3.0)])
            alpha = rng.uniform(0.2, 2.0, K * (nloc + 1))
            c.set(api.F_ALPHA, alpha)
        c.set(api.F_Q, Q)
        c.set(api.F_LOCPRIOR, lp)
        c.set(api.F_REP, np.array([rep], np.int32))
        c.UpdateLocPrior()
        assert c.sync() == 0
        mine, _, _ = orc.update_locprior(myloc, Q, alpha, lp, noadmix, 0.2, 0.3, 20.0, SEED, rep)
        np.testing.assert_allclose(c.get(api.F_LOCPRIOR), mine, rtol=1e-12, atol=0)
        moves += int(np.sum(mine != lp))
    assert moves > 5
    np.testing.assert_array_equal(c.get(api.F_SUMLOCPRIOR), 0.0)
    c.close(); data.close()


def test_alpha_locprior_matches_oracle(ctx, orc):
    geno, na, myloc, nloc, data, c = _setup(ctx, 0)
    K, N = c.K, c.N
    rng = np.random.default_rng(9)
    moved = 0
    for trial in range(10):
        rep = 1 + trial
        Q = rng.dirichlet(np.full(K, 0.7), N).astype(np.float32)
        alpha = rng.uniform(0.2, 3.0, K * (nloc + 1))
        r = rng.uniform(0.5, 4.0)
        c.set(api.F_Q, Q)
        c.set(api.F_ALPHA, alpha)
        c.set(api.F_LOCPRIOR, np.array([r]))
        c.set(api.F_REP, np.array([rep], np.int32))
        c.UpdateAlpha()                                      # UpdateAlphaLocPrior
        assert c.sync() == 0
        lq = c.get(api.F_LOGQ).astype(np.float64)
        mine, _, _ = orc.update_alpha_locprior(myloc, lq, alpha, r, 0.2, 10.0, SEED, rep)
        np.testing.assert_allclose(c.get(api.F_ALPHA), mine, rtol=1e-12, atol=0)
        moved += int(np.sum(mine != alpha))
    assert moved > 10
    c.close(); data.close()


@pytest.mark.parametrize("noadmix", [0, 1])
def test_collecting_sweep_adds_location_sums(ctx, noadmix):
    _, _, _, nloc, data, c = _setup(ctx, noadmix)
    c.sweep(5)                                               # burn-in: nothing summed
    np.testing.assert_array_equal(c.get(api.F_SUMLOCPRIOR), 0.0)
    c.sweep(1)
    assert c.sync() == 0
    np.testing.assert_array_equal(c.get(api.F_SUMLOCPRIOR), c.get(api.F_LOCPRIOR))
    if not noadmix:
        np.testing.assert_array_equal(c.get(api.F_SUMALPHA), c.get(api.F_ALPHA))
    else:
        np.testing.assert_array_equal(c.get(api.F_SUMALPHA), 0.0)
    c.sweep(14)
    assert c.sync() == 0
    assert c.get(api.F_SUMLOCPRIOR)[0] > 0
    c.close(); data.close()
