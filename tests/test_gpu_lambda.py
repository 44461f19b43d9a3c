"""INFERLAMBDA on the device (st_update_lambda; lambda between P and eps in
the fused sweep) against the oracle's restatement of UpdateLambda /
UpdatePopLambda (itself pinned to the reference in test_oracle_pins.py).
The device sums the log ratio over loci in blocks of 256, the oracle in one
pass: ratios agree to 1e-9 relative and the moves are the same."""
import numpy as np
import pytest

from structure_b200 import api, synth

pytestmark = pytest.mark.gpu

SEED = 0x1A4BDA


@pytest.mark.parametrize("freqscorr,popspecific", [(0, 0), (1, 0), (0, 1)])
def test_update_lambda_matches_oracle(ctx, orc, freqscorr, popspecific):
    d = synth.microsat(N=60, L=700, K=4, seed=31)
    data = api.Data(ctx, d["numalleles"], geno=d["geno"])
    K = 4
    m = api.model_defaults(maxpops=K, burnin=0, numreps=10, freqscorr=freqscorr, inferlambda=1,
                           popspecificlambda=popspecific)
    c = api.Chain(ctx, data, m, SEED)
    c.UpdateP()       # a P drawn from the initial counts
    rng = np.random.default_rng(popspecific)
    lam0 = rng.uniform(0.4, 2.5, K) if popspecific else np.full(K, 1.7)
    c.set(api.F_LAMBDA, lam0)
    logP, eps = c.get(api.F_LOGP), c.get(api.F_EPS)
    c.UpdateLambda()
    assert c.sync() == 0
    lam1 = c.get(api.F_LAMBDA)
    npop = K if popspecific else 1
    lpd = c.get(api.F_STATS)[api.ST_LAMBDA_LPD:api.ST_LAMBDA_LPD + npop]
    mine, lpo = orc.update_lambda(d["numalleles"], logP, eps, freqscorr, popspecific, lam0, SEED,
                                  c.get(api.F_REP))
    lpo = lpo[:npop]
    ok = np.isfinite(lpo)
    np.testing.assert_allclose(lpd[ok], lpo[ok], rtol=1e-9, atol=1e-9)
    np.testing.assert_array_equal(lam1, mine)
    c.close(); data.close()


def test_sweeps_with_inferlambda_move_lambda(ctx):
    d = synth.microsat(N=80, L=200, K=3, seed=5)
    data = api.Data(ctx, d["numalleles"], geno=d["geno"])
    m = api.model_defaults(maxpops=3, burnin=5, numreps=40, freqscorr=0, inferlambda=1)
    c = api.Chain(ctx, data, m, SEED + 1)
    c.sweep(45)
    assert c.sync() == 0
    lam = c.get(api.F_LAMBDA)
    assert np.all(lam == lam[0]) and 0 < lam[0] < 10 and lam[0] != 1.0
    s = c.get(api.F_SUMLAMBDA)
    assert 0 < s[0] / 40 < 10
    c.close(); data.close()
