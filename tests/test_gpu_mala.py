"""The optional Metropolis-adjusted Langevin move on Q (Z summed out, P
fixed; st_update_q_mala) against the oracle's FP64 restatement
(oracle/st_oracle.c orc_mala_step) on the same state and Philox draws.

The device evaluates ll_i in FP32, so its log acceptance ratio differs from
the oracle's by ~1e-3; decisions must agree outside a band of 0.05 around
the acceptance threshold, accepted Q within 1e-5, adapted steps within 5e-3.
"""
import numpy as np
import pytest

from structure_b200 import api, synth
from oracle.oracle import S_MALA

pytestmark = pytest.mark.gpu

SEED = 0x4D414C41


def _u01(hi, lo):
    x = ((int(hi) >> 6) << 26) | (int(lo) >> 6)
    return (x + 0.5) / 4503599627370496.0


@pytest.mark.parametrize("K,popalphas", [(4, 0), (7, 1)])
def test_mala_step_matches_oracle(ctx, orc, K, popalphas):
    N, L = 200, 1500
    d = synth.snp_fmodel(N, L, K, np.linspace(0.05, 0.3, K), 0.4, 0.03, 60 + K)
    geno = d["geno"]
    data = api.Data(ctx, d["numalleles"], packed=d["packed"], layout=api.LAYOUT_B2G,
                    num_inds=N, num_loci=L)
    m = api.model_defaults(maxpops=K, burnin=10, numreps=10, mala=1, popalphas=popalphas,
                           alpha=0.7)
    c = api.Chain(ctx, data, m, SEED)
    rng = np.random.default_rng(K)
    Q = rng.dirichlet(np.full(K, 0.8), N).astype(np.float32)
    p1 = rng.beta(0.7, 0.7, (L, K)).astype(np.float32)
    P = np.stack([1 - p1, p1], axis=2).astype(np.float32)
    c.set(api.F_Q, Q)
    c.set(api.F_P, P)
    if popalphas:
        c.set(api.F_ALPHA, np.linspace(0.4, 1.2, K))
    eps0 = rng.permutation(np.geomspace(0.01, 0.5, N)).astype(np.float32)   # accepts and rejects
    c.set(api.F_MALA_EPS, eps0)
    Q0, lQ0, alpha = c.get(api.F_Q), c.get(api.F_LOGQ), c.get(api.F_ALPHA)
    c.UpdateQMala()
    assert c.sync() == 0
    Qd, lQd, ed = c.get(api.F_Q), c.get(api.F_LOGQ), c.get(api.F_MALA_EPS)
    st = c.get(api.F_STATS)
    Qo, lQo, eo, logr, acc = orc.mala_step(geno, Q0, lQ0, c.get(api.F_P), alpha, popalphas, eps0,
                                           SEED, 0, 10, 0.574)
    acc_d = (Qd != Q0).any(1)
    logu = np.array([np.log(_u01(*orc.stream(i, 0, 0, S_MALA, SEED)[:2])) for i in range(N)])
    clear = np.abs(logr - logu) > 0.05
    assert clear.sum() > 0.9 * N
    np.testing.assert_array_equal(acc_d[clear], acc[clear].astype(bool))
    both = clear & acc_d
    assert both.sum() > 20 and (~acc_d[clear]).sum() > 0
    np.testing.assert_allclose(Qd[both], Qo[both], rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(lQd[both], lQo[both], rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(Qd[~acc_d], Q0[~acc_d])
    np.testing.assert_allclose(ed[clear], eo[clear], rtol=5e-3)
    assert st[api.ST_MALA_TRIES] == N and st[api.ST_MALA_ACC] == acc_d.sum()
    c.close(); data.close()


def test_mala_sweeps_adapt_and_mix(ctx):
    """Inside st_sweep: steps adapt during burn-in toward the target rate."""
    N, L, K = 300, 3000, 5
    d = synth.snp_fmodel(N, L, K, np.linspace(0.05, 0.25, K), 0.3, 0.03, 71)
    data = api.Data(ctx, d["numalleles"], packed=d["packed"], layout=api.LAYOUT_B2G,
                    num_inds=N, num_loci=L)
    m = api.model_defaults(maxpops=K, burnin=150, numreps=100, mala=1, freqscorr=1)
    c = api.Chain(ctx, data, m, SEED + 1)
    c.sweep(150)
    st0 = c.get(api.F_STATS)
    c.sweep(100)
    assert c.sync() == 0
    st = c.get(api.F_STATS)
    rate = (st[api.ST_MALA_ACC] - st0[api.ST_MALA_ACC]) / (st[api.ST_MALA_TRIES] - st0[api.ST_MALA_TRIES])
    assert 0.3 < rate < 0.85, rate
    e = c.get(api.F_MALA_EPS)
    assert np.isfinite(e).all() and (e > 0).all()
    q = c.get(api.F_Q)
    np.testing.assert_allclose(q.sum(1), 1.0, rtol=1e-5)
    c.close(); data.close()
