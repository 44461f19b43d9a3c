"""NOADMIX on the device: the one-population Q update (thread = individual,
FP64 sums of log P over locus chunks, then the reference's PickAnOption rule)
against the oracle's restatement (itself pinned to the reference's
UpdateQNoAdmix in test_oracle_pins.py), on both genotype layouts; and the
schedule (admixture Gibbs with alpha before ADMBURNIN, one population after)."""
import numpy as np
import pytest

from structure_b200 import api, synth

pytestmark = pytest.mark.gpu

SEED = 0x4E4F4144


@pytest.mark.parametrize("layout", [api.LAYOUT_U8, api.LAYOUT_B2G])
def test_noadmix_q_matches_oracle(ctx, orc, layout):
    if layout == api.LAYOUT_U8:
        d = synth.microsat(N=300, L=400, K=5, seed=8)
        geno, na = d["geno"], d["numalleles"]
        data = api.Data(ctx, na, geno=geno, layout=layout)
    else:
        d = synth.snp_fmodel(300, 1200, 5, np.linspace(0.05, 0.3, 5), 0.2, 0.03, 9)
        geno, na = d["geno"], d["numalleles"]
        data = api.Data(ctx, na, packed=d["packed"], layout=layout, num_inds=300, num_loci=1200)
    K = 5
    m = api.model_defaults(maxpops=K, burnin=10, numreps=10, noadmix=1, admburnin=2)
    c = api.Chain(ctx, data, m, SEED)
    rng = np.random.default_rng(layout)
    A = c.A
    P = np.zeros((c.L, K, A), np.float32)
    for l in range(c.L):
        if na[l] > 0:
            P[l, :, :na[l]] = rng.dirichlet(np.full(na[l], 0.7), K)
    c.set(api.F_P, P)
    c.set(api.F_REP, np.array([5], np.int32))      # past ADMBURNIN: one-population update
    c.UpdateQ()
    assert c.sync() == 0
    Q, lQ = c.get(api.F_Q), c.get(api.F_LOGQ)
    Qo, lQo, pick = orc.update_q_noadmix(geno, c.get(api.F_LOGP), SEED, 5)
    np.testing.assert_array_equal(Q, Qo)
    np.testing.assert_array_equal(lQ, lQo)
    assert len(set(pick)) > 2
    c.close(); data.close()


def test_noadmix_schedule_and_sums(ctx):
    d = synth.microsat(N=100, L=150, K=3, seed=4)
    data = api.Data(ctx, d["numalleles"], geno=d["geno"])
    m = api.model_defaults(maxpops=3, burnin=20, numreps=30, noadmix=1, admburnin=10,
                           alphapropsd=0.2)
    c = api.Chain(ctx, data, m, SEED + 1)
    c.sweep(10)                       # reps 0..9: admixture Gibbs, alpha moves
    q = c.get(api.F_Q)
    assert ((q > 0) & (q < 1)).any()
    alpha_early = c.get(api.F_ALPHA).copy()
    assert alpha_early[0] != 1.0
    c.sweep(40)                       # rep 10: Gibbs without alpha; then one population
    assert c.sync() == 0
    q = c.get(api.F_Q)
    assert set(np.unique(q)) <= {0.0, 1.0} and (q.sum(1) == 1).all()
    np.testing.assert_array_equal(c.get(api.F_ALPHA), alpha_early)
    qs = c.get(api.F_QSUM)
    np.testing.assert_allclose(qs.sum(1), 30)
    assert (c.get(api.F_SUMALPHA) == 0).all()       # no alpha sums under NOADMIX
    c.close(); data.close()
