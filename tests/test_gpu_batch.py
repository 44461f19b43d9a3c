"""Batched chains of uneven shape: chains over several data sets (different N
and L), with K from 1 to 16 (several K classes, so several Z launches per step)
and per-chain model options, advanced together by st_batch_sweep, give the same
state as each chain advanced alone by st_sweep.

Random draws are keyed by (chain seed, sweep, update, element), never by the
launch, so batching changes no draw: Z counts, P, Q, eps, F, alpha and every
sum must agree exactly.  The Metropolis log ratio is a sum over locus groups
whose partition follows the Z-pass tile, which a tuned batch may change; it is
compared to 1e-12.
"""
import numpy as np
import pytest

from structure_b200 import api, synth

pytestmark = pytest.mark.gpu

DATASETS = [(64, 600), (200, 1100), (150, 700), (330, 450)]
KS = [1, 2, 3, 4, 5, 7, 10, 13, 16]
EXACT = [api.F_Q, api.F_LOGQ, api.F_P, api.F_LOGP, api.F_EPS, api.F_F, api.F_ALPHA,
         api.F_N, api.F_M, api.F_QSUM, api.F_PSUM, api.F_SUMEPS, api.F_FSTSUM,
         api.F_SUMALPHA, api.F_REP, api.F_ERR]


def _datasets(ctx):
    out = []
    for j, (N, L) in enumerate(DATASETS):
        d = synth.snp_fmodel(N, L, 4, np.linspace(0.02, 0.2, 4), 0.5, 0.03, 300 + j)
        out.append(api.Data(ctx, d["numalleles"], packed=d["packed"], layout=api.LAYOUT_B2G,
                            num_inds=N, num_loci=L))
    return out


def _model(K, s):
    return api.model_defaults(maxpops=K, burnin=1, numreps=10, freqscorr=1, metrofreq=2,
                              alpha=1.0, alphapropsd=0.05, popalphas=(K + s) % 2,
                              fpriormean=0.01, fpriorsd=0.05)


def _specs():
    return [(K, s, (K + s) % len(DATASETS)) for K in KS for s in range(2)]


@pytest.mark.parametrize("graphs", [True, False])
def test_batched_uneven_chains_equal_plain_chains(ctx, graphs):
    data = _datasets(ctx)
    batched = [api.Chain(ctx, data[di], _model(K, s), 4000 + 10 * K + s) for K, s, di in _specs()]
    plain = [api.Chain(ctx, data[di], _model(K, s), 4000 + 10 * K + s) for K, s, di in _specs()]
    b = api.Batch(ctx, batched)
    b.graphs(graphs)
    l0 = ctx.launches()
    b.sweep(4)
    # one locus, one or two individual, one count-clearing and one Z launch per
    # K class per sweep
    nclass = len({api.fast_class(K) for K, _, _ in _specs()})
    assert ctx.launches() - l0 == 4 * (3 + nclass) + 2 * (1 + nclass)
    for c in plain:
        c.sweep(4)
    for cb, cp in zip(batched, plain):
        assert cb.sync() == 0 and cp.sync() == 0
        for f in EXACT:
            np.testing.assert_array_equal(cb.get(f), cp.get(f), err_msg=f"K={cb.K} field {f}")
        sb, sp = cb.get(api.F_STATS), cp.get(api.F_STATS)
        np.testing.assert_array_equal(sb[:4], sp[:4])   # like, sumlikes, sumsqlikes, count
        assert sb[api.ST_NLIKE] == 3
        np.testing.assert_allclose(cb.get(api.F_LOGDIFF), cp.get(api.F_LOGDIFF), rtol=1e-12,
                                   atol=1e-9)
        if cb.K == 1:
            assert (cb.get(api.F_Q) == 1.0).all()
            m = cb.get(api.F_M)
            assert m[:, 0].sum() == cb.get(api.F_N).sum()
    b.close()
    for c in batched + plain:
        c.close()
    for d in data:
        d.close()


def test_autotuned_batch_samples_the_same_chains(ctx):
    """st_batch_autotune changes the Z-pass tiles only: the tuned batch and an
    untuned twin (same seeds) end in the same state after sweeps that include
    Metropolis steps; a batch of the same shapes created afterwards starts
    from the remembered tiles."""
    data = _datasets(ctx)
    specs = [(K, s, d) for (K, s, d) in _specs() if K in (2, 5, 10)]
    mk = lambda: [api.Chain(ctx, data[d], _model(K, s), 500 + 10 * K + s) for (K, s, d) in specs]
    tuned, plain = mk(), mk()
    bt, bp = api.Batch(ctx, tuned), api.Batch(ctx, plain)
    bt.sweep(2)
    bp.sweep(2)
    before = [c.get(api.F_DIMS)[6:8].copy() for c in tuned]
    bt.autotune(2)
    after = [c.get(api.F_DIMS)[6:8].copy() for c in tuned]
    bt.sweep(9)
    bp.sweep(9)
    for ct, cp in zip(tuned, plain):
        assert ct.sync() == 0 and cp.sync() == 0
        for f in EXACT:
            a, b = ct.get(f), cp.get(f)
            if f == api.F_REP or f == api.F_ERR:
                assert a == b
            else:
                np.testing.assert_array_equal(a, b, err_msg=str(f))
        sa, sp = ct.get(api.F_STATS), cp.get(api.F_STATS)
        assert sa[api.ST_SUMLIKES] == pytest.approx(sp[api.ST_SUMLIKES], rel=1e-12)
    # the remembered tiles apply to a new batch of the same shapes
    again = mk()
    ba = api.Batch(ctx, again)
    np.testing.assert_array_equal([c.get(api.F_DIMS)[6:8] for c in again], after)
    print("tiles (nchunks, ngroups) before", before[:3], "after", after[:3])
    for b in (bt, bp, ba):
        b.close()
    for c in tuned + plain + again:
        c.close()
    for d in data:
        d.close()
