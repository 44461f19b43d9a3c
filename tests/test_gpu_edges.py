"""Edge cases of the device path against the oracle: the smallest shapes
(one individual, one locus, rows that are not a multiple of the 16
genotypes of a packed word), the K limits (one population; the widest
classes 16-32), individuals and loci with every copy missing, monomorphic
loci, the allele limit, and inputs the boundary must refuse with a status
instead of running."""
import numpy as np
import pytest

from structure_b200 import api, synth

pytestmark = pytest.mark.gpu

SEED = 0xED6E5


def _snp(N, L, K=3, seed=3, missing=0.03):
    d = synth.snp_fmodel(N, L, K, np.linspace(0.05, 0.25, K), 0.4, missing, seed)
    return d["geno"], d["numalleles"]


def _rand_state(rng, N, L, K, na):
    A = int(max(1, na.max()))
    Q = rng.dirichlet(np.full(K, 0.7), N).astype(np.float32)
    P = np.zeros((L, K, A), np.float32)
    for l in range(L):
        if na[l] > 0:
            P[l, :, :na[l]] = rng.dirichlet(np.ones(na[l]), K)
    return Q, P


def _model(K, **kw):
    return api.model_defaults(maxpops=K, burnin=2, numreps=6, freqscorr=0, metrofreq=3,
                              store_z=1, **kw)


def _z(c):
    z = c.get(api.F_Z).astype(np.int32)
    z[z == 255] = -9
    return z


def _check_z_pass(ctx, orc, geno, na, K, layout, rep=4):
    """One Z pass on random Q, P: Z and counts bit-exact, ln P(D) within 1e-5."""
    N, _, L = geno.shape
    d = api.Data(ctx, na, geno=geno, layout=layout)
    c = api.Chain(ctx, d, _model(K), SEED)
    Q, P = _rand_state(np.random.default_rng(N * 1000 + L + K), N, L, K, na)
    c.set(api.F_Q, Q)
    c.set(api.F_P, P)
    c.set(api.F_REP, np.array([rep], np.int32))
    c.UpdateZ()
    assert c.sync() == 0
    zo = orc.zupdate_f32(geno, Q, P, SEED, rep)
    assert (_z(c) == zo).all()
    n_o, m_o = orc.counts(geno, zo, K, c.A)
    assert (c.get(api.F_N) == n_o).all() and (c.get(api.F_M) == m_o).all()
    like = c.CalcLike()
    lo = orc.calc_like(geno, Q, P)
    assert abs(like - lo) <= 1e-5 * max(1.0, abs(lo))
    # and whole sweeps run clean from there (Gibbs and Metropolis)
    c.sweep(6)
    assert c.sync() == 0 and c.get(api.F_ERR) == 0
    assert np.isfinite(c.get(api.F_Q)).all() and np.isfinite(c.get(api.F_P)).all()
    c.close()
    d.close()


@pytest.mark.parametrize("layout", [api.LAYOUT_U8, api.LAYOUT_B2G])
@pytest.mark.parametrize("N,L", [(1, 1), (1, 37), (17, 1), (16, 16), (33, 5), (47, 129)])
def test_small_and_ragged_shapes(ctx, orc, layout, N, L):
    geno, na = _snp(N, L, seed=N + L)
    _check_z_pass(ctx, orc, geno, na, 3, layout)


@pytest.mark.parametrize("K", [1, 16, 20, 24, 32])
def test_k_limits(ctx, orc, K):
    """K = 1 (every copy from population 0, Q = 1) and the widest classes."""
    geno, na = _snp(90, 200, K=min(K, 4), seed=K)
    _check_z_pass(ctx, orc, geno, na, K, api.LAYOUT_B2G)
    if K == 1:
        d = api.Data(ctx, na, geno=geno, layout=api.LAYOUT_B2G)
        c = api.Chain(ctx, d, _model(1), SEED)
        c.sweep(4)
        np.testing.assert_array_equal(c.get(api.F_Q), 1.0)
        M = c.get(api.F_M)
        np.testing.assert_array_equal(M[:, 0], (geno >= 0).sum((1, 2)))
        c.close()
        d.close()


@pytest.mark.parametrize("layout", [api.LAYOUT_U8, api.LAYOUT_B2G])
def test_all_missing_individual_and_locus(ctx, orc, layout):
    """An individual and a locus with every copy missing: no draws, no counts,
    no ln P(D) terms; the locus's P comes from the prior and stays finite."""
    geno, na = _snp(70, 90, seed=9)
    geno = geno.copy()
    geno[5] = -9
    geno[:, :, 11] = -9
    na = na.copy()
    _check_z_pass(ctx, orc, geno, na, 4, layout)
    d = api.Data(ctx, na, geno=geno, layout=layout)
    c = api.Chain(ctx, d, _model(4), SEED)
    c.sweep(5)
    assert c.sync() == 0
    z = _z(c)
    assert (z[5] == -9).all() and (z[:, :, 11] == -9).all()
    assert (c.get(api.F_M)[5] == 0).all() and (c.get(api.F_N)[11] == 0).all()
    P = c.get(api.F_P)
    assert np.isfinite(P).all()
    if na[11] > 0:
        np.testing.assert_allclose(P[11, :, :na[11]].sum(1), 1.0, rtol=1e-5)
    c.close()
    d.close()


def test_monomorphic_loci_and_allele_limit(ctx, orc):
    """Loci with one allele (P = 1) next to a locus with the maximum 64 alleles
    (multi-allelic data take the one-byte-per-copy layout)."""
    N, L = 80, 12
    rng = np.random.default_rng(4)
    na = np.array([1, 2, 64, 1, 5, 64, 3, 1, 2, 10, 64, 1], np.int32)
    geno = np.zeros((N, 2, L), np.int32)
    for l in range(L):
        geno[:, :, l] = rng.integers(0, na[l], (N, 2))
    geno[rng.random((N, 2, L)) < 0.05] = -9
    geno[:64, 0, 2] = np.arange(64)          # every allele of the 64-allele locus seen
    _check_z_pass(ctx, orc, geno, na, 3, api.LAYOUT_U8)
    d = api.Data(ctx, na, geno=geno)
    c = api.Chain(ctx, d, _model(3), SEED)
    c.sweep(3)
    P = c.get(api.F_P)
    np.testing.assert_array_equal(P[na == 1][:, :, 0], 1.0)
    c.close()
    d.close()


def test_invalid_inputs_are_refused(ctx):
    geno, na = _snp(40, 30, seed=2)

    def code(fn):
        with pytest.raises(api.StError) as e:
            fn()
        return e.value.code

    bad = geno.copy()
    bad[0, 0, 0] = 2                                  # allele >= num_alleles (2)
    assert code(lambda: api.Data(ctx, na, geno=bad)) == api.ST_ERR_ARG
    bad[0, 0, 0] = -5                                 # neither an allele nor -9
    assert code(lambda: api.Data(ctx, na, geno=bad)) == api.ST_ERR_ARG
    na65 = np.full(30, 65, np.int32)                  # over the allele limit
    assert code(lambda: api.Data(ctx, na65, geno=geno)) == api.ST_ERR_UNSUPPORTED
    loc = np.zeros(40, np.int32)
    loc[3] = -1                                       # negative location (Util.c:241-246)
    assert code(lambda: api.Data(ctx, na, geno=geno, location=loc)) == api.ST_ERR_ARG
    d = api.Data(ctx, na, geno=geno)
    for kw, want in [(dict(maxpops=0), api.ST_ERR_UNSUPPORTED),
                     (dict(maxpops=33), api.ST_ERR_UNSUPPORTED),
                     (dict(maxpops=3, linkage=1), api.ST_ERR_UNSUPPORTED),
                     (dict(maxpops=3, recessivealleles=1), api.ST_ERR_UNSUPPORTED),
                     (dict(maxpops=3, noadmix=1, admburnin=50, burnin=50), api.ST_ERR_ARG),
                     (dict(maxpops=3, locprior=1), api.ST_ERR_ARG),
                     (dict(maxpops=3, usepopinfo=1), api.ST_ERR_ARG),
                     (dict(maxpops=1, locprior=1, noadmix=1), api.ST_ERR_UNSUPPORTED)]:
        m = api.model_defaults(**kw)
        assert code(lambda: api.Chain(ctx, d, m, 1)) == want, kw
    d.close()


def test_reused_device_blocks_give_identical_chains(ctx):
    """A chain created in the device blocks a destroyed chain left in the
    context's cache starts from the same state as one in fresh memory: same
    seed, same sweeps, same result; the cached blocks are not counted as in use."""
    geno, na = _snp(120, 400, seed=21)
    base, _ = ctx.memory()
    d = api.Data(ctx, na, geno=geno, layout=api.LAYOUT_B2G)
    m = api.model_defaults(maxpops=3, burnin=3, numreps=6, freqscorr=1, metrofreq=2)
    runs = []
    for _ in range(2):
        c = api.Chain(ctx, d, m, 4242)
        c.sweep(6)
        assert c.sync() == 0
        runs.append([c.get(f) for f in (api.F_Q, api.F_P, api.F_QSUM, api.F_STATS)])
        used, _ = ctx.memory()
        c.close()
    for a, b in zip(*runs):
        np.testing.assert_array_equal(a, b)
    d.close()
    assert ctx.memory()[0] == base
    assert used > base


def test_get_into_caller_array(ctx):
    """Chain.get(f, out=...) fills a caller-owned (here page-locked) array with
    the same bytes as a fresh copy, and refuses an array of the wrong size or type."""
    import torch
    geno, na = _snp(60, 300, seed=23)
    d = api.Data(ctx, na, geno=geno, layout=api.LAYOUT_B2G)
    c = api.Chain(ctx, d, api.model_defaults(maxpops=4, burnin=1, numreps=4, freqscorr=1), 99)
    c.sweep(4)
    for f in (api.F_QSUM, api.F_PSUM, api.F_STATS, api.F_ALPHA, api.F_F):
        ref = c.get(f)
        buf = torch.empty(ref.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(ref.dtype)
        got = c.get(f, out=buf)
        np.testing.assert_array_equal(got, ref)
        assert np.shares_memory(got, buf)
    q = c.get(api.F_QSUM)
    with pytest.raises(api.StError):
        c.get(api.F_QSUM, out=np.zeros(q.size + 1, q.dtype))
    with pytest.raises(api.StError):
        c.get(api.F_QSUM, out=np.zeros(q.size, np.float32))
    c.close()
    d.close()


@pytest.mark.parametrize("N", [1, 17, 130])
def test_packed_upload_counts_match_int32_upload(ctx, N):
    """Allele counts of 2-bit words (counted on the device, padding genotypes of
    the last word masked) equal those of the int32 upload of the same data: the
    initial eps (lambda + n_a) / (A lambda + n) agree exactly."""
    L = 257
    d = synth.snp_fmodel(N, L, 3, np.linspace(0.05, 0.25, 3), 0.4, 0.05, 31 + N)
    m = api.model_defaults(maxpops=3, freqscorr=1, burnin=1, numreps=2)
    a = api.Data(ctx, d["numalleles"], geno=d["geno"], layout=api.LAYOUT_B2G)
    b = api.Data(ctx, d["numalleles"], packed=d["packed"], layout=api.LAYOUT_B2G,
                 num_inds=N, num_loci=L)
    ca, cb = api.Chain(ctx, a, m, 5), api.Chain(ctx, b, m, 5)
    ea = ca.get(api.F_EPS)
    np.testing.assert_array_equal(ea, cb.get(api.F_EPS))
    two = np.asarray(d["numalleles"]) == 2
    assert ((ea[two] > 0) & (ea[two] < 1)).all()
    np.testing.assert_allclose(ea[two].sum(1), 1.0, rtol=1e-12)
    for x in (ca, cb, a, b):
        x.close()


@pytest.mark.parametrize("layout", [api.LAYOUT_B2G, api.LAYOUT_U8])
@pytest.mark.parametrize("K,store_z", [(3, 1), (5, 0), (10, 1), (13, 0)])
def test_pfrompopflagonly_counts(orc, layout, K, store_z):
    """PFROMPOPFLAGONLY (src/Updates/UpdateP.c GetNumFromPops): only individuals
    whose POPFLAG is 1 add to the allele counts n; every individual adds to the
    ancestry counts m.  One Z pass on a fixed state against the oracle's Z and
    its counts with the same flags, with and without the stored Z."""
    N, L = 203, 517
    geno, na = _snp(N, L, K, seed=11 + K)
    rng = np.random.default_rng(7 * K + store_z)
    popflags = (rng.random(N) < 0.4).astype(np.int32)
    ctx = api.Context(0)
    d = api.Data(ctx, na, geno=geno, layout=layout, popflags=popflags)
    m = api.model_defaults(maxpops=K, burnin=2, numreps=6, freqscorr=0, metrofreq=3,
                           store_z=store_z, pfrompopflagonly=1)
    c = api.Chain(ctx, d, m, SEED)
    Q, P = _rand_state(np.random.default_rng(N + L + K), N, L, K, na)
    c.set(api.F_Q, Q)
    c.set(api.F_P, P)
    rep = 4
    c.set(api.F_REP, np.array([rep], np.int32))
    c.UpdateZ()
    assert c.sync() == 0
    zo = orc.zupdate_f32(geno, Q, P, SEED, rep)
    if store_z:
        assert (_z(c) == zo).all()
    n_o, m_o = orc.counts(geno, zo, K, c.A, popflags=popflags, pfrompopflagonly=1)
    n_all, _ = orc.counts(geno, zo, K, c.A)
    assert n_o.sum() < n_all.sum()          # the flags leave some copies out of n
    assert (c.get(api.F_N) == n_o).all()
    assert (c.get(api.F_M) == m_o).all()
    c.close()
    d.close()
    ctx.close()
