"""Checkpoint / resume: a chain saved at sweep s and loaded into a fresh chain
of the same shape continues bit for bit like the original (counter-based
draws keyed by seed, sweep, update and element)."""
import numpy as np
import pytest

from structure_b200 import api, synth

pytestmark = pytest.mark.gpu

FIELDS = [api.F_Q, api.F_LOGQ, api.F_P, api.F_LOGP, api.F_EPS, api.F_F, api.F_ALPHA, api.F_N,
          api.F_M, api.F_QSUM, api.F_PSUM, api.F_SUMEPS, api.F_FSTSUM, api.F_SUMALPHA,
          api.F_STATS, api.F_REP, api.F_ERR]


@pytest.mark.parametrize("kind", ["snp-mala", "microsat"])
def test_resume_continues_exactly(ctx, tmp_path, kind):
    if kind == "microsat":
        d = synth.microsat(N=80, L=60, K=3, seed=3)
        data = api.Data(ctx, d["numalleles"], geno=d["geno"])
        K, extra = 3, {}
    else:
        d = synth.snp_fmodel(150, 800, 4, np.linspace(0.05, 0.2, 4), 0.4, 0.03, 8)
        data = api.Data(ctx, d["numalleles"], packed=d["packed"], layout=api.LAYOUT_B2G,
                        num_inds=150, num_loci=800)
        K, extra = 4, {"mala": 1, "ancestdist": 1, "numboxes": 50}
    m = api.model_defaults(maxpops=K, burnin=2, numreps=20, freqscorr=1, metrofreq=3, **extra)
    a = api.Chain(ctx, data, m, 1111)
    a.sweep(3)
    path = str(tmp_path / "chain.ckpt")
    a.save(path)
    a.sweep(4)
    b = api.Chain(ctx, data, m, 2222)     # another seed: the file brings the key
    b.load(path)
    assert b.get(api.F_REP) == 3
    b.sweep(4)
    assert a.sync() == 0 and b.sync() == 0
    fields = FIELDS + ([api.F_MALA_EPS, api.F_ANCESTDIST] if kind != "microsat" else [])
    for f in fields:
        np.testing.assert_array_equal(a.get(f), b.get(f), err_msg=f"field {f}")
    # a chain of another shape refuses the file
    c = api.Chain(ctx, data, api.model_defaults(maxpops=K + 1, burnin=2, numreps=20), 1)
    with pytest.raises(api.StError):
        c.load(path)
    for x in (a, b, c):
        x.close()
    data.close()


def test_resume_into_a_chain_with_another_tile(ctx, tmp_path):
    """A chain saved after st_batch_autotune changed its Z-pass tile loads into
    a fresh chain with the starting tile and continues exactly: nothing saved
    depends on the tile."""
    d = synth.snp_fmodel(300, 3000, 3, np.linspace(0.05, 0.2, 3), 0.4, 0.03, 12)
    data = api.Data(ctx, d["numalleles"], packed=d["packed"], layout=api.LAYOUT_B2G,
                    num_inds=300, num_loci=3000)
    m = api.model_defaults(maxpops=3, burnin=2, numreps=20, freqscorr=1, metrofreq=3)
    a = api.Chain(ctx, data, m, 77)
    b = api.Batch(ctx, [a])
    b.sweep(2)
    b.autotune(1)
    b.sweep(2)
    path = str(tmp_path / "tuned.ckpt")
    a.save(path)
    b.sweep(4)
    fresh = api.Chain(ctx, data, m, 1)
    fresh.load(path)
    fresh.sweep(4)
    assert a.sync() == 0 and fresh.sync() == 0
    for f in FIELDS:
        if f == api.F_STATS:
            # ln P(D) partial sums follow the tile's locus grouping
            np.testing.assert_allclose(a.get(f), fresh.get(f), rtol=1e-12)
        else:
            np.testing.assert_array_equal(a.get(f), fresh.get(f), err_msg=f"field {f}")
    b.close()
    for x in (a, fresh):
        x.close()
    data.close()


def test_bad_checkpoints_leave_the_chain_unchanged(ctx, tmp_path):
    """A truncated file, a file with trailing bytes and a file saved under other
    model options are refused with ST_ERR_STATE before any device memory of
    the chain is written: its state afterwards equals its state before."""
    d = synth.snp_fmodel(120, 500, 3, np.linspace(0.05, 0.2, 3), 0.4, 0.03, 19)
    data = api.Data(ctx, d["numalleles"], packed=d["packed"], layout=api.LAYOUT_B2G,
                    num_inds=120, num_loci=500)
    mk = lambda burnin, numreps: api.model_defaults(maxpops=3, burnin=burnin, numreps=numreps,
                                                    freqscorr=1, metrofreq=3)
    src = api.Chain(ctx, data, mk(2, 20), 31)
    src.sweep(5)
    path = str(tmp_path / "good.ckpt")
    src.save(path)
    raw = open(path, "rb").read()
    dst = api.Chain(ctx, data, mk(2, 20), 32)
    dst.sweep(2)
    before = {f: dst.get(f) for f in FIELDS}
    for name, blob in (("truncated", raw[:len(raw) - 100]), ("trailing", raw + b"\0\0\0\0")):
        p = str(tmp_path / f"{name}.ckpt")
        with open(p, "wb") as fh:
            fh.write(blob)
        with pytest.raises(api.StError) as e:
            dst.load(p)
        assert e.value.code == api.ST_ERR_STATE, name
    # the same shape but another BURNIN: refused as well
    other = api.Chain(ctx, data, mk(7, 20), 33)
    with pytest.raises(api.StError) as e:
        other.load(path)
    assert e.value.code == api.ST_ERR_STATE
    for f in FIELDS:
        a, b = dst.get(f), before[f]
        if isinstance(a, int):
            assert a == b, f
        else:
            np.testing.assert_array_equal(a, b, err_msg=f"field {f}")
    # NUMREPS alone may differ (it only says where st_run stops)
    more = api.Chain(ctx, data, mk(2, 50), 34)
    more.load(path)
    assert more.get(api.F_REP) == 5
    for x in (src, dst, other, more):
        x.close()
    data.close()
