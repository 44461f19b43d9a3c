"""The injected-array parity modes of UpdateP and UpdateQMetro against the
reference's own array-fed functions (src/Updates/UpdateP.c:106-199,
src/Updates/UpdateQ.c:199-307) on the same chain state and the same uniform
array: the device runs the reference's sampler (RGammaDisc, src/ran.c:
1094-1188) in FP64 and stores P, Q and TestQ in FP32, so values agree to the
FP32 rounding of the reference's FP64 ones (one FP32 step where CUDA's and
the C library's log/exp round an FP64 value differently).  The reference's
reads past a 64-value block are counted by the oracle build (never fatal
there); the tests check that none happened, so both sides read the same
values."""
import numpy as np
import pytest

from structure_b200 import api, synth

pytestmark = pytest.mark.gpu

SEED = 0x1A7EC7ED


def _chain(ctx, d, K, **kw):
    data = api.Data(ctx, d["numalleles"], geno=d["geno"], layout=api.LAYOUT_U8)
    m = api.model_defaults(maxpops=K, burnin=0, numreps=10, store_z=1, **kw)
    return data, api.Chain(ctx, data, m, SEED)


def _f32_close(dev, ref64):
    """Device FP32 values equal the FP32 rounding of the reference's FP64 ones,
    or differ from it by at most one FP32 step; returns the exact fraction."""
    r32 = ref64.astype(np.float32)
    ulp = np.spacing(np.abs(r32))
    d = np.abs(dev.astype(np.float64) - r32.astype(np.float64))
    assert (d <= ulp).all(), float((d / np.maximum(ulp, 1e-45)).max())
    return float(np.mean(dev == r32))


@pytest.mark.parametrize("freqscorr", [0, 1])
def test_updatep_injected_matches_reference(ctx, ref, freqscorr):
    d = synth.microsat(N=70, L=45, K=3, seed=5 + freqscorr)
    geno, na = d["geno"], d["numalleles"]
    N, _, L = geno.shape
    K, A = 3, int(na.max())
    data, c = _chain(ctx, d, K, freqscorr=freqscorr, fpriormean=0.1, fpriorsd=0.1)
    rng = np.random.default_rng(11 + freqscorr)
    z = rng.integers(0, K, size=geno.shape).astype(np.int32)
    z[geno < 0] = -9
    zb = z.astype(np.int16)
    zb[zb < 0] = 255
    c.set(api.F_Z, zb.astype(np.uint8))          # recounts n from this Z
    eps = np.zeros((L, A))
    for l in range(L):
        eps[l, :na[l]] = rng.dirichlet(np.ones(na[l]))
    F = np.array([0.05, 0.2, 0.45])
    lam = np.array([1.0, 1.0, 1.0]) if freqscorr else np.array([0.7, 1.0, 1.6])
    c.set(api.F_EPS, eps)
    c.set(api.F_F, F)
    c.set(api.F_LAMBDA, lam)
    u = rng.random(L * K * A * 64)
    c.UpdatePInjected(u)
    assert c.sync() == 0
    Pd = c.get(api.F_P)

    ref.set_globals(N=N, L=L, K=K, maxalleles=A, freqscorr=freqscorr, fpriormean=0.1,
                    fpriorsd=0.1)
    g0 = ref.lib.stref_guard_hits()
    Pr = np.zeros(L * K * A)
    ref.lib.UpdateP(Pr, eps.reshape(-1).copy(), F.copy(), na.astype(np.int32), geno.copy(),
                    z.copy(), lam.copy(), ref.individuals(N), u)
    assert ref.lib.stref_guard_hits() == g0, "the reference read past a block"
    Pr = Pr.reshape(L, K, A)
    mask = np.broadcast_to(np.arange(A)[None, None, :] < na[:, None, None], Pr.shape)
    exact = _f32_close(Pd[mask], Pr[mask])
    assert exact > 0.99
    with np.errstate(divide="ignore"):      # an allele frequency that underflowed to 0
        np.testing.assert_allclose(c.get(api.F_LOGP)[mask], np.log(Pr[mask]), rtol=1e-6,
                                   atol=1e-6)
    c.close()
    data.close()


@pytest.mark.parametrize("alpha", [0.35, 1.0, 2.7])
def test_updateqmetro_injected_matches_reference(ctx, ref, alpha):
    """TestQ from the reference's Dirichlet sampler (shapes below one, one and
    above 2.5 take the sampler's three branches), the log ratio of the FP64
    data pass, and the accept decisions."""
    d = synth.microsat(N=64, L=50, K=4, seed=17)
    geno, na = d["geno"], d["numalleles"]
    N, _, L = geno.shape
    K, A = 4, int(na.max())
    data, c = _chain(ctx, d, K, metrofreq=1, popalphas=1)
    rng = np.random.default_rng(int(alpha * 100))
    Q = rng.dirichlet(np.full(K, 0.8), N).astype(np.float32)
    P = np.zeros((L, K, A), np.float32)
    for l in range(L):
        P[l, :, :na[l]] = rng.dirichlet(np.ones(na[l]), K)
    al = np.array([alpha, alpha * 0.5, alpha, alpha * 1.5]) if alpha != 1.0 else np.ones(K)
    c.set(api.F_Q, Q)
    c.set(api.F_P, P)
    c.set(api.F_ALPHA, al)
    u = rng.random(N * 64)
    c.UpdateQMetroInjected(u)
    assert c.sync() == 0
    Qd, Td, ld = c.get(api.F_Q), c.get(api.F_TESTQ), c.get(api.F_LOGDIFF)

    ref.set_globals(N=N, L=L, K=K, maxalleles=A, popalphas=1, metrofreq=1)
    g0 = ref.lib.stref_guard_hits()
    Qr = Q.astype(np.float64).copy()
    ref.lib.UpdateQMetro(geno.copy(), None, Qr, P.astype(np.float64), al.copy(), 1,
                         ref.individuals(N), None, u)
    assert ref.lib.stref_guard_hits() == g0, "the reference read past a block"
    acc_r = np.any(Qr != Q.astype(np.float64), axis=1)
    acc_d = np.all(Qd == Td, axis=1) & np.any(Td != Q, axis=1)
    # the log ratio of each individual on the device's TestQ, by the reference
    ld_r = np.array([ref.lib.CalcLikeIndDiff(geno, None, Td[i].astype(np.float64),
                                             Q[i].astype(np.float64), P.astype(np.float64), i,
                                             None) for i in range(N)])
    np.testing.assert_allclose(ld, ld_r, rtol=1e-11, atol=1e-9)
    # decisions: the same (the ratios differ only by the FP32 storage of
    # TestQ, far below the distance of log u from them here)
    np.testing.assert_array_equal(acc_d, acc_r)
    # accepted rows hold the reference's TestQ (FP32 rounding); rejected rows
    # keep Q exactly
    if acc_r.any():
        _f32_close(Qd[acc_r], Qr[acc_r])
    np.testing.assert_array_equal(Qd[~acc_d], Q[~acc_d])
    c.close()
    data.close()
