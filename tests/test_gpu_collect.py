"""DataCollection on a fixed state against the reference's own UpdateSums
(src/output.c:654-707) and DataCollection's alpha sums (output.c:76-85).

The device (st_collect) and the reference are fed the same Q, P, eps, F,
alpha and lambda (the device's FP32 Q and P upcast for the reference), twice
in a row, so every accumulator is compared after two additions: QSum, PSum,
SumEpsilon, FstSum, sumAlpha, sumlambda exactly (one FP64 addition of the
same values in the same order per element), and AncestDist (the histogram of
Q in NUMBOXES boxes) exactly, since both sides bin the same FP32 value in FP64.

A chain of the reference keeps Q in FP64, the device in FP32.  For the same
posterior draw the two can fall in different boxes only when the FP64 value
and its FP32 rounding straddle a box edge k/NUMBOXES; the last test counts
how often that happens for Dirichlet draws (about 2 NUMBOXES 2^-24 per entry).
"""
import numpy as np
import pytest

from structure_b200 import api, synth

SEED = 0xC011EC7


@pytest.mark.gpu
@pytest.mark.parametrize("freqscorr,K", [(1, 5), (0, 3)])
def test_collect_matches_reference_updatesums(ctx, ref, freqscorr, K):
    if freqscorr:
        s = synth.snp_fmodel(150, 300, K, np.linspace(0.05, 0.25, K), 0.4, 0.03, 41)
    else:
        s = synth.microsat(N=150, L=80, K=K, seed=41 + K)
    geno, na = s["geno"], s["numalleles"]
    N, _, L = geno.shape
    A = int(na.max())
    numboxes = 1000
    m = api.model_defaults(maxpops=K, burnin=0, numreps=10, freqscorr=freqscorr, ancestdist=1,
                           numboxes=numboxes, computeprob=1, inferalpha=1, popalphas=1)
    data = api.Data(ctx, na, geno=geno)
    c = api.Chain(ctx, data, m, SEED)
    rng = np.random.default_rng(K)
    Q = rng.dirichlet(np.full(K, 0.4), N).astype(np.float32)
    # entries exactly on, and one FP32 step below, box edges; Q = 1
    Q[0, 0] = np.float32(0.5)
    Q[1, 0] = np.nextafter(np.float32(0.25), np.float32(0))
    Q[2, 0] = np.float32(1.0)
    Q[2, 1:] = 0.0
    Q[3, 0] = np.float32(0.001)
    P = np.zeros((L, K, A), np.float32)
    for l in range(L):
        P[l, :, :na[l]] = rng.dirichlet(np.ones(na[l]), K)
    eps = np.zeros((L, A))
    for l in range(L):
        eps[l, :na[l]] = rng.dirichlet(np.ones(na[l]))
    F = rng.uniform(0.01, 0.4, K)
    alpha = rng.uniform(0.2, 2.0, K)
    lam = rng.uniform(0.5, 1.5, K)
    c.set(api.F_Q, Q)
    c.set(api.F_P, P)
    c.set(api.F_EPS, eps)
    c.set(api.F_F, F)
    c.set(api.F_ALPHA, alpha)
    c.set(api.F_LAMBDA, lam)
    for f in (api.F_QSUM, api.F_PSUM, api.F_SUMEPS, api.F_FSTSUM, api.F_SUMALPHA,
              api.F_SUMLAMBDA, api.F_ANCESTDIST):
        assert not c.get(f).any()
    c.DataCollection()
    c.DataCollection()
    assert c.sync() == 0

    ref.set_globals(N=N, L=L, K=K, maxalleles=A, freqscorr=freqscorr, ancestdist=1,
                    numboxes=numboxes, popalphas=1)
    Q64, P64 = Q.astype(np.float64), P.astype(np.float64).reshape(-1)
    QSum = np.zeros(N * K)
    PSum = np.zeros(L * K * A)
    FstSum = np.zeros(K)
    SumEps = np.zeros(L * A)
    sumlam = np.zeros(K)
    AD = np.zeros(N * K * numboxes, np.int32)
    Z = np.zeros(N * 2 * L, np.int32)
    eps_r = eps.reshape(-1).copy()
    for _ in range(2):
        ref.lib.UpdateSums(Q64.reshape(-1), QSum, Z, P64, PSum, F.copy(), FstSum,
                           na.astype(np.int32), AD.ctypes.data, eps_r, SumEps, lam.copy(),
                           sumlam, None, None, 0)
    sumAlpha = alpha + alpha          # output.c:81-85: sumAlpha[pop] += Alpha[pop]

    np.testing.assert_array_equal(c.get(api.F_QSUM).reshape(-1), QSum)
    np.testing.assert_array_equal(c.get(api.F_PSUM).reshape(-1), PSum)
    np.testing.assert_array_equal(c.get(api.F_SUMLAMBDA), sumlam)
    np.testing.assert_array_equal(c.get(api.F_SUMALPHA)[:K], sumAlpha)
    if freqscorr:
        np.testing.assert_array_equal(c.get(api.F_FSTSUM), FstSum)
        np.testing.assert_array_equal(c.get(api.F_SUMEPS).reshape(-1), SumEps)
    ad = c.get(api.F_ANCESTDIST)
    np.testing.assert_array_equal(ad.reshape(-1), AD)
    assert ad[2, 0, numboxes - 1] == 2     # Q = 1 goes to the last box, as in the reference
    assert ad[0, 0, 500] == 2 and ad[1, 0, 249] == 2 and ad[3, 0, 1] == 2
    c.close()
    data.close()


def test_ancestdist_fp32_fp64_edge_rate():
    """How often the FP32 rounding of an FP64 Q moves it across a box edge of
    AncestDist (the only way the device's histogram of a chain can differ from
    one kept in FP64 for the same draws): measured on 10^6 Dirichlet draws and
    bounded by 4 NUMBOXES 2^-24 per entry, about 2.4e-4."""
    rng = np.random.default_rng(5)
    q64 = rng.dirichlet(np.full(5, 0.3), 200000).reshape(-1)
    nb = 1000
    b64 = np.minimum((q64 * nb).astype(np.int64), nb - 1)
    b32 = np.minimum((q64.astype(np.float32).astype(np.float64) * nb).astype(np.int64), nb - 1)
    rate = float(np.mean(b64 != b32))
    print(f"AncestDist boxes moved by FP32 rounding: {rate:.2e} per entry")
    assert rate <= 4 * nb * 2.0 ** -24
