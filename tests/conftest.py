import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def orc():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import RefLib, ref_available
    if not ref_available():
        pytest.skip("reference CPU library not built")
    return RefLib()


@pytest.fixture(scope="session")
def ctx():
    from structure_b200 import Context
    return Context(0)


# ---------------------------------------------------------------------------
# Error bound of the device's Metropolis log ratio (used by the parity tests)
# ---------------------------------------------------------------------------
U32 = 2.0 ** -24            # unit roundoff of FP32


def _log_err(x):
    """Bound on the error of the device's fast FP32 log (__logf) at x: an
    absolute 2^-21.41 on [0.5, 2], else 3 ulp of the result (CUDA's documented
    bounds for the intrinsic), taken as the larger of the two everywhere."""
    return np.maximum(2.0 ** -21.41, 3.0 * 2.0 ** -23 * np.abs(np.log(x)))


def metro_terms_and_bound(geno, Q, T, P, chunk=2048):
    """Per individual: the FP64 log ratio sum_l log(T_i.P_l,g / Q_i.P_l,g) (the
    oracle's value), sum_l |term|, and a bound on the error of the device's
    FP32 form of it (the biallelic data pass; the one-byte layout's pass runs
    in FP64 and is far inside it).  Per genotype with both copies present the
    device forms tp = (T.P_a0)(T.P_a1) and tm = (Q.P_a0)(Q.P_a1) in FP32 from
    K-term multiply-add chains (relative error <= (2K+1) u each), takes one
    fast log of each and subtracts; per genotype the bound is
    2(2K+1)u + e_log(tp) + e_log(tm) + u|term|.  The FP32 sums over a warp's
    loci and locus blocks add at most 80 u sum|term| (5 butterfly levels and
    at most 64 locus blocks, with margin); the rest is summed in FP64.
    Half-missing genotypes (one-byte layout only) are bounded per copy."""
    N, _, L = geno.shape
    K = Q.shape[1]
    Q64, T64, P64 = (np.asarray(x, np.float64) for x in (Q, T, P))
    ld = np.zeros(N)
    mag = np.zeros(N)
    bnd = np.zeros(N)
    for l0 in range(0, L, chunk):
        l1 = min(L, l0 + chunk)
        g0 = geno[:, 0, l0:l1]
        g1 = geno[:, 1, l0:l1]
        Pc = P64[l0:l1]                                      # [n, K, A]
        n, A = Pc.shape[0], Pc.shape[2]
        Pk = Pc.transpose(1, 0, 2).reshape(K, n * A)
        qa = (Q64 @ Pk).reshape(N, n, A)                     # Q_i . P_l,:,a
        ta = (T64 @ Pk).reshape(N, n, A)
        ii = np.arange(N)[:, None]
        ll = np.arange(n)[None, :]
        ok0, ok1 = g0 >= 0, g1 >= 0
        a0, a1 = np.where(ok0, g0, 0), np.where(ok1, g1, 0)
        q0, q1 = qa[ii, ll, a0], qa[ii, ll, a1]
        t0, t1 = ta[ii, ll, a0], ta[ii, ll, a1]
        both = ok0 & ok1
        one = ok0 ^ ok1
        tp = np.where(both, t0 * t1, 1.0)
        tm = np.where(both, q0 * q1, 1.0)
        term = np.where(both, np.log(tp) - np.log(tm), 0.0)
        eb = np.where(both, 2 * (2 * K + 1) * U32 + _log_err(tp) + _log_err(tm)
                      + U32 * np.abs(term), 0.0)
        # one copy present: that copy's ratio alone
        qs = np.where(one, np.where(ok0, q0, q1), 1.0)
        ts = np.where(one, np.where(ok0, t0, t1), 1.0)
        tone = np.where(one, np.log(ts) - np.log(qs), 0.0)
        eone = np.where(one, 2 * K * U32 + _log_err(ts) + _log_err(qs) + U32 * np.abs(tone), 0.0)
        term = term + tone
        ld += term.sum(1)
        mag += np.abs(term).sum(1)
        bnd += (eb + eone).sum(1)
    bnd += 80 * U32 * mag
    return ld, mag, bnd


def metro_uniforms(orc, N, seed, rep):
    """The accept uniforms u_i of the Metropolis Q step (accept iff
    u_i < exp(logdiff_i)), from the oracle's stream as orc_metro_accept draws
    them: block (i, 0) of stream 6 at sweep rep, 52 bits of words 0 and 1."""
    from oracle.oracle import S_QMA
    u = np.empty(N)
    for i in range(N):
        w = orc.stream(i, 0, rep, S_QMA, seed)
        x = ((int(w[0]) >> 6) << 26) | (int(w[1]) >> 6)
        u[i] = (x + 0.5) / 4503599627370496.0
    return u


def check_metro_decisions(ld_dev, ld_o, bound, u):
    """Every decision outside the error band |log u - ld| <= bound must be the
    same for the device's and the oracle's log ratios.  Returns (number of
    individuals inside the band, number of decisions that differ)."""
    lu = np.log(u)
    acc_d = lu < ld_dev
    acc_o = lu < ld_o
    band = np.abs(lu - ld_o) <= bound
    assert np.array_equal(acc_d[~band], acc_o[~band])
    return int(band.sum()), int((acc_d != acc_o).sum())
