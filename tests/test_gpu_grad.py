"""Gradient of ln P(D|Q,P) (Z summed out) with respect to the softmax logits
of Q and P: the device (st_loglik_grad, FP32 and FP64) against the oracle's
FP64 restatement of CalcLikeInd without clamps (oracle/st_oracle.c
orc_loglik_grad), and torch.autograd.gradcheck (finite differences) on a
64-individual x 256-locus slice through the torch.autograd.Function shim.

Tolerances: FP64 1e-10 relative; FP32 ln P(D) 1e-5 relative and each
gradient entry within a derived bound: every entry is p * (g - <p, g>) with
g a sum of n positive terms (n = 2L allele copies for Q, 2N for P), so with
unit roundoff u = 2^-24 its error is at most (n + K + 16) u times
p * (g + <p, g>) (the summation, the K products of S, the reciprocal and
the softmax, each a few u).
"""
import numpy as np
import pytest

from structure_b200 import api, synth
from structure_b200.grad import LogLikGrad, loglik

pytestmark = pytest.mark.gpu


def _data(ctx, N, L, K, seed):
    d = synth.snp_fmodel(N, L, K, np.linspace(0.05, 0.3, K), 0.3, 0.03, seed)
    data = api.Data(ctx, d["numalleles"], packed=d["packed"], layout=api.LAYOUT_B2G,
                    num_inds=N, num_loci=L)
    return d["geno"], data


def _logits(rng, N, L, K, scale=1.5):
    return rng.normal(0, scale, (N, K)), rng.normal(0, scale, (L, K, 2))


@pytest.mark.parametrize("K", [1, 3, 8, 13])
def test_grad_fp64_matches_oracle(ctx, orc, K):
    import torch
    N, L = 150, 700
    geno, data = _data(ctx, N, L, max(K, 2), 40 + K)
    rng = np.random.default_rng(K)
    ql, pl = _logits(rng, N, L, K)
    ev = LogLikGrad(ctx, data, K, precision=64)
    ll, dq, dp, lli = ev(torch.tensor(ql, device="cuda"), torch.tensor(pl, device="cuda"),
                         per_individual=True)
    torch.cuda.synchronize()
    llo, dqo, dpo, llio = orc.loglik_grad(geno, ql, pl)
    assert abs(ll.item() - llo) <= 1e-10 * abs(llo)
    np.testing.assert_allclose(lli.cpu().numpy(), llio, rtol=1e-10)
    np.testing.assert_allclose(dq.cpu().numpy(), dqo, rtol=1e-9, atol=1e-9 * np.abs(dqo).max())
    np.testing.assert_allclose(dp.cpu().numpy(), dpo, rtol=1e-9, atol=1e-9 * np.abs(dpo).max())
    ev.close(); data.close()


def test_grad_fp32_matches_oracle(ctx, orc):
    import torch
    N, L, K = 300, 2000, 8
    geno, data = _data(ctx, N, L, K, 77)
    rng = np.random.default_rng(5)
    ql, pl = _logits(rng, N, L, K)
    ev = LogLikGrad(ctx, data, K, precision=32)
    ll, dq, dp = ev(torch.tensor(ql, dtype=torch.float32, device="cuda"),
                    torch.tensor(pl, dtype=torch.float32, device="cuda"))
    torch.cuda.synchronize()
    # the oracle runs on the logits the device saw (rounded to float)
    llo, dqo, dpo, _ = orc.loglik_grad(geno, ql.astype(np.float32).astype(np.float64),
                                       pl.astype(np.float32).astype(np.float64))
    assert abs(ll.item() - llo) <= 1e-5 * abs(llo)
    sq, sp = _grad_scales(geno, ql.astype(np.float32).astype(np.float64),
                          pl.astype(np.float32).astype(np.float64))
    u = 2.0 ** -24
    worst = {}
    for name, dev, ref, scale, n in (("Q", dq, dqo, sq, 2 * L), ("P", dp, dpo, sp, 2 * N)):
        err = np.abs(dev.cpu().numpy().astype(np.float64) - ref)
        bound = (n + K + 16) * u * scale
        assert (err <= bound).all(), (name, (err / bound).max())
        worst[name] = float((err / scale).max())
    print("FP32 gradient, largest error / (p (g + <p, g>)):", worst)
    ev.close(); data.close()


def _grad_scales(geno, ql, pl):
    """p * (g + <p, g>) for the Q and P logits, g the gradient with respect to
    Q and P themselves (sums of positive terms)."""
    Q = np.exp(ql - ql.max(1, keepdims=True))
    Q /= Q.sum(1, keepdims=True)
    P = np.exp(pl - pl.max(2, keepdims=True))
    P /= P.sum(2, keepdims=True)
    N, _, L = geno.shape
    gq, gp = np.zeros_like(Q), np.zeros_like(P)
    for c in range(2):
        a = geno[:, c, :]                              # [N][L]
        ok = a >= 0
        Pa = P[np.arange(L)[None, :], :, np.where(ok, a, 0)]    # [N][L][K]
        S = np.einsum("ik,ilk->il", Q, Pa)
        w = np.where(ok, 1.0 / np.where(ok, S, 1.0), 0.0)        # [N][L]
        gq += np.einsum("ilk,il->ik", Pa, w)
        for al in range(P.shape[2]):
            gp[:, :, al] += np.einsum("ik,il->lk", Q, w * (a == al))
    sq = Q * (gq + (Q * gq).sum(1, keepdims=True))
    sp = P * (gp + (P * gp).sum(2, keepdims=True))
    return sq, sp


def test_gradcheck_on_a_slice(ctx):
    """Finite differences of the FP64 device likelihood on 64 x 256."""
    import torch
    N, L, K = 64, 256, 4
    _, data = _data(ctx, N, L, K, 91)
    ev = LogLikGrad(ctx, data, K, precision=64)
    rng = np.random.default_rng(3)
    ql, pl = _logits(rng, N, L, K, scale=1.0)
    q = torch.tensor(ql, device="cuda", requires_grad=True)
    p = torch.tensor(pl, device="cuda", requires_grad=True)
    assert torch.autograd.gradcheck(lambda a, b: loglik(a, b, ev), (q, p), eps=1e-6, atol=1e-5,
                                    rtol=1e-6, nondet_tol=1e-9)
    out = loglik(q, p, ev)
    out.backward()
    _, dq, dp = ev(q.detach(), p.detach())
    torch.testing.assert_close(q.grad, dq)
    torch.testing.assert_close(p.grad, dp)
    ev.close(); data.close()


def test_grad_rejects_unsupported(ctx):
    import ctypes as C
    geno = synth.microsat(N=20, L=10, K=2, seed=1)
    data = api.Data(ctx, geno["numalleles"], geno=geno["geno"])
    h = C.c_void_p()
    assert api.lib().st_grad_create(ctx.h, data.h, 2, 32, C.byref(h)) == api.ST_ERR_UNSUPPORTED
    data.close()
    _, d2 = _data(ctx, 32, 40, 2, 5)
    assert api.lib().st_grad_create(ctx.h, d2.h, 17, 32, C.byref(h)) == api.ST_ERR_UNSUPPORTED
    assert api.lib().st_grad_create(ctx.h, d2.h, 4, 16, C.byref(h)) == api.ST_ERR_ARG
    d2.close()
