"""Gradient of ln P(D|Q,P) (Z summed out) with respect to the softmax logits
of Q and P: the device (st_loglik_grad, FP32 and FP64) against the oracle's
FP64 restatement of CalcLikeInd without clamps (oracle/st_oracle.c
orc_loglik_grad), and torch.autograd.gradcheck (finite differences) on a
64-individual x 256-locus slice through the torch.autograd.Function shim.

Tolerances: FP64 1e-10 relative; FP32 ln P(D) 1e-5 relative and gradients
within 2e-4 of the largest entry's magnitude.
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
    for dev, ref in ((dq, dqo), (dp, dpo)):
        err = np.abs(dev.cpu().numpy().astype(np.float64) - ref)
        assert err.max() <= 2e-4 * np.abs(ref).max(), (err.max(), np.abs(ref).max())
    ev.close(); data.close()


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
