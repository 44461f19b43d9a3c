"""ln P(D|Q,P) with Z summed out, and its gradient, as a torch.autograd.Function.

Test and experiment shim over the C ABI (st_grad_create / st_loglik_grad): the
forward pass evaluates ln P(D|softmax(q_logits), softmax(p_logits)) on the
device and keeps the gradient that the same call computed; the backward pass
scales it by the incoming gradient.  Torch supplies device memory and the
stream; the arithmetic is the library's (structure_b200/csrc/st_grad.cu).

q_logits: [N, K] over populations; p_logits: [L, K, 2] over the two alleles of
each biallelic locus.  float32 or float64 (the precision of the evaluator).
"""
import ctypes as C

from . import api


class LogLikGrad:
    """Evaluator bound to one data set and K (st_grad_create)."""

    def __init__(self, ctx, data, K, precision=32):
        self.ctx, self.data, self.K, self.precision = ctx, data, K, precision
        self.h = C.c_void_p()
        ctx.check(api.lib().st_grad_create(ctx.h, data.h, K, precision, C.byref(self.h)))

    def __call__(self, q_logits, p_logits, per_individual=False):
        """Returns (loglik [1] float64, dq, dp[, ll_ind [N] float64]) as tensors."""
        import torch
        dt = torch.float64 if self.precision == 64 else torch.float32
        assert q_logits.dtype == dt and p_logits.dtype == dt
        q = q_logits.detach().contiguous()
        p = p_logits.detach().contiguous()
        N, K = q.shape
        assert K == self.K and p.shape[1:] == (K, 2)
        dq, dp = torch.empty_like(q), torch.empty_like(p)
        ll = torch.empty(1, dtype=torch.float64, device=q.device)
        lli = torch.empty(N, dtype=torch.float64, device=q.device) if per_individual else None
        # launch on torch's current stream; its legacy default stream (handle 0)
        # is passed as cudaStreamLegacy, since NULL selects the context's own
        # (the context's own stream is selected again afterwards)
        self.ctx.set_stream(torch.cuda.current_stream(q.device).cuda_stream or 1)
        try:
            self.ctx.check(api.lib().st_loglik_grad(self.h, q.data_ptr(), p.data_ptr(),
                                                    dq.data_ptr(), dp.data_ptr(), ll.data_ptr(),
                                                    lli.data_ptr() if lli is not None else None))
        finally:
            self.ctx.set_stream(None)
        return (ll, dq, dp, lli) if per_individual else (ll, dq, dp)

    def close(self):
        if self.h:
            api.lib().st_grad_destroy(self.h)
            self.h = C.c_void_p()


def _function():
    import torch

    class LogLik(torch.autograd.Function):
        @staticmethod
        def forward(fctx, q_logits, p_logits, evaluator):
            ll, dq, dp = evaluator(q_logits, p_logits)
            fctx.save_for_backward(dq, dp)
            return ll[0].to(q_logits.dtype)

        @staticmethod
        def backward(fctx, grad_out):
            dq, dp = fctx.saved_tensors
            return grad_out * dq, grad_out * dp, None

    return LogLik


_LOGLIK = None


def loglik(q_logits, p_logits, evaluator):
    """ln P(D|softmax(q_logits), softmax(p_logits)), differentiable in both."""
    global _LOGLIK
    if _LOGLIK is None:
        _LOGLIK = _function()
    return _LOGLIK.apply(q_logits, p_logits, evaluator)
