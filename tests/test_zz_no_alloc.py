"""st_update_z_noalloc: the Z update with counts and ln P(D) that allocates
no device memory, checked against the chain API's st_update_z (counts) and
st_collect (ln P(D)) on the same state.

Some callers cannot let a library call cudaMalloc: a host program that owns
every device allocation through its own pool, one that runs under a fixed
device-memory budget, or one on a path where an allocation would synchronise
the device.  This entry point keeps its count partials in one static device
array instead, and the caller passes device inputs and outputs.

The file is named so pytest collects it last.  It must pass alone in a fresh
process and after the other GPU tests (which leave the static array holding
their own contents, if they called it).

Tolerances are those of the other GPU tests: counts bit-exact, ln P(D) within
1e-5 relative.
"""
import ctypes as C

import numpy as np
import pytest

from structure_b200 import api, synth

pytestmark = pytest.mark.gpu

SEED = 0x5EED1234ABCD
NOALLOC_SCRATCH_BYTES = 32 << 20   # ST_NOALLOC_SCRATCH_BYTES in include/stgpu.h


def _entry():
    f = api.lib().st_update_z_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                  C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_size_t)]
    return f


def _state_and_reference(c):
    """Current Q, P, sweep index of a chain, and the chain API's results on them."""
    Q, P, rep = c.get(api.F_Q), c.get(api.F_P), c.get(api.F_REP)
    c.UpdateZ()
    n, m = c.get(api.F_N), c.get(api.F_M)
    c.DataCollection()
    like = c.get(api.F_STATS)[api.ST_LIKE]
    return Q, P, rep, n, m, like


@pytest.mark.parametrize("K,with_like", [(2, True), (5, True), (9, True), (20, False)])
def test_noalloc_matches_chain_update_z_on_two_calls_in_a_row(orc, K, with_like):
    """Two calls back to back on one stream, against the chain API's results
    on the same state and against the oracle (Z drawn by the oracle from the
    same Q, P and stream, then counted; ln P(D) of the same Q and P).  K=2 and
    5 read the per-class allele table, 9 the one-pair-per-population table and
    its two-half word loop, 20 the two-warp CTAs of the wide classes; the K=20
    case passes no ln P(D) output, which skips the last-CTA reduction."""
    import torch

    N, L = 700, 2600
    d = synth.snp_fmodel(N, L, K, np.linspace(0.05, 0.25, K), 0.4, 0.03, 21 + K)
    packed, na = np.ascontiguousarray(d["packed"], np.uint32), d["numalleles"]
    wpr = (N + 15) // 16
    assert packed.shape == (L, wpr)

    ctx = api.Context(0)
    data = api.Data(ctx, na, packed=packed, layout=api.LAYOUT_B2G, num_inds=N, num_loci=L)
    model = api.model_defaults(maxpops=K, burnin=0, numreps=10, freqscorr=1, metrofreq=10,
                               alpha=1.0, alphapropsd=0.025, computeprob=1)
    chain = api.Chain(ctx, data, model, SEED)
    assert chain.A == 2

    # two chain states, each with the chain API's counts and ln P(D)
    chain.sweep(2)
    s1 = _state_and_reference(chain)
    chain.sweep(1)
    s2 = _state_and_reference(chain)
    assert s1[2] != s2[2]

    dev = torch.device("cuda:0")
    g2 = torch.from_numpy(packed.view(np.int32)).to(dev)
    ins, outs = [], []
    for Q, P, _, _, _, _ in (s1, s2):
        ins.append((torch.from_numpy(Q).to(dev), torch.from_numpy(np.ascontiguousarray(P)).to(dev)))
        outs.append((torch.full((L, K, 2), -1, dtype=torch.int32, device=dev),
                     torch.full((N, K), -1, dtype=torch.int32, device=dev),
                     torch.full((1,), float("nan"), dtype=torch.float64, device=dev),
                     torch.full((1,), -1, dtype=torch.int32, device=dev)))
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)

    f = _entry()
    need = C.c_size_t(0)
    # the two calls back to back on one stream, no host sync between them
    for (q, p), (n_o, m_o, like_o, err_o), s in zip(ins, outs, (s1, s2)):
        rc = f(0, g2.data_ptr(), wpr, N, L, K, q.data_ptr(), p.data_ptr(), SEED, s[2],
               n_o.data_ptr(), m_o.data_ptr(), like_o.data_ptr() if with_like else None,
               err_o.data_ptr(), C.c_void_p(stream.cuda_stream), C.byref(need))
        assert rc == api.ST_OK, rc
        assert 0 < need.value <= NOALLOC_SCRATCH_BYTES
    torch.cuda.synchronize(dev)

    geno = d["geno"]
    for (n_o, m_o, like_o, err_o), (Q, P, rep, n_ref, m_ref, like_ref) in zip(outs, (s1, s2)):
        assert int(err_o.item()) == 0
        np.testing.assert_array_equal(n_o.cpu().numpy(), n_ref)
        np.testing.assert_array_equal(m_o.cpu().numpy(), m_ref)
        # the oracle: Z from the same Q, P and stream, then GetNumFromPops /
        # GetNumLociPop on it
        zo = orc.zupdate_f32(geno, Q, P, SEED, rep)
        n_orc, m_orc = orc.counts(geno, zo, K, 2)
        np.testing.assert_array_equal(n_o.cpu().numpy(), n_orc)
        np.testing.assert_array_equal(m_o.cpu().numpy(), m_orc)
        if with_like:
            like = float(like_o.item())
            assert abs(like - like_ref) <= 1e-5 * abs(like_ref), (like, like_ref)
            like_orc = orc.calc_like(geno, Q, P)
            assert abs(like - like_orc) <= 1e-5 * abs(like_orc), (like, like_orc)
        else:
            assert np.isnan(float(like_o.item()))   # not written

    # every observed allele copy is counted once in n and once in m
    copies = int(2 * N * L - 2 * np.count_nonzero(synth.unpack_int32(packed, N)[:, 0, :] < 0))
    for n_o, m_o, _, _ in outs:
        assert int(n_o.sum()) == copies == int(m_o.sum())

    chain.close()
    data.close()
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_static_scratch():
    import torch

    dev = torch.device("cuda:0")
    tiny_i = torch.zeros(16, dtype=torch.int32, device=dev)
    tiny_f = torch.zeros(16, dtype=torch.float32, device=dev)
    f = _entry()
    need = C.c_size_t(0)
    N, L, K = 10000, 500000, 10
    # rejected on the host before any device work, so the tiny buffers are never read
    rc = f(0, tiny_i.data_ptr(), (N + 15) // 16, N, L, K, tiny_f.data_ptr(), tiny_f.data_ptr(),
           SEED, 0, tiny_i.data_ptr(), tiny_i.data_ptr(), None, None, None, C.byref(need))
    assert rc == api.ST_ERR_ADMISSION
    assert need.value > NOALLOC_SCRATCH_BYTES
    rc = f(0, tiny_i.data_ptr(), 1, 32, 64, K, tiny_f.data_ptr(), tiny_f.data_ptr(),
           SEED, 0, tiny_i.data_ptr(), tiny_i.data_ptr(), None, None, None, None)
    assert rc == api.ST_ERR_ARG   # row stride shorter than ceil(num_inds/16) words
