"""Regenerate tests/golden/*.npz from the reference's own CPU functions.

    python tests/golden/make_golden.py

Needs oracle/_ref/libstref.so (built by oracle/Makefile from the reference
sources).  Each fixture stores its inputs and the reference's outputs, so the
oracle can be checked on machines without the reference tree.  Random streams
fed to the reference are the Philox streams the device uses, written as the
values rand()/RNormal() returned.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from structure_b200 import synth  # noqa: E402
from oracle.oracle import Oracle, RefLib, S_ALPHA, S_EPS, S_INITZ, rnd_words  # noqa: E402

KEY = 0x600DF00D1234


def main():
    orc, ref = Oracle(), RefLib()
    out = {}

    # -- UpdateZ (FP64, uniforms injected), counts, CalcLike on microsat data --
    d = synth.microsat(N=24, L=16, K=3, seed=77)
    geno, na = d["geno"], d["numalleles"]
    N, _, L = geno.shape
    K, A = 3, int(na.max())
    rng = np.random.default_rng(77)
    Q = rng.dirichlet(np.full(K, 0.7), N).astype(np.float32).astype(np.float64)
    P = np.zeros((L, K, A))
    for l in range(L):
        P[l, :, :na[l]] = rng.dirichlet(np.ones(na[l]), K)
    P = P.astype(np.float32).astype(np.float64)
    u = rng.random(N * L * 2)
    ref.set_globals(N=N, L=L, K=K, maxalleles=A)
    Z = np.zeros_like(geno)
    ref.lib.UpdateZ(Z, Q, P, geno.copy(), u)
    n = np.zeros(L * K * A, np.int32)
    ref.lib.GetNumFromPops(n, geno.copy(), Z, na.astype(np.int32), ref.individuals(N))
    m = np.zeros((N, K), np.int32)
    tmp = np.zeros(K, np.int32)
    for i in range(N):
        ref.lib.GetNumLociPop(tmp, Z, i)
        m[i] = tmp
    like = ref.lib.CalcLike(geno.copy(), None, Q, P, None, None, None)
    zi_vals = []
    for i in range(N):
        for line in range(2):
            for l in range(L):
                if geno[i, line, l] >= 0:
                    w = orc.stream(l, i >> 1, 0, S_INITZ, KEY)
                    zi_vals.append(int(w[2 * (i & 1) + line]) >> 1)
    ref.rand_queue(zi_vals)
    Zi = np.zeros_like(geno)
    ref.lib.InitializeZ(geno.copy(), ref.individuals(N), Zi)
    ref.rand_queue(None)
    np.savez_compressed(os.path.join(HERE, "z_counts_like.npz"), geno=geno, numalleles=na, Q=Q,
                        P=P, u=u, Z=Z, n=n.reshape(L, K, A), m=m, like=like, key=KEY, Zinit=Zi,
                        raw=d["geno_raw"])

    # -- UpdateAlpha (POPALPHAS=1) fed fixed normals and rand() values ---------
    Nq, Kq = 40, 3
    Qa = rng.dirichlet(np.full(Kq, 0.6), Nq).astype(np.float32)
    logQ = np.log(Qa.astype(np.float64)).astype(np.float32)
    Qd = np.exp(logQ.astype(np.float64))
    alpha0 = np.array([0.6, 1.1, 0.9])
    normals = np.array([orc.normal(p, 5, S_ALPHA, KEY) for p in range(Kq)])
    rands = []
    for p in range(Kq):
        na_ = alpha0[p] + 0.2 * normals[p]
        if 0 < na_ < 10.0:
            rands += rnd_words(orc.stream(p, 1, 5, S_ALPHA, KEY))
    ref.set_globals(N=Nq, L=1, K=Kq, maxalleles=2, popalphas=1, alphapropsd=0.2, alphamax=10.0)
    ar = alpha0.copy()
    ref.normal_queue(normals)
    ref.rand_queue(rands)
    ref.lib.UpdateAlpha(Qd.copy(), ar, ref.individuals(Nq), 5)
    ref.rand_queue(None)
    ref.normal_queue(None)
    np.savez_compressed(os.path.join(HERE, "alpha_popalphas.npz"), logQ=logQ, alpha0=alpha0,
                        alpha1=ar, rep=5, key=KEY, sd=0.2, amax=10.0)

    # -- NonIndependenceUpdateEpsilon fed fixed rand() values -------------------
    Le, Ke = 12, 3
    nae = na[:Le].copy()
    Ae = int(nae.max())
    Pe = np.zeros((Le, Ke, Ae))
    for l in range(Le):
        Pe[l, :, :nae[l]] = rng.dirichlet(np.ones(nae[l]), Ke)
    logP = np.log(np.maximum(Pe, 1e-300)).astype(np.float32)
    logP[Pe == 0] = 0
    Pd = np.where(Pe > 0, np.exp(logP.astype(np.float64)), 0)
    eps0 = np.zeros((Le, Ae))
    for l in range(Le):
        eps0[l, :nae[l]] = rng.dirichlet(np.ones(nae[l]) * 5)
    Fe = np.array([0.05, 0.2, 0.4])
    inv = float(N) ** -0.5
    vals = []
    for l in range(Le):
        if nae[l] > 1:
            w = orc.stream(l, 0, 2, S_EPS, KEY)
            a1 = int(((int(w[0]) >> 1) / 2147483648.0) * nae[l])
            a2 = int(((int(w[1]) >> 1) / 2147483648.0) * (nae[l] - 1))
            a2 = a2 + 1 if a2 >= a1 else a2
            dl = ((int(w[2]) >> 1) / 2147483648.0) * inv
            vals += [int(w[0]) >> 1, int(w[1]) >> 1, int(w[2]) >> 1]
            if eps0[l, a1] + dl < 1.0 and eps0[l, a2] - dl > 0.0:
                vals += rnd_words(orc.stream(l, 1, 2, S_EPS, KEY))
    ref.set_globals(N=N, L=Le, K=Ke, maxalleles=Ae, freqscorr=1)
    er = eps0.copy()
    ref.rand_queue(vals)
    ref.lib.UpdateEpsilon(Pd, er, Fe.copy(), nae.astype(np.int32), 1.0)
    ref.rand_queue(None)
    np.savez_compressed(os.path.join(HERE, "epsilon.npz"), numalleles=nae, logP=logP, eps0=eps0,
                        eps1=er, F=Fe, inv=inv, rep=2, key=KEY)
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
