"""ctypes bindings for the test oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py.  The product (structure_b200) never
imports this module.

* ``Oracle``  -- liboracle.so, the CPU restatement of the hot path (st_oracle.c).
* ``RefLib``  -- _ref/libstref.so, the reference's own CPU code
  (pmelsted/structure src/*.c) driven by ref_driver.c.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's src/ directory; STRUCTURE_REF_SRC overrides the default
REF_SRC = os.environ.get("STRUCTURE_REF_SRC", "/root/reference/src")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_ci, _cd, _cu32, _cu64 = C.c_int, C.c_double, C.c_uint32, C.c_uint64

(S_INITZ, S_Z, S_P, S_QG, S_QM, S_QMA, S_ALPHA, S_EPS, S_FST, S_MALA, S_LAMBDA,
 S_NOADMIX, S_POPINFO, S_LOCPRIOR, S_LOCALPHA) = range(1, 16)


def rnd_words(w):
    """The rand() values the reference's rnd() (ran.c:152-161) consumes when
    it reproduces rnd31 of one Philox block: leading zeros, then the first
    non-zero 31-bit word."""
    out = []
    for x in w:
        out.append(int(x) >> 1)
        if out[-1] != 0:
            break
    return out


def build(ref=True):
    """Compile liboracle.so (and, when the reference tree is present, libstref.so)."""
    targets = ["oracle"]
    if ref and os.path.isdir(REF_SRC):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, "REF=" + REF_SRC] + targets, check=True)


def _load(path):
    if not os.path.exists(path):
        build(ref=path.endswith("libstref.so"))
    return C.CDLL(path)


class Oracle:
    def __init__(self):
        lib = self.lib = _load(os.path.join(HERE, "liboracle.so"))
        lib.orc_philox.argtypes = [_u32p, _cu64, _u32p]
        lib.orc_stream.argtypes = [_cu32, _cu32, _cu32, _cu32, _cu64, _u32p]
        lib.orc_seed32.argtypes = [_cu64]
        lib.orc_seed32.restype = _cu32
        lib.orc_lgamma.argtypes = [_cd]
        lib.orc_lgamma.restype = _cd
        lib.orc_loggamma.argtypes = [_cd, _cu32, _cu32, _cu32, _cu64, C.POINTER(_ci)]
        lib.orc_loggamma.restype = _cd
        lib.orc_loggamma_f32.argtypes = [C.c_float, _cu32, _cu32, _cu32, _cu64, C.POINTER(_ci)]
        lib.orc_loggamma_f32.restype = C.c_float
        lib.orc_ln_f32.argtypes = [C.c_float]
        lib.orc_ln_f32.restype = C.c_float
        lib.orc_sincos_2pi_f32.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        lib.orc_normal.argtypes = [_cu32, _cu32, _cu32, _cu64]
        lib.orc_normal.restype = _cd
        lib.orc_init_z.argtypes = [_ci, _ci, _ci, _i32p, _cu64, _i32p]
        lib.orc_zupdate_f32.argtypes = [_ci, _ci, _ci, _ci, _i32p, _f32p, _f32p, _cu64, _cu32, _i32p]
        lib.orc_zupdate_f64_injected.argtypes = [_ci, _ci, _ci, _ci, _i32p, _f64p, _f64p, _f64p, _i32p, _i32p]
        lib.orc_counts.argtypes = [_ci, _ci, _ci, _ci, _i32p, _i32p, _ci, _i32p, _i32p, _i32p]
        lib.orc_update_p.argtypes = [_ci, _ci, _ci, _i32p, _i32p, _ci, _f64p, _f64p, _f64p,
                                     _cu64, _cu32, _f32p, _f32p, C.POINTER(_ci)]
        lib.orc_update_q_gibbs.argtypes = [_ci, _ci, _i32p, _f64p, _cu64, _cu32, _f32p, _f32p,
                                           C.POINTER(_ci), C.c_void_p]
        lib.orc_metro_propose.argtypes = [_ci, _ci, _f64p, _cu64, _cu32, _f32p, _f32p,
                                          C.POINTER(_ci), C.c_void_p]
        lib.orc_update_locprior.argtypes = [_ci, _ci, _ci, _ci, _i32p, _f32p, _f64p, _f64p, _cd,
                                            _cd, _cd, _cu64, _cu32, C.c_void_p]
        lib.orc_update_alpha_locprior.argtypes = [_ci, _ci, _ci, _i32p, _f64p, _f64p, _cd, _cd,
                                                  _cd, _cu64, _cu32, C.c_void_p]
        lib.orc_metro_logdiff.argtypes = [_ci, _ci, _ci, _ci, _i32p, _f32p, _f32p, _f32p, _f64p]
        lib.orc_metro_accept.argtypes = [_ci, _ci, _f64p, _cu64, _cu32, _f32p, _f32p, _f32p, _f32p, _u8p]
        lib.orc_metro_accept.restype = _ci
        lib.orc_alpha_sums.argtypes = [_ci, _ci, _f32p, _f64p, C.POINTER(_cd)]
        lib.orc_update_alpha.argtypes = [C.c_void_p, _f64p, _cd, _f64p, _cu64, _cu32, _f64p]
        lib.orc_update_eps.argtypes = [_ci, _ci, _ci, _i32p, _f32p, _f64p, _f64p, _cd, _cd, _cu64, _cu32, _u8p]
        lib.orc_fst_diffs.argtypes = [_ci, _ci, _ci, _i32p, _f32p, _f64p, _f64p, _ci, _cd, _cu64, _cu32, _f64p, _f64p]
        lib.orc_update_fst.argtypes = [_ci, _ci, _cd, _cd, _ci, _f64p, _f64p, _f64p, _cu64, _cu32, _f64p]
        lib.orc_calc_like.argtypes = [_ci, _ci, _ci, _ci, _i32p, _f64p, _f64p]
        lib.orc_calc_like.restype = _cd
        lib.orc_calc_like_f.argtypes = [_ci, _ci, _ci, _ci, _i32p, _f32p, _f32p]
        lib.orc_calc_like_f.restype = _cd
        lib.orc_init_eps.argtypes = [_ci, _ci, _ci, _i32p, _i32p, _ci, _cd, _cd, _ci, _f64p, _f64p]
        lib.orc_est_logprob.argtypes = [_cd, _cd, _ci]
        lib.orc_est_logprob.restype = _cd
        lib.orc_loglik_grad.argtypes = [_ci, _ci, _ci, _ci, _i32p, _f64p, _f64p, _f64p, _f64p,
                                        _f64p]
        lib.orc_loglik_grad.restype = _cd
        lib.orc_update_q_noadmix.argtypes = [_ci, _ci, _ci, _ci, _i32p, _f32p, _cu64, _cu32,
                                             _f32p, _f32p, _i32p, C.c_void_p, C.c_void_p]
        lib.orc_update_q_withpops.argtypes = [_ci, _ci, _ci, _ci, _i32p, _f32p, _i32p, _i32p,
                                              _ci, _cd, _cu64, _cu32, _ci, _f32p, _f32p, _f64p]
        lib.orc_update_lambda.argtypes = [_ci, _ci, _ci, _i32p, _f32p, _f64p, _ci, _ci, _f64p,
                                          _cu64, _cu32, _f64p]
        lib.orc_mala_step.argtypes = [_ci, _ci, _ci, _i32p, _f32p, _f32p, _f32p, _f64p, _ci, _f32p,
                                      _cu64, _cu32, _ci, _cd, _f64p, _u8p]

    # -- RNG ---------------------------------------------------------------
    def philox(self, ctr, key):
        out = np.zeros(4, np.uint32)
        self.lib.orc_philox(np.ascontiguousarray(ctr, np.uint32), key, out)
        return out

    def stream(self, a, b, rep, stream, seed):
        """Four words of block (a, b) of a chain's stream at a sweep."""
        out = np.zeros(4, np.uint32)
        self.lib.orc_stream(a, b, rep, stream, seed, out)
        return out

    def lgamma(self, z):
        return self.lib.orc_lgamma(float(z))

    def loggamma(self, a, e, rep, stream, key):
        err = _ci(0)
        v = self.lib.orc_loggamma(a, e, rep, stream, key, C.byref(err))
        return v, err.value

    def loggamma_f32(self, a, e, rep, stream, key):
        """The FP32 draw the P update uses (ln of a Gamma(a, 1) variate)."""
        err = _ci(0)
        v = self.lib.orc_loggamma_f32(a, e, rep, stream, key, C.byref(err))
        return v, err.value

    def ln_f32(self, x):
        return self.lib.orc_ln_f32(x)

    def sincos_2pi_f32(self, u):
        sn, cs = C.c_float(), C.c_float()
        self.lib.orc_sincos_2pi_f32(u, C.byref(sn), C.byref(cs))
        return sn.value, cs.value

    def normal(self, idx, rep, stream, key):
        return self.lib.orc_normal(idx, rep, stream, key)

    # -- Z -----------------------------------------------------------------
    def init_z(self, geno, K, key):
        N, _, L = geno.shape
        Z = np.zeros_like(geno)
        self.lib.orc_init_z(N, L, K, geno, key, Z)
        return Z

    def zupdate_f32(self, geno, Q, P, key, rep):
        N, _, L = geno.shape
        K = Q.shape[1]
        A = P.shape[2]
        Z = np.zeros_like(geno)
        self.lib.orc_zupdate_f32(N, L, K, A, geno, Q, P, key, rep, Z)
        return Z

    def zupdate_f64_injected(self, geno, Q, P, rnd):
        N, _, L = geno.shape
        K = Q.shape[1]
        A = P.shape[2]
        Z = np.zeros_like(geno)
        flags = np.zeros(1, np.int32)
        self.lib.orc_zupdate_f64_injected(N, L, K, A, geno, Q, P, rnd, Z, flags)
        return Z, int(flags[0])

    def counts(self, geno, Z, K, A, popflags=None, pfrompopflagonly=0):
        N, _, L = geno.shape
        n = np.zeros((L, K, A), np.int32)
        m = np.zeros((N, K), np.int32)
        pf = np.zeros(N, np.int32) if popflags is None else np.ascontiguousarray(popflags, np.int32)
        self.lib.orc_counts(N, L, K, A, geno, Z, pfrompopflagonly, pf, n, m)
        return n, m

    # -- P / Q -------------------------------------------------------------
    def update_p(self, numalleles, n, freqscorr, eps, F, lam, key, rep):
        L, K, A = n.shape
        P = np.zeros((L, K, A), np.float32)
        logP = np.zeros((L, K, A), np.float32)
        err = _ci(0)
        self.lib.orc_update_p(L, K, A, numalleles, n, int(freqscorr), eps, F, lam, key, rep,
                              P, logP, C.byref(err))
        return P, logP, err.value

    def update_q_gibbs(self, m, alpha, key, rep, arow=None):
        """arow [N]: row of alpha [rows][K] per individual (LOCPRIOR)."""
        N, K = m.shape
        Q = np.zeros((N, K), np.float32)
        logQ = np.zeros((N, K), np.float32)
        err = _ci(0)
        ar = None if arow is None else np.ascontiguousarray(arow, np.int32)
        self.lib.orc_update_q_gibbs(N, K, m, np.ascontiguousarray(alpha, np.float64).reshape(-1),
                                    key, rep, Q, logQ, C.byref(err),
                                    None if ar is None else ar.ctypes.data)
        return Q, logQ, err.value

    def metro_propose(self, N, alpha, key, rep, arow=None):
        K = alpha.shape[-1]
        T = np.zeros((N, K), np.float32)
        lT = np.zeros((N, K), np.float32)
        err = _ci(0)
        ar = None if arow is None else np.ascontiguousarray(arow, np.int32)
        self.lib.orc_metro_propose(N, K, np.ascontiguousarray(alpha, np.float64).reshape(-1), key,
                                   rep, T, lT, C.byref(err), None if ar is None else ar.ctypes.data)
        return T, lT, err.value

    def update_locprior(self, myloc, Q, alpha, locp, noadmix, alphapropsd, step, maxlp, key,
                        rep):
        """UpdateLocPrior restated; returns (locp, rand words, normals) where
        the words are the rand() values the reference would consume."""
        N, K = Q.shape
        nloc = int(np.max(myloc)) + 1
        lp = np.ascontiguousarray(locp, np.float64).copy()
        tr, keep = _trace(nloc, K)
        self.lib.orc_update_locprior(N, K, nloc, int(noadmix), np.ascontiguousarray(myloc, np.int32),
                                     np.ascontiguousarray(Q, np.float32),
                                     np.ascontiguousarray(alpha, np.float64), lp, alphapropsd,
                                     step, maxlp, key, rep, C.byref(tr))
        return lp, keep[0][:tr.nr].copy(), keep[1][:tr.nn].copy()

    def update_alpha_locprior(self, myloc, logQ, alpha, r, alphapropsd, alphamax, key, rep):
        """UpdateAlphaLocPrior restated; logQ FP64.  Returns (alpha, words,
        normals)."""
        N, K = logQ.shape
        nloc = int(np.max(myloc)) + 1
        al = np.ascontiguousarray(alpha, np.float64).copy()
        tr, keep = _trace(nloc, K)
        self.lib.orc_update_alpha_locprior(N, K, nloc, np.ascontiguousarray(myloc, np.int32),
                                           np.ascontiguousarray(logQ, np.float64), al, r,
                                           alphapropsd, alphamax, key, rep, C.byref(tr))
        return al, keep[0][:tr.nr].copy(), keep[1][:tr.nn].copy()

    def metro_logdiff(self, geno, Q, TestQ, P):
        N, _, L = geno.shape
        out = np.zeros(N, np.float64)
        self.lib.orc_metro_logdiff(N, L, Q.shape[1], P.shape[2], geno, Q, TestQ, P, out)
        return out

    def metro_accept(self, logdiff, key, rep, Q, logQ, TestQ, logTestQ):
        N, K = Q.shape
        Q, logQ = Q.copy(), logQ.copy()
        acc = np.zeros(N, np.uint8)
        self.lib.orc_metro_accept(N, K, logdiff, key, rep, Q, logQ, TestQ, logTestQ, acc)
        return Q, logQ, acc

    # -- alpha / eps / F ---------------------------------------------------
    class AlphaParams(C.Structure):
        _fields_ = [("K", _ci), ("N", _ci), ("popalphas", _ci), ("unifprioralpha", _ci),
                    ("alphamax", _cd), ("alphapropsd", _cd), ("alphapriora", _cd),
                    ("alphapriorb", _cd)]

    def alpha_sums(self, logQ):
        N, K = logQ.shape
        S = np.zeros(K, np.float64)
        T = _cd(0)
        self.lib.orc_alpha_sums(N, K, logQ, S, C.byref(T))
        return S, T.value

    def update_alpha(self, N, S, T, alpha, key, rep, popalphas, unifprioralpha,
                     alphamax, alphapropsd, alphapriora, alphapriorb):
        K = alpha.shape[0]
        p = self.AlphaParams(K, N, popalphas, unifprioralpha, alphamax, alphapropsd,
                             alphapriora, alphapriorb)
        a = alpha.copy()
        lpd = np.full(K, np.nan)
        self.lib.orc_update_alpha(C.byref(p), np.ascontiguousarray(S, np.float64), T, a, key, rep, lpd)
        return a, lpd

    def update_eps(self, numalleles, logP, eps, F, lambda0, invsqrtnuminds, key, rep):
        L, K, A = logP.shape
        e = eps.copy()
        acc = np.zeros(L, np.uint8)
        self.lib.orc_update_eps(L, K, A, numalleles, logP, e, F, lambda0, invsqrtnuminds,
                                key, rep, acc)
        return e, acc

    def fst_diffs(self, numalleles, logP, eps, F, onefst, fpriorsd, key, rep):
        L, K, A = logP.shape
        nf = np.zeros(K, np.float64)
        d = np.zeros(K, np.float64)
        self.lib.orc_fst_diffs(L, K, A, numalleles, logP, eps, F, onefst, fpriorsd, key, rep, nf, d)
        return nf, d

    def update_fst(self, F, onefst, fpriormean, fpriorsd, Leff, diff, newf, key, rep):
        K = F.shape[0]
        Fo = F.copy()
        lpd = np.full(K, np.nan)
        self.lib.orc_update_fst(K, onefst, fpriormean, fpriorsd, Leff, diff, newf, Fo, key, rep, lpd)
        return Fo, lpd

    # -- likelihood ------------------------------------------------------------
    def calc_like(self, geno, Q, P):
        N, _, L = geno.shape
        if Q.dtype == np.float32:
            return self.lib.orc_calc_like_f(N, L, Q.shape[1], P.shape[2], geno, Q, P)
        return self.lib.orc_calc_like(N, L, Q.shape[1], P.shape[2], geno, Q, P)

    def init_eps(self, geno, numalleles, A, freqscorr, lam, fpriormean, K):
        N, _, L = geno.shape
        eps = np.zeros((L, A), np.float64)
        F = np.zeros(K, np.float64)
        self.lib.orc_init_eps(N, L, A, geno, numalleles, int(freqscorr), lam, fpriormean, K, eps, F)
        return eps, F

    def est_logprob(self, s, ss, reps):
        return self.lib.orc_est_logprob(s, ss, reps)

    def update_q_noadmix(self, geno, logP, key, rep, locp=None, myloc=None):
        N, _, L = geno.shape
        _, K, A = logP.shape
        Q, lQ = np.zeros((N, K), np.float32), np.zeros((N, K), np.float32)
        pick = np.zeros(N, np.int32)
        lp = None if locp is None else np.ascontiguousarray(locp, np.float64)
        ml = None if myloc is None else np.ascontiguousarray(myloc, np.int32)
        self.lib.orc_update_q_noadmix(N, L, K, A, np.ascontiguousarray(geno, np.int32),
                                      np.ascontiguousarray(logP, np.float32), key, rep, Q, lQ, pick,
                                      None if lp is None else lp.ctypes.data,
                                      None if ml is None else ml.ctypes.data)
        return Q, lQ, pick

    def update_q_withpops(self, geno, P, population, popflags, gensback, migrprior, key, rep,
                          burnin, Q, logQ, usepop=None):
        """USEPOPINFO migrant-model Q of the flagged individuals (others untouched)."""
        N, _, L = geno.shape
        _, K, A = P.shape
        Qo = np.ascontiguousarray(Q, np.float32).copy()
        lQo = np.ascontiguousarray(logQ, np.float32).copy()
        up = np.zeros((N, K, gensback + 1)) if usepop is None else np.array(usepop, np.float64)
        self.lib.orc_update_q_withpops(N, L, K, A, np.ascontiguousarray(geno, np.int32),
                                       np.ascontiguousarray(P, np.float32),
                                       np.ascontiguousarray(population, np.int32),
                                       np.ascontiguousarray(popflags, np.int32), gensback,
                                       migrprior, key, rep, burnin, Qo, lQo, up)
        return Qo, lQo, up

    def update_lambda(self, numalleles, logP, eps, freqscorr, popspecific, lam, key, rep):
        L, K, A = logP.shape
        out = np.ascontiguousarray(lam, np.float64).copy()
        lpd = np.full(K, np.nan)
        self.lib.orc_update_lambda(L, K, A, np.ascontiguousarray(numalleles, np.int32),
                                   np.ascontiguousarray(logP, np.float32),
                                   np.ascontiguousarray(eps, np.float64), int(freqscorr),
                                   int(popspecific), out, key, rep, lpd)
        return out, lpd

    def mala_step(self, geno, Q, logQ, P, alpha, popalphas, eps, key, rep, burnin, target):
        """One Langevin move on every Q_i; returns (Q, logQ, eps, logr, acc)."""
        N, _, L = geno.shape
        K = Q.shape[1]
        Qo = np.ascontiguousarray(Q, np.float32).copy()
        lQo = np.ascontiguousarray(logQ, np.float32).copy()
        eo = np.ascontiguousarray(eps, np.float32).copy()
        logr, acc = np.zeros(N), np.zeros(N, np.uint8)
        self.lib.orc_mala_step(N, L, K, np.ascontiguousarray(geno, np.int32), Qo, lQo,
                               np.ascontiguousarray(P, np.float32), np.ascontiguousarray(alpha, np.float64),
                               int(popalphas), eo, key, rep, burnin, target, logr, acc)
        return Qo, lQo, eo, logr, acc

    def loglik_grad(self, geno, qlog, plog):
        """ln P(D|softmax(qlog), softmax(plog)) and its gradient w.r.t. the
        logits, FP64, no clamps.  qlog [N][K], plog [L][K][A]."""
        N, _, L = geno.shape
        K, A = qlog.shape[1], plog.shape[2]
        qlog = np.ascontiguousarray(qlog, np.float64)
        plog = np.ascontiguousarray(plog, np.float64)
        dq, dp, lli = np.zeros_like(qlog), np.zeros_like(plog), np.zeros(N)
        ll = self.lib.orc_loglik_grad(N, L, K, A, np.ascontiguousarray(geno, np.int32), qlog,
                                      plog, dq, dp, lli)
        return ll, dq, dp, lli


class Trace(C.Structure):
    _fields_ = [("rw", C.c_void_p), ("nr", _ci), ("nv", C.c_void_p), ("nn", _ci)]


def _trace(nloc, K):
    rw = np.zeros(8 + 4 * (nloc + 1), np.int32)
    nv = np.zeros((nloc + 1) * K + 4, np.float64)
    return Trace(rw.ctypes.data, 0, nv.ctypes.data, 0), (rw, nv)


class RefModel(C.Structure):
    _fields_ = [(n, _ci) for n in ("N", "L", "K", "maxalleles", "freqscorr", "onefst",
                                   "inferalpha", "popalphas", "unifprioralpha", "metrofreq",
                                   "burnin", "numreps", "computeprob", "pfrompopflagonly",
                                   "ancestdist", "numboxes")] + \
              [(n, _cd) for n in ("alpha", "alphamax", "alphapropsd", "alphapriora",
                                  "alphapriorb", "lambda_", "fpriormean", "fpriorsd")] + \
              [("inferlambda", _ci), ("popspecificlambda", _ci), ("noadmix", _ci),
               ("admburnin", _ci), ("usepopinfo", _ci), ("gensback", _ci), ("popflag", _ci),
               ("migrprior", _cd), ("locprior", _ci), ("updatelocprior", _ci),
               ("locpriorinit", _cd), ("maxlocprior", _cd), ("locpriorstep", _cd),
               ("startatpopinfo", _ci)]


class RefView(C.Structure):
    _fields_ = [(n, C.POINTER(_ci)) for n in ("Geno", "Z", "NumAlleles", "Translation", "AncestDist")] + \
              [(n, C.POINTER(_cd)) for n in ("Q", "P", "Eps", "SumEps", "Fst", "FstSum", "Alpha",
                                            "sumAlpha", "PSum", "QSum", "like", "sumlikes",
                                            "sumsqlikes")] + \
              [("maxalleles", _ci), ("rep", _ci)] + \
              [(n, C.POINTER(_cd)) for n in ("lambda_", "sumlambda", "UsePopProbs", "LocPrior",
                                            "sumLocPrior")] + \
              [("LocPriorLen", _ci), ("numlocations", _ci)]


def ref_model(**kw):
    d = dict(N=0, L=0, K=1, maxalleles=2, freqscorr=0, onefst=0, inferalpha=1, popalphas=0,
             unifprioralpha=1, metrofreq=10, burnin=0, numreps=1, computeprob=1,
             pfrompopflagonly=0, ancestdist=0, numboxes=1000, alpha=1.0, alphamax=10.0,
             alphapropsd=0.025, alphapriora=0.05, alphapriorb=0.001, lambda_=1.0,
             fpriormean=0.01, fpriorsd=0.05, inferlambda=0, popspecificlambda=0, noadmix=0,
             admburnin=0, usepopinfo=0, gensback=2, popflag=0, migrprior=0.05, locprior=0,
             updatelocprior=1, locpriorinit=1.0, maxlocprior=20.0, locpriorstep=0.1,
             startatpopinfo=0)
    d.update(kw)
    return RefModel(**d)


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libstref.so")) or os.path.isdir(REF_SRC)


class RefLib:
    """The reference's CPU functions (compiled from its sources)."""

    def __init__(self):
        lib = self.lib = _load(os.path.join(HERE, "_ref", "libstref.so"))
        lib.stref_set_globals.argtypes = [C.POINTER(RefModel)]
        lib.stref_rand_queue.argtypes = [C.c_void_p, C.c_long]
        lib.stref_normal_queue.argtypes = [C.c_void_p, C.c_long]
        lib.stref_rand_consumed.restype = C.c_long
        lib.stref_rand_overrun.restype = C.c_long
        lib.stref_normal_consumed.restype = C.c_long
        lib.stref_free_seed.argtypes = [_cu64]
        lib.stref_individuals.argtypes = [_ci, C.c_void_p]
        lib.stref_individuals.restype = C.c_void_p
        lib.stref_free.argtypes = [C.c_void_p]
        lib.stref_chain_new.argtypes = [C.POINTER(RefModel), _i32p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, _cu64]
        lib.stref_individuals_loc.argtypes = [_ci, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.stref_individuals_loc.restype = C.c_void_p
        lib.stref_numlocations.restype = _ci
        lib.stref_set_numlocations.argtypes = [_ci]
        lib.UpdateLocPrior.argtypes = [_f64p, _f64p, _f64p, C.c_void_p]
        lib.UpdateAlphaLocPrior.argtypes = [_f64p, _f64p, _f64p, C.c_void_p]
        lib.UpdateQAdmixture.argtypes = [_f64p, _i32p, _f64p, C.c_void_p, C.c_void_p]
        lib.UpdateQMetro.argtypes = [_i32p, C.c_void_p, _f64p, _f64p, _f64p, _ci, C.c_void_p,
                                     C.c_void_p, _f64p]
        lib.stref_individuals_pop.argtypes = [_ci, C.c_void_p, C.c_void_p]
        lib.stref_individuals_pop.restype = C.c_void_p
        lib.UpdateQWithPops.argtypes = [_i32p, _f64p, _f64p, C.c_void_p, _f64p, _ci, C.c_void_p,
                                        _f64p, C.c_void_p]
        lib.stref_chain_new.restype = C.c_void_p
        lib.stref_chain_sweeps.argtypes = [C.c_void_p, _ci]
        lib.stref_chain_sweeps.restype = _ci
        lib.stref_chain_view.argtypes = [C.c_void_p, C.POINTER(RefView)]
        lib.stref_chain_free.argtypes = [C.c_void_p]
        lib.mylgamma.argtypes = [_cd]
        lib.mylgamma.restype = _cd
        lib.UpdateZ.argtypes = [_i32p, _f64p, _f64p, _i32p, _f64p]
        lib.GetNumFromPops.argtypes = [_i32p, _i32p, _i32p, _i32p, C.c_void_p]
        lib.GetNumLociPop.argtypes = [_i32p, _i32p, _ci]
        lib.CalcLike.argtypes = [_i32p, C.c_void_p, _f64p, _f64p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.CalcLike.restype = _cd
        lib.CalcLikeIndDiff.argtypes = [_i32p, C.c_void_p, _f64p, _f64p, _f64p, _ci, C.c_void_p]
        lib.CalcLikeIndDiff.restype = _cd
        lib.LogProbQ.argtypes = [_f64p, _cd, C.c_void_p]
        lib.LogProbQ.restype = _cd
        lib.LogProbQonepop.argtypes = [_f64p, _cd, _cd, C.c_void_p, _ci]
        lib.LogProbQonepop.restype = _cd
        lib.AlphaPriorDiff.argtypes = [_cd, _cd]
        lib.AlphaPriorDiff.restype = _cd
        lib.FlikeFreqs.argtypes = [_cd, _f64p, _f64p, _i32p, _ci]
        lib.FlikeFreqs.restype = _cd
        lib.FPriorDiff.argtypes = [_cd, _cd]
        lib.FPriorDiff.restype = _cd
        lib.UpdateAlpha.argtypes = [_f64p, _f64p, C.c_void_p, _ci]
        lib.UpdateLambda.argtypes = [_f64p, _f64p, _f64p, _i32p]
        lib.UpdatePopLambda.argtypes = [_f64p, _f64p, _i32p]
        lib.UpdateQNoAdmix.argtypes = [_i32p, _f64p, _f64p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.UpdateP.argtypes = [_f64p, _f64p, _f64p, _i32p, _i32p, _i32p, _f64p, C.c_void_p, _f64p]
        lib.stref_guard_hits.restype = C.c_long
        lib.UpdateEpsilon.argtypes = [_f64p, _f64p, _f64p, _i32p, _cd]
        lib.UpdateFst.argtypes = [_f64p, _f64p, _f64p, _i32p]
        lib.InitializeZ.argtypes = [_i32p, C.c_void_p, _i32p]
        lib.InitFreqPriors.argtypes = [_f64p, _f64p, _i32p, _i32p]
        lib.CountAlleles.argtypes = [_i32p, _i32p, _i32p, C.c_void_p]
        lib.EstLogProb.argtypes = [_cd, _cd, _ci]
        lib.EstLogProb.restype = _cd
        lib.UpdateSums.argtypes = [_f64p, _f64p, _i32p, _f64p, _f64p, _f64p, _f64p, _i32p,
                                   C.c_void_p, _f64p, _f64p, _f64p, _f64p, C.c_void_p,
                                   C.c_void_p, _ci]
        self._keep = []

    def set_globals(self, **kw):
        self.model = ref_model(**kw)
        self.lib.stref_set_globals(C.byref(self.model))

    def individuals(self, N, popflags=None):
        pf = None if popflags is None else np.ascontiguousarray(popflags, np.int32)
        self._keep.append(pf)
        return self.lib.stref_individuals(N, None if pf is None else pf.ctypes.data)

    def rand_queue(self, vals):
        """Feed rand(); None -> free-running generator."""
        if vals is None:
            self.lib.stref_rand_queue(None, -1)
            return
        v = np.ascontiguousarray(vals, np.int32)
        self._rq = v
        self.lib.stref_rand_queue(v.ctypes.data, v.size)

    def normal_queue(self, vals):
        if vals is None:
            self.lib.stref_normal_queue(None, -1)
            return
        v = np.ascontiguousarray(vals, np.float64)
        self._nq = v
        self.lib.stref_normal_queue(v.ctypes.data, v.size)

    # -- chain -----------------------------------------------------------------
    def chain_new(self, model, geno, popflags=None, seed=1, population=None, location=None):
        pf = None if popflags is None else np.ascontiguousarray(popflags, np.int32)
        pp = None if population is None else np.ascontiguousarray(population, np.int32)
        lc = None if location is None else np.ascontiguousarray(location, np.int32)
        self._keep += [pf, pp, lc]
        return self.lib.stref_chain_new(C.byref(model), np.ascontiguousarray(geno, np.int32),
                                        None if pf is None else pf.ctypes.data,
                                        None if pp is None else pp.ctypes.data,
                                        None if lc is None else lc.ctypes.data, seed)

    def individuals_loc(self, N, location, popflags=None, population=None):
        """Individuals with locations; runs GetNumLocations (NUMLOCATIONS,
        myloc).  Returns (handle, NUMLOCATIONS)."""
        pf = np.zeros(N, np.int32) if popflags is None else np.ascontiguousarray(popflags, np.int32)
        pp = np.zeros(N, np.int32) if population is None else np.ascontiguousarray(population, np.int32)
        lc = np.ascontiguousarray(location, np.int32)
        self._keep += [pf, pp, lc]
        h = self.lib.stref_individuals_loc(N, pf.ctypes.data, pp.ctypes.data, lc.ctypes.data)
        return h, self.lib.stref_numlocations()

    def individuals_pop(self, N, popflags, population):
        pf = np.ascontiguousarray(popflags, np.int32)
        pp = np.ascontiguousarray(population, np.int32)
        self._keep += [pf, pp]
        return self.lib.stref_individuals_pop(N, pf.ctypes.data, pp.ctypes.data)

    def chain_view(self, ch, N, L, K, gensback=2):
        v = RefView()
        self.lib.stref_chain_view(ch, C.byref(v))
        A = v.maxalleles

        def arr(p, n, dt=np.float64):
            return np.ctypeslib.as_array(p, shape=(n,)).copy()

        # LOCPRIOR with admixture: alpha global + one row per location
        na = K * (v.numlocations + 1) if v.LocPriorLen == 1 else K

        return dict(
            A=A, rep=v.rep,
            Q=arr(v.Q, N * K).reshape(N, K), P=arr(v.P, L * K * A).reshape(L, K, A),
            Z=arr(v.Z, N * 2 * L).reshape(N, 2, L), Geno=arr(v.Geno, N * 2 * L).reshape(N, 2, L),
            NumAlleles=arr(v.NumAlleles, L), Eps=arr(v.Eps, L * A).reshape(L, A),
            Fst=arr(v.Fst, K), Alpha=arr(v.Alpha, na), QSum=arr(v.QSum, N * K).reshape(N, K),
            PSum=arr(v.PSum, L * K * A).reshape(L, K, A), SumEps=arr(v.SumEps, L * A).reshape(L, A),
            FstSum=arr(v.FstSum, K), sumAlpha=arr(v.sumAlpha, na),
            like=v.like[0], sumlikes=v.sumlikes[0], sumsqlikes=v.sumsqlikes[0],
            lambda_=arr(v.lambda_, K), sumlambda=arr(v.sumlambda, K),
            usepop=(arr(v.UsePopProbs, N * K * (gensback + 1)).reshape(N, K, gensback + 1)
                    if v.UsePopProbs else None),
            LocPrior=arr(v.LocPrior, v.LocPriorLen) if v.LocPriorLen else None,
            sumLocPrior=arr(v.sumLocPrior, v.LocPriorLen) if v.LocPriorLen else None,
            numlocations=v.numlocations)
