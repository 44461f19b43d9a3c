"""The oracle against golden outputs of the reference's own CPU functions
(tests/golden/*.npz, written by tests/golden/make_golden.py), and the host
helpers against the reference's recoding.  CPU only; no reference tree needed."""
import os

import numpy as np

from structure_b200 import synth

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_golden_z_counts_like(orc):
    g = np.load(os.path.join(G, "z_counts_like.npz"))
    geno, Q, P, u = g["geno"], g["Q"], g["P"], g["u"]
    Z, flags = orc.zupdate_f64_injected(geno, Q, P, u)
    assert flags == 0 and (Z == g["Z"]).all()
    K, A = Q.shape[1], P.shape[2]
    n, m = orc.counts(geno, Z, K, A)
    assert (n == g["n"]).all() and (m == g["m"]).all()
    assert orc.calc_like(geno, Q, P) == float(g["like"])
    assert (orc.init_z(geno, K, int(g["key"])) == g["Zinit"]).all()


def test_golden_recoding():
    """datain.c:824-904 CountAlleles: codes in order of first appearance."""
    g = np.load(os.path.join(G, "z_counts_like.npz"))
    rec, na = synth.recode(g["raw"])
    assert (rec == g["geno"]).all() and (na == g["numalleles"]).all()


def test_golden_alpha(orc):
    g = np.load(os.path.join(G, "alpha_popalphas.npz"))
    logQ = g["logQ"]
    S, T = orc.alpha_sums(logQ)
    a1, _ = orc.update_alpha(logQ.shape[0], S, T, g["alpha0"], int(g["key"]), int(g["rep"]),
                             1, 1, float(g["amax"]), float(g["sd"]), 1.0, 2.0)
    np.testing.assert_allclose(a1, g["alpha1"], rtol=1e-13)


def test_golden_epsilon(orc):
    g = np.load(os.path.join(G, "epsilon.npz"))
    e1, _ = orc.update_eps(g["numalleles"], g["logP"], g["eps0"], g["F"], 1.0, float(g["inv"]),
                           int(g["key"]), int(g["rep"]))
    np.testing.assert_allclose(e1, g["eps1"], rtol=1e-12, atol=1e-15)
