"""The structure_b200 front end (libstfront.so, include/stfront.h) against the
reference's own front-end code (params.c, datain.c, output.c compiled into
oracle/_ref/libstref.so and driven by oracle/ref_front.py):

* parameter files and command-line flags give the same values;
* data files give the same recoded genotypes, allele tables, individual
  records and marker names, for several layouts;
* the same sums give a byte-identical OUTFILE_f (and OUTFILE_q).

Data files and parameter files are written by the tests (seeded); the
reference's own example parameter files are read from its tree when present.
"""
import ctypes as C
import json
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from structure_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FRONT_LIB = os.path.join(ROOT, "structure_b200", "libstfront.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libstref.so")
from oracle.oracle import REF_SRC  # noqa: E402  (STRUCTURE_REF_SRC overrides it)

needs_ref = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference library not built")


def _front():
    if not os.path.exists(FRONT_LIB):
        from structure_b200 import build
        build.build_frontend()
    L = C.CDLL(FRONT_LIB)
    vp = C.c_void_p
    L.stf_open.argtypes = [C.c_int, vp, C.POINTER(vp)]
    L.stf_last_error.restype = C.c_char_p
    L.stf_last_error.argtypes = [vp]
    L.stf_param_int.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int)]
    L.stf_param_double.argtypes = [vp, C.c_char_p, C.POINTER(C.c_double)]
    L.stf_param_str.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_size_t]
    L.stf_read_data.argtypes = [vp]
    L.stf_dims.argtypes = [vp, vp]
    L.stf_geno.argtypes = [vp, vp, vp, vp]
    L.stf_individuals.argtypes = [vp, vp, vp, vp, vp, vp]
    L.stf_write_results.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, C.c_double,
                                    C.c_double]
    L.stf_check_pop_priors.argtypes = [vp, vp]
    L.stf_num_locations.argtypes = [vp]
    L.stf_set_locprior_sums.argtypes = [vp, vp, C.c_size_t]
    L.stf_set_usepopprobs.argtypes = [vp, vp]
    L.stf_format_update.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, C.c_double, vp, vp,
                                    C.c_size_t]
    L.stf_echo_data.argtypes = [vp, vp, C.c_size_t]
    L.stf_close.argtypes = [vp]
    return L


class Ours:
    """One stf_run, opened in `workdir` with `argv`."""

    def __init__(self, workdir, argv):
        self.L = _front()
        self.cwd = os.getcwd()
        os.chdir(workdir)
        self.argv = [a.encode() for a in argv]
        self._c = (C.c_char_p * len(argv))(*self.argv)
        self.h = C.c_void_p()
        self.rc = self.L.stf_open(len(argv), self._c, C.byref(self.h))

    def int(self, k):
        v = C.c_int()
        assert self.L.stf_param_int(self.h, k.encode(), C.byref(v)) == 0, k
        return v.value

    def real(self, k):
        v = C.c_double()
        assert self.L.stf_param_double(self.h, k.encode(), C.byref(v)) == 0, k
        return v.value

    def str(self, k):
        b = C.create_string_buffer(256)
        assert self.L.stf_param_str(self.h, k.encode(), b, 256) == 0
        return b.value.decode()

    def data(self):
        rc = self.L.stf_read_data(self.h)
        assert rc == 0, self.L.stf_last_error(self.h)
        d = np.zeros(4, np.int32)
        self.L.stf_dims(self.h, d.ctypes.data)
        N, L, LINES, A = map(int, d)
        geno = np.zeros((N, LINES, L), np.int32)
        na = np.zeros(L, np.int32)
        tr = np.zeros((L, max(A, 1)), np.int32)
        self.L.stf_geno(self.h, geno.ctypes.data, na.ctypes.data, tr.ctypes.data)
        pop, pf, loc, ph = (np.zeros(N, np.int32) for _ in range(4))
        lab = C.create_string_buffer(12 * N)
        self.L.stf_individuals(self.h, pop.ctypes.data, pf.ctypes.data, loc.ctypes.data,
                               ph.ctypes.data, lab)
        labels = [lab.raw[12 * i:12 * (i + 1)].split(b"\0")[0].decode() for i in range(N)]
        return dict(A=A, geno=geno, numalleles=na, translation=tr, pop=pop, popflag=pf,
                    labels=labels)

    def check_pop_priors(self):
        n = np.zeros(1, np.int32)
        rc = self.L.stf_check_pop_priors(self.h, n.ctypes.data)
        assert rc == 0, self.L.stf_last_error(self.h)
        return int(n[0])

    def write(self, rep, z):
        f = lambda a: np.ascontiguousarray(a, np.float64)
        if "usepop" in z:
            self._up = f(z["usepop"])
            assert self.L.stf_set_usepopprobs(self.h, self._up.ctypes.data) == 0
        if "sumLocPrior" in z:
            self._lp = f(z["sumLocPrior"])
            assert self.L.stf_set_locprior_sums(self.h, self._lp.ctypes.data, self._lp.size) == 0, \
                self.L.stf_last_error(self.h)
        self._keep = {k: f(z[k]) for k in ("QSum", "PSum", "SumEps", "FstSum", "sumAlpha",
                                           "sumlambda")}
        ad = np.ascontiguousarray(z["AncestDist"], np.int32) if "AncestDist" in z else None
        k = self._keep
        rc = self.L.stf_write_results(self.h, rep, k["QSum"].ctypes.data, k["PSum"].ctypes.data,
                                      k["SumEps"].ctypes.data, k["FstSum"].ctypes.data,
                                      k["sumAlpha"].ctypes.data, k["sumlambda"].ctypes.data,
                                      ad.ctypes.data if ad is not None else None,
                                      float(z["sumlikes"]), float(z["sumsqlikes"]))
        assert rc == 0, self.L.stf_last_error(self.h)

    def update(self, rep, a):
        """stf_format_update of one trace line from the arrays of `a`."""
        f = lambda x: np.ascontiguousarray(x, np.float64)
        args = [f(a[k]) for k in ("Q", "P", "alpha", "F", "lambda")]
        lp = f(a["locprior"])
        call = lambda buf, n: self.L.stf_format_update(
            self.h, rep, *[x.ctypes.data for x in args], float(a["like"]), lp.ctypes.data, buf, n)
        n = call(None, 0)
        assert n >= 0, n
        buf = C.create_string_buffer(n + 1)
        assert call(buf, n + 1) == n
        return buf.value

    def echo(self):
        n = self.L.stf_echo_data(self.h, None, 0)
        assert n >= 0
        buf = C.create_string_buffer(n + 1)
        self.L.stf_echo_data(self.h, buf, n + 1)
        return buf.value

    def close(self):
        self.L.stf_close(self.h)
        os.chdir(self.cwd)


def _ref(workdir, argv, read_data=False, sums=None, rep=0, trace=None):
    spec = os.path.join(workdir, "spec.json")
    with open(spec, "w") as f:
        json.dump({"argv": argv, "read_data": read_data, "sums": sums, "rep": rep,
                   "trace": trace}, f)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "ref_front.py"), workdir,
                        spec], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    with open(os.path.join(workdir, "ref_out.json")) as f:
        out = json.load(f)
    if read_data:
        out["data"] = dict(np.load(os.path.join(workdir, "ref_data.npz")))
    return out


MAIN_TMPL = """KEY PARAMETERS (written by the test)

Basic Program Parameters

#define MAXPOPS    {K}      // (int) number of populations assumed
#define BURNIN    {burnin}   // (int) length of burnin period
#define NUMREPS   {numreps}   // (int) number of MCMC reps after burnin

#define INFILE   {infile}   // (str) name of input data file
#define OUTFILE  {outfile}  //(str) name of output data file

#define NUMINDS    {N}    // (int)
#define NUMLOCI    {L}    // (int)
#define PLOIDY       2    // (int) ploidy of data
#define MISSING     {missing}    // (int) value given to missing genotype data
#define ONEROWPERIND {onerow}    // (B) store data for individuals in a single line
#define LABEL     {label}     // (B) Input file contains individual labels
#define POPDATA   {popdata}     // (B) Input file contains a population identifier
#define POPFLAG   {popflag}     // (B) whether to use popinfo when USEPOPINFO==1
#define LOCDATA   {locdata}     // (B) Input file contains a location identifier
#define PHENOTYPE 0     // (B)
#define EXTRACOLS {extracols}     // (int) Number of additional columns
#define MARKERNAMES      {markernames}  // (B) data file contains row of marker names
#define RECESSIVEALLELES 0  // (B)
#define MAPDISTANCES     {mapdist}  // (B)
"""

EXTRA_TMPL = """EXTRA PARAMS (written by the test)
#define NOADMIX     {noadmix} // (B)
#define ADMBURNIN   {admburnin} // (int)
#define LINKAGE     0 // (B)
#define USEPOPINFO  {usepopinfo} // (B)
#define MIGRPRIOR {migrprior} // (d)
#define GENSBACK  {gensback} // (int)
#define LOCPRIOR    {locprior} //(B)
#define LOCISPOP    {locispop} //(B)
#define FREQSCORR   {freqscorr} // (B)
#define ONEFST      {onefst} // (B)
#define INFERALPHA  1 // (B)
#define POPALPHAS   {popalphas} // (B)
#define ALPHA     1.0 // (d)
#define INFERLAMBDA 0 // (B)
#define LAMBDA    1.0 // (d)
#define FPRIORMEAN 0.01 // (d)
#define FPRIORSD   0.05  // (d)
#define UNIFPRIORALPHA 1 // (B)
#define ALPHAMAX     10.0 // (d)
#define ALPHAPROPSD 0.025 // (d)
#define UPDATEFREQ   {updatefreq}  // (int)
#define INTERMEDSAVE {intermedsave}  // (int)
#define PRINTLIKES   {printlikes}  // (B)
#define PRINTQHAT  {printqhat}  // (B)
#define ANCESTDIST   {ancestdist}  // (B)
#define NUMBOXES   {numboxes} // (int)
#define ANCESTPINT 0.90 // (d)
#define PRINTQSUM  {printqsum}  // (B)
#define PRINTNET   {printnet}  // (B)
#define PRINTLAMBDA {printlambda}  // (B)
#define POPSPECIFICLAMBDA {popspecificlambda}  // (B)
#define ECHODATA   {echodata}  // (B)
#define COMPUTEPROB {computeprob}     // (B)
#define METROFREQ    10   // (int)
#define RANDOMIZE      0  // (B)
#define SEED        {seed}  // (int)
#define NOTAKEY     5  // an unknown name: ignored with a warning
# a comment line with a hash that is not a definition
"""


def _scenario(d, **kw):
    p = dict(K=3, burnin=100, numreps=400, infile="data file.str", outfile="results", N=40, L=25,
             missing=-9, onerow=0, label=1, popdata=1, popflag=0, extracols=0, markernames=1,
             mapdist=0, freqscorr=1, onefst=0, popalphas=0, updatefreq=0, printqhat=0,
             ancestdist=0, numboxes=100, seed=4242, noadmix=0, usepopinfo=0, migrprior=0.05,
             gensback=2, locdata=0, locprior=0, locispop=0, admburnin=50, intermedsave=0,
             printlikes=0, printqsum=0, printnet=0, printlambda=0, popspecificlambda=0,
             echodata=0, computeprob=1)
    p.update(kw)
    with open(os.path.join(d, "mainparams"), "w") as f:
        f.write(MAIN_TMPL.format(**p))
    with open(os.path.join(d, "extraparams"), "w") as f:
        f.write(EXTRA_TMPL.format(**p))
    g = synth.microsat(N=p["N"], L=p["L"], K=3, seed=p["seed"])["geno_raw"]
    if p["missing"] != -9:
        g = np.where(g == -9, p["missing"], g)
    rng = np.random.default_rng(p["seed"])
    rows = []
    if p["markernames"]:
        names = [f"loc{l}" for l in range(p["L"])]
        names[1] = "a_marker_name_longer_than_fourteen"
        rows.append("\t".join(names))
    if p["mapdist"]:
        rows.append(" ".join(["-1"] + [f"{x:.2f}" for x in rng.random(p["L"] - 1)]))
    for i in range(p["N"]):
        lab = f"ind{i}" if i != 3 else "a_long_individual_label"
        head = []
        if p["label"]:
            head.append(lab)
        if p["popdata"]:
            head.append(str(1 + i % 4))
        if p["popflag"]:
            head.append(str(i % 2))
        if p["locdata"]:
            head.append(str(3 * (i % 3) + 5))          # location ids 5, 8, 11
        head += ["7"] * p["extracols"]
        if p["onerow"]:
            rows.append(" ".join(head + [str(v) for v in g[i].T.reshape(-1)]))
        else:
            for line in range(2):
                rows.append(" ".join(head + [str(v) for v in g[i, line]]))
    with open(os.path.join(d, p["infile"]), "w") as f:
        f.write("\n".join(rows) + "\n")
    return p


def _random_sums(p, A, seed=1):
    rng = np.random.default_rng(seed)
    K, N, L, reps = p["K"], p["N"], p["L"], p["numreps"]
    Q = rng.dirichlet(np.ones(K), N) * reps
    P = rng.dirichlet(np.ones(A), (L, K)) * reps
    z = dict(QSum=Q, PSum=P, SumEps=rng.random((L, A)) * reps, FstSum=rng.random(K) * 0.3 * reps,
             sumAlpha=rng.random(K) * reps, sumlambda=np.ones(K) * reps,
             sumlikes=-1234.56 * reps, sumsqlikes=1234.56 ** 2 * reps + 50.0 * (reps - 1))
    if p["locprior"]:
        nloc = 4 if p["locispop"] else 3               # populations 1..4 or locations 5, 8, 11
        if not p["noadmix"]:
            z["sumAlpha"] = rng.random(K * (nloc + 1)) * reps
        n = 1 + K * (nloc + 1) if p["noadmix"] else 1
        z["sumLocPrior"] = rng.random(n) * reps
    if p["usepopinfo"]:
        u = rng.dirichlet(np.ones(K * (p["gensback"] + 1)), N) * reps
        z["usepop"] = u.reshape(N, K, p["gensback"] + 1)
        z["usepop"][:5, :, 0] = 0.0    # low posterior of the given population: stars
    if p["ancestdist"]:
        ad = np.zeros((N, K, p["numboxes"]), np.int32)
        for i in range(N):
            for k in range(K):
                ad[i, k] = rng.multinomial(reps, np.ones(p["numboxes"]) / p["numboxes"])
        z["AncestDist"] = ad
    return z


@needs_ref
def test_params_match_reference(tmp_path):
    d = str(tmp_path)
    _scenario(d)
    argv = ["structure", "-K", "4", "-L", "25", "-D", "77", "-o", "other_out"]
    ref = _ref(d, argv)
    ours = Ours(d, argv)
    assert ours.rc == 0
    for k, v in ref["int"].items():
        assert ours.int(k) == v, k
    for k, v in ref["real"].items():
        assert ours.real(k) == pytest.approx(v, rel=1e-15), k
    for k, v in ref["str"].items():
        assert ours.str(k) == v, k
    ours.close()


@needs_ref
@pytest.mark.skipif(not os.path.isdir(REF_SRC), reason="reference tree not present")
def test_reference_example_params_read_alike(tmp_path):
    """The reference's own example mainparams/extraparams."""
    d = str(tmp_path)
    for f in ("mainparams", "extraparams"):
        shutil.copy(os.path.join(REF_SRC, f), os.path.join(d, f))
    argv = ["structure"]
    ref = _ref(d, argv)
    ours = Ours(d, argv)
    assert ours.rc == 0
    for k, v in ref["int"].items():
        assert ours.int(k) == v, k
    for k, v in ref["real"].items():
        assert ours.real(k) == pytest.approx(v, rel=1e-15), k
    for k, v in ref["str"].items():
        assert ours.str(k) == v, k
    ours.close()


LAYOUTS = [dict(), dict(onerow=1), dict(missing=0, markernames=0), dict(label=0, popdata=0),
           dict(popflag=1, extracols=2, mapdist=1)]


@needs_ref
@pytest.mark.parametrize("layout", LAYOUTS, ids=["rows", "onerow", "missing0", "bare", "extra"])
def test_data_matches_reference(tmp_path, layout):
    d = str(tmp_path)
    p = _scenario(d, **layout)
    argv = ["structure"]
    ref = _ref(d, argv, read_data=True)
    ours = Ours(d, argv)
    assert ours.rc == 0
    o = ours.data()
    r = ref["data"]
    assert o["A"] == ref["A"]
    np.testing.assert_array_equal(o["geno"], r["geno"])
    np.testing.assert_array_equal(o["numalleles"], r["numalleles"])
    np.testing.assert_array_equal(o["translation"], r["translation"])
    if p["label"]:
        assert o["labels"] == list(r["labels"])
    if p["popdata"]:
        np.testing.assert_array_equal(o["pop"], r["pop"])
    if p["popflag"]:
        np.testing.assert_array_equal(o["popflag"], r["popflag"])
    ours.close()


OUTPUTS = [dict(), dict(freqscorr=0, popalphas=1), dict(onefst=1, printqhat=1),
           dict(ancestdist=1, label=0), dict(popdata=0, markernames=0, K=2),
           dict(usepopinfo=1, popflag=1, migrprior=0.1), dict(usepopinfo=1, gensback=1),
           dict(usepopinfo=1, K=4, ancestdist=1), dict(noadmix=1),
           dict(locprior=1, locdata=1), dict(locprior=1, locdata=1, noadmix=1, popalphas=1),
           dict(locprior=1, locispop=1, noadmix=1)]


@needs_ref
@pytest.mark.parametrize("opts", OUTPUTS, ids=["f", "indep-popalphas", "onefst-qhat", "ancest",
                                                "nopop", "usepop-flags", "usepop-all",
                                                "usepop-noalpha", "noadmix", "locprior",
                                                "locprior-noadmix", "locispop"])
def test_results_file_matches_reference_byte_for_byte(tmp_path, opts):
    d = str(tmp_path)
    p = _scenario(d, **opts)
    argv = ["structure", "-K", str(p["K"])]
    ours = Ours(d, argv)
    o = ours.data()
    dropped = ours.check_pop_priors()
    if p["usepopinfo"]:
        # populations are 1..4 in the file: 4 is outside 1..K for K=3
        flagged = (o["popflag"] == 1) if p["popflag"] else np.ones(p["N"], bool)
        assert dropped == int((flagged & (o["pop"] > p["K"])).sum())
        if p["K"] == 4 and not p["popflag"]:
            assert ours.int("INFERALPHA") == 0      # NOALPHA: everybody has prior info
    z = _random_sums(p, o["A"])
    np.savez(os.path.join(d, "sums.npz"), **z)
    rep = p["burnin"] + p["numreps"]
    ours.write(rep, z)
    ours.close()
    mine = open(os.path.join(d, "results_f"), "rb").read()
    q_mine = open(os.path.join(d, "results_q"), "rb").read() if p["printqhat"] else None
    os.rename(os.path.join(d, "results_f"), os.path.join(d, "ours_f"))
    _ref(d, argv, read_data=True, sums="sums.npz", rep=rep)
    theirs = open(os.path.join(d, "results_f"), "rb").read()
    assert mine == theirs
    if p["printqhat"]:
        assert q_mine == open(os.path.join(d, "results_q"), "rb").read()


def test_front_end_reports_errors(tmp_path):
    d = str(tmp_path)
    _scenario(d)
    ours = Ours(d, ["structure", "-m", "missing_file"])
    assert ours.rc == -4 and b"missing_file" in ours.L.stf_last_error(ours.h)
    ours.close()
    with open(os.path.join(d, "mainparams"), "a") as f:
        f.write("#define NUMINDS 41\n")          # more individuals than the file holds
    ours = Ours(d, ["structure"])
    assert ours.rc == 0
    assert ours.L.stf_read_data(ours.h) == -3
    ours.close()


TRACES = [dict(), dict(printqsum=1, printnet=1, K=4), dict(freqscorr=0, popalphas=1, K=12),
          dict(onefst=1, printlambda=1, popspecificlambda=1, printqsum=1, popdata=0),
          dict(noadmix=1, admburnin=70, popalphas=1), dict(noadmix=1, admburnin=30),
          dict(locprior=1, locdata=1, printlambda=1), dict(computeprob=0, burnin=150),
          dict(usepopinfo=1, K=4), dict(burnin=130000, numreps=2000)]


@needs_ref
@pytest.mark.parametrize("opts", TRACES, ids=["default", "qsum-net", "popalphas-k12",
                                               "onefst-lambda", "noadmix-admburnin",
                                               "noadmix-early", "locprior", "noprob",
                                               "usepop-noalpha", "six-digit-reps"])
def test_screen_trace_matches_reference(tmp_path, opts):
    """The screen trace of a run (src/output.c:218-454 PrintUpdate and
    PrintBanner), line for line at the sweeps where the run loop prints it
    (src/structure.c:669-702), from the same alpha, F, lambda, r, like, Q and
    P: identical text."""
    d = str(tmp_path)
    p = _scenario(d, updatefreq=10, **opts)
    argv = ["structure", "-K", str(p["K"])]
    ours = Ours(d, argv)
    o = ours.data()
    ours.check_pop_priors()
    K, A, N, L = p["K"], o["A"], p["N"], p["L"]
    total = p["burnin"] + p["numreps"]
    every = ours.int("UPDATEFREQ")
    reps = list(range(every, total + 1, every))
    if p["burnin"] > 1000:       # a few sweeps on each side of the banners
        reps = [r for r in reps if r < 60 or abs(r - p["burnin"]) <= 30 or r > total - 120]
    if total % every:
        reps.append(total)
    rng = np.random.default_rng(5)
    U = len(reps)
    z = dict(rep=np.array(reps), like=-rng.random(U) * 5000.0 - 1000.5,
             alpha=rng.random((U, K)) * 3.0, F=rng.random((U, K)) * 0.5,
             **{"lambda": rng.random((U, K)) * 2.0}, locprior=rng.random((U, 1)) * 4.0,
             Q=rng.dirichlet(np.ones(K), (U, N)), P=rng.dirichlet(np.ones(A), (U, L, K)))
    np.savez(os.path.join(d, "trace.npz"), **z)
    mine = b"".join(ours.update(int(r), {k: z[k][u] for k in z}) for u, r in enumerate(reps))
    ours.close()
    out = _ref(d, argv, read_data=True, trace="trace.npz")
    theirs = open(os.path.join(d, "ref_stdout.txt"), "rb").read()
    theirs = theirs[out["trace_at"]:out["trace_end"]]
    assert mine == theirs


@needs_ref
@pytest.mark.parametrize("layout", [dict(), dict(N=5, L=4, popflag=1), dict(label=0, popdata=0),
                                    dict(missing=0, onerow=1, N=7)],
                         ids=["default", "few", "bare", "onerow-missing0"])
def test_echo_data_matches_reference(tmp_path, layout):
    """ECHODATA=1: the data echo of src/datain.c:514-571 PrintSomeData."""
    d = str(tmp_path)
    p = _scenario(d, echodata=1, **layout)
    argv = ["structure"]
    ours = Ours(d, argv)
    ours.data()
    mine = ours.echo()
    ours.close()
    out = _ref(d, argv, read_data=True)
    theirs = open(os.path.join(d, "ref_stdout.txt"), "rb").read()[out["read_at"]:out["read_end"]]
    head = b'Reading file "%s".\n' % p["infile"].encode()
    assert theirs.startswith(head)
    assert mine == theirs[len(head):]
