"""The reference's own front end, for checking the structure_b200 front end.

TEST INFRASTRUCTURE ONLY (the checker, never the product): runs, in this
process, the reference's parameter reader (src/params.c GetParams), data
reader and recoder (src/datain.c ReadInputFile, FindMaxAlleles and
CountAlleles, as src/structure.c:266-320 and src/Init.c:392-396 call them) and
result writer (src/output.c OutPutResults), all compiled from the reference
sources into oracle/_ref/libstref.so.  The reference keeps its state in
process globals and exits on errors, so each scenario runs in its own process:

    python oracle/ref_front.py <workdir> <spec.json>

spec: {"argv": [...], "read_data": bool, "sums": "<npz in workdir>" or null,
       "rep": int, "trace": "<npz in workdir>" or null}; with USEPOPINFO=1 the sums carry "usepop" [N][K][GENSBACK+1]
and CheckPopPriors (src/Init.c:15-70) runs before OutPutResults; with
LOCPRIOR=1 they carry "sumLocPrior" (and sumAlpha of K * (locations + 1)
values with admixture).  "trace" holds, per screen-trace line, rep, like,
alpha, F, lambda, locprior, Q and P, each passed to PrintUpdate
(src/output.c:218-374) after the data are read.  The working directory is
<workdir> (the reference opens its files relative to it).  Results go to
<workdir>/ref_out.json and <workdir>/ref_data.npz; OutPutResults writes
OUTFILE_f (and OUTFILE_q).  What the reference prints goes to
<workdir>/ref_stdout.txt; ref_out.json gives the offsets in it where the data
reading ("read_at", "read_end") and the trace ("trace_at") start and end.
"""
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

INT_KEYS = ["NUMINDS", "NUMLOCI", "MISSING", "LABEL", "POPDATA", "MARKERNAMES", "PHASEINFO",
            "MAPDISTANCES", "MARKOVPHASE", "LINES", "ONEROWPERIND", "RECESSIVEALLELES",
            "NOTAMBIGUOUS", "POPFLAG", "PHENOTYPE", "EXTRACOLS", "MAXPOPS", "BURNIN", "NUMREPS",
            "USEPOPINFO", "PFROMPOPFLAGONLY", "INFERALPHA", "INFERLAMBDA", "POPSPECIFICLAMBDA",
            "POPALPHAS", "COMPUTEPROB", "NOADMIX", "ADMBURNIN", "PHASED", "PRINTQHAT",
            "PRINTQSUM", "UPDATEFREQ", "PRINTLIKES", "INTERMEDSAVE", "PRINTKLD", "PRINTNET",
            "PRINTLAMBDA", "ECHODATA", "ANCESTDIST", "NUMBOXES", "GENSBACK", "FREQSCORR",
            "ONEFST", "UNIFPRIORALPHA", "STARTATPOPINFO", "RANDOMIZE", "LINKAGE", "METROFREQ",
            "REPORTHITRATE", "NOQS", "POSTERIOR", "PICTUREFILE", "INDIVIDUALR", "NUMSIMSTATS",
            "POOLFREQ", "LOCUSxONLY", "PHENOTYPECOL", "MISSINGPHENO", "LOCPRIOR",
            "UPDATELOCPRIOR", "LOCISPOP", "LOCDATA", "SEED"]
REAL_KEYS = ["ANCESTPINT", "MIGRPRIOR", "ALPHA", "LOG10RPROPSD", "LOG10RMIN", "LOG10RMAX",
             "LOG10RSTART", "FPRIORMEAN", "FPRIORSD", "LAMBDA", "ALPHAMAX", "ALPHAPRIORA",
             "ALPHAPRIORB", "ALPHAPROPSD", "EMERROR", "LOCPRIORINIT", "MAXLOCPRIOR",
             "LOCPRIORSTEP"]


class IND(C.Structure):
    _fields_ = [("Label", C.c_char * 12), ("Population", C.c_int), ("PopFlag", C.c_int),
                ("Phenotype", C.c_int), ("Location", C.c_int), ("myloc", C.c_int)]


def _stdout_pos():
    C.CDLL(None).fflush(None)
    return os.lseek(1, 0, os.SEEK_CUR)


def _trace(lib, g, spec, workdir, geno, na, inds, out):
    """PrintUpdate for each line of the trace file (src/structure.c:681-702
    passes the current Alpha, Fst, P, Q, like, sums, NumAlleles, R, lambda,
    Individual and LocPrior)."""
    z = np.load(os.path.join(workdir, spec["trace"]))
    N = g("NUMINDS").value
    if g("LOCDATA").value > 0 or g("LOCISPOP").value:
        lib.GetNumLocations.argtypes = [C.c_void_p]
        lib.GetNumLocations(inds)
    if g("USEPOPINFO").value:
        lib.CheckPopPriors.argtypes = [C.c_void_p]
        lib.CheckPopPriors(inds)     # sets NOALPHA when every individual is flagged
    vp = C.c_void_p
    lib.PrintUpdate.argtypes = [C.c_int, vp, vp, vp, vp, vp, vp, C.c_double, C.c_double,
                                C.c_double, vp, vp, vp, vp, C.c_double, vp, vp, C.c_int]
    R = np.zeros(N)
    keep = []
    out["trace_at"] = _stdout_pos()
    for u in range(len(z["rep"])):
        a = {k: np.ascontiguousarray(z[k][u], np.float64)
             for k in ("alpha", "F", "lambda", "locprior", "Q", "P")}
        keep.append(a)
        P = lambda x: x.ctypes.data_as(vp)
        lib.PrintUpdate(int(z["rep"][u]), geno, None, P(a["alpha"]), P(a["F"]), P(a["P"]),
                        P(a["Q"]), float(z["like"][u]), 0.0, 0.0, na, P(R), P(a["lambda"]),
                        inds, 0.0, None, P(a["locprior"]), a["locprior"].size)
    out["trace_end"] = _stdout_pos()


def main(workdir, specpath):
    with open(specpath) as f:
        spec = json.load(f)
    lib = C.CDLL(os.path.join(HERE, "_ref", "libstref.so"))
    os.chdir(workdir)
    argv = [a.encode() for a in spec["argv"]]
    cargv = (C.c_char_p * len(argv))(*argv)
    lib.GetParams.argtypes = [C.c_int, C.c_int, C.c_void_p]
    lib.GetParams(0, len(argv), cargv)
    g = lambda n, t=C.c_int: t.in_dll(lib, n)
    out = {"int": {k: g(k).value for k in INT_KEYS},
           "real": {k: g(k, C.c_double).value for k in REAL_KEYS},
           "str": {k: (C.c_char * 201).in_dll(lib, k).value.decode() for k in ("DATAFILE", "OUTFILE")}}
    if spec.get("read_data"):
        N, L, LINES = g("NUMINDS").value, g("NUMLOCI").value, g("LINES").value
        geno = (C.c_int * (N * LINES * L))()
        mapd = (C.c_double * L)()
        names = (C.c_char * (L * 15))()
        inds = (IND * N)()
        phase = (C.c_double * (N * L))()
        rec = (C.c_int * L)()
        out["read_at"] = _stdout_pos()
        lib.ReadInputFile(geno, mapd, names, inds, phase, rec)
        out["read_end"] = _stdout_pos()
        lib.FindMaxAlleles.restype = C.c_int
        A = lib.FindMaxAlleles(geno, rec)
        g("MAXALLELES").value = A
        na = (C.c_int * L)()
        tr = (C.c_int * (L * max(A, 1)))()
        lib.CountAlleles(geno, na, tr, rec)
        out["A"] = A
        out["int"]["MISSING_AFTER"] = g("MISSING").value
        np.savez(os.path.join(workdir, "ref_data.npz"),
                 geno=np.ctypeslib.as_array(geno).reshape(N, LINES, L).copy(),
                 numalleles=np.ctypeslib.as_array(na).copy(),
                 translation=np.ctypeslib.as_array(tr).reshape(L, max(A, 1)).copy(),
                 labels=np.array([x.Label.decode() for x in inds]),
                 pop=np.array([x.Population for x in inds]),
                 popflag=np.array([x.PopFlag for x in inds]),
                 location=np.array([x.Location for x in inds]),
                 phenotype=np.array([x.Phenotype for x in inds]),
                 names=np.array([bytes(names[l * 15:(l + 1) * 15]).split(b"\0")[0].decode()
                                 for l in range(L)]))
        if spec.get("trace"):
            _trace(lib, g, spec, workdir, geno, na, inds, out)
        if spec.get("sums"):
            z = np.load(os.path.join(workdir, spec["sums"]))
            K = g("MAXPOPS").value
            usepop = None
            slp, lplen = None, 0
            if g("LOCDATA").value > 0 or g("LOCISPOP").value:
                # src/structure.c:350-352
                lib.GetNumLocations.argtypes = [C.c_void_p]
                lib.GetNumLocations(inds)
            if g("LOCPRIOR").value:
                slp = np.ascontiguousarray(z["sumLocPrior"], np.float64)
                lplen = slp.size
            if g("USEPOPINFO").value:
                # src/Init.c:417: the prior-population checks run before the
                # chain and decide which individuals print the migrant model
                lib.CheckPopPriors.argtypes = [C.c_void_p]
                lib.CheckPopPriors(inds)
                usepop = np.ascontiguousarray(z["usepop"], np.float64)
            d = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(C.c_void_p)
            keep = {k: np.ascontiguousarray(z[k], np.float64) for k in
                    ("QSum", "PSum", "SumEps", "FstSum", "sumAlpha", "sumlambda")}
            ad = np.ascontiguousarray(z["AncestDist"], np.int32) if "AncestDist" in z.files else None
            zeros = {k: np.zeros(n) for k, n in (("sumR", N + 1), ("varR", N + 1), ("R", N),
                                                  ("lambda", K), ("sil", N), ("iln", N))}
            P = lambda a: a.ctypes.data_as(C.c_void_p)
            lib.OutPutResults.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_void_p]
            lib.OutPutResults(geno, int(spec["rep"]), 1, inds, P(keep["PSum"]), P(keep["QSum"]),
                              P(keep["FstSum"]), P(ad) if ad is not None else None,
                              P(usepop) if usepop is not None else None,
                              float(z["sumlikes"]), float(z["sumsqlikes"]), P(keep["sumAlpha"]),
                              P(zeros["sumR"]), P(zeros["varR"]), na, tr, 1, names,
                              P(zeros["R"]), P(keep["SumEps"]), P(zeros["lambda"]),
                              P(keep["sumlambda"]), P(slp) if slp is not None else None, lplen,
                              P(zeros["sil"]), P(zeros["iln"]),
                              len(argv), cargv)
    C.CDLL(None).fflush(None)
    with open(os.path.join(workdir, "ref_out.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    # the reference prints progress on stdout: keep it for the tests
    fd = os.open(os.path.join(sys.argv[1], "ref_stdout.txt"),
                 os.O_WRONLY | os.O_CREAT | os.O_TRUNC, 0o644)
    os.dup2(fd, 1)
    main(sys.argv[1], sys.argv[2])
