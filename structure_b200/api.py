"""Python host mirror of the C ABI in include/stgpu.h.

Names follow the reference's update functions (UpdateP, UpdateQ, UpdateZ,
UpdateAlpha, UpdateEpsilon, UpdateFst, DataCollection: pmelsted/structure
src/Updates/*.h, src/output.h) on a chain handle whose state lives in HBM.
Every call goes through libstgpu.so; there is no CPU fallback -- a missing
library or device raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# STGPU_LIB selects another build of the library (e.g. one installed elsewhere)
LIB_PATH = os.environ.get("STGPU_LIB") or os.path.join(HERE, "libstgpu.so")

ST_OK, ST_ERR_ARG, ST_ERR_CUDA, ST_ERR_NOMEM, ST_ERR_ADMISSION = 0, -1, -2, -3, -4
ST_ERR_STATE, ST_ERR_DEVICE, ST_ERR_UNSUPPORTED, ST_ERR_NODEVICE = -5, -6, -7, -8
LAYOUT_AUTO, LAYOUT_U8, LAYOUT_B2G = 0, 1, 2

(F_Q, F_LOGQ, F_TESTQ, F_LOGTESTQ, F_P, F_LOGP, F_EPS, F_F, F_ALPHA, F_LAMBDA, F_Z, F_N,
 F_M, F_LOGDIFF, F_QSUM, F_PSUM, F_SUMEPS, F_FSTSUM, F_SUMALPHA, F_SUMLAMBDA, F_ANCESTDIST,
 F_STATS, F_REP, F_ERR, F_DIMS, F_MALA_EPS, F_USEPOPPROBS, F_LOCPRIOR, F_SUMLOCPRIOR,
 F_MYLOC) = range(1, 31)

# stats block offsets (csrc/st_types.h)
ST_LIKE, ST_SUMLIKES, ST_SUMSQ, ST_NLIKE, ST_METROHITS = 0, 1, 2, 3, 4
ST_ALPHA_T, ST_ALPHA_S = 6, 8
ST_FST_DIFF, ST_FST_NEW, ST_ALPHA_LPD, ST_FST_LPD, ST_ALPHA_NEW = 40, 72, 104, 136, 168
ST_MALA_ACC, ST_MALA_TRIES, ST_LAMBDA_LPD = 200, 201, 202


class StError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"stgpu error {code}: {msg}")
        self.code = code


class DataDesc(C.Structure):
    _fields_ = [("num_inds", C.c_int32), ("num_loci", C.c_int32), ("lines", C.c_int32),
                ("layout", C.c_int32), ("geno", C.c_void_p), ("packed", C.c_void_p),
                ("num_alleles", C.c_void_p), ("popflags", C.c_void_p),
                ("population", C.c_void_p), ("location", C.c_void_p)]


class Model(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "maxpops", "burnin", "numreps", "noadmix", "linkage", "usepopinfo", "locprior",
        "freqscorr", "onefst", "inferalpha", "popalphas", "inferlambda", "popspecificlambda",
        "unifprioralpha", "computeprob", "pfrompopflagonly", "ancestdist", "numboxes",
        "metrofreq", "recessivealleles")] + \
        [(n, C.c_double) for n in ("alpha", "alphamax", "alphapropsd", "alphapriora",
                                   "alphapriorb", "lambda_", "fpriormean", "fpriorsd")] + \
        [(n, C.c_int32) for n in ("store_z", "precision", "tile_t", "tile_w", "tile_r", "mala",
                                  "mala_target", "admburnin", "gensback", "popflag_given")] + \
        [("updatelocprior", C.c_int32), ("startatpopinfo", C.c_int32), ("migrprior", C.c_double),
         ("locpriorinit", C.c_double), ("maxlocprior", C.c_double),
         ("locpriorstep", C.c_double)]


_lib = None


def lib():
    """Load libstgpu.so (build it if this checkout has none yet)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if os.environ.get("STGPU_LIB"):
            raise OSError(f"STGPU_LIB={LIB_PATH} does not exist")
        from . import build
        build.build()
    L = C.CDLL(LIB_PATH)
    vp, i32, u64, sz = C.c_void_p, C.c_int32, C.c_uint64, C.c_size_t
    sig = {
        "st_version": ([], C.c_int),
        "st_ctx_create": ([C.c_int, sz, C.POINTER(vp)], C.c_int),
        "st_ctx_destroy": ([vp], C.c_int),
        "st_last_error": ([vp], C.c_char_p),
        "st_ctx_memory": ([vp, C.POINTER(sz), C.POINTER(sz)], C.c_int),
        "st_ctx_set_stream": ([vp, vp], C.c_int),
        "st_ctx_profile": ([vp, C.c_int], C.c_int),
        "st_ctx_profile_read": ([vp, C.POINTER(C.c_double), C.POINTER(C.c_int64)], C.c_int),
        "st_ctx_launches": ([vp], C.c_int64),
        "st_data_upload": ([vp, C.POINTER(DataDesc), C.POINTER(vp)], C.c_int),
        "st_data_destroy": ([vp], C.c_int),
        "st_data_layout": ([vp], C.c_int),
        "st_model_defaults": ([C.POINTER(Model)], C.c_int),
        "st_chain_create": ([vp, vp, C.POINTER(Model), u64, C.POINTER(vp)], C.c_int),
        "st_chain_destroy": ([vp], C.c_int),
        "st_update_p": ([vp], C.c_int), "st_update_q": ([vp], C.c_int),
        "st_update_z": ([vp], C.c_int), "st_update_alpha": ([vp], C.c_int),
        "st_update_eps": ([vp], C.c_int), "st_update_fst": ([vp], C.c_int),
        "st_collect": ([vp], C.c_int),
        "st_update_q_mala": ([vp], C.c_int),
        "st_update_lambda": ([vp], C.c_int),
        "st_update_locprior": ([vp], C.c_int),
        "st_calc_like": ([vp, C.POINTER(C.c_double)], C.c_int),
        "st_batch_autotune": ([vp, C.c_int], C.c_int),
        "st_chain_save": ([vp, C.c_char_p], C.c_int),
        "st_chain_load": ([vp, C.c_char_p], C.c_int),
        "st_update_z_injected": ([vp, vp, sz, C.c_int], C.c_int),
        "st_update_p_injected": ([vp, vp, sz], C.c_int),
        "st_update_q_metro_injected": ([vp, vp, sz], C.c_int),
        "st_sweep": ([vp, C.c_int], C.c_int), "st_run": ([vp], C.c_int),
        "st_sync": ([vp], C.c_int),
        "st_batch_create": ([vp, C.POINTER(vp), C.c_int, C.POINTER(vp)], C.c_int),
        "st_batch_sweep": ([vp, C.c_int], C.c_int),
        "st_batch_graphs": ([vp, C.c_int], C.c_int),
        "st_batch_destroy": ([vp], C.c_int),
        "st_get_state": ([vp, C.c_int, vp, sz], C.c_int),
        "st_set_state": ([vp, C.c_int, vp, sz], C.c_int),
        "st_field_bytes": ([vp, C.c_int], sz),
        "st_get_timing": ([vp, C.POINTER(C.c_double)], C.c_int),
        "st_grad_create": ([vp, vp, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
        "st_grad_destroy": ([vp], C.c_int),
        "st_loglik_grad": ([vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "st_update_z_noalloc": ([C.c_int, vp, i32, i32, i32, i32, vp, vp, u64, i32, vp, vp, vp,
                                 vp, vp, C.POINTER(sz)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


FAST_K_CLASSES = (1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 16, 20, 24, 32)


def fast_class(K):
    """K capacity class of the biallelic Z pass (K is zero-padded up to it)."""
    return next(k for k in FAST_K_CLASSES if k >= K)


def model_defaults(**kw):
    m = Model()
    lib().st_model_defaults(C.byref(m))
    for k, v in kw.items():
        setattr(m, "lambda_" if k == "lambda" else k, v)
    return m


class Context:
    """One CUDA device with an HBM budget (admission control)."""

    def __init__(self, device=0, hbm_budget=0):
        self.h = C.c_void_p()
        rc = lib().st_ctx_create(device, hbm_budget, C.byref(self.h))
        if rc != ST_OK:
            raise StError(rc, "st_ctx_create failed (no CUDA device?)")

    def check(self, rc):
        if rc != ST_OK:
            raise StError(rc, lib().st_last_error(self.h).decode())
        return rc

    def memory(self):
        a, b = C.c_size_t(), C.c_size_t()
        lib().st_ctx_memory(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def set_stream(self, stream_handle):
        """Launch on a caller's cudaStream_t (int handle, e.g. torch's
        Stream.cuda_stream); None restores the context's own stream."""
        self.check(lib().st_ctx_set_stream(self.h, stream_handle or None))

    def profile(self, enable=True):
        self.check(lib().st_ctx_profile(self.h, 1 if enable else 0))

    def profile_read(self):
        """{kind: (ms, launches)} since the last read (kinds: locus, ind, zpass,
        metro, other)."""
        ms = (C.c_double * 5)()
        n = (C.c_int64 * 5)()
        self.check(lib().st_ctx_profile_read(self.h, ms, n))
        return {k: (ms[j], n[j]) for j, k in enumerate(("locus", "ind", "zpass", "metro", "other"))}

    def launches(self):
        return lib().st_ctx_launches(self.h)

    def close(self):
        if self.h:
            lib().st_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Data:
    """Genotypes in HBM (reference layout in, packed on the device)."""

    def __init__(self, ctx, num_alleles, geno=None, packed=None, popflags=None, layout=LAYOUT_AUTO,
                 num_inds=None, num_loci=None, population=None, location=None):
        self.ctx = ctx
        na = np.ascontiguousarray(num_alleles, np.int32)
        d = DataDesc()
        if geno is not None:
            g = np.ascontiguousarray(geno, np.int32)
            d.num_inds, _, d.num_loci = g.shape
            d.geno = g.ctypes.data
            self._g = g
        else:
            p = np.ascontiguousarray(packed, np.uint32)
            d.num_inds, d.num_loci = num_inds, num_loci
            d.packed = p.ctypes.data
            self._p = p
        d.lines = 2
        d.layout = layout
        d.num_alleles = na.ctypes.data
        pf = pp = None
        if popflags is not None:
            pf = np.ascontiguousarray(popflags, np.int32)
            d.popflags = pf.ctypes.data
        if population is not None:
            pp = np.ascontiguousarray(population, np.int32)
            d.population = pp.ctypes.data
        if location is not None:
            lc = np.ascontiguousarray(location, np.int32)
            d.location = lc.ctypes.data
        self.N, self.L = d.num_inds, d.num_loci
        self.A = int(max(1, na.max()))
        self.num_alleles = na
        self.h = C.c_void_p()
        ctx.check(lib().st_data_upload(ctx.h, C.byref(d), C.byref(self.h)))
        self.layout = lib().st_data_layout(self.h)
        self._g = self._p = None

    def close(self):
        if self.h:
            lib().st_data_destroy(self.h)
            self.h = C.c_void_p()


_DT = {F_Q: np.float32, F_LOGQ: np.float32, F_TESTQ: np.float32, F_LOGTESTQ: np.float32,
       F_P: np.float32, F_LOGP: np.float32, F_EPS: np.float64, F_F: np.float64,
       F_ALPHA: np.float64, F_LAMBDA: np.float64, F_Z: np.uint8, F_N: np.int32, F_M: np.int32,
       F_LOGDIFF: np.float64, F_QSUM: np.float64, F_PSUM: np.float64, F_SUMEPS: np.float64,
       F_FSTSUM: np.float64, F_SUMALPHA: np.float64, F_SUMLAMBDA: np.float64,
       F_ANCESTDIST: np.int32, F_STATS: np.float64, F_REP: np.int32, F_ERR: np.int32,
       F_DIMS: np.int32, F_MALA_EPS: np.float32, F_USEPOPPROBS: np.float64,
       F_LOCPRIOR: np.float64, F_SUMLOCPRIOR: np.float64, F_MYLOC: np.int32}


class Chain:
    """One MCMC chain; methods mirror the reference's *CL update twins."""

    def __init__(self, ctx, data, model, seed):
        self.ctx, self.data, self.model = ctx, data, model
        self.h = C.c_void_p()
        ctx.check(lib().st_chain_create(ctx.h, data.h, C.byref(model), seed, C.byref(self.h)))
        dims = self.get(F_DIMS)
        self.N, self.L, self.K, self.A, self.layout, self.G, self.nchunks, self.ngroups = map(int, dims)

    def _shape(self, f):
        N, L, K, A = self.N, self.L, self.K, self.A
        return {F_Q: (N, K), F_LOGQ: (N, K), F_TESTQ: (N, K), F_LOGTESTQ: (N, K),
                F_P: (L, K, A), F_LOGP: (L, K, A), F_EPS: (L, A), F_SUMEPS: (L, A),
                F_Z: (N, 2, L), F_N: (L, K, A), F_M: (N, K), F_LOGDIFF: (N,),
                F_QSUM: (N, K), F_PSUM: (L, K, A), F_STATS: (256,), F_DIMS: (8,),
                F_MALA_EPS: (N,), F_USEPOPPROBS: (N, K, -1)}.get(f, None)

    def get(self, f, out=None):
        """Copy field f to the host.  `out`, if given, is a C-contiguous array of
        the field's type and size (page-locked memory makes the copy a direct DMA)
        and is filled and returned in the field's shape."""
        n = lib().st_field_bytes(self.h, f)
        if out is None:
            out = np.zeros(n // np.dtype(_DT[f]).itemsize, _DT[f])
        elif (out.dtype != np.dtype(_DT[f]) or out.nbytes != n
              or not out.flags["C_CONTIGUOUS"]):
            raise StError(ST_ERR_ARG, "field %d: output array must be C-contiguous %s of %d bytes"
                          % (f, np.dtype(_DT[f]).name, n))
        self.ctx.check(lib().st_get_state(self.h, f, out.ctypes.data, n))
        shp = self._shape(f) if f != F_DIMS else (8,)
        if f == F_ANCESTDIST:
            return out.reshape(self.N, self.K, -1)
        if f in (F_REP, F_ERR):
            return int(out[0])
        return out.reshape(shp) if shp else out

    def set(self, f, arr):
        a = np.ascontiguousarray(arr, _DT[f])
        self.ctx.check(lib().st_set_state(self.h, f, a.ctypes.data, a.nbytes))

    # reference-named updates
    def UpdateP(self): self.ctx.check(lib().st_update_p(self.h))
    def UpdateQ(self): self.ctx.check(lib().st_update_q(self.h))
    def UpdateZ(self): self.ctx.check(lib().st_update_z(self.h))
    def UpdateAlpha(self): self.ctx.check(lib().st_update_alpha(self.h))
    def UpdateEpsilon(self): self.ctx.check(lib().st_update_eps(self.h))
    def UpdateFst(self): self.ctx.check(lib().st_update_fst(self.h))
    def DataCollection(self): self.ctx.check(lib().st_collect(self.h))
    def UpdateQMala(self): self.ctx.check(lib().st_update_q_mala(self.h))
    def UpdateLambda(self): self.ctx.check(lib().st_update_lambda(self.h))
    def UpdateLocPrior(self): self.ctx.check(lib().st_update_locprior(self.h))

    def CalcLike(self):
        """ln P(D|Q,P) of the current state (st_calc_like)."""
        v = C.c_double()
        self.ctx.check(lib().st_calc_like(self.h, C.byref(v)))
        return v.value

    def save(self, path):
        """Checkpoint the whole chain state to `path` (st_chain_save)."""
        self.ctx.check(lib().st_chain_save(self.h, os.fsencode(path)))

    def load(self, path):
        """Resume from a checkpoint of a chain of the same shape (st_chain_load)."""
        self.ctx.check(lib().st_chain_load(self.h, os.fsencode(path)))

    def UpdateZInjected(self, uniforms, precision=64):
        u = np.ascontiguousarray(uniforms, np.float64)
        self.ctx.check(lib().st_update_z_injected(self.h, u.ctypes.data, u.size, precision))

    def UpdatePInjected(self, uniforms):
        """UpdateP with the reference's sampler on the reference's randomArr
        slots (L*K*A*64 uniforms)."""
        u = np.ascontiguousarray(uniforms, np.float64)
        self.ctx.check(lib().st_update_p_injected(self.h, u.ctypes.data, u.size))

    def UpdateQMetroInjected(self, uniforms):
        """UpdateQMetro with the reference's sampler on its randomArr slots
        (N*64 uniforms)."""
        u = np.ascontiguousarray(uniforms, np.float64)
        self.ctx.check(lib().st_update_q_metro_injected(self.h, u.ctypes.data, u.size))

    def sweep(self, n=1):
        self.ctx.check(lib().st_sweep(self.h, n))

    def run(self):
        self.ctx.check(lib().st_run(self.h))

    def sync(self):
        return lib().st_sync(self.h)

    def timing_ms(self):
        v = C.c_double()
        lib().st_get_timing(self.h, C.byref(v))
        return v.value

    def close(self):
        if self.h:
            lib().st_chain_destroy(self.h)
            self.h = C.c_void_p()


class Batch:
    """Chains advanced together, one launch per update step."""

    def __init__(self, ctx, chains):
        self.ctx, self.chains = ctx, chains
        arr = (C.c_void_p * len(chains))(*[c.h.value for c in chains])
        self.h = C.c_void_p()
        ctx.check(lib().st_batch_create(ctx.h, arr, len(chains), C.byref(self.h)))

    def sweep(self, n=1):
        self.ctx.check(lib().st_batch_sweep(self.h, n))

    def graphs(self, enable=True):
        """Replay captured CUDA graphs of the sweep (default on)."""
        self.ctx.check(lib().st_batch_graphs(self.h, int(enable)))

    def autotune(self, reps=3):
        """Time candidate Z-pass tiles on these chains and keep the fastest."""
        self.ctx.check(lib().st_batch_autotune(self.h, int(reps)))

    def close(self):
        if self.h:
            lib().st_batch_destroy(self.h)
            self.h = C.c_void_p()
