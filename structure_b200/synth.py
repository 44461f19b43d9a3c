"""Seeded synthetic STRUCTURE datasets (the benchmark shapes).

No dataset ships with the reference for these shapes, so benchmarks and tests
draw their inputs from the generative model STRUCTURE itself assumes:
Q_i ~ Dirichlet, per-population allele frequencies (independent Dirichlet, or
the F model Beta(p(1-F)/F, (1-p)(1-F)/F) around an ancestral frequency p),
each allele copy drawn by first sampling its population from Q_i and then its
allele from that population's frequencies.

Genotypes come back in the reference's layout Geno[ind][line][loc] (int32,
alleles already recoded to 0..k-1 in order of first appearance, missing = -9),
or packed 2 bits per genotype, locus-major, for the biallelic fast path.
"""
import numpy as np

MISSING = -9

# data seed = 20261203 + config number; chain seed = 1000 * config + replicate
DATA_SEED_BASE = 20261203


def recode(geno):
    """Recode raw allele values to 0..k-1 in order of first appearance, scanning
    individuals then lines (datain.c:824-904 CountAlleles).  Returns
    (recoded int32 geno, numalleles int32[L])."""
    N, lines, L = geno.shape
    flat = geno.transpose(2, 0, 1).reshape(L, N * lines)
    out = np.full_like(flat, MISSING)
    numalleles = np.zeros(L, np.int32)
    for l in range(L):
        row = flat[l]
        ok = row != MISSING
        vals = row[ok]
        if vals.size == 0:
            continue
        uniq, first = np.unique(vals, return_index=True)
        order = np.argsort(first)
        code = np.empty(uniq.size, np.int32)
        code[order] = np.arange(uniq.size, dtype=np.int32)
        out[l, ok] = code[np.searchsorted(uniq, vals)]
        numalleles[l] = uniq.size
    return out.reshape(L, N, lines).transpose(1, 2, 0).copy(), numalleles


def canonical_biallelic(geno):
    """Sort the two copies of each genotype (smaller code on line 0).  For
    unphased data this changes nothing in the model; after recoding it keeps
    the codes (0 is still seen first) and makes the data packable at 2 bits
    per genotype."""
    a, b = geno[:, 0, :], geno[:, 1, :]
    lo = np.where((a == MISSING) | (b == MISSING), np.maximum(a, b), np.minimum(a, b))
    hi = np.where((a == MISSING) | (b == MISSING), np.minimum(a, b), np.maximum(a, b))
    out = np.stack([lo, hi], axis=1)
    # keep "missing" on line 1 when only one copy is missing
    return np.ascontiguousarray(out.astype(np.int32))


def _draw_z(rng, Q, L):
    """Population of origin for each allele copy: [N, 2, L] int8."""
    N, K = Q.shape
    cq = np.cumsum(Q, axis=1)
    cq[:, -1] = 1.0
    u = rng.random((N, 2, L), dtype=np.float64)
    z = np.zeros((N, 2, L), np.int8)
    for k in range(K - 1):
        z += (u > cq[:, k][:, None, None]).astype(np.int8)
    return z


def microsat(N=200, L=100, K=3, amin=2, amax=10, qalpha=0.5, missing=0.05, seed=None):
    """Config 1: multi-allelic loci, A_l ~ U{amin..amax}, P ~ Dir(1), copies
    missing i.i.d."""
    rng = np.random.default_rng(DATA_SEED_BASE + 1 if seed is None else seed)
    Q = rng.dirichlet(np.full(K, qalpha), size=N)
    A = rng.integers(amin, amax + 1, size=L)
    z = _draw_z(rng, Q, L)
    geno = np.empty((N, 2, L), np.int32)
    for l in range(L):
        Pl = rng.dirichlet(np.ones(A[l]), size=K)          # [K, A_l]
        cp = np.cumsum(Pl, axis=1)
        cp[:, -1] = 1.0
        u = rng.random((N, 2))
        zz = z[:, :, l]
        allele = (u[..., None] > cp[zz][..., :-1]).sum(-1)
        geno[:, :, l] = 100 + 3 * allele                    # raw microsatellite-like codes
    geno[rng.random((N, 2, L)) < missing] = MISSING
    rec, na = recode(geno)
    return dict(geno_raw=geno, geno=rec, numalleles=na, Q=Q, K=K)


def snp_fmodel(N, L, K, F, qalpha, missing, seed, p_beta=(1.0, 1.0), chunk=1024,
               want_int32=True, indep_beta=None):
    """Configs 2/3/5: biallelic SNPs under the F model; whole genotypes missing.
    Genotype code g = copies of allele 1 (0,1,2; 3 = missing).  At each locus the
    allele labels are chosen so that the first non-missing copy (scanning
    individuals, then lines) is allele 0, so the reference's recoding
    (datain.c:824-904) leaves the codes unchanged; heterozygotes are stored
    0 on line 0, 1 on line 1.  indep_beta=(a, b): independent frequencies
    P_kl ~ Beta(a, b) instead of the F model (config 4)."""
    rng = np.random.default_rng(seed)
    F = np.asarray(F, np.float64)
    Q = rng.dirichlet(np.full(K, qalpha), size=N)
    cq = np.cumsum(Q, axis=1)
    cq[:, -1] = 1.0
    cq32 = cq.astype(np.float32)
    geno = np.empty((N, 2, L), np.int32) if want_int32 else None
    numalleles = np.zeros(L, np.int32)
    wpr = (N + 15) // 16
    packed = np.zeros((L, wpr), np.uint32)
    fr = (1.0 - F) / F
    for l0 in range(0, L, chunk):
        l1 = min(L, l0 + chunk)
        n = l1 - l0
        p = np.clip(rng.beta(p_beta[0], p_beta[1], size=n), 1e-4, 1 - 1e-4)
        if indep_beta is None:
            P1 = rng.beta(p[None, :] * fr[:, None], (1 - p[None, :]) * fr[:, None])  # [K, n]
        else:
            P1 = rng.beta(indep_beta[0], indep_beta[1], size=(K, n))
        u = rng.random((N, 2, n), dtype=np.float32)
        z = np.zeros((N, 2, n), np.int8)
        for k in range(K - 1):
            z += u > cq32[:, k][:, None, None]
        v = rng.random((N, 2, n), dtype=np.float32)
        a = v < P1.astype(np.float32)[z, np.arange(n)[None, None, :]]
        g = a.sum(axis=1, dtype=np.uint8)                     # [N, n]
        g[rng.random((N, n), dtype=np.float32) < missing] = 3
        ok = g != 3
        first = np.where(ok.any(0), ok.argmax(0), 0)
        flip = ok.any(0) & (g[first, np.arange(n)] == 2)
        g = np.where(flip[None, :] & ok, 2 - g, g).astype(np.uint8)
        has0 = ((g == 0) | (g == 1)).any(0)
        has1 = ((g == 1) | (g == 2)).any(0)
        numalleles[l0:l1] = has0.astype(np.int32) + has1.astype(np.int32)
        if want_int32:
            lo = np.where(g == 2, 1, 0).astype(np.int32)
            hi = np.where(g >= 1, 1, 0).astype(np.int32)
            lo[g == 3] = MISSING
            hi[g == 3] = MISSING
            geno[:, 0, l0:l1] = lo
            geno[:, 1, l0:l1] = hi
        packed[l0:l1] = pack_codes(g)
    out = dict(Q=Q, K=K, F=F, packed=packed, numalleles=numalleles, N=N, L=L)
    if want_int32:
        out["geno"] = geno
    return out


def pack_codes(g):
    """g: [N, n] genotype codes -> [n, ceil(N/16)] uint32, 16 individuals/word,
    individual j of a word in bits 2j..2j+1.  Padding individuals are 3."""
    N, n = g.shape
    wpr = (N + 15) // 16
    gp = np.full((wpr * 16, n), 3, np.uint32)
    gp[:N] = g
    gp = gp.reshape(wpr, 16, n)
    w = np.zeros((wpr, n), np.uint32)
    for j in range(16):
        w |= gp[:, j, :] << np.uint32(2 * j)
    return np.ascontiguousarray(w.T)


def unpack_int32(packed, N, l0=0, l1=None):
    """Inverse of pack_codes for loci [l0, l1): reference-layout int32 geno
    [N][2][l1-l0] with -9 for missing."""
    l1 = packed.shape[0] if l1 is None else l1
    w = packed[l0:l1]                                      # [n, wpr]
    j = np.arange(N)
    g = (w[:, j >> 4] >> (2 * (j & 15)).astype(np.uint32)) & np.uint32(3)   # [n, N]
    g = g.T.astype(np.int8)
    lo = (g == 2).astype(np.int32)
    hi = (g >= 1).astype(np.int32)
    lo[g == 3] = MISSING
    hi[g == 3] = MISSING
    return np.ascontiguousarray(np.stack([lo, hi], axis=1))


def repack_from_int32(geno):
    """Pack canonical biallelic recoded genotypes (line0 <= line1, whole
    genotypes missing) at 2 bits/genotype: 0 = 0/0, 1 = 0/1, 2 = 1/1, 3 = missing."""
    a, b = geno[:, 0, :], geno[:, 1, :]
    g = np.where((a < 0) | (b < 0), 3, a + b).astype(np.uint8)
    return pack_codes(g)


def config2(N=2000, L=50000, seed=None, want_int32=True):
    return snp_fmodel(N, L, 5, [0.05, 0.10, 0.15, 0.20, 0.25], 0.3, 0.03,
                      DATA_SEED_BASE + 2 if seed is None else seed, want_int32=want_int32)


def config3_datasets(seed=None, want_int32=True):
    base = DATA_SEED_BASE + 3 if seed is None else seed
    shapes = [(300, 5000), (1000, 10000), (2500, 20000), (4000, 8000)]
    out = []
    for s, (N, L) in enumerate(shapes):
        rng = np.random.default_rng(base * 10 + s)
        F = rng.uniform(0.02, 0.2, size=4)
        out.append(snp_fmodel(N, L, 4, F, 0.3, 0.03, base * 10 + s + 100, want_int32=want_int32))
    return out


def config4(N=5000, L=100000, seed=None, want_int32=False):
    """Config 4: N=5000, L=100,000 biallelic SNPs, K=8, Q ~ Dir(0.2), independent
    frequencies P ~ Beta(0.5, 0.5), no missing data."""
    return snp_fmodel(N, L, 8, np.full(8, 0.5), 0.2, 0.0,
                      DATA_SEED_BASE + 4 if seed is None else seed, want_int32=want_int32,
                      indep_beta=(0.5, 0.5))


def config5(N=10000, L=500000, seed=None, want_int32=False):
    """Config 5: N=10,000, L=500,000 biallelic SNPs, 2% missing, K=10 F model with
    F_k ~ U[0.01, 0.3], Q ~ Dir(0.1)."""
    rng = np.random.default_rng(DATA_SEED_BASE + 5 if seed is None else seed)
    F = rng.uniform(0.01, 0.3, 10)
    return snp_fmodel(N, L, 10, F, 0.1, 0.02, int(rng.integers(1 << 31)), want_int32=want_int32)


def snp_fmodel_device(N, L, K, F, qalpha, missing, seed, p_beta=(1.0, 1.0), indep_beta=None,
                      chunk=2048, device="cuda"):
    """snp_fmodel's generative model drawn on a CUDA device with torch's
    generator (seeded), for the large shapes where the NumPy version takes
    minutes (N=10,000 x L=500,000 is 5e9 genotypes).  Same model and the same
    canonical coding (first non-missing copy of a locus is allele 0,
    heterozygotes 0/1, whole genotypes missing); different random numbers.
    Returns dict(packed [L][ceil(N/16)] uint32, numalleles, N, L, K)."""
    import torch
    dev = torch.device(device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed))
    torch.manual_seed(int(seed))       # torch._standard_gamma draws from the default generator
    F = torch.as_tensor(np.asarray(F, np.float64), device=dev)
    fr = (1.0 - F) / F
    gq = torch._standard_gamma(torch.full((N, K), float(qalpha), dtype=torch.float64, device=dev))
    Q = gq / gq.sum(1, keepdim=True).clamp_min(1e-300)
    cq = torch.cumsum(Q, 1)[:, :K - 1].float().contiguous()           # [N, K-1]
    wpr = (N + 15) // 16
    packed = np.zeros((L, wpr), np.uint32)
    numalleles = np.zeros(L, np.int32)
    shifts = (2 * torch.arange(16, device=dev, dtype=torch.int64)).view(1, 16, 1)
    for l0 in range(0, L, chunk):
        l1 = min(L, l0 + chunk)
        n = l1 - l0
        if tuple(p_beta) == (1.0, 1.0):
            p = torch.rand(n, generator=gen, device=dev, dtype=torch.float64)
        else:
            a = torch._standard_gamma(torch.full((n,), p_beta[0], dtype=torch.float64, device=dev))
            b = torch._standard_gamma(torch.full((n,), p_beta[1], dtype=torch.float64, device=dev))
            p = a / (a + b)
        p = p.clamp(1e-4, 1 - 1e-4)
        if indep_beta is None:
            ca = (p[None, :] * fr[:, None]).clamp_min(1e-300)
            cb = ((1 - p)[None, :] * fr[:, None]).clamp_min(1e-300)
        else:
            ca = torch.full((K, n), float(indep_beta[0]), dtype=torch.float64, device=dev)
            cb = torch.full((K, n), float(indep_beta[1]), dtype=torch.float64, device=dev)
        ga, gb = torch._standard_gamma(ca), torch._standard_gamma(cb)
        P1 = (ga / (ga + gb).clamp_min(1e-300)).float().t().contiguous()  # [n, K]
        u = torch.rand((N, 2 * n), generator=gen, device=dev)
        z = torch.searchsorted(cq, u, right=False).view(N, 2, n)          # #(cq_k < u)
        v = torch.rand((N, 2, n), generator=gen, device=dev)
        lidx = torch.arange(n, device=dev).view(1, 1, n)
        a1 = v < P1[lidx, z]
        g = a1.sum(1, dtype=torch.uint8)                                   # [N, n]
        g[torch.rand((N, n), generator=gen, device=dev) < missing] = 3
        ok = g != 3
        anyok = ok.any(0)
        first = ok.to(torch.uint8).argmax(0)
        flip = anyok & (g[first, torch.arange(n, device=dev)] == 2)
        g = torch.where(flip[None, :] & ok, 2 - g, g)
        has0 = ((g == 0) | (g == 1)).any(0)
        has1 = ((g == 1) | (g == 2)).any(0)
        numalleles[l0:l1] = (has0.int() + has1.int()).cpu().numpy()
        gp = torch.full((wpr * 16, n), 3, dtype=torch.int64, device=dev)
        gp[:N] = g.to(torch.int64)
        w = (gp.view(wpr, 16, n) << shifts).sum(1)                         # [wpr, n]
        packed[l0:l1] = w.t().contiguous().cpu().numpy().astype(np.uint32)
        del u, z, v, a1, g, gp, w
    return dict(packed=packed, numalleles=numalleles, N=N, L=L, K=K)
