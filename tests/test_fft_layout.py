"""The split-row FFT's index arithmetic (csrc/fft.cuh) checked on the CPU.

`Geo` below restates fft.cuh's Geo (samples per CTA, runs of G samples per CTA on split
rows, rows of NL/G in shared memory, the padded and skewed shared offsets, the combined
frequency layout), and `_forward` / `_inverse` restate the kernels' passes with their exact
indices: the Stockham passes over the G rows (`stockham_pass`, `local_fft`) and the one
radix-(C G) butterfly across the cluster (`combine_fwd`, `combine_inv`). For every geometry
the library builds, the time and frequency maps are bijections onto the row and every
shared offset stays inside the CTA's array; for the geometries up to 4096 samples per
row, the 2-CTA rows of 8192 and one 4- and one 8-CTA row in each precision the whole
transform is run and compared with numpy.fft."""
import numpy as np
import pytest


def pad(i):
    return i + (i >> 5)


class Geo:
    def __init__(self, fp64, logn, xc):
        logsz = 4 if fp64 else 3
        self.N = 1 << logn
        self.LOGC = (logn + logsz - 17 if logn + logsz > 17 else 0) + xc
        self.C = 1 << self.LOGC
        self.LOGL = logn - self.LOGC
        self.NL = 1 << self.LOGL
        self.LOGG = 5 - logsz if self.LOGC > 0 else 0
        self.G = 1 << self.LOGG
        self.LOGNLG = self.LOGL - self.LOGG
        self.NLG = 1 << self.LOGNLG
        pref = 5 if (not fp64 and self.LOGL >= 13) else 4
        cap = self.LOGL - 5 if self.LOGL - 5 > 1 else 1
        self.LOGE = min(pref, cap)
        self.E = 1 << self.LOGE
        self.NTHR = self.NL // self.E
        self.LOGCH = self.LOGNLG - self.LOGC
        self.CH = 1 << self.LOGCH
        self.SKEW = 4 if self.LOGG > 0 else 0
        self.NDATA = self.NL + (self.NL >> 5) + (self.G - 1) * self.SKEW
        assert self.LOGE >= self.LOGC + self.LOGG          # static_asserts of Geo
        assert self.LOGNLG - self.LOGE >= 5 or self.LOGG == 0
        assert 32 <= self.NTHR <= 1024

    def sidx(self, i):
        return pad(i) + (i >> self.LOGNLG) * self.SKEW

    def freq_of(self, rank, i):
        return i if self.C == 1 else rank * self.CH + (i & (self.CH - 1)) + self.NLG * (i >> self.LOGCH)

    def time_of_w(self, rank, w):
        if self.C == 1:
            return w
        return ((((w >> self.LOGG) << self.LOGC) + rank) << self.LOGG) + (w & (self.G - 1))

    def local_of_w(self, w):
        return w if self.C == 1 else ((w & (self.G - 1)) << self.LOGNLG) + (w >> self.LOGG)


# (fp64, log2 N, row split): every kernel set the library builds
GEOMETRIES = ([(False, n, 0) for n in range(6, 17)] + [(False, n, 1) for n in range(12, 17)] +
              [(True, n, 0) for n in range(6, 17)] + [(True, n, 1) for n in range(11, 15)])


def _dft(v, inv):
    r = v.shape[-1]
    k = np.arange(r)
    return v @ np.exp((2j if inv else -2j) * np.pi * np.outer(k, k) / r).T


def _stockham(gm, s, logns, logr, inv):
    nb, r = gm.NLG, 1 << logr
    logj = gm.LOGNLG - logr
    tid = np.arange(gm.NTHR)
    out = s.copy()
    for bf in range(gm.E // r):
        ja = tid + bf * gm.NTHR
        base, j = (ja >> logj) << gm.LOGNLG, ja & ((1 << logj) - 1)
        v = np.stack([s[gm.sidx(base + j + q * (nb // r))] for q in range(r)], axis=1)
        jm = j & ((1 << logns) - 1)
        if logns > 0:
            step = jm << (gm.LOGNLG - logns - logr)
            for q in range(1, r):
                v[:, q] *= np.exp((2j if inv else -2j) * np.pi * q * step / nb)
        v = _dft(v, inv)
        idx = ((j >> logns) << (logns + logr)) + jm
        for q in range(r):
            out[gm.sidx(base + idx + (q << logns))] = v[:, q]
    return out


def _local(gm, s, inv):
    logns = 0
    for _ in range(gm.LOGNLG // gm.LOGE):
        s = _stockham(gm, s, logns, gm.LOGE, inv)
        logns += gm.LOGE
    if gm.LOGNLG % gm.LOGE:
        s = _stockham(gm, s, logns, gm.LOGNLG % gm.LOGE, inv)
    return s


def _forward(gm, S):
    S = [_local(gm, x, False) for x in S]
    if gm.C == 1:
        return S
    cg, tid = gm.C * gm.G, np.arange(gm.NTHR)
    new = [x.copy() for x in S]
    for jj in range(gm.E // cg):
        for rank in range(gm.C):
            i = tid + jj * gm.NTHR
            kl = rank * gm.CH + i
            v = np.zeros((gm.NTHR, cg), complex)
            for c in range(gm.C):
                for g in range(gm.G):
                    n = g + gm.G * c
                    v[:, n] = S[c][gm.sidx(g * gm.NLG + kl)] * np.exp(-2j * np.pi * n * kl / gm.N)
            v = _dft(v, False)
            for j in range(cg):
                new[rank][gm.sidx(j * gm.CH + i)] = v[:, j]
    return new


def _inverse(gm, S):
    if gm.C > 1:
        cg, tid = gm.C * gm.G, np.arange(gm.NTHR)
        new = [x.copy() for x in S]
        for jj in range(gm.E // cg):
            for rank in range(gm.C):
                i = tid + jj * gm.NTHR
                kl = rank * gm.CH + i
                v = _dft(np.stack([S[rank][gm.sidx(j * gm.CH + i)] for j in range(cg)], axis=1), True)
                for n in range(cg):
                    v[:, n] *= np.exp(2j * np.pi * n * kl / gm.N)
                for c in range(gm.C):
                    for g in range(gm.G):
                        new[c][gm.sidx(g * gm.NLG + kl)] = v[:, g + gm.G * c]
        S = new
    return [_local(gm, x, True) for x in S]


@pytest.mark.parametrize("fp64,logn,xc", GEOMETRIES)
def test_maps_cover_the_row_once_and_offsets_stay_in_the_array(fp64, logn, xc):
    gm = Geo(fp64, logn, xc)
    off = np.array([gm.sidx(i) for i in range(gm.NL)])
    assert len(set(off.tolist())) == gm.NL and off.min() >= 0 and off.max() < gm.NDATA
    times = [gm.time_of_w(r, w) for r in range(gm.C) for w in range(gm.NL)]
    freqs = [gm.freq_of(r, i) for r in range(gm.C) for i in range(gm.NL)]
    assert sorted(times) == list(range(gm.N)) and sorted(freqs) == list(range(gm.N))
    assert sorted(gm.local_of_w(w) for w in range(gm.NL)) == list(range(gm.NL))
    # a warp walking time in order touches runs of G consecutive samples (whole sectors)
    if gm.C > 1:
        t = np.array([gm.time_of_w(0, w) for w in range(32)])
        assert (t.reshape(-1, gm.G) - t.reshape(-1, gm.G)[:, :1] == np.arange(gm.G)).all()


@pytest.mark.parametrize("fp64,logn,xc", [g for g in GEOMETRIES if g[1] <= 12 or (g[2] == 1 and g[1] <= 13)] +
                         [(True, 14, 1), (False, 15, 1), (True, 16, 0), (False, 16, 1)])  # 4- and 8-CTA rows
def test_transform_matches_numpy(fp64, logn, xc):
    gm = Geo(fp64, logn, xc)
    rng = np.random.default_rng(logn + 32 * xc + 64 * fp64)
    x = rng.standard_normal(gm.N) + 1j * rng.standard_normal(gm.N)
    S = [np.zeros(gm.NDATA, complex) for _ in range(gm.C)]
    for r in range(gm.C):
        for w in range(gm.NL):
            S[r][gm.sidx(gm.local_of_w(w))] = x[gm.time_of_w(r, w)]
    S = _forward(gm, S)
    X = np.zeros(gm.N, complex)
    for r in range(gm.C):
        for i in range(gm.NL):
            X[gm.freq_of(r, i)] = S[r][gm.sidx(i)]
    ref = np.fft.fft(x)
    assert np.abs(X - ref).max() <= 1e-12 * np.abs(ref).max()
    S = _inverse(gm, S)
    y = np.zeros(gm.N, complex)
    for r in range(gm.C):
        for w in range(gm.NL):
            y[gm.time_of_w(r, w)] = S[r][gm.sidx(gm.local_of_w(w))]
    assert np.abs(y / gm.N - x).max() <= 1e-12 * np.abs(x).max()


@pytest.mark.parametrize("fp64,logn,xc", GEOMETRIES)
def test_pass_offsets_by_constant_stride(fp64, logn, xc):
    # stockham_pass computes one padded offset per butterfly and steps by a constant where
    # the elements lie a multiple of 32 apart (reads: stride NB/R when it is one; writes:
    # Ns = 2^logns from 32 up, and R consecutive elements at logns = 0)
    gm = Geo(fp64, logn, xc)
    passes = [gm.LOGE] * (gm.LOGNLG // gm.LOGE) + ([gm.LOGNLG % gm.LOGE] if gm.LOGNLG % gm.LOGE else [])
    sidx = np.vectorize(gm.sidx)
    tid = np.arange(gm.NTHR)
    logns = 0
    for logr in passes:
        r, logj = 1 << logr, gm.LOGNLG - logr
        stride = gm.NLG // r
        for bf in range(gm.E // r):
            ja = tid + bf * gm.NTHR
            base, j = (ja >> logj) << gm.LOGNLG, ja & ((1 << logj) - 1)
            if stride % 32 == 0:
                a0 = sidx(base + j)
                for q in range(r):
                    assert (a0 + q * (stride + stride // 32) == sidx(base + j + q * stride)).all()
            jm = j & ((1 << logns) - 1)
            idx = ((j >> logns) << (logns + logr)) + jm
            w0 = sidx(base + idx)
            for q in range(r):
                ref = sidx(base + idx + (q << logns))
                if logns >= 5:
                    assert (w0 + q * ((1 << logns) + (1 << (logns - 5))) == ref).all()
                elif logns == 0:
                    assert (w0 + q == ref).all()
        logns += logr
