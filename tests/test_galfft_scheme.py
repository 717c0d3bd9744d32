"""The radix-2 shared-memory FFT scheme of the reference-mode galaxy render
(``smem_fft_lines`` / ``fft2_*`` in uph_internal.cuh, used by k_gal_fft and
k_sp_gal) restated in numpy with the kernels' index arithmetic -- bit-
reversed loads, iterative decimation-in-time stages with twiddles j P/len
from a float32 table, row transforms of the T non-zero rows, column
transforms of the P/2 + 1 half-spectrum columns, the inverse columns cropped
to T rows and the Hermitian real inverse of those rows -- agrees with the
oracle's numpy FFT render (sersic_mog.py:153-207) on every row the Gauss-
Newton step uses.  The GPU parity tests check the kernels themselves."""
import numpy as np
import pytest

import oracle.island_oracle as O
from test_oracle_pins import _mini_island


def brev(k, logP):
    r = 0
    for b in range(logP):
        r = (r << 1) | ((k >> b) & 1)
    return r

def fft_lines(buf, P, sign, cw, sw):
    """buf: (nl, P) complex64; in-place iterative DIT as the kernel does."""
    logP = P.bit_length() - 1
    nl = buf.shape[0]
    perm = np.array([brev(k, logP) for k in range(P)])
    buf[:] = buf[:, perm]
    length = 2
    while length <= P:
        half = length // 2
        step = P // length
        for grp in range(P // length):
            for j in range(half):
                i0 = grp * length + j
                i1 = i0 + half
                m = j * step
                w = np.complex64(cw[m] + 1j * sign * sw[m])
                t = w * buf[:, i1]
                u = buf[:, i0].copy()
                buf[:, i0] = u + t
                buf[:, i1] = u - t
        length <<= 1
    return buf

def _fft_render(psf, gal, T, PP, need, psfx=None, psfy=None):
    amps, vars_, core, da, dv, dcore, dndu, cg, dcg = gal
    H = PP // 2 + 1
    m = np.arange(PP)
    cw = np.cos(2 * np.pi * m / PP).astype(np.float32)
    sw = np.sin(2 * np.pi * m / PP).astype(np.float32)
    imgs = [psf, psfx, psfy]
    X = [None] * 3
    for im in range(3):
        if not need[im]:
            continue
        # row FFTs of the zero-padded rows i < T
        lines = np.zeros((T, PP), np.complex64)
        lines[:, :T] = imgs[im]
        fft_lines(lines, PP, -1, cw, sw)
        R = lines[:, :H]
        # column FFTs of the H columns (rows >= T are zero)
        cols = np.zeros((H, PP), np.complex64)
        cols[:, :T] = R.T
        fft_lines(cols, PP, -1, cw, sw)
        X[im] = cols.T            # (P, H)
    u = np.arange(H)[None, :]; w = np.arange(PP)[:, None]
    nu = u / PP
    nw = np.where(w < PP // 2, w, w - PP) / PP
    ex = -2 * np.pi ** 2 * (cg[0] * nu * nu + cg[1] * nw * nw + 2 * cg[2] * nu * nw)
    F = sum(amps[g] * np.exp(vars_[g] * ex) for g in range(len(amps)))
    F1 = sum(amps[g] * vars_[g] * np.exp(vars_[g] * ex) for g in range(len(amps)))
    dF = sum((da[g] + amps[g] * dv[g] * ex) * np.exp(vars_[g] * ex) for g in range(len(amps)))
    out = {}
    for s in range(7):
        if not need[s]:
            continue
        Xb = X[s if s < 3 else 0]
        if s < 3:
            fac = F
        elif s < 6:
            q = s - 3
            fac = F1 * (-2 * np.pi ** 2) * (dcg[q][0] * nu * nu + dcg[q][1] * nw * nw + 2 * dcg[q][2] * nu * nw)
        else:
            fac = dF
        Q = (Xb * fac.astype(np.float32)).astype(np.complex64)     # (P, H)
        cols = np.ascontiguousarray(Q.T)                           # (H, P)
        fft_lines(cols, PP, +1, cw, sw)
        C = cols[:, :T].T                                          # (T, H)
        lines = np.zeros((T, PP), np.complex64)
        lines[:, 0] = C[:, 0].real
        lines[:, PP // 2] = C[:, H - 1].real
        for uu in range(1, PP // 2):
            lines[:, uu] = C[:, uu]
            lines[:, PP - uu] = np.conj(C[:, uu])
        fft_lines(lines, PP, +1, cw, sw)
        r = lines[:, :T].real.astype(np.float64) / (PP * PP)
        if s == 0: r = r + core * psf
        elif s == 1: r = r + core * psfx
        elif s == 2: r = r + core * psfy
        elif s == 6: r = (r + dcore * psf) * dndu
        out[s] = r
    return out


@pytest.mark.parametrize("T", [31, 55])
def test_radix2_scheme_matches_the_fft_render(T):
    isl, _ = _mini_island("reference", n_src=2, seed=3, T=T, B=48)
    isl.stype[:] = np.array([0, 3])
    isl.free_n[:] = [False, True]
    isl.keep[1, 2:6] = True
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64)
    gal = s._gal_params(1, p)
    x, y = float(p[6]), float(p[7])
    S, Sx, Sy, Ssh, Su = s._galaxy_fft(0, x, y, gal, True)
    psf, _, _ = s._star_unshifted(0, x, y)
    # the position partials of a varying PSF take the PSF's path with
    # another base image: feed the PSF itself and expect row 0
    out = _fft_render(psf, gal, T, O.fft_pad_for(T), [1] * 7, psf, psf)
    ref = {0: S, 1: S, 2: S, 3: Ssh[0], 4: Ssh[1], 5: Ssh[2], 6: Su}
    for q, r in ref.items():
        assert np.abs(out[q] - r).max() <= 1e-6 * np.abs(r).max(), q
