"""The radix-2 shared-memory FFT scheme of the reference-mode galaxy render
(``smem_fft_lines`` / ``fft2_*`` in uph_internal.cuh, used by k_gal_fft and
k_sp_gal) restated in numpy with the kernels' index arithmetic -- bit-
reversed loads, decimation-in-time stages fused in pairs with twiddles from
a float32 table, row transforms of the T non-zero rows, column
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

def _bfly(u, v, wr, wi):
    """The kernel's butterfly: t = w v, (u + t, u - t)."""
    w = np.complex64(wr + 1j * wi)
    t = w * v
    return u + t, u - t


def fft_lines(buf, P, sign, cw, sw):
    """buf: (nl, P) complex64; in place, as the kernel does: the lines are
    filled in bit-reversed order, then the decimation-in-time stages run in
    pairs -- for half-lengths h and 2h, the four elements j, j+h, j+2h,
    j+3h of each group of 4h take stage h's butterflies (twiddle j P/(2h))
    and then stage 2h's (twiddles j P/(4h) and (j+h) P/(4h)) -- with a last
    single stage when log2 P is odd."""
    logP = P.bit_length() - 1
    perm = np.array([brev(k, logP) for k in range(P)])
    loaded = np.empty_like(buf)
    loaded[:, perm] = buf          # element k goes to position brev(k)
    buf[:] = loaded
    h = 1
    while 4 * h <= P:
        sA, sB = P // (2 * h), P // (4 * h)
        for grp in range(P // (4 * h)):
            for j in range(h):
                i0 = grp * 4 * h + j
                x0, x1 = buf[:, i0].copy(), buf[:, i0 + h].copy()
                x2, x3 = buf[:, i0 + 2 * h].copy(), buf[:, i0 + 3 * h].copy()
                mA = j * sA
                x0, x1 = _bfly(x0, x1, cw[mA], sign * sw[mA])
                x2, x3 = _bfly(x2, x3, cw[mA], sign * sw[mA])
                mB0, mB1 = j * sB, (j + h) * sB
                x0, x2 = _bfly(x0, x2, cw[mB0], sign * sw[mB0])
                x1, x3 = _bfly(x1, x3, cw[mB1], sign * sw[mB1])
                buf[:, i0], buf[:, i0 + h], buf[:, i0 + 2 * h], buf[:, i0 + 3 * h] = \
                    x0, x1, x2, x3
        h *= 4
    if 2 * h == P:
        step = P // (2 * h)
        for j in range(h):
            m = j * step
            buf[:, j], buf[:, j + h] = _bfly(buf[:, j].copy(), buf[:, j + h].copy(),
                                             cw[m], sign * sw[m])
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
