"""The dense-DFT scheme of the reference-mode galaxy render (k_gal_fft in
uph_galfft.cu) restated in numpy with the kernel's index arithmetic -- row
transforms of the T non-zero rows to P/2 + 1 frequencies, column transforms
against P frequencies, twiddles (j u) mod P from a float32 table, the
inverse cropped to T x T with the Hermitian row sum -- agrees with the
oracle's numpy FFT render (sersic_mog.py:153-207) on every row the Gauss-
Newton step uses.  The GPU parity test checks the kernel itself."""
import numpy as np
import pytest

import oracle.island_oracle as O
from test_oracle_pins import _mini_island


def _dft_render(psf, psfx, psfy, gal, T, PP, need):
    amps, vars_, core, da, dv, dcore, dndu, cg, dcg = gal
    H = PP // 2 + 1
    msk = PP - 1
    m = np.arange(PP)
    cw = np.cos(2 * np.pi * m / PP).astype(np.float32)
    sw = np.sin(2 * np.pi * m / PP).astype(np.float32)
    imgs = [psf, psfx, psfy]
    X = [None] * 3
    for im in range(3):
        if not need[im]:
            continue
        a = imgs[im].astype(np.float64)
        i = np.arange(T)[:, None]; u = np.arange(H)[None, :]
        j = np.arange(T)
        # R[i][u] = sum_j a[i][j] (cw - i sw)[(j u) & msk]
        idx = (j[:, None] * np.arange(H)[None, :]) & msk        # (T_j, H)
        R = a @ (cw[idx] - 1j * sw[idx])                        # (T_i, H)
        idx2 = (np.arange(T)[None, :] * np.arange(PP)[:, None]) & msk   # (P_w, T_i)
        X[im] = (cw[idx2] - 1j * sw[idx2]) @ R                   # (P, H)
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
        Q = Xb * fac
        idx3 = (np.arange(T)[:, None] * np.arange(PP)[None, :]) & msk   # (T_i, P_w)
        C = (cw[idx3] + 1j * sw[idx3]) @ Q                       # (T, H)
        jj = np.arange(T)
        v = C[:, 0].real[:, None] + np.where(jj % 2 == 1, -1, 1)[None, :] * C[:, H - 1].real[:, None]
        idx4 = (jj[None, :] * np.arange(1, H - 1)[:, None]) & msk   # (H-2, T_j)
        acc = C[:, 1:H - 1].real @ cw[idx4] - C[:, 1:H - 1].imag @ sw[idx4]
        r = (v + 2 * acc) / (PP * PP)
        if s == 0: r = r + core * psf
        elif s == 1: r = r + core * psfx
        elif s == 2: r = r + core * psfy
        elif s == 6: r = (r + dcore * psf) * dndu
        out[s] = r
    return out


@pytest.mark.parametrize("T", [31, 55, 63])
def test_dense_dft_scheme_matches_the_fft_render(T):
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
    out = _dft_render(psf, psf, psf, gal, T, O.fft_pad_for(T), [1, 1, 1, 1, 1, 1, 1])
    ref = {0: S, 1: S, 2: S, 3: Ssh[0], 4: Ssh[1], 5: Ssh[2], 6: Su}
    for q, r in ref.items():
        assert np.abs(out[q] - r).max() <= 1e-6 * np.abs(r).max(), q
