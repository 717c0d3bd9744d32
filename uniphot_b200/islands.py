"""Island decomposition: coupling radii, connected components, bucketing.

Host-side numpy/scipy, same contract as the reference's
``fit/grid_gpu/islands.py`` (``coupling_radii`` :82, ``flux_aware_radii``
:234, ``build_islands`` :423, ``bucket_islands`` :614): two sources share an
island iff ``dist < r_i + r_j``; islands are numbered by their minimum member
index; the bbox is the half-open integer hull of the member coupling disks;
classes are the smallest (bbox, nsrc) class that holds the island.  Membership
must be identical to the reference's, which the golden fixtures pin.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy import sparse
from scipy.sparse.csgraph import connected_components
from scipy.spatial import cKDTree

SOURCE_STAR = 0
RE_MIN, RE_MAX = 0.3, 200.0
SERSIC_B1 = 1.6783469900166605

# Bucket classes used by the island stage (island_stage.py:133-134).
ISLAND_BBOX_CLASSES = (32, 48, 64, 96, 128, 192, 256, 384)
ISLAND_NSRC_CLASSES = (1, 2, 4, 8, 16, 32, 64)


def nre_multiplier(sersic_n) -> np.ndarray:
    n = np.asarray(sersic_n, dtype=np.float64)
    n = np.where(np.isfinite(n), n, 1.0)
    return np.where(n < 1.5, 4.0, np.where(n < 3.0, 6.0, 8.0))


def coupling_radii(source_type, logre, sersic_n, r_psf: float) -> np.ndarray:
    """Stars: r_psf; extended: nre(n) * clip(exp(logre)) + r_psf."""
    if r_psf <= 0:
        raise ValueError(f"r_psf must be positive, got {r_psf}")
    st = np.asarray(source_type)
    re = np.exp(np.asarray(logre, dtype=np.float64))
    re = np.clip(np.where(np.isfinite(re), re, RE_MIN), RE_MIN, RE_MAX)
    r_ext = nre_multiplier(sersic_n) * re + float(r_psf)
    return np.where(st == SOURCE_STAR, float(r_psf), r_ext)


def psf_radial_profile(stamp: np.ndarray, bin_width: float = 0.5):
    """Monotone (running-min) annulus-mean profile of a unit-sum stamp."""
    s = np.asarray(stamp, dtype=np.float64)
    tot = s.sum()
    if not np.isfinite(tot) or tot <= 0:
        raise ValueError("psf_radial_profile: stamp must have positive sum")
    s = s / tot
    H, W = s.shape
    yy, xx = np.mgrid[0:H, 0:W]
    rr = np.hypot(yy - (H - 1) / 2.0, xx - (W - 1) / 2.0).ravel()
    nbin = int(np.ceil(rr.max() / bin_width)) + 1
    idx = np.minimum((rr / bin_width).astype(np.int64), nbin - 1)
    sums = np.bincount(idx, weights=s.ravel(), minlength=nbin)
    cnts = np.bincount(idx, minlength=nbin)
    ok = cnts > 0
    r = (np.nonzero(ok)[0] + 0.5) * bin_width
    p = np.minimum.accumulate(np.maximum(sums[ok] / cnts[ok], 1e-12))
    return np.concatenate([[0.0], r]), np.concatenate([[p[0]], p])


def _invert_profile(psf_r, psf_p, thresh):
    lp = np.log(psf_p[::-1])
    rr = psf_r[::-1]
    t = np.asarray(thresh, dtype=np.float64)
    out = np.full(t.shape, psf_r[-1], dtype=np.float64)
    pos = np.isfinite(t) & (t > 0)
    tc = np.clip(np.log(np.where(pos, t, 1.0)), lp[0], lp[-1])
    out[pos] = np.interp(tc, lp, rr)[pos]
    out[np.isfinite(t) & (t >= psf_p[0])] = 0.0
    out[np.isinf(t) & (t > 0)] = 0.0
    return out


def flux_aware_radii(source_type, logre, sersic_n, flux, sigma_sky, kappa,
                     psf_r, psf_p, r_psf, r_core=None) -> np.ndarray:
    """Radius where flux * unit_profile(r) = kappa * sigma_sky, floored at the
    PSF FWHM and capped at the geometric coupling radius."""
    from scipy.special import gamma
    if sigma_sky <= 0 or not np.isfinite(sigma_sky):
        raise ValueError(f"sigma_sky must be positive, got {sigma_sky}")
    if kappa <= 0:
        raise ValueError(f"kappa must be positive, got {kappa}")
    st = np.asarray(source_type)
    lr = np.asarray(logre, dtype=np.float64)
    sn = np.asarray(sersic_n, dtype=np.float64)
    flux = np.asarray(flux, dtype=np.float64)
    if r_core is None:
        r_core = 2.0 * float(_invert_profile(psf_r, psf_p,
                                             np.array([0.5 * psf_p[0]]))[0])
    if r_core <= 0:
        raise ValueError(f"r_core must be positive, got {r_core}")
    good = np.isfinite(flux) & (flux > 0)
    thresh = np.where(good, kappa * float(sigma_sky) / np.where(good, flux, 1.0),
                      np.inf)
    r_star = _invert_profile(psf_r, psf_p, thresh)
    re = np.clip(np.where(np.isfinite(lr), np.exp(lr), RE_MIN), RE_MIN, RE_MAX)
    n = np.where(np.isfinite(sn), sn, 1.0)
    n_eff = np.where(n < 1.5, 1.0, n)
    b = np.where(n_eff < 1.5, SERSIC_B1, 2.0 * n_eff - 1.0 / 3.0)
    i0 = b ** (2.0 * n_eff) / (2.0 * np.pi * n_eff * gamma(2.0 * n_eff) * re ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        arg = np.log(i0 / thresh)
    r_ext = np.where(arg > 0, re * (np.maximum(arg, 0.0) / b) ** n_eff, 0.0)
    cap = coupling_radii(st, lr, sn, r_psf)
    return np.clip(np.where(st == SOURCE_STAR, r_star, r_ext), r_core, cap)


@dataclass
class IslandSet:
    n_sources: int
    n_islands: int
    labels: np.ndarray
    radius: np.ndarray
    members: list = field(repr=False)
    n_src: np.ndarray = field(repr=False)
    bbox: np.ndarray = field(repr=False)
    r_psf: float = 0.0

    @property
    def bbox_size(self) -> np.ndarray:
        return np.maximum(self.bbox[:, 2] - self.bbox[:, 0],
                          self.bbox[:, 3] - self.bbox[:, 1])


def _coupled_pairs(x, y, r):
    """All i<j with (x_i-x_j)^2 + (y_i-y_j)^2 < (r_i + r_j)^2.

    Candidates come from one KD-tree pair query at twice the largest radius
    per radius octave band, then the exact predicate filters them."""
    n = x.shape[0]
    if n < 2:
        return np.empty(0, np.int64), np.empty(0, np.int64)
    octave = np.floor(np.log2(r / r.min())).astype(np.int64)
    bands = np.unique(octave)
    xy = np.column_stack([x, y])
    trees = {b: (cKDTree(xy[octave == b]), np.nonzero(octave == b)[0],
                 float(r[octave == b].max())) for b in bands}
    gi_all, gj_all = [], []
    for a_i, a in enumerate(bands):
        ta, ia, ra = trees[a]
        for b in bands[a_i:]:
            tb, ib, rb = trees[b]
            if b == a:
                pr = ta.query_pairs(r=2.0 * ra, output_type="ndarray")
                if pr.size == 0:
                    continue
                gi, gj = ia[pr[:, 0]], ia[pr[:, 1]]
            else:
                sm = ta.sparse_distance_matrix(tb, ra + rb, output_type="coo_matrix")
                if sm.nnz == 0:
                    continue
                gi, gj = ia[sm.row], ib[sm.col]
            d2 = (x[gi] - x[gj]) ** 2 + (y[gi] - y[gj]) ** 2
            rs = r[gi] + r[gj]
            ok = d2 < rs * rs
            gi_all.append(gi[ok])
            gj_all.append(gj[ok])
    if not gi_all:
        return np.empty(0, np.int64), np.empty(0, np.int64)
    return np.concatenate(gi_all), np.concatenate(gj_all)


def build_islands(pos_x, pos_y, source_type, logre, sersic_n, r_psf, *,
                  radius=None, forced_singleton=None, context=None) -> IslandSet:
    """Coupling islands of a catalog (islands.py:423-560).  With
    ``context`` (a ``uniphot_b200._lib.Context``) the coupled-pair search
    and the connected components run on its GPU (``uph_island_roots``);
    the labels, member lists and boxes are the same."""
    x = np.asarray(pos_x, dtype=np.float64)
    y = np.asarray(pos_y, dtype=np.float64)
    n = x.shape[0]
    if y.shape[0] != n:
        raise ValueError("pos_x and pos_y must have the same length")
    if not (np.all(np.isfinite(x)) and np.all(np.isfinite(y))):
        raise ValueError("build_islands requires finite positions; "
                         "filter the catalog first")
    if source_type is None:
        source_type = np.zeros(n, np.int32)
    if logre is None:
        logre = np.zeros(n)
    if sersic_n is None:
        sersic_n = np.ones(n)
    if radius is not None:
        radius = np.asarray(radius, dtype=np.float64)
        if radius.shape[0] != n:
            raise ValueError("radius must have the same length as pos_x")
        if n and not (np.all(np.isfinite(radius)) and np.all(radius > 0)):
            raise ValueError("radius override must be finite and positive")
    else:
        radius = coupling_radii(source_type, logre, sersic_n, r_psf)
    if n == 0:
        return IslandSet(0, 0, np.empty(0, np.int32), radius, [],
                         np.empty(0, np.int32), np.empty((0, 4), np.int64),
                         float(r_psf))
    if forced_singleton is not None and np.asarray(forced_singleton).shape[0] != n:
        raise ValueError("forced_singleton must have the same length as pos_x")
    if context is not None:
        # component roots are minimum member indices: their ascending order
        # is the order of islands by minimum member
        _, raw = np.unique(context.island_roots(x, y, radius, forced_singleton),
                           return_inverse=True)
    else:
        gi, gj = _coupled_pairs(x, y, radius)
        if forced_singleton is not None and gi.size:
            fs = np.asarray(forced_singleton, dtype=bool)
            ok = ~(fs[gi] | fs[gj])
            gi, gj = gi[ok], gj[ok]
        if gi.size:
            g = sparse.coo_matrix((np.ones(gi.size, np.int8), (gi, gj)), shape=(n, n))
            _, raw = connected_components(g, directed=False)
        else:
            raw = np.arange(n)
    n_isl = int(raw.max()) + 1
    first = np.full(n_isl, n, dtype=np.int64)
    np.minimum.at(first, raw, np.arange(n))
    remap = np.empty(n_isl, np.int64)
    remap[np.argsort(first, kind="stable")] = np.arange(n_isl)
    labels = remap[raw].astype(np.int32)
    order = np.argsort(labels, kind="stable")
    counts = np.bincount(labels, minlength=n_isl).astype(np.int32)
    starts = np.concatenate([[0], np.cumsum(counts[:-1])]).astype(np.int64)
    members = [order[s:s + c].astype(np.int32) for s, c in zip(starts, counts)]
    bbox = np.empty((n_isl, 4), np.int64)
    bbox[:, 0] = np.floor(np.minimum.reduceat((x - radius)[order], starts))
    bbox[:, 1] = np.floor(np.minimum.reduceat((y - radius)[order], starts))
    bbox[:, 2] = np.ceil(np.maximum.reduceat((x + radius)[order], starts))
    bbox[:, 3] = np.ceil(np.maximum.reduceat((y + radius)[order], starts))
    return IslandSet(n, n_isl, labels, radius, members, counts, bbox, float(r_psf))


@dataclass
class IslandBucket:
    bbox_class: int
    nsrc_class: int
    island_ids: np.ndarray
    member_idx: np.ndarray = field(repr=False)
    member_mask: np.ndarray = field(repr=False)
    bbox: np.ndarray = field(repr=False)

    @property
    def n_islands(self) -> int:
        return int(self.island_ids.shape[0])


@dataclass
class BucketedIslands:
    bbox_classes: tuple
    nsrc_classes: tuple
    buckets: dict
    giant_ids: np.ndarray

    @property
    def n_giant(self) -> int:
        return int(self.giant_ids.shape[0])


def bucket_islands(island_set, bbox_classes=ISLAND_BBOX_CLASSES,
                   nsrc_classes=ISLAND_NSRC_CLASSES) -> BucketedIslands:
    bcs = tuple(sorted(int(c) for c in bbox_classes))
    ncs = tuple(sorted(int(c) for c in nsrc_classes))
    bi = np.searchsorted(np.asarray(bcs), island_set.bbox_size, side="left")
    ni = np.searchsorted(np.asarray(ncs), island_set.n_src, side="left")
    giant = (bi >= len(bcs)) | (ni >= len(ncs))
    buckets = {}
    ok_ids = np.nonzero(~giant)[0]
    if ok_ids.size:
        keys = bi[ok_ids] * len(ncs) + ni[ok_ids]
        for key in np.unique(keys):
            sel = ok_ids[keys == key]
            bc, nc = bcs[int(key) // len(ncs)], ncs[int(key) % len(ncs)]
            midx = np.full((sel.size, nc), -1, np.int32)
            mmask = np.zeros((sel.size, nc), bool)
            for row, isl in enumerate(sel):
                m = island_set.members[isl]
                midx[row, :m.size] = m
                mmask[row, :m.size] = True
            buckets[(bc, nc)] = IslandBucket(bc, nc, sel.astype(np.int32),
                                             midx, mmask, island_set.bbox[sel])
    return BucketedIslands(bcs, ncs, buckets,
                           np.nonzero(giant)[0].astype(np.int32))
