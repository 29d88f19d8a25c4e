"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No survey data, mock catalogue or random-field realisation ships with this
project; these generators stand in for them:

* ``forest_catalog`` — quasar sightlines with Lyman-alpha forest pixels:
  positions uniform on the sphere inside a mask, z_q ~ U[2.1, 3.5], pixels on
  the global log10(lambda) grid k * 1e-4 over rest frame 1040-1200 A clipped to
  observed >= 3600 A, delta ~ N(0, 0.2^2) drawn in float64 and stored as
  float32, weights ~ U[0.5, 2], comoving distances from flat LCDM
  (Omega_m = 0.3) stored as float32 (h5healxi.cc:196-203).
* ``small_patch`` — 2,000 sightlines on a 10 x 10 degree patch.
* ``full_survey`` — 160,000 sightlines (16 per deg^2) over the union of the
  HEALPix nside=8 cells whose centres lie in a seeded ~10,000 deg^2 cap.
* ``mock_batch`` — mock catalogues with sightline counts log-uniform in
  [2k, 40k], each on its own seeded cap at 16 sightlines per deg^2, merged
  into one catalogue with one sightline group per mock (``merge_groups``).
* ``grf_grid`` — 64^3 Gaussian random field with P(k) ~ k^-2 on a 256 Mpc/h
  periodic box, unit variance, points at cell centres, w = 1.
"""
from __future__ import annotations

import math

import numpy as np

from . import PIXEL_DTYPE, PLATE_DTYPE, SIGHTLINE_DTYPE

LYA = 1216.0
LOG_LYA = math.log10(LYA)
HUBBLE_DISTANCE = 2997.92458  # c / (100 km/s/Mpc), Mpc/h
LOGLAM_STEP = 1e-4


def comoving_distance_fp64(z: np.ndarray, omega_m: float = 0.3) -> np.ndarray:
    """Flat LCDM D_C(z) in Mpc/h, FP64 (Gauss-Legendre, 64 nodes per unit z)."""
    z = np.asarray(z, dtype=np.float64)
    out = np.empty_like(z)
    xg, wg = np.polynomial.legendre.leggauss(64)
    flat = z.ravel()
    res = out.ravel()
    for k, zz in enumerate(flat):
        if zz <= 0:
            res[k] = 0.0
            continue
        n = max(1, int(math.ceil(zz)))
        acc = 0.0
        for p in range(n):
            a, b = zz * p / n, zz * (p + 1) / n
            t = 0.5 * (b - a) * xg + 0.5 * (b + a)
            acc += 0.5 * (b - a) * np.sum(wg / np.sqrt(omega_m * (1 + t) ** 3 + (1 - omega_m)))
        res[k] = HUBBLE_DISTANCE * acc
    return out


def _pixel_index_range(zq: np.ndarray):
    """Global loglam grid indices [k0, k1] of each forest."""
    lo = np.log10(np.maximum(1040.0 * (1.0 + zq), 3600.0))
    hi = np.log10(1200.0 * (1.0 + zq))
    k0 = np.ceil(lo / LOGLAM_STEP - 1e-9).astype(np.int64)
    k1 = np.floor(hi / LOGLAM_STEP + 1e-9).astype(np.int64)
    return k0, k1


def forest_catalog(ra: np.ndarray, dec: np.ndarray, seed: int, omega_m: float = 0.3,
                   delta_sigma: float = 0.2, zq_range=(2.1, 3.5)):
    """Sightlines at (ra, dec) [radians] with seeded forests.

    Returns (sightlines, pixels, meta) where sightlines/pixels are numpy arrays
    of the engine's C structs and meta has the transverse comoving scale at the
    lowest pixel redshift (the XiEstimator ``scale``)."""
    rng = np.random.default_rng(seed)
    n = len(ra)
    zq = rng.uniform(zq_range[0], zq_range[1], n)
    k0, k1 = _pixel_index_range(zq)
    npx = (k1 - k0 + 1).astype(np.int64)
    total = int(npx.sum())
    # distance per global loglam index (few thousand distinct values)
    kmin, kmax = int(k0.min()), int(k1.max())
    kk = np.arange(kmin, kmax + 1)
    loglam_k = (kk * LOGLAM_STEP).astype(np.float32)
    zpix = 10.0 ** (loglam_k.astype(np.float64) - LOG_LYA) - 1.0
    dist_k = comoving_distance_fp64(zpix, omega_m).astype(np.float32)
    offsets = np.zeros(n, dtype=np.int64)
    offsets[1:] = np.cumsum(npx)[:-1]
    # pixel -> global index
    rep = np.repeat(np.arange(n), npx)
    local = np.arange(total) - offsets[rep]
    gidx = k0[rep] + local - kmin
    pixels = np.zeros(total, dtype=PIXEL_DTYPE)
    pixels["loglam"] = loglam_k[gidx]
    pixels["distance"] = dist_k[gidx]
    pixels["value"] = rng.normal(0.0, delta_sigma, total).astype(np.float32)
    pixels["weight"] = rng.uniform(0.5, 2.0, total).astype(np.float32)
    los = np.zeros(n, dtype=SIGHTLINE_DTYPE)
    los["ra"] = ra
    los["dec"] = dec
    los["forest_id"] = np.arange(n, dtype=np.int32)
    los["plate"] = 0
    los["pixel_offset"] = offsets.astype(np.uint64)
    los["num_pixels"] = npx.astype(np.uint32)
    # scale = transverse comoving distance at the lowest first-pixel redshift (h5healxi.cc:237-239)
    zmin = 10.0 ** (float(loglam_k[k0.min() - kmin]) - LOG_LYA) - 1.0
    scale = float(comoving_distance_fp64(np.array([zmin]), omega_m)[0])
    meta = {"zq": zq, "scale": scale, "zmin": zmin, "num_pixels": total,
            "pixels_per_sightline": (int(npx.min()), float(npx.mean()), int(npx.max()))}
    return los, pixels, meta


def small_patch(n: int = 2000, seed: int = 1, ra0_deg: float = 180.0, dec0_deg: float = 20.0,
                size_deg: float = 10.0, **kw):
    """Sightlines uniform (in ra and sin dec) on a size x size degree patch."""
    rng = np.random.default_rng(seed)
    ra = np.deg2rad(rng.uniform(ra0_deg, ra0_deg + size_deg, n))
    s0, s1 = math.sin(math.radians(dec0_deg)), math.sin(math.radians(dec0_deg + size_deg))
    dec = np.arcsin(rng.uniform(s0, s1, n))
    return forest_catalog(ra, dec, seed + 1000, **kw)


def plate_tiling(sightlines: np.ndarray, spacing_deg: float = 2.0, first_plate: int = 3000):
    """BOSS-like plates over a catalogue: centres on a lattice of the given
    spacing (in dec, and in ra scaled by 1/cos dec) covering the sightlines,
    each sightline on the plate of the nearest centre (a BOSS plate's fibres
    lie within 1.49 degrees of its centre).  Returns (sightlines with their
    `plate` set, the platelist as PLATE_DTYPE rows of every lattice plate,
    ids first_plate, first_plate + 1, ...; plates may hold no sightline)."""
    ra = np.degrees(np.asarray(sightlines["ra"], dtype=np.float64))
    dec = np.degrees(np.asarray(sightlines["dec"], dtype=np.float64))
    d0, d1 = dec.min() - spacing_deg, dec.max() + spacing_deg
    cra, cdec = [], []
    for dc in np.arange(d0, d1 + 1e-9, spacing_deg):
        step = spacing_deg / max(math.cos(math.radians(dc)), 0.05)
        for rc in np.arange(ra.min() - step, ra.max() + step + 1e-9, step):
            cra.append(rc % 360.0)
            cdec.append(dc)
    plates = np.zeros(len(cra), dtype=PLATE_DTYPE)
    plates["plate"] = first_plate + np.arange(len(cra))
    plates["ra_center"] = np.asarray(cra, dtype=np.float32)
    plates["dec_center"] = np.asarray(cdec, dtype=np.float32)
    # nearest centre on the sphere
    u = np.stack([np.cos(np.radians(dec)) * np.cos(np.radians(ra)), np.cos(np.radians(dec)) * np.sin(np.radians(ra)),
                  np.sin(np.radians(dec))], 1)
    pr, pd = np.radians(plates["ra_center"].astype(np.float64)), np.radians(plates["dec_center"].astype(np.float64))
    v = np.stack([np.cos(pd) * np.cos(pr), np.cos(pd) * np.sin(pr), np.sin(pd)], 1)
    out = np.array(sightlines, copy=True)
    out["plate"] = plates["plate"][np.argmax(u @ v.T, axis=1)]
    return out, plates


def _healpix_centres_nside8():
    """Centres (theta, phi) of the 768 RING pixels of nside = 8."""
    nside = 8
    npix = 12 * nside * nside
    ncap = 2 * nside * (nside - 1)
    th = np.empty(npix)
    ph = np.empty(npix)
    for p in range(npix):
        if p < ncap:
            r = int((1 + math.isqrt(1 + 2 * p)) // 2)
            while 2 * r * (r - 1) > p:
                r -= 1
            while 2 * (r + 1) * r <= p:
                r += 1
            iphi = p + 1 - 2 * r * (r - 1)
            z = 1 - r * r * 4.0 / npix
            phi = (iphi - 0.5) * (math.pi / 2) / r
        elif p < npix - ncap:
            ip = p - ncap
            ring = ip // (4 * nside) + nside
            iphi = ip % (4 * nside) + 1
            fodd = 1.0 if (ring + nside) & 1 else 0.5
            z = (2 * nside - ring) * 2.0 / (3 * nside)
            phi = (iphi - fodd) * math.pi / (2 * nside)
        else:
            ip = npix - p
            r = int((1 + math.isqrt(max(2 * ip - 1, 0))) // 2)
            r = max(r, 1)
            while 2 * r * (r - 1) >= ip:
                r -= 1
            while 2 * (r + 1) * r < ip:
                r += 1
            iphi = 4 * r + 1 - (ip - 2 * r * (r - 1))
            z = -1 + r * r * 4.0 / npix
            phi = (iphi - 0.5) * (math.pi / 2) / r
        th[p] = math.acos(z)
        ph[p] = phi
    return th, ph


def survey_mask(seed: int, area_deg2: float = 10000.0):
    """Set of nside=8 RING cells whose centres lie in a seeded cap of the given area."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=3)
    v /= np.linalg.norm(v)
    cap = math.acos(1.0 - area_deg2 * (math.pi / 180.0) ** 2 / (2 * math.pi))
    th, ph = _healpix_centres_nside8()
    cv = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)
    return np.nonzero(cv @ v >= math.cos(cap))[0], v, cap


def ang2pix_ring(nside: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """Vectorised RING ang2pix (Gorski et al. 2005 formulas)."""
    theta = np.asarray(theta, dtype=np.float64)
    phi = np.asarray(phi, dtype=np.float64)
    z = np.cos(theta)
    za = np.abs(z)
    tt = np.mod(phi * (2 / math.pi), 4.0)
    out = np.empty(theta.shape, dtype=np.int64)
    eq = za <= 2.0 / 3.0
    nl4 = 4 * nside
    t1 = nside * (0.5 + tt[eq])
    t2 = nside * z[eq] * 0.75
    jp = (t1 - t2).astype(np.int64)
    jm = (t1 + t2).astype(np.int64)
    ir = nside + 1 + jp - jm
    ks = 1 - (ir & 1)
    ip = ((jp + jm - nside + ks + 1 + 2 * nl4) // 2) % nl4
    out[eq] = 2 * nside * (nside - 1) + (ir - 1) * nl4 + ip
    pc = ~eq
    tp = tt[pc] - np.floor(tt[pc])
    tmp = nside * np.sqrt(3 * (1 - za[pc]))
    jp = (tp * tmp).astype(np.int64)
    jm = ((1 - tp) * tmp).astype(np.int64)
    ir = jp + jm + 1
    ip = (tt[pc] * ir).astype(np.int64)
    ip = np.where(ip >= 4 * ir, ip - 4 * ir, ip)
    npix = 12 * nside * nside
    out[pc] = np.where(z[pc] > 0, 2 * ir * (ir - 1) + ip, npix - 2 * ir * (ir + 1) + ip)
    return out


def full_survey(n: int = 160000, seed: int = 7, area_deg2: float = 10000.0, **kw):
    """n sightlines uniform over a seeded ~area_deg2 mask made of nside=8 cells."""
    cells, v, cap = survey_mask(seed, area_deg2)
    keep = np.zeros(768, dtype=bool)
    keep[cells] = True
    rng = np.random.default_rng(seed + 1)
    ra_out, dec_out = [], []
    got = 0
    # sample inside a slightly larger cap around v, keep points in masked cells
    big = min(math.pi, cap + math.radians(8.0))
    # orthonormal frame around v
    a = np.array([1.0, 0, 0]) if abs(v[0]) < 0.9 else np.array([0, 1.0, 0])
    e1 = np.cross(v, a)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(v, e1)
    while got < n:
        m = 2 * (n - got) + 1000
        cz = rng.uniform(math.cos(big), 1.0, m)
        az = rng.uniform(0, 2 * math.pi, m)
        sz = np.sqrt(1 - cz * cz)
        p = (cz[:, None] * v[None, :] + (sz * np.cos(az))[:, None] * e1[None, :]
             + (sz * np.sin(az))[:, None] * e2[None, :])
        th = np.arccos(np.clip(p[:, 2], -1, 1))
        ph = np.mod(np.arctan2(p[:, 1], p[:, 0]), 2 * math.pi)
        ok = keep[ang2pix_ring(8, th, ph)]
        th, ph = th[ok], ph[ok]
        take = min(len(th), n - got)
        ra_out.append(ph[:take])
        dec_out.append(0.5 * math.pi - th[:take])
        got += take
    ra = np.concatenate(ra_out)
    dec = np.concatenate(dec_out)
    return forest_catalog(ra, dec, seed + 2000, **kw)


def cap_patch(n: int, seed: int, area_deg2: float, **kw):
    """n sightlines uniform in a spherical cap of the given area around a
    seeded random centre."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=3)
    v /= np.linalg.norm(v)
    cap = math.acos(max(-1.0, 1.0 - area_deg2 * (math.pi / 180.0) ** 2 / (2 * math.pi)))
    a = np.array([1.0, 0, 0]) if abs(v[0]) < 0.9 else np.array([0, 1.0, 0])
    e1 = np.cross(v, a)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(v, e1)
    cz = rng.uniform(math.cos(cap), 1.0, n)
    az = rng.uniform(0, 2 * math.pi, n)
    sz = np.sqrt(1 - cz * cz)
    p = (cz[:, None] * v[None, :] + (sz * np.cos(az))[:, None] * e1[None, :]
         + (sz * np.sin(az))[:, None] * e2[None, :])
    dec = np.arcsin(np.clip(p[:, 2], -1, 1))
    ra = np.mod(np.arctan2(p[:, 1], p[:, 0]), 2 * math.pi)
    return forest_catalog(ra, dec, seed + 3000, **kw)


def merge_groups(parts):
    """One batched catalogue from a list of (sightlines, pixels): part k's
    sightlines get group k and pixel offsets past the earlier parts' pixels."""
    los_all, px_all, off = [], [], 0
    for k, (los, px) in enumerate(parts):
        lk = los.copy()
        lk["group"] = k
        lk["pixel_offset"] += np.uint64(off)
        los_all.append(lk)
        px_all.append(px)
        off += len(px)
    return np.concatenate(los_all), np.concatenate(px_all)


def mock_counts(n_mocks: int = 256, seed: int = 11, n_range=(2000, 40000)) -> np.ndarray:
    """Seeded sightline counts log-uniform in n_range."""
    rng = np.random.default_rng(seed)
    lo, hi = math.log(n_range[0]), math.log(n_range[1])
    return np.exp(rng.uniform(lo, hi, n_mocks)).astype(np.int64)


def mock_batch(n_mocks: int = 256, seed: int = 11, n_range=(2000, 40000), density: float = 16.0,
               first: int = 0, **kw):
    """Mocks first .. first+n_mocks-1 of the seeded draw of mock_counts(seed):
    each on its own cap of area count/density deg^2 (seed seed*1000 + k).
    Returns (parts, scale): parts a list of (sightlines, pixels) and the
    smallest per-mock scale (every mock with a quasar below z = 2.46 reaches
    the 3600 A clip, so the scales agree)."""
    counts = mock_counts(first + n_mocks, seed, n_range)[first:]
    parts, scale = [], None
    for k, n in enumerate(counts):
        los, px, meta = cap_patch(int(n), seed * 1000 + first + k, float(n) / density, **kw)
        parts.append((los, px))
        scale = meta["scale"] if scale is None else min(scale, meta["scale"])
    return parts, scale


def mock_batch_stratified(n_pick: int = 32, n_mocks: int = 256, seed: int = 11, n_range=(2000, 40000),
                          density: float = 16.0, **kw):
    """A size-stratified sample of the seeded n_mocks-mock draw: the mocks at
    ranks 0, s, 2s, ... of the draw sorted by sightline count (s = n_mocks /
    n_pick), so the sample holds the smallest mock and spans the range.  Each
    mock is generated exactly as in mock_batch (its own seed and cap).
    Returns (parts, scale, indices) with the mocks' indices in the draw."""
    counts = mock_counts(n_mocks, seed, n_range)
    order = np.argsort(counts, kind="stable")
    step = max(1, n_mocks // n_pick)
    idx = np.sort(order[::step][:n_pick])
    parts, scale = [], None
    for k in idx:
        n = int(counts[k])
        los, px, meta = cap_patch(n, seed * 1000 + int(k), float(n) / density, **kw)
        parts.append((los, px))
        scale = meta["scale"] if scale is None else min(scale, meta["scale"])
    return parts, scale, idx


def grf_grid(n: int = 64, box: float = 256.0, seed: int = 3, index: float = -2.0) -> np.ndarray:
    """Gaussian random field with P(k) ~ k^index on an n^3 periodic box, unit
    variance, as (n^3, 5) float32 rows x, y, z, delta, w at cell centres."""
    rng = np.random.default_rng(seed)
    white = rng.normal(size=(n, n, n))
    fk = np.fft.rfftn(white)
    kx = np.fft.fftfreq(n, d=box / n) * 2 * math.pi
    kz = np.fft.rfftfreq(n, d=box / n) * 2 * math.pi
    k2 = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    amp = np.zeros_like(k2)
    nz = k2 > 0
    amp[nz] = k2[nz] ** (index / 4.0)  # sqrt(P) with P ~ k^index
    field = np.fft.irfftn(fk * amp, s=(n, n, n), axes=(0, 1, 2))
    field /= field.std()
    cell = box / n
    c = (np.arange(n) + 0.5) * cell
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    pts = np.empty((n ** 3, 5), dtype=np.float32)
    pts[:, 0] = X.ravel()
    pts[:, 1] = Y.ravel()
    pts[:, 2] = Z.ravel()
    pts[:, 3] = field.ravel().astype(np.float32)
    pts[:, 4] = 1.0
    return pts
