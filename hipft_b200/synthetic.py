"""Seeded synthetic inputs for the benchmark workloads.

No public benchmark suite is involved: the workloads are flux-transport runs
on generated maps with the shapes and parameter distributions of the
benchmark configurations.

* ``refined_theta(ntm)``: theta scale 0..pi whose spacing is halved within
  15 degrees of each pole (smooth tanh transition); HipFT takes nonuniform
  theta from the map file's dim2 scale.
* ``bipole_map``: N flux-balanced bipolar Gaussian pairs, latitudes
  +-N(15, 7) deg, longitudes U(0, 360), peak |B| lognormal(ln 300 G, 0.8),
  separation U(3, 10) deg, Joy's-law tilt 0.5|lat|.
* ``batched_params``: per-realization diffusion D log-U(100, 1000) km^2/s,
  meridional-flow amplitude v0 U(10, 20) m/s, differential-rotation B, C
  scaled by U(0.9, 1.1).
* ``observed_map``: the axisymmetric dipole 10 cos(theta) G plus N(0, 2 G)
  noise, with mu = cosine of the angle from a disk centre that rotates at
  the Carrington rate, in the [data, weight, mu] slice order of HipFT's
  assimilation maps.

* ``supergranular_flow``: a random divergent velocity v = grad(psi), psi a
  sum of Gaussian cells of correlation length 30 Mm with random signs and
  centres, differenced onto HipFT's staggered faces (vt on theta faces, vp on
  phi faces), scaled to 300 m/s rms and returned in the layouts of HipFT's
  flow files (use_flow_from_files, src/hipft.f90:3525-3873).  A new field per
  day: ``supergranular_flow(..., day=d)`` seeds with (seed, d).

Flow-model conversion (HipFT's analytic models, src/hipft.f90:7219-7285):
Omega = A + B cos^2 + C cos^4 deg/day becomes vp = st (p0 + p2 ct^2 + p4 ct^4)
m/s with p = (pi/180)/86400 * 6.96e8 * (A, B, C); v0 sin(2 lat) cos^2(lat)
becomes vt = -sth (p1 c + p3 c^3) with p1 = 2 v0, p3 = -2 v0.
"""
from __future__ import annotations

import numpy as np

DEG_DAY_TO_M_S = (np.pi / 180.0) / 86400.0 * 6.96e8  # 140.596...
CARRINGTON_DEG_PER_HOUR = 360.0 / (25.38 * 24.0)


def refined_theta(ntm: int, band_deg: float = 15.0, factor: float = 2.0, width_deg: float = 2.0) -> np.ndarray:
    """ntm theta points on [0, pi] with spacing / factor within band_deg of each pole."""
    x = np.linspace(0.0, np.pi, 20001)
    lat_from_pole = np.minimum(x, np.pi - x)
    b, w = np.deg2rad(band_deg), np.deg2rad(width_deg)
    density = 1.0 + (factor - 1.0) * 0.5 * (1.0 - np.tanh((lat_from_pole - b) / w))
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (density[1:] + density[:-1]) * np.diff(x))])
    cdf /= cdf[-1]
    t = np.interp(np.linspace(0.0, 1.0, ntm), cdf, x)
    t[0], t[-1] = 0.0, np.pi
    return t


def uniform_phi(npm1: int) -> np.ndarray:
    return np.linspace(0.0, 2.0 * np.pi, npm1)


def _gauss(t, p, t0, p0, width):
    """Gaussian of angular distance on the sphere, evaluated in a window of
    +-8 widths around (t0, p0).  Returns (row slice, column indices, values)."""
    rows = slice(np.searchsorted(t, t0 - 8 * width), np.searchsorted(t, t0 + 8 * width))
    tt = t[rows]
    dp = np.deg2rad(8.0) + 8 * width / max(np.sin(t0), 0.1)
    cols = np.nonzero(np.abs(((p - p0 + np.pi) % (2 * np.pi)) - np.pi) <= dp)[0]
    pp = p[cols]
    ct = np.cos(tt)[:, None] * np.cos(t0) + np.sin(tt)[:, None] * np.sin(t0) * np.cos(pp[None, :] - p0)
    ang = np.arccos(np.clip(ct, -1.0, 1.0))
    return rows, cols, np.exp(-(ang / width) ** 2)


def bipole_map(t: np.ndarray, p: np.ndarray, seed: int, n_pairs: int = 200, width_deg: float = 1.0) -> np.ndarray:
    """Br (ntm, npm1) in Gauss from n_pairs flux-balanced bipoles."""
    rng = np.random.Generator(np.random.PCG64(seed))
    st = np.sin(t)
    br = np.zeros((len(t), len(p)))
    w = np.deg2rad(width_deg)
    for _ in range(n_pairs):
        hemi = 1.0 if rng.random() < 0.5 else -1.0
        lat = hemi * abs(rng.normal(15.0, 7.0))
        lon = rng.uniform(0.0, 360.0)
        peak = rng.lognormal(np.log(300.0), 0.8)
        sep = rng.uniform(3.0, 10.0)
        tilt = np.deg2rad(0.5 * abs(lat)) * hemi
        lat_r, lon_r = np.deg2rad(lat), np.deg2rad(lon)
        dlat = 0.5 * np.deg2rad(sep) * np.sin(tilt)
        dlon = 0.5 * np.deg2rad(sep) * np.cos(tilt) / max(np.cos(lat_r), 0.2)
        sign = hemi  # Hale's law: leading polarity flips between hemispheres
        rl, cl, lead = _gauss(t, p, np.pi / 2 - (lat_r - dlat), lon_r + dlon, w)
        rt, ctr, trail = _gauss(t, p, np.pi / 2 - (lat_r + dlat), lon_r - dlon, w)
        fl = (lead * st[rl][:, None]).sum()
        ft = (trail * st[rt][:, None]).sum()
        br[rl.start:rl.stop][:, cl] += sign * peak * lead
        br[rt.start:rt.stop][:, ctr] -= sign * peak * trail * (fl / ft if ft > 0 else 1.0)
    # one-point overlap in phi: the 2*pi column repeats the 0 column
    br[:, -1] = br[:, 0] = 0.5 * (br[:, 0] + br[:, -1])
    return br


def batched_params(nr: int, seed: int) -> dict:
    """Per-realization coefficients of the batched configuration."""
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    D = np.exp(rng.uniform(np.log(100.0), np.log(1000.0), nr))
    v0 = rng.uniform(10.0, 20.0, nr)
    sB = rng.uniform(0.9, 1.1, nr)
    sC = rng.uniform(0.9, 1.1, nr)
    return dict(
        diffusion_coef_constants=D,
        dr_p0=np.zeros(nr), dr_p2=-2.40 * DEG_DAY_TO_M_S * sB, dr_p4=-1.80 * DEG_DAY_TO_M_S * sC,
        mf_p1=2.0 * v0, mf_p3=-2.0 * v0, mf_p5=np.zeros(nr),
        mu_power=np.full(nr, 4.0), mu_limit=np.full(nr, 0.1), lat_limit=np.zeros(nr),
    )


def plain_params() -> dict:
    """Coefficients of the plain (one realization) configuration: D = 300
    km^2/s, v0 = 15 m/s, differential rotation B = -2.40, C = -1.80 deg/day."""
    v0 = 15.0
    return dict(
        diffusion_coef_constants=np.array([300.0]),
        dr_p0=np.zeros(1), dr_p2=np.array([-2.40 * DEG_DAY_TO_M_S]), dr_p4=np.array([-1.80 * DEG_DAY_TO_M_S]),
        mf_p1=np.array([2.0 * v0]), mf_p3=np.array([-2.0 * v0]), mf_p5=np.zeros(1),
        mu_power=np.full(1, 4.0), mu_limit=np.full(1, 0.1), lat_limit=np.zeros(1),
    )


def observed_map(t: np.ndarray, p: np.ndarray, time_hr: float, seed: int, noise_g: float = 2.0) -> np.ndarray:
    """(3, ntm, npm1) assimilation map [data, weight, mu] at model time time_hr."""
    rng = np.random.Generator(np.random.PCG64(seed + int(time_hr * 16)))
    data = 10.0 * np.cos(t)[:, None] * np.ones((1, len(p))) + rng.normal(0.0, noise_g, (len(t), len(p)))
    lon0 = np.deg2rad((-CARRINGTON_DEG_PER_HOUR * time_hr) % 360.0)
    mu = np.sin(t)[:, None] * np.cos(p[None, :] - lon0)
    weight = np.where(mu > 0.1, mu ** 4, 0.0)
    return np.stack([data, weight, mu])


RSUN_MM = 696.0  # solar radius, Mm


def supergranular_psi(t: np.ndarray, p: np.ndarray, seed: int, day: int = 0, corr_mm: float = 30.0,
                      window: float = 5.0) -> np.ndarray:
    """The random potential of supergranular_flow at the nodes t x p,
    (ntm, npm1): psi = sum_n a_n exp(-d_n^2 / (2 L^2)), d_n the chord distance
    to centre n on the unit sphere, L = corr_mm / 696 Mm, a_n = +-1, centres
    uniform on the sphere with one per L^2 of area, each cell evaluated within
    `window` L of its centre."""
    rng = np.random.Generator(np.random.PCG64([seed, day]))
    L = corr_mm / RSUN_MM
    n = int(4.0 * np.pi / (L * L))
    z = rng.uniform(-1.0, 1.0, n)
    lon = rng.uniform(0.0, 2.0 * np.pi, n)
    amp = rng.choice([-1.0, 1.0], n)
    R = window * L
    psi = np.zeros((len(t), len(p)))
    for c_z, c_lon, a in zip(z, lon, amp):
        c_t = np.arccos(c_z)
        r0, r1 = np.searchsorted(t, c_t - R), np.searchsorted(t, c_t + R)
        if r1 <= r0:
            continue
        st, ct = np.sin(t[r0:r1]), np.cos(t[r0:r1])
        smin = min(np.sin(c_t - R), np.sin(c_t + R)) if R < c_t < np.pi - R else 0.0
        if smin > R:
            dphi = np.abs(((p - c_lon + np.pi) % (2.0 * np.pi)) - np.pi)
            cols = np.nonzero(dphi <= R / smin)[0]
        else:
            cols = np.arange(len(p))
        s_c = np.sqrt(max(1.0 - c_z * c_z, 0.0))
        dot = st[:, None] * s_c * np.cos(p[cols][None, :] - c_lon) + ct[:, None] * c_z
        psi[r0:r1, cols] += a * np.exp(-(2.0 - 2.0 * dot) / (2.0 * L * L))
    return psi


def supergranular_flow(t: np.ndarray, p: np.ndarray, seed: int, day: int = 0, corr_mm: float = 30.0,
                       rms_m_s: float = 300.0, coarse=None):
    """Random divergent flow v = grad(psi) for the day `day` (psi of
    supergranular_psi), scaled to rms_m_s: returns (vt, vp) in m/s in the
    flow-file layouts, vt (nt, npm1) on theta faces x phi nodes and vp
    (ntm, np) on theta nodes x phi faces (C order, phi fastest: the files'
    Fortran (npm1, nt) and (np, ntm)).  vt(j) = (psi(t_j) - psi(t_{j-1})) / (t_j - t_{j-1}) on the
    interior faces (zero on the faces beyond the poles), vp(k) = (psi(p_k) -
    psi(p_{k-1})) / (sin t (p_k - p_{k-1})) (zero on the pole rows), phi
    periodic.  coarse = (ntc, npc): evaluate psi on a uniform ntc x npc grid
    and interpolate it (cubic) to the nodes, for large grids."""
    if coarse is None:
        psi = supergranular_psi(t, p, seed, day, corr_mm)
    else:
        from scipy.interpolate import RegularGridInterpolator
        tc = np.linspace(0.0, np.pi, coarse[0])
        pc = np.linspace(0.0, 2.0 * np.pi, coarse[1])
        pc_ext = np.concatenate([pc[-4:-1] - 2.0 * np.pi, pc, pc[1:4] + 2.0 * np.pi])
        psic = supergranular_psi(tc, pc, seed, day, corr_mm)
        psic = np.concatenate([psic[:, -4:-1], psic, psic[:, 1:4]], axis=1)
        f = RegularGridInterpolator((tc, pc_ext), psic, method="cubic")
        T, P = np.meshgrid(t, p, indexing="ij")
        psi = f(np.stack([T.ravel(), P.ravel()], axis=1)).reshape(len(t), len(p))
    ntm, npm1 = psi.shape
    vt = np.zeros((ntm + 1, npm1))
    vt[1:ntm] = (psi[1:] - psi[:-1]) / (t[1:] - t[:-1])[:, None]
    vp = np.zeros((ntm, npm1 + 1))
    st = np.sin(t)
    dps = (psi[:, 1:] - psi[:, :-1]) / (p[1:] - p[:-1])[None, :]
    inner = slice(1, ntm - 1)
    vp[inner, 1:npm1] = dps[inner] / st[inner, None]
    vp[:, 0] = vp[:, npm1 - 1]
    vp[:, npm1] = vp[:, 1]
    rms = np.sqrt(0.5 * (np.mean(vt ** 2) + np.mean(vp ** 2)))
    scale = (rms_m_s / rms) if rms > 0 else 0.0
    return vt * scale, vp * scale
