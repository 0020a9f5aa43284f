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
