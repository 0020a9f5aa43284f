"""ctypes driver for the CPU oracle (test infrastructure only).

The oracle restates HipFT's flux-transport step (src/hipft.f90) in C
(oracle/hipft_oracle.c).  This module parses a ``hipft.in`` namelist the way
``read_input_file``/``process_input_parameters`` do (src/hipft.f90:8307-8614),
fills the oracle's parameter struct and returns the history rows and the
final field.  Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline use it; the hipft_b200 product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
MAX_REALIZATIONS = 2000  # src/hipft.f90:236

# ---------------------------------------------------------------- namelist
# Defaults of the namelist variables this path reads (src/hipft.f90:493-726).
DEFAULTS = dict(
    verbose=0, res_nt=0, res_np=0, n_realizations=1,
    validation_run=0, validation_run_width=0.03,
    initial_map_filename="", initial_map_flux_balance=False,
    initial_map_mult_fac=1.0,
    output_map_idx_start=1, output_map_idx_cadence=0,
    output_map_time_cadence=0.0, output_history_time_cadence=0.0,
    output_single_precision=True, output_map_flux_balance=False, output_map_2d=True,
    output_map_root_filename="hipft_brmap", output_map_directory="output_maps",
    flow_list_filename="", flow_root_dir=".",
    time_start=0.0, time_end=1.0, dt_min=1.0e-15,
    dt_max=float(np.finfo(np.float64).max),
    strang_splitting=False, pole_flux_lat_limit=30.0,
    advance_flow=False, flow_vp_rigid_omega=0.0, flow_rigid_omega=0.0,
    flow_vt_const=0.0, flow_attenuate=False, flow_attenuate_value=500.0,
    flow_dr_model=0, flow_mf_model=0,
    flow_dr_coef_p0_value=46.0, flow_dr_coef_p2_value=-262.0,
    flow_dr_coef_p4_value=-379.0,
    flow_mf_coef_p1_value=22.0, flow_mf_coef_p3_value=11.0,
    flow_mf_coef_p5_value=-28.0,
    use_flow_from_files=False, flow_num_method=4, upwind=1.0, weno_eps=0.0,
    advance_diffusion=False, diffusion_coef_constant=0.0,
    diffusion_coef_filename="", diffusion_coef_grid=False,
    diffusion_coef_factor=7.43162901307967e-09,
    diffusion_num_method=3, diffusion_subcycles=0,
    advance_source=False, source_rfe_model=0, source_rfe_seed=-9999, source_rfe_lifetime=0.3,
    source_rfe_total_unsigned_flux_per_hour=0.0, source_from_file=False, source_filename="",
    assimilate_data=False, assimilate_data_balance_flux=False,
    assimilate_data_mult_fac=1.0, assimilate_data_map_list_filename="",
    assimilate_data_map_root_dir=".", assimilate_data_add=False,
    assimilate_data_custom_from_mu=False,
    assimilate_data_lat_limit=0.0, assimilate_data_mu_power=4.0,
    assimilate_data_mu_limit=0.1,
)

# per-realization vectors: name -> (scalar default name, sentinel test)
RVECS = {
    "diffusion_coef_constants": ("diffusion_coef_constant", lambda v: v < 0.0),
    "flow_attenuate_values": ("flow_attenuate_value", lambda v: v < 0.0),
    "flow_dr_coef_p0_values": ("flow_dr_coef_p0_value", lambda v: v < -100000.0),
    "flow_dr_coef_p2_values": ("flow_dr_coef_p2_value", lambda v: v < -100000.0),
    "flow_dr_coef_p4_values": ("flow_dr_coef_p4_value", lambda v: v < -100000.0),
    "flow_mf_coef_p1_values": ("flow_mf_coef_p1_value", lambda v: v < -100000.0),
    "flow_mf_coef_p3_values": ("flow_mf_coef_p3_value", lambda v: v < -100000.0),
    "flow_mf_coef_p5_values": ("flow_mf_coef_p5_value", lambda v: v < -100000.0),
    "assimilate_data_lat_limits": ("assimilate_data_lat_limit", lambda v: v < 0.0),
    "assimilate_data_mu_powers": ("assimilate_data_mu_power", lambda v: v < 0.0),
    "assimilate_data_mu_limits": ("assimilate_data_mu_limit", lambda v: v < 0.0),
    "source_rfe_total_unsigned_flux_per_hours": ("source_rfe_total_unsigned_flux_per_hour", lambda v: v < 0.0),
}
RVEC_SENTINEL = {k: (-1000000.0 if "coef_p" in k else -1.0) for k in RVECS}


def _value(tok: str):
    t = tok.strip()
    tl = t.lower()
    if tl in (".true.", "t", ".t."):
        return True
    if tl in (".false.", "f", ".f."):
        return False
    if (t.startswith("'") and t.endswith("'")) or (t.startswith('"') and t.endswith('"')):
        return t[1:-1]
    tl = tl.replace("d", "e")
    try:
        if re.fullmatch(r"[+-]?\d+", tl):
            return int(tl)
        return float(tl)
    except ValueError:
        return t


def parse_namelist(text: str) -> dict:
    """Parse the ``&hipft_input_parameters`` group into a dict of raw values."""
    body = []
    inside = False
    for line in text.splitlines():
        s = line.split("!", 1)[0].strip()
        if not s:
            continue
        if s.lower().startswith("&hipft_input_parameters"):
            inside = True
            continue
        if inside and s.startswith("/"):
            break
        if inside:
            body.append(s)
    raw = {}
    for s in body:
        if "=" not in s:
            continue
        k, v = s.split("=", 1)
        k = k.strip().lower()
        vals = [x for x in v.split(",") if x.strip()]
        raw[k] = [_value(x) for x in vals] if len(vals) > 1 or k in RVECS else _value(v)
    return raw


def process_parameters(raw: dict) -> dict:
    """Apply defaults and per-realization fill-in (src/hipft.f90:8542-8579)."""
    p = dict(DEFAULTS)
    for k, v in raw.items():
        if k in RVECS:
            continue
        p[k] = v
    nr = int(p["n_realizations"])
    for name, (scal, is_sentinel) in RVECS.items():
        vec = [RVEC_SENTINEL[name]] * MAX_REALIZATIONS
        given = raw.get(name, [])
        if not isinstance(given, list):
            given = [given]
        for i, v in enumerate(given):
            vec[i] = float(v)
        p[name] = [float(p[scal]) if is_sentinel(x) else x for x in vec[:nr]]
    if p["initial_map_filename"] and p["res_nt"] * p["res_np"] > 0:
        p["res_nt"] = p["res_np"] = 0
    return p


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("verbose", ctypes.c_int), ("res_nt", ctypes.c_int), ("res_np", ctypes.c_int),
        ("n_realizations", ctypes.c_int), ("validation_run", ctypes.c_int),
        ("validation_run_width", ctypes.c_double),
        ("initial_map_flux_balance", ctypes.c_int), ("initial_map_mult_fac", ctypes.c_double),
        ("output_map_time_cadence", ctypes.c_double),
        ("output_map_idx_cadence", ctypes.c_long), ("output_map_idx_start", ctypes.c_long),
        ("output_history_time_cadence", ctypes.c_double),
        ("time_start", ctypes.c_double), ("time_end", ctypes.c_double),
        ("dt_min", ctypes.c_double), ("dt_max", ctypes.c_double),
        ("strang_splitting", ctypes.c_int), ("pole_flux_lat_limit", ctypes.c_double),
        ("advance_flow", ctypes.c_int), ("flow_vp_rigid_omega", ctypes.c_double),
        ("flow_rigid_omega", ctypes.c_double), ("flow_vt_const", ctypes.c_double),
        ("flow_attenuate", ctypes.c_int), ("flow_dr_model", ctypes.c_int),
        ("flow_mf_model", ctypes.c_int), ("flow_num_method", ctypes.c_int),
        ("upwind", ctypes.c_double), ("weno_eps", ctypes.c_double),
        ("advance_diffusion", ctypes.c_int), ("diffusion_coef_factor", ctypes.c_double),
        ("diffusion_coef_grid", ctypes.c_int), ("diffusion_num_method", ctypes.c_int),
        ("diffusion_subcycles", ctypes.c_int),
        ("assimilate_data", ctypes.c_int), ("assimilate_data_balance_flux", ctypes.c_int),
        ("assimilate_data_add", ctypes.c_int), ("assimilate_data_custom_from_mu", ctypes.c_int),
        ("assimilate_data_mult_fac", ctypes.c_double),
    ] + [(name, ctypes.POINTER(ctypes.c_double)) for name in (
        "diffusion_coef_constants", "flow_attenuate_values",
        "flow_dr_coef_p0_values", "flow_dr_coef_p2_values", "flow_dr_coef_p4_values",
        "flow_mf_coef_p1_values", "flow_mf_coef_p3_values", "flow_mf_coef_p5_values",
        "assimilate_data_lat_limits", "assimilate_data_mu_powers", "assimilate_data_mu_limits")] + [
        ("output_map_flux_balance", ctypes.c_int),
        ("use_flow_from_files", ctypes.c_int), ("n_flows", ctypes.c_int),
        ("flow_jd", ctypes.POINTER(ctypes.c_double)), ("flow_vt", ctypes.POINTER(ctypes.c_double)),
        ("flow_vp", ctypes.POINTER(ctypes.c_double)),
        ("advance_source", ctypes.c_int), ("source_rfe_model", ctypes.c_int), ("source_rfe_seed", ctypes.c_long),
        ("source_rfe_lifetime", ctypes.c_double),
        ("source_rfe_total_unsigned_flux_per_hours", ctypes.POINTER(ctypes.c_double)),
        ("source_from_file", ctypes.c_int), ("source_nfp", ctypes.c_int), ("source_nft", ctypes.c_int),
        ("source_data", ctypes.POINTER(ctypes.c_double)), ("source_pf", ctypes.POINTER(ctypes.c_double)),
        ("source_tf", ctypes.POINTER(ctypes.c_double))]
# set by run(flows=..., source=...)
FLOW_FILE_FIELDS = ("n_flows", "flow_jd", "flow_vt", "flow_vp", "source_nfp", "source_nft", "source_data",
                    "source_pf", "source_tf")


class OrcHist(ctypes.Structure):
    _fields_ = [("cap", ctypes.c_long), ("nrows", ctypes.c_long),
                ("sol", ctypes.POINTER(ctypes.c_double)),
                ("num", ctypes.POINTER(ctypes.c_double)),
                ("map_cap", ctypes.c_long), ("n_maps", ctypes.c_long),
                ("map_idx", ctypes.POINTER(ctypes.c_long)),
                ("map_time", ctypes.POINTER(ctypes.c_double)),
                ("maps", ctypes.POINTER(ctypes.c_double)),
                ("map_initial", ctypes.POINTER(ctypes.c_double)),
                ("map_final", ctypes.POINTER(ctypes.c_double))]


_lib = None
_fast = None
FAST_PATH = os.path.join(HERE, "liboracle_fast.so")
FAST_FLAGS = "-O3 -march=x86-64-v3 -fopenmp (contraction allowed)"


def build():
    """Compile liboracle.so (parity build) and liboracle_fast.so (timing
    build) from hipft_oracle.c (gcc; no GPU needed)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def _load(path, target):
    src = os.path.join(HERE, "hipft_oracle.c")
    if not os.path.exists(path) or (os.path.exists(src) and os.path.getmtime(src) > os.path.getmtime(path)):
        subprocess.run(["make", "-s", "-C", HERE, target], check=True)
    L = ctypes.CDLL(path)
    L.orc_run.restype = ctypes.c_int
    L.orc_run.argtypes = [
        ctypes.POINTER(OrcParams), ctypes.c_int, ctypes.c_int,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.POINTER(OrcHist), ctypes.c_long, ctypes.c_void_p]
    return L


def lib():
    """The parity build (-O2 -ffp-contract=off), the oracle of every test."""
    global _lib
    if _lib is None:
        _lib = _load(LIB_PATH, "liboracle.so")
    return _lib


def lib_fast():
    """The timing build of the same source, for the CPU baseline only."""
    global _fast
    if _fast is None:
        _fast = _load(FAST_PATH, "liboracle_fast.so")
    return _fast


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _params_struct(p: dict):
    keep = []
    c = OrcParams()
    for name, typ in OrcParams._fields_:
        if name in FLOW_FILE_FIELDS:
            continue
        if name in RVECS:
            arr = np.ascontiguousarray(np.asarray(p[name], dtype=np.float64))
            keep.append(arr)
            setattr(c, name, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        elif typ in (ctypes.c_int, ctypes.c_long):
            setattr(c, name, int(p[name]))
        else:
            setattr(c, name, float(p[name]))
    return c, keep


def run(p: dict, map_pt=None, s1=None, s2=None, da_times=None, da_maps=None,
        max_steps: int = 0, hist_cap: int = 0, want_field: bool = True, map_cap: int = 0, flows=None,
        source=None, fast: bool = False):
    """Run the oracle on processed parameters ``p``.

    map_pt: (nr, ntm, npm1) C-order array (i.e. Fortran (npm1,ntm,nr)), or None.
    Returns dict(sol=(rows,nr,16), num=(rows,nr,8), f=(nr,npm,ntm) or None).
    With map_cap > 0 also maps=(n,nr,npm,ntm), map_idx, map_time (the numbered
    map outputs, at most map_cap) and map_initial, map_final (nr,npm,ntm): the
    fields write_map writes, flux-balanced when output_map_flux_balance.
    flows (use_flow_from_files): dict(jd=(n,), vt=(n, nt, npm1), vp=(n, ntm, np)),
    the flow list's Julian days and the files' data in C order, m/s.
    source (source_from_file): dict(data=(nft, nfp) C order, pf=(nfp,), tf=(nft,)).
    fast: run the timing build (lib_fast) instead of the parity build.
    """
    L = lib_fast() if fast else lib()
    nr = int(p["n_realizations"])
    c, keep = _params_struct(p)
    if flows is not None:
        fa = [np.ascontiguousarray(flows[k], dtype=np.float64) for k in ("jd", "vt", "vp")]
        keep.extend(fa)
        c.n_flows = len(fa[0])
        c.flow_jd, c.flow_vt, c.flow_vp = (a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in fa)
    if source is not None:
        sa = [np.ascontiguousarray(source[k], dtype=np.float64) for k in ("data", "pf", "tf")]
        keep.extend(sa)
        c.source_nft, c.source_nfp = sa[0].shape
        c.source_data, c.source_pf, c.source_tf = (a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in sa)
    if map_pt is not None:
        map_pt = np.ascontiguousarray(map_pt, dtype=np.float64)
        n2, n1 = map_pt.shape[-2], map_pt.shape[-1]
        s1 = np.ascontiguousarray(s1, dtype=np.float64)
        s2 = np.ascontiguousarray(s2, dtype=np.float64)
    else:
        n1, n2 = int(p["res_np"]), int(p["res_nt"])
    ntm, npm = n2, n1 + 1
    if hist_cap <= 0:
        dtm = max(float(p["dt_max"]), 1e-300)
        est = (float(p["time_end"]) - float(p["time_start"])) / dtm if dtm < 1e300 else 1
        hist_cap = int(min(est * 64, 4_000_000 // max(nr, 1))) + 4096
    h = OrcHist()
    sol = np.zeros((hist_cap, nr, 16))
    num = np.zeros((hist_cap, nr, 8))
    h.cap = hist_cap
    h.sol = sol.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    h.num = num.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    maps = None
    if map_cap > 0:
        maps = np.zeros((map_cap, nr, npm, ntm))
        map_idx = np.zeros(map_cap, dtype=np.int64)
        map_time = np.zeros(map_cap)
        map_initial = np.zeros((nr, npm, ntm))
        map_final = np.zeros((nr, npm, ntm))
        dptr = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        h.map_cap = map_cap
        h.map_idx = map_idx.ctypes.data_as(ctypes.POINTER(ctypes.c_long))
        h.map_time, h.maps = dptr(map_time), dptr(maps)
        h.map_initial, h.map_final = dptr(map_initial), dptr(map_final)
    f = np.zeros((nr, npm, ntm)) if want_field else None
    n_da = 0
    if da_times is not None:
        da_times = np.ascontiguousarray(da_times, dtype=np.float64)
        da_maps = np.ascontiguousarray(da_maps, dtype=np.float64)
        n_da = len(da_times)
    tinfo = np.zeros(4)
    rc = L.orc_run(ctypes.byref(c), n1 if map_pt is not None else 0,
                   n2 if map_pt is not None else 0, _ptr(s1), _ptr(s2), _ptr(map_pt),
                   n_da, _ptr(da_times), _ptr(da_maps), _ptr(f), ctypes.byref(h),
                   int(max_steps), _ptr(tinfo))
    if rc != 0:
        raise RuntimeError(f"oracle failed with code {rc}")
    n = min(h.nrows, hist_cap)
    out = dict(sol=sol[:n].copy(), num=num[:n].copy(), f=f, nsteps=int(tinfo[0]),
               time=float(tinfo[1]), cell_updates=float(tinfo[2]))
    if maps is not None:
        m = int(h.n_maps)
        out.update(maps=maps[:m], map_idx=map_idx[:m], map_time=map_time[:m], map_initial=map_initial,
                   map_final=map_final)
    return out


def da_blend(p: dict, t, ph, f, map3):
    """One assimilation blend of map3 (3, ntm, npm1) into f (nr, npm, ntm) (in place)."""
    L = lib()
    L.orc_da_blend.restype = ctypes.c_int
    L.orc_da_blend.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    c, keep = _params_struct(p)
    t = np.ascontiguousarray(t, dtype=np.float64)
    ph = np.ascontiguousarray(ph, dtype=np.float64)
    m = np.ascontiguousarray(map3, dtype=np.float64)
    assert f.flags["C_CONTIGUOUS"] and f.dtype == np.float64
    rc = L.orc_da_blend(ctypes.byref(c), len(t), len(ph), _ptr(t), _ptr(ph), _ptr(f), _ptr(m))
    if rc:
        raise RuntimeError("oracle da_blend failed")
    return f


def get_flux(t, ph, f):
    """get_flux of every realization of f (nr, npm, ntm) on the mesh of the
    scales t (ntm) and ph (npm1); returns (flux_p, flux_m), nr values each."""
    L = lib()
    L.orc_get_flux.restype = ctypes.c_int
    L.orc_get_flux.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 5
    t = np.ascontiguousarray(t, dtype=np.float64)
    ph = np.ascontiguousarray(ph, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    nr = f.shape[0]
    assert f.shape[1:] == (len(ph) + 1, len(t))
    fp, fm = np.zeros(nr), np.zeros(nr)
    if L.orc_get_flux(len(t), len(ph), nr, _ptr(t), _ptr(ph), _ptr(f), _ptr(fp), _ptr(fm)):
        raise RuntimeError("oracle get_flux failed")
    return fp, fm


def read_history(path: str) -> np.ndarray:
    """Read a hipft_history_{sol,num}_rNNNNNN.out file into an array."""
    rows = []
    with open(path) as fh:
        next(fh)
        for line in fh:
            if line.strip():
                rows.append([float(x.replace("D", "E")) for x in line.split()])
    return np.array(rows)
