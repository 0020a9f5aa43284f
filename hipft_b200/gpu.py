"""ctypes binding of the hipft_b200 C ABI (include/hipft_gpu.h).

Each method wraps one entry point, which in turn replaces one routine of the
reference solver (src/hipft.f90); the method docstrings name it.  Arrays use
NumPy's C order, so a field of Fortran shape f(ntm, npm, nr) is the array
``f[nr, npm, ntm]`` here.  There is no CPU fallback: if the CUDA library is
missing the import of :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Callable, Optional

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libhipft_gpu.so")

HIPFT_OK, HIPFT_EINVAL, HIPFT_ECUDA, HIPFT_ETIMEOUT, HIPFT_ENAN, HIPFT_ESTATE, HIPFT_EIO, HIPFT_ENOMEM, HIPFT_ECOMM = \
    range(9)
STATUS = {0: "OK", 1: "EINVAL", 2: "ECUDA", 3: "ETIMEOUT", 4: "ENAN", 5: "ESTATE", 6: "EIO", 7: "ENOMEM", 8: "ECOMM"}

DPTR = ctypes.POINTER(ctypes.c_double)


class HipftError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str = ""):
        self.code = code
        super().__init__(f"{where}: {STATUS.get(code, code)} {msg}".strip())


class Grid(ctypes.Structure):
    _fields_ = [("ntm", ctypes.c_int), ("npm1", ctypes.c_int), ("nr", ctypes.c_int), ("device", ctypes.c_int),
                ("t", DPTR), ("p", DPTR)]


class Params(ctypes.Structure):
    _fields_ = [("advance_flow", ctypes.c_int), ("flow_num_method", ctypes.c_int), ("upwind", ctypes.c_double),
                ("weno_eps", ctypes.c_double), ("strang_splitting", ctypes.c_int),
                ("advance_diffusion", ctypes.c_int), ("diffusion_num_method", ctypes.c_int),
                ("diffusion_subcycles", ctypes.c_int), ("diffusion_coef_grid", ctypes.c_int),
                ("diffusion_coef_factor", ctypes.c_double), ("diffusion_coef_constants", DPTR),
                ("pole_flux_lat_limit", ctypes.c_double), ("verbose", ctypes.c_int),
                ("advance_source", ctypes.c_int)]


ALLREDUCE_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double))
GATHER_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int64,
                             ctypes.POINTER(ctypes.c_double))


class Shard(ctypes.Structure):
    _fields_ = [("rank", ctypes.c_int), ("nranks", ctypes.c_int), ("allreduce", ALLREDUCE_CB),
                ("gather", GATHER_CB), ("user", ctypes.c_void_p)]


class FlowDef(ctypes.Structure):
    _fields_ = [("flow_dr_model", ctypes.c_int), ("flow_mf_model", ctypes.c_int),
                ("dr_p0", DPTR), ("dr_p2", DPTR), ("dr_p4", DPTR), ("mf_p1", DPTR), ("mf_p3", DPTR),
                ("mf_p5", DPTR), ("flow_vp_rigid_omega", ctypes.c_double), ("flow_vt_const", ctypes.c_double),
                ("flow_rigid_omega", ctypes.c_double), ("flow_attenuate", ctypes.c_int),
                ("flow_attenuate_values", DPTR)]


class DAOpts(ctypes.Structure):
    _fields_ = [("add", ctypes.c_int), ("custom_from_mu", ctypes.c_int), ("balance_flux", ctypes.c_int),
                ("mult_fac", ctypes.c_double), ("mu_power", DPTR), ("mu_limit", DPTR), ("lat_limit", DPTR)]


class DiffusionInfo(ctypes.Structure):
    _fields_ = [("dtime_diffusion_euler", ctypes.c_double), ("sts_s", ctypes.c_int64),
                ("subcycles", ctypes.c_int64), ("total_stages", ctypes.c_int64)]


class Info(ctypes.Structure):
    _fields_ = [("ntm", ctypes.c_int), ("npm", ctypes.c_int), ("nr", ctypes.c_int), ("ldt", ctypes.c_int),
                ("dtime_diffusion_euler", ctypes.c_double), ("sts_s", ctypes.c_int64),
                ("kernel_launches", ctypes.c_int64), ("cell_stage_updates", ctypes.c_int64),
                ("device_bytes", ctypes.c_size_t), ("rkg2_stages", ctypes.c_int64),
                ("rkg2_cell_stages", ctypes.c_int64)]


CYCLE_CB = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                            ctypes.c_int64)

# (name, restype, argtypes) of every exported entry point
_H = ctypes.c_void_p
SIGNATURES = [
    ("hipft_gpu_create", ctypes.c_int, [ctypes.POINTER(Grid), ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_void_p)]),
    ("hipft_gpu_destroy", ctypes.c_int, [_H]),
    ("hipft_gpu_last_error", ctypes.c_int, [_H, ctypes.c_char_p, ctypes.c_size_t]),
    ("hipft_gpu_version", ctypes.c_char_p, []),
    ("hipft_gpu_set_field", ctypes.c_int, [_H, DPTR]),
    ("hipft_gpu_get_field", ctypes.c_int, [_H, DPTR]),
    ("hipft_gpu_load_initial_map", ctypes.c_int, [_H, DPTR, ctypes.c_int, ctypes.c_double]),
    ("hipft_gpu_set_flow", ctypes.c_int, [_H, ctypes.POINTER(FlowDef)]),
    ("hipft_gpu_update_flow", ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int)]),
    ("hipft_gpu_flow_dtmax", ctypes.c_int, [_H, DPTR]),
    ("hipft_gpu_advection_step", ctypes.c_int, [_H, ctypes.c_double]),
    ("hipft_gpu_diffusion_step", ctypes.c_int, [_H, ctypes.c_double, CYCLE_CB, ctypes.c_void_p,
                                                ctypes.POINTER(DiffusionInfo)]),
    ("hipft_gpu_flux_transport_step", ctypes.c_int, [_H, ctypes.c_double, CYCLE_CB, ctypes.c_void_p,
                                                     ctypes.POINTER(DiffusionInfo)]),
    ("hipft_gpu_assimilate", ctypes.c_int, [_H, DPTR, ctypes.POINTER(DAOpts)]),
    ("hipft_gpu_set_validation", ctypes.c_int, [_H, ctypes.c_int, DPTR, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_double]),
    ("hipft_gpu_analysis", ctypes.c_int, [_H, ctypes.c_double, DPTR]),
    ("hipft_gpu_get_flux", ctypes.c_int, [_H, DPTR, DPTR]),
    ("hipft_gpu_balance_flux", ctypes.c_int, [_H]),
    ("hipft_gpu_info", ctypes.c_int, [_H, ctypes.POINTER(Info)]),
    ("hipft_gpu_set_profiling", ctypes.c_int, [_H, ctypes.c_int]),
    ("hipft_gpu_kernel_time", ctypes.c_int, [_H, ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
                                             ctypes.POINTER(ctypes.c_double)]),
    ("hipft_gpu_set_stream", ctypes.c_int, [_H, ctypes.c_void_p]),
    ("hipft_gpu_synchronize", ctypes.c_int, [_H]),
    ("hipft_run", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]),
    ("hipft_run_field", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, DPTR, ctypes.c_size_t]),
    ("hipft_get_flux_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              DPTR, DPTR, DPTR, DPTR, ctypes.c_void_p, ctypes.c_char_p,
                                              ctypes.c_size_t]),
    ("hipft_h5_read", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64),
                                     DPTR, DPTR, DPTR, DPTR]),
    ("hipft_gpu_set_flow_from_files", ctypes.c_int, [_H, DPTR, DPTR, ctypes.c_int]),
    ("hipft_gpu_set_allreduce", ctypes.c_int, [_H, ALLREDUCE_CB, ctypes.c_void_p]),
    ("hipft_gpu_field_device_ptr", ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int)]),
    ("hipft_gpu_check_bounded_wait", ctypes.c_int, [_H, ctypes.c_uint]),
    ("hipft_adj_step", ctypes.c_int, [_H, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]),
    ("hipft_gpu_set_field_device", ctypes.c_int, [_H, ctypes.c_void_p]),
    ("hipft_adj_tape_fields", ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int64)]),
    ("hipft_adj_record", ctypes.c_int, [_H, ctypes.c_double]),
    ("hipft_adj_reverse", ctypes.c_int, [_H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("hipft_adj_recorded", ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    ("hipft_adj_clear", ctypes.c_int, [_H]),
    ("hipft_run_shard", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(Shard), DPTR,
                                       ctypes.c_size_t]),
    ("hipft_gpu_set_source_file", ctypes.c_int, [_H, DPTR]),
    ("hipft_gpu_set_rfe_frame", ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, DPTR, DPTR]),
    ("hipft_gpu_update_source", ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_double]),
    ("hipft_gpu_source_step", ctypes.c_int, [_H, ctypes.c_double]),
    ("hipft_h5_write", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int64), DPTR, DPTR,
                                      DPTR, DPTR, ctypes.c_int]),
    ("hipft_adj_set_tape_limit", ctypes.c_int, [_H, ctypes.c_int64, ctypes.c_int64]),
    ("hipft_adj_release", ctypes.c_int, [_H]),
    ("hipft_adj_assimilate", ctypes.c_int, [_H, DPTR, ctypes.POINTER(DAOpts), ctypes.c_void_p]),
    ("hipft_adj_assimilate_at", ctypes.c_int, [_H, DPTR, ctypes.POINTER(DAOpts), ctypes.c_void_p,
                                               ctypes.c_void_p]),
    ("hipft_gpu_describe", ctypes.c_int, [_H, ctypes.c_char_p, ctypes.c_size_t]),
    ("hipft_gpu_set_ragged", ctypes.c_int, [_H, ctypes.c_int]),
    ("hipft_gpu_set_graph", ctypes.c_int, [_H, ctypes.c_int]),
    ("hipft_gpu_flow_dtmax_each", ctypes.c_int, [_H, DPTR]),
    ("hipft_gpu_ragged_schedule", ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                                 ctypes.POINTER(ctypes.c_int64), DPTR]),
]

_lib = None


def lib() -> ctypes.CDLL:
    """Load libhipft_gpu.so (built by hipft_b200.build); raises if absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -m hipft_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(DPTR)


def _vec(x, n: int) -> np.ndarray:
    a = np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=np.float64), (n,)))
    return a


def h5_read(path: str):
    """Read a HipFT HDF5 map: returns (data, [scales]) with data in C order
    (i.e. Fortran (n1, n2[, n3]) becomes shape (n3, n2, n1))."""
    L = lib()
    nd = ctypes.c_int(0)
    dims = (ctypes.c_int64 * 3)()
    rc = L.hipft_h5_read(path.encode(), ctypes.byref(nd), dims, None, None, None, None)
    if rc:
        raise HipftError(rc, "hipft_h5_read", path)
    n = [int(dims[i]) for i in range(3)]
    data = np.zeros(n[0] * n[1] * n[2])
    sc = [np.zeros(n[i]) for i in range(3)]
    rc = L.hipft_h5_read(path.encode(), ctypes.byref(nd), dims, _p(data), _p(sc[0]),
                         _p(sc[1]) if nd.value > 1 else None, _p(sc[2]) if nd.value > 2 else None)
    if rc:
        raise HipftError(rc, "hipft_h5_read", path)
    shape = tuple(reversed(n[: nd.value]))
    return data.reshape(shape), sc[: nd.value]


def h5_write(path: str, data: np.ndarray, scales, single_precision: bool = True) -> None:
    """Write a HipFT HDF5 map as the reference's wrh5 does.  ``data`` is in
    C order (shape (n3, n2, n1) for Fortran (n1, n2, n3)); ``scales`` lists
    the Fortran-order scales (n1 values first)."""
    L = lib()
    a = np.ascontiguousarray(data, dtype=np.float64)
    nd = a.ndim
    if not 1 <= nd <= 3 or len(scales) != nd:
        raise ValueError("data must have 1-3 dimensions and one scale per dimension")
    fdims = list(reversed(a.shape))
    sc = [np.ascontiguousarray(x, dtype=np.float64) for x in scales]
    for x, n in zip(sc, fdims):
        if x.shape != (n,):
            raise ValueError("scale length does not match its dimension")
    dims = (ctypes.c_int64 * 3)(*(fdims + [1] * (3 - nd)))
    ptr = [_p(x) for x in sc] + [None] * (3 - nd)
    rc = L.hipft_h5_write(path.encode(), nd, dims, _p(a), ptr[0], ptr[1], ptr[2], 1 if single_precision else 0)
    if rc:
        raise HipftError(rc, "hipft_h5_write", path)


def run(namelist: str, run_dir: str, device: int = 0) -> int:
    """``program HIPFT`` (src/hipft.f90:869-968) through hipft_run."""
    rc = lib().hipft_run(namelist.encode(), run_dir.encode(), int(device))
    if rc:
        raise HipftError(rc, "hipft_run", namelist)
    return rc


def run_field(namelist: str, run_dir: str, shape, device: int = 0) -> np.ndarray:
    """hipft_run, returning the final field as an (nr, npm, ntm) array."""
    f = np.zeros(shape)
    rc = lib().hipft_run_field(namelist.encode(), run_dir.encode(), int(device), _p(f), f.size)
    if rc:
        raise HipftError(rc, "hipft_run_field", namelist)
    return f


class HipftGPU:
    """Device state for ``nr`` realizations on one GPU (one handle)."""

    def __init__(self, t: np.ndarray, p: np.ndarray, nr: int, *, device: int = 0, advance_flow: bool = False,
                 flow_num_method: int = 4, upwind: float = 1.0, weno_eps: float = 0.0,
                 strang_splitting: bool = False, advance_diffusion: bool = False, diffusion_num_method: int = 3,
                 diffusion_subcycles: int = 0, diffusion_coef_grid: bool = False,
                 diffusion_coef_factor: float = 7.43162901307967e-09, diffusion_coef_constants=None,
                 pole_flux_lat_limit: float = 30.0, verbose: int = 0):
        self.L = lib()
        self.t = np.ascontiguousarray(t, dtype=np.float64)
        self.p = np.ascontiguousarray(p, dtype=np.float64)
        self.nr = int(nr)
        self.ntm, self.npm1 = len(self.t), len(self.p)
        self.npm = self.npm1 + 1
        self._dc = _vec(diffusion_coef_constants if diffusion_coef_constants is not None else 0.0, self.nr)
        g = Grid(self.ntm, self.npm1, self.nr, int(device), _p(self.t), _p(self.p))
        prm = Params(int(advance_flow), int(flow_num_method), float(upwind), float(weno_eps), int(strang_splitting),
                     int(advance_diffusion), int(diffusion_num_method), int(diffusion_subcycles),
                     int(diffusion_coef_grid), float(diffusion_coef_factor), _p(self._dc),
                     float(pole_flux_lat_limit), int(verbose))
        self.file_flow = False  # a 2-D flow from files is set
        self.h = ctypes.c_void_p()
        rc = self.L.hipft_gpu_create(ctypes.byref(g), ctypes.byref(prm), ctypes.byref(self.h))
        if rc:
            raise HipftError(rc, "hipft_gpu_create")
        self._keep = []

    # -- helpers
    def _ck(self, rc: int, where: str):
        if rc:
            buf = ctypes.create_string_buffer(512)
            self.L.hipft_gpu_last_error(self.h, buf, 512)
            raise HipftError(rc, where, buf.value.decode(errors="replace"))

    def close(self):
        if self.h:
            self.L.hipft_gpu_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- field
    def set_field(self, f: np.ndarray):
        """!$omp target enter data map(to:f) (src/hipft.f90:2159); f is (nr, npm, ntm)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        assert f.shape == (self.nr, self.npm, self.ntm), f.shape
        self._ck(self.L.hipft_gpu_set_field(self.h, _p(f)), "set_field")

    def get_field(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """!$omp target update from(f) (src/hipft.f90:2844)."""
        if out is None:
            out = np.empty((self.nr, self.npm, self.ntm))
        self._ck(self.L.hipft_gpu_get_field(self.h, _p(out)), "get_field")
        return out

    def field_tensor(self):
        """Zero-copy torch view (nr, npm, ldt) of the current field on the GPU
        (theta padded to ldt); valid until the field next changes."""
        import torch
        ptr, ldt = ctypes.c_void_p(), ctypes.c_int()
        self._ck(self.L.hipft_gpu_field_device_ptr(self.h, ctypes.byref(ptr), ctypes.byref(ldt)), "field_device_ptr")

        class _View:
            __cuda_array_interface__ = {"shape": (self.nr, self.npm, ldt.value), "typestr": "<f8",
                                        "data": (ptr.value, False), "version": 2}
        return torch.as_tensor(_View(), device="cuda")

    def load_initial_map(self, map_pt: np.ndarray, flux_balance: bool = False, mult_fac: float = 1.0):
        """load_initial_condition's transpose/seam/pole steps (src/hipft.f90:2116-2172); map is (nr, ntm, npm1)."""
        m = np.ascontiguousarray(np.broadcast_to(map_pt, (self.nr, self.ntm, self.npm1)), dtype=np.float64)
        self._ck(self.L.hipft_gpu_load_initial_map(self.h, _p(m), int(flux_balance), float(mult_fac)),
                 "load_initial_map")

    # -- flows
    def set_flow(self, *, dr_model: int = 0, mf_model: int = 0, dr_p0=0.0, dr_p2=0.0, dr_p4=0.0, mf_p1=0.0,
                 mf_p3=0.0, mf_p5=0.0, vp_rigid_omega: float = 0.0, vt_const: float = 0.0,
                 rigid_omega: float = 0.0, attenuate: bool = False, attenuate_values=500.0):
        v = [_vec(x, self.nr) for x in (dr_p0, dr_p2, dr_p4, mf_p1, mf_p3, mf_p5, attenuate_values)]
        self._keep = v
        d = FlowDef(int(dr_model), int(mf_model), *[_p(a) for a in v[:6]], float(vp_rigid_omega), float(vt_const),
                    float(rigid_omega), int(attenuate), _p(v[6]))
        self._ck(self.L.hipft_gpu_set_flow(self.h, ctypes.byref(d)), "set_flow")

    def set_flow_from_files(self, vt: np.ndarray, vp: np.ndarray, at_load: bool = True):
        """The 2-D flow of HipFT's flow files (add_flow_from_files / load_flow_from_files,
        src/hipft.f90:3525-3800), shared by all realizations, in m/s: vt (nt, npm1) and
        vp (ntm, np) in C order (the files' Fortran (npm1, nt) and (np, ntm))."""
        a = np.ascontiguousarray(vt, dtype=np.float64)
        b = np.ascontiguousarray(vp, dtype=np.float64)
        assert a.shape == (self.ntm + 1, self.npm1) and b.shape == (self.ntm, self.npm1 + 1), (a.shape, b.shape)
        self._ck(self.L.hipft_gpu_set_flow_from_files(self.h, _p(a), _p(b), int(at_load)), "set_flow_from_files")
        self.file_flow = True

    def update_flow(self) -> bool:
        """update_flow (src/hipft.f90:3371); True when the flow changed."""
        u = ctypes.c_int(0)
        self._ck(self.L.hipft_gpu_update_flow(self.h, ctypes.byref(u)), "update_flow")
        return bool(u.value)

    def flow_dtmax(self) -> float:
        """get_flow_dtmax (src/hipft.f90:7287)."""
        d = ctypes.c_double(0.0)
        self._ck(self.L.hipft_gpu_flow_dtmax(self.h, ctypes.byref(d)), "flow_dtmax")
        return d.value

    def flow_dtmax_each(self) -> np.ndarray:
        """get_flow_dtmax (src/hipft.f90:7287) of each realization alone."""
        d = np.zeros(self.nr)
        self._ck(self.L.hipft_gpu_flow_dtmax_each(self.h, _p(d)), "flow_dtmax_each")
        return d

    # -- ragged batches
    def set_ragged(self, on: bool = True):
        """Ragged batching: each realization keeps the schedule it would have
        alone (Euler limit, PTL subcycles, stage counts, advection substeps)."""
        self._ck(self.L.hipft_gpu_set_ragged(self.h, int(on)), "set_ragged")

    def set_graph(self, on: bool = True):
        """Run every flux_transport_step as one launch of a captured CUDA graph
        whose loops (subcycles, stage pairs, advection substeps) are sized on
        the device; same field, bit for bit, as the host-driven step."""
        self._ck(self.L.hipft_gpu_set_graph(self.h, int(on)), "set_graph")

    def ragged_schedule(self) -> dict:
        """Per-realization schedule of the last ragged step."""
        I64 = ctypes.POINTER(ctypes.c_int64)
        s, c, a = (np.zeros(self.nr, dtype=np.int64) for _ in range(3))
        e = np.zeros(self.nr)
        self._ck(self.L.hipft_gpu_ragged_schedule(self.h, s.ctypes.data_as(I64), c.ctypes.data_as(I64),
                                                  a.ctypes.data_as(I64), _p(e)), "ragged_schedule")
        return dict(sts_s=s, subcycles=c, adv_substeps=a, dt_euler=e)

    # -- steps
    def advection_step(self, dt: float):
        """advection_step (src/hipft.f90:4509)."""
        self._ck(self.L.hipft_gpu_advection_step(self.h, float(dt)), "advection_step")

    def diffusion_step(self, dt: float, cb: Optional[Callable] = None) -> DiffusionInfo:
        """diffusion_step (src/hipft.f90:4551)."""
        info = DiffusionInfo()
        ccb = CYCLE_CB(lambda u, c, ts, dc, s, sc: cb(c, ts, dc, s, sc)) if cb else CYCLE_CB()
        self._ck(self.L.hipft_gpu_diffusion_step(self.h, float(dt), ccb, None, ctypes.byref(info)),
                 "diffusion_step")
        return info

    def flux_transport_step(self, dt: float, cb: Optional[Callable] = None) -> DiffusionInfo:
        """flux_transport_step (src/hipft.f90:4463)."""
        info = DiffusionInfo()
        ccb = CYCLE_CB(lambda u, c, ts, dc, s, sc: cb(c, ts, dc, s, sc)) if cb else CYCLE_CB()
        self._ck(self.L.hipft_gpu_flux_transport_step(self.h, float(dt), ccb, None, ctypes.byref(info)),
                 "flux_transport_step")
        return info

    # -- assimilation / diagnostics
    def assimilate(self, data3: np.ndarray, *, add: bool = False, custom_from_mu: bool = False,
                   balance_flux: bool = False, mult_fac: float = 1.0, mu_power=4.0, mu_limit=0.1, lat_limit=0.0):
        """apply_data_assimilation + assimilate_new_data (src/hipft.f90:4148, 4083); data3 is (3, ntm, npm1)."""
        d = np.ascontiguousarray(data3, dtype=np.float64)
        assert d.shape == (3, self.ntm, self.npm1), d.shape
        v = [_vec(x, self.nr) for x in (mu_power, mu_limit, lat_limit)]
        o = DAOpts(int(add), int(custom_from_mu), int(balance_flux), float(mult_fac), *[_p(a) for a in v])
        self._ck(self.L.hipft_gpu_assimilate(self.h, _p(d), ctypes.byref(o)), "assimilate")

    def set_validation(self, mode: int, fval_u0_pt: Optional[np.ndarray] = None, width: float = 0.03,
                       vt_const: float = 0.0, vp_omega: float = 0.0, time_start: float = 0.0):
        f = None if fval_u0_pt is None else np.ascontiguousarray(fval_u0_pt, dtype=np.float64)
        self._ck(self.L.hipft_gpu_set_validation(self.h, int(mode), _p(f), float(width), float(vt_const),
                                                 float(vp_omega), float(time_start)), "set_validation")

    def analysis(self, time: float) -> np.ndarray:
        """analysis_step (src/hipft.f90:3098): (nr, 14) diagnostics."""
        out = np.zeros((self.nr, 14))
        self._ck(self.L.hipft_gpu_analysis(self.h, float(time), _p(out)), "analysis")
        return out

    def get_flux(self):
        """get_flux (src/hipft.f90:8672) per realization."""
        fp, fm = np.zeros(self.nr), np.zeros(self.nr)
        self._ck(self.L.hipft_gpu_get_flux(self.h, _p(fp), _p(fm)), "get_flux")
        return fp, fm

    def balance_flux(self):
        """balance_flux (src/hipft.f90:8752) on every realization."""
        self._ck(self.L.hipft_gpu_balance_flux(self.h), "balance_flux")

    def info(self) -> Info:
        i = Info()
        self._ck(self.L.hipft_gpu_info(self.h, ctypes.byref(i)), "info")
        return i

    def set_profiling(self, on: bool):
        """Per-kernel CUDA-event timing on the handle's stream (resets the counters)."""
        self._ck(self.L.hipft_gpu_set_profiling(self.h, int(on)), "set_profiling")

    def kernel_time(self, kind: int):
        """(launches, total ms) of kernel kind 0 STS stage, 1 advection stage, 2 ring sums, 3 other."""
        n, ms = ctypes.c_int64(0), ctypes.c_double(0.0)
        self._ck(self.L.hipft_gpu_kernel_time(self.h, int(kind), ctypes.byref(n), ctypes.byref(ms)), "kernel_time")
        return n.value, ms.value

    def describe(self) -> str:
        """Schedule and the two-stage kernel the autotuner picked."""
        buf = ctypes.create_string_buffer(256)
        self._ck(self.L.hipft_gpu_describe(self.h, buf, 256), "describe")
        return buf.value.decode()

    def set_stream(self, stream_ptr: int):
        self._ck(self.L.hipft_gpu_set_stream(self.h, ctypes.c_void_p(stream_ptr)), "set_stream")

    def synchronize(self):
        self._ck(self.L.hipft_gpu_synchronize(self.h), "synchronize")
