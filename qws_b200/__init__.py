"""qws_b200: B200-native domain-decomposed Wilson-clover solver.

Python mirror of the C ABI in include/qwsg.h (ctypes over the in-tree
qws_b200/libqws_b200.so).  The compute path is the CUDA library; this module
only moves arrays and calls it.  It raises if the library is missing: there
is no CPU fallback.

Device buffers are torch CUDA tensors used as raw memory (one spinor =
24 * pad reals in the library's DD-order planes); host arrays are numpy in
the natural layout documented in include/qwsg.h.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

__all__ = ["load_library", "Lattice", "QwsgError", "SolveStats", "LIB_PATH", "gen_gauge",
           "gen_clover", "gen_source", "plaquette"]

LIB_PATH = Path(__file__).resolve().parent / "libqws_b200.so"
_lib = None


class QwsgError(RuntimeError):
    pass


class SolveStats(ctypes.Structure):
    _fields_ = [("outer_iters", ctypes.c_int), ("inner_iters", ctypes.c_long),
                ("rel_resid_recursive", ctypes.c_double), ("rel_resid_true", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GroupItem(ctypes.Structure):
    _fields_ = [("lat", ctypes.c_void_p), ("x", ctypes.c_void_p), ("b", ctypes.c_void_p),
                ("tol", ctypes.c_double), ("maxiter", ctypes.c_int), ("tol_s", ctypes.c_double),
                ("maxiter_s", ctypes.c_int), ("nsap", ctypes.c_int), ("nm", ctypes.c_int),
                ("reliable", ctypes.c_int), ("stats", SolveStats), ("status", ctypes.c_int)]


class GroupStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_long), ("merged_launches", ctypes.c_long),
                ("member_launches", ctypes.c_long), ("t_members", ctypes.c_double),
                ("t_merge", ctypes.c_double), ("t_launch", ctypes.c_double),
                ("t_gpu_wait", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def load_library(path: str | os.PathLike | None = None):
    """Load libqws_b200.so (build it with `python -m qws_b200.build`)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise QwsgError(f"{p} not found: build the CUDA library with `python -m qws_b200.build`")
    lib = ctypes.CDLL(str(p), mode=os.RTLD_LOCAL)
    vp, ip, dp, fp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, ctypes.c_void_p
    c_int, c_double = ctypes.c_int, ctypes.c_double
    lib.qwsg_last_error.restype = ctypes.c_char_p
    lib.qwsg_version.restype = ctypes.c_char_p
    sig = {
        "qwsg_create": [ctypes.POINTER(vp), ip, ip, c_int],
        "qwsg_destroy": [vp],
        "qwsg_set_stream": [vp, vp],
        "qwsg_own_stream": [vp, c_int, ctypes.POINTER(vp)],
        "qwsg_set_kappa": [vp, c_double],
        "qwsg_geometry": [vp, ip, ip],
        "qwsg_sync": [vp],
        "qwsg_create_batch": [ctypes.POINTER(vp), vp, c_int],
        "qwsg_nrhs": [vp, ip],
        "qwsg_batch_set_kappas": [vp, vp, c_double],
        "qwsg_batch_set_tols": [vp, vp],
        "qwsg_inject_breakdown": [vp, c_int],
        "qwsg_batch_stats": [vp, ctypes.POINTER(SolveStats), ip],
        "qwsg_build_clover": [vp, c_double],
        "qwsg_set_graphs": [vp, c_int],
        "qwsg_set_hop_threads": [vp, c_int],
        "qwsg_set_link_compression": [vp, c_int],
        "qwsg_link_compression": [vp, ip],
        "qwsg_mtdagmt_d": [vp, vp, vp],
        "qwsg_load_gauge_bqcd": [vp, vp, vp],
        "qwsg_load_clover_bqcd": [vp, vp, vp],
        "qwsg_spinor_from_bqcd_d": [vp, vp, vp, vp, vp],
        "qwsg_spinor_from_bqcd_s": [vp, vp, vp, vp, vp],
        "qwsg_spinor_to_bqcd_d": [vp, vp, vp, vp, vp],
        "qwsg_spinor_to_bqcd_s": [vp, vp, vp, vp, vp],
        "qwsg_cg_vm": [vp, vp, vp, c_int, ip],
        "qwsg_mcg_vm": [vp, vp, vp, c_int, dp, c_int, ip],
        "qwsg_gen_gauge_device": [vp, ctypes.c_ulonglong, c_int, c_double,
                                  ctypes.POINTER(c_double)],
        "qwsg_load_gauge": [vp, dp],
        "qwsg_load_clover": [vp, dp],
        "qwsg_load_gauge_s": [vp, fp],
        "qwsg_load_clover_s": [vp, fp],
        "qwsg_spinor_to_device_d": [vp, vp, dp],
        "qwsg_spinor_to_host_d": [vp, dp, vp],
        "qwsg_spinor_to_device_s": [vp, vp, fp],
        "qwsg_spinor_to_host_s": [vp, fp, vp],
        "qwsg_ddd_d": [vp, vp, vp],
        "qwsg_ddd_s": [vp, vp, vp],
        "qwsg_ddd_in_d": [vp, vp, vp, c_int],
        "qwsg_ddd_in_s": [vp, vp, vp, c_int],
        "qwsg_ddd_out_d": [vp, vp, vp, c_int, c_double],
        "qwsg_ddd_out_s": [vp, vp, vp, c_int, c_double],
        "qwsg_jinv_s": [vp, vp, vp, c_int, c_int],
        "qwsg_prec_ddd_s": [vp, vp, vp, c_int, c_int],
        "qwsg_prec_s": [vp, vp, vp, c_int, c_int],
        "qwsg_bicgstab_precdd_s": [vp, vp, vp, c_double, c_int, c_int, c_int, ip,
                                   ctypes.POINTER(c_double)],
        "qwsg_bicgstab_dd_mix": [vp, vp, vp, c_double, c_int, c_double, c_int, c_int, c_int,
                                 ctypes.POINTER(SolveStats)],
        "qwsg_true_residual": [vp, vp, vp, ctypes.POINTER(c_double)],
        "qwsg_set_parities": [vp, c_int, c_int],
        "qwsg_deo_d": [vp, vp, vp, c_int, c_int, c_int, c_int, c_int, c_double, vp],
        "qwsg_deo_s": [vp, vp, vp, c_int, c_int, c_int, c_int, c_int, c_double, vp],
        "qwsg_clv_d": [vp, vp, vp, c_int],
        "qwsg_clv_s": [vp, vp, vp, c_int],
        "qwsg_mtilde_d": [vp, vp, vp],
        "qwsg_mtilde_dag_d": [vp, vp, vp],
        "qwsg_mtilde_s": [vp, vp, vp],
        "qwsg_bicgstab_vm": [vp, vp, vp, c_int, ip],
        "qwsg_prec_s_h": [vp, vp, vp, c_int, c_int],
        "qwsg_ddd_in_h": [vp, vp, vp, c_int],
        "qwsg_jinv_h": [vp, vp, vp, c_int, c_int],
        "qwsg_ddd_out_h": [vp, vp, vp, c_int, c_double],
        "qwsg_sap_update_s": [vp, vp, vp, vp, c_int],
        "qwsg_sap_update_h": [vp, vp, vp, vp, c_int],
        "qwsg_store_h": [vp, vp, vp],
        "qwsg_bicgstab_precdd_s_h": [vp, vp, vp, c_double, c_int, c_int, c_int, ip,
                                     ctypes.POINTER(c_double)],
        "qwsg_bicgstab_dd_mix2_hf": [vp, vp, vp, c_double, c_int, c_double, c_int, c_int, c_int,
                                     c_int, ctypes.POINTER(SolveStats)],
        "qwsg_batch_set_parent": [vp, vp],
        "qwsg_group_bicgstab_dd_mix2_hf": [ctypes.POINTER(GroupItem), c_int, vp,
                                           ctypes.POINTER(GroupStats)],
        "qwsg_counters": [vp] + [ctypes.POINTER(ctypes.c_long)] * 5,
        "qwsg_kernel_timing": [vp, c_int],
        "qwsg_kernel_stats": [vp, ip, vp, vp, vp],
        "qwsg_gen_gauge": [vp, ip, ctypes.c_ulonglong, c_int, c_double, ctypes.POINTER(c_double)],
        "qwsg_plaquette": [vp, ip, ctypes.POINTER(c_double)],
        "qwsg_gen_clover": [vp, vp, ip, c_double, c_double, vp],
        "qwsg_gen_source": [vp, ip, ctypes.c_ulonglong, c_int, c_int],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = c_int
    lib.qwsg_launch_count.restype = ctypes.c_long
    lib.qwsg_launch_count.argtypes = []
    lib.qwsg_kernel_name.restype = ctypes.c_char_p
    lib.qwsg_kernel_name.argtypes = [c_int]
    _lib = lib
    return lib


def _L4(L):
    return (ctypes.c_int * 4)(*map(int, L))


def gen_gauge(L, seed=1, n_smear=5, alpha=0.36):
    """Seeded SU(3) links smoothed by n_smear APE-style steps (natural layout
    [4, V, 18] FP64).  Returns (U, plaquette)."""
    lib = load_library()
    V = int(np.prod(L))
    U = np.empty((4, V, 18), np.float64)
    p = ctypes.c_double()
    _check(lib.qwsg_gen_gauge(U.ctypes.data_as(ctypes.c_void_p), _L4(L), int(seed), int(n_smear),
                              float(alpha), ctypes.byref(p)))
    return U, p.value


def plaquette(U, L):
    lib = load_library()
    U = np.ascontiguousarray(U, np.float64)
    p = ctypes.c_double()
    _check(lib.qwsg_plaquette(U.ctypes.data_as(ctypes.c_void_p), _L4(L), ctypes.byref(p)))
    return p.value


def gen_clover(U, L, csw, kappa, with_T=False):
    """Clover-leaf clover term; returns the packed inverse [V, 72] (and T)."""
    lib = load_library()
    V = int(np.prod(L))
    U = np.ascontiguousarray(U, np.float64)
    C = np.empty((V, 72), np.float64)
    T = np.empty((V, 12, 12, 2), np.float64) if with_T else None
    _check(lib.qwsg_gen_clover(C.ctypes.data_as(ctypes.c_void_p), U.ctypes.data_as(ctypes.c_void_p),
                               _L4(L), float(csw), float(kappa),
                               T.ctypes.data_as(ctypes.c_void_p) if with_T else None))
    return (C, T) if with_T else C


def gen_source(L, seed=2, kind="gauss", arg=0):
    """Sources in natural layout [V, 24]: kind gauss | point (arg = 4*colour+spin) | z2."""
    lib = load_library()
    V = int(np.prod(L))
    S = np.empty((V, 24), np.float64)
    k = {"gauss": 0, "point": 1, "z2": 2}[kind]
    _check(lib.qwsg_gen_source(S.ctypes.data_as(ctypes.c_void_p), _L4(L), int(seed), k, int(arg)))
    return S


def group_solve(solves, stream=None, check=True):
    """Solve several lattices together (qwsg_group_bicgstab_dd_mix2_hf): each
    kernel step is one launch over all of them.  solves: dicts with keys
    lattice (a one-RHS Lattice), x, b (device tensors; x holds the initial
    guess), tol, maxiter, tol_s, maxiter_s and optionally nsap (4), nm (2),
    reliable (0).  Returns (per-solve stats dicts with a 'status' key, group
    stats).  check: raise on the first failed solve, else report statuses."""
    lib = load_library()
    n = len(solves)
    items = (GroupItem * max(n, 1))()
    for i, s in enumerate(solves):
        lat = s["lattice"]
        if lat.nr != 1:
            raise QwsgError("group_solve: one-RHS lattices only")
        items[i].lat = lat.h
        items[i].x = _ptr(s["x"]).value
        items[i].b = _ptr(s["b"]).value
        items[i].tol = float(s["tol"])
        items[i].maxiter = int(s["maxiter"])
        items[i].tol_s = float(s["tol_s"])
        items[i].maxiter_s = int(s["maxiter_s"])
        items[i].nsap = int(s.get("nsap", 4))
        items[i].nm = int(s.get("nm", 2))
        items[i].reliable = int(s.get("reliable", 0))
    gs = GroupStats()
    st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    rc = lib.qwsg_group_bicgstab_dd_mix2_hf(items, n, st, ctypes.byref(gs))
    if check:
        _check(rc)
    out = []
    for i in range(n):
        d = items[i].stats.as_dict()
        d["status"] = items[i].status
        out.append(d)
    return out, gs.as_dict()


def launch_count():
    """Kernels the library has launched in this process (graph replays included)."""
    return load_library().qwsg_launch_count()


def _check(rc):
    if rc != 0:
        raise QwsgError(f"qwsg error {rc}: {_lib.qwsg_last_error().decode()}")


def _ptr(t):
    """Device pointer of a torch tensor (or an int address)."""
    if isinstance(t, int):
        return ctypes.c_void_p(t)
    return ctypes.c_void_p(t.data_ptr())


def _host(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a, a.ctypes.data_as(ctypes.c_void_p)


class Lattice:
    """One lattice resident on the current CUDA device.

    L: global extents (x, y, z, t); NB: SAP block grid (NB[0] even;
    the reference's partition on rank grid npe is (2*npe0, npe1, npe2, npe3));
    tbc: +1/-1 time boundary; kappa: hopping parameter.
    """

    def __init__(self, L, NB=(2, 1, 1, 1), tbc=-1, kappa=0.0, stream=None):
        import torch
        self.torch = torch
        self.lib = load_library()
        self.L, self.NB = tuple(map(int, L)), tuple(map(int, NB))
        h = ctypes.c_void_p()
        arr = lambda v: (ctypes.c_int * 4)(*v)
        _check(self.lib.qwsg_create(ctypes.byref(h), arr(self.L), arr(self.NB), int(tbc)))
        self.h = h
        V, pad = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.qwsg_geometry(self.h, ctypes.byref(V), ctypes.byref(pad)))
        self.V, self.pad = V.value, pad.value
        self.nr = 1
        self.set_kappa(kappa)
        self.set_stream(stream if stream is not None else torch.cuda.current_stream())

    def batch(self, nrhs, stream=None):
        """A multi-RHS handle on this lattice's fields (qwsg_create_batch)."""
        return BatchLattice(self, nrhs, stream)

    def close(self):
        if getattr(self, "h", None):
            self.lib.qwsg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- configuration -----------------------------------------------------
    def set_stream(self, stream):
        """Run this handle's work on `stream` (a torch stream, kept here, or a
        raw cudaStream_t)."""
        handle = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _check(self.lib.qwsg_set_stream(self.h, ctypes.c_void_p(handle)))
        self.stream = stream

    def use_own_stream(self, priority=0):
        """A private CUDA stream of this priority, made and owned by the
        library (qwsg_own_stream), as a torch ExternalStream.  torch's own
        streams come from a small pool that hands the same stream to several
        owners; handles used from several threads must not share one (a graph
        captured on a stream takes in every launch made into it meanwhile)."""
        p = ctypes.c_void_p()
        _check(self.lib.qwsg_own_stream(self.h, int(priority), ctypes.byref(p)))
        self.stream = self.torch.cuda.ExternalStream(p.value)
        return self.stream

    def set_kappa(self, kappa):
        self.kappa = float(kappa)
        _check(self.lib.qwsg_set_kappa(self.h, self.kappa))

    def load_fields(self, U, C, Us=None, Cs=None):
        """U natural [4,V,3,3,2] FP64, C natural [V,72] FP64 (inverse clover, QWS packing)."""
        U, pu = _host(U, np.float64)
        C, pc = _host(C, np.float64)
        assert U.size == 72 * self.V and C.size == 72 * self.V
        _check(self.lib.qwsg_load_gauge(self.h, pu))
        _check(self.lib.qwsg_load_clover(self.h, pc))
        if Us is not None:
            Us, p = _host(Us, np.float32)
            _check(self.lib.qwsg_load_gauge_s(self.h, p))
        if Cs is not None:
            Cs, p = _host(Cs, np.float32)
            _check(self.lib.qwsg_load_clover_s(self.h, p))

    def load_gauge(self, U):
        """Gauge field only (natural [4,V,3,3,2] FP64); see build_clover."""
        U, pu = _host(U, np.float64)
        assert U.size == 72 * self.V
        _check(self.lib.qwsg_load_gauge(self.h, pu))

    # ---- BQCD-format arrays (reordered on the device) ------------------------
    @staticmethod
    def _map(site_map):
        if site_map is None:
            return None, None
        m = np.ascontiguousarray(site_map, np.int32)
        return m, ctypes.c_void_p(m.ctypes.data)

    def load_fields_bqcd(self, u, c, site_map=None):
        """BQCD gauge u (4*V*18 reals) and clover c (V*72 reals), FP64."""
        u, pu = _host(u, np.float64)
        c, pc = _host(c, np.float64)
        assert u.size == 72 * self.V and c.size == 72 * self.V
        m, pm = self._map(site_map)
        _check(self.lib.qwsg_load_gauge_bqcd(self.h, pu, pm))
        _check(self.lib.qwsg_load_clover_bqcd(self.h, pc, pm))

    def from_bqcd(self, even, odd, dtype="f64", site_map=None, out=None):
        """BQCD even/odd spinor arrays (FP64, V/2*24 reals each per RHS) -> device."""
        e, pe_ = _host(even, np.float64)
        o, po = _host(odd, np.float64)
        assert e.size == o.size == 12 * self.V * self.nr
        out = self.empty(dtype) if out is None else out
        m, pm = self._map(site_map)
        fn = self.lib.qwsg_spinor_from_bqcd_d if out.dtype == self.torch.float64 else \
            self.lib.qwsg_spinor_from_bqcd_s
        _check(fn(self.h, _ptr(out), pe_, po, pm))
        return out

    def to_bqcd(self, t, site_map=None):
        """device spinor -> (even, odd) BQCD arrays, FP64."""
        even = np.empty(12 * self.V * self.nr, np.float64)
        odd = np.empty_like(even)
        m, pm = self._map(site_map)
        fn = self.lib.qwsg_spinor_to_bqcd_d if t.dtype == self.torch.float64 else \
            self.lib.qwsg_spinor_to_bqcd_s
        _check(fn(self.h, ctypes.c_void_p(even.ctypes.data), ctypes.c_void_p(odd.ctypes.data),
                  _ptr(t), pm))
        return even, odd

    def gen_gauge_device(self, seed, n_smear=5, alpha=0.36):
        """Seeded SU(3) + APE gauge field generated on the GPU; returns the
        plaquette.  The FP64 clover planes serve as scratch: build or load
        the clover term afterwards."""
        p = ctypes.c_double()
        _check(self.lib.qwsg_gen_gauge_device(self.h, int(seed), int(n_smear), float(alpha),
                                              ctypes.byref(p)))
        return p.value

    def build_clover(self, csw):
        """Clover term of the loaded gauge field for this kappa, built on the GPU."""
        _check(self.lib.qwsg_build_clover(self.h, float(csw)))

    # ---- buffers -----------------------------------------------------------
    def empty(self, dtype="f32"):
        t = self.torch.float32 if dtype in ("f32", np.float32) else self.torch.float64
        return self.torch.zeros(24 * self.pad * self.nr, dtype=t, device="cuda")

    def to_device(self, v, out=None):
        """Host natural-layout spinor(s) ([V,24], or [nrhs,V,24] on a multi-RHS handle)."""
        v = np.asarray(v)
        assert v.size == 24 * self.V * self.nr
        if v.dtype == np.float64:
            out = self.empty("f64") if out is None else out
            a, p = _host(v, np.float64)
            _check(self.lib.qwsg_spinor_to_device_d(self.h, _ptr(out), p))
        else:
            out = self.empty("f32") if out is None else out
            a, p = _host(v, np.float32)
            _check(self.lib.qwsg_spinor_to_device_s(self.h, _ptr(out), p))
        return out

    def to_host(self, t, out=None):
        """Device planes -> host natural layout (into `out` if given, e.g. pinned)."""
        shape = (self.V, 24) if self.nr == 1 else (self.nr, self.V, 24)
        n = 24 * self.V * self.nr
        if t.dtype == self.torch.float64:
            a = np.empty(shape, np.float64) if out is None else out
            assert a.dtype == np.float64 and a.flags.c_contiguous and a.size == n
            _check(self.lib.qwsg_spinor_to_host_d(self.h, a.ctypes.data_as(ctypes.c_void_p), _ptr(t)))
        else:
            a = np.empty(shape, np.float32) if out is None else out
            assert a.dtype == np.float32 and a.flags.c_contiguous and a.size == n
            _check(self.lib.qwsg_spinor_to_host_s(self.h, a.ctypes.data_as(ctypes.c_void_p), _ptr(t)))
        return a

    def sync(self):
        _check(self.lib.qwsg_sync(self.h))

    # ---- operators (device tensors in, device tensors out) -----------------
    def _out(self, x, out):
        return self.torch.zeros_like(x) if out is None else out

    def ddd(self, x, out=None):
        out = self._out(x, out)
        fn = self.lib.qwsg_ddd_d if x.dtype == self.torch.float64 else self.lib.qwsg_ddd_s
        _check(fn(self.h, _ptr(out), _ptr(x)))
        return out

    def ddd_in(self, x, colour, out=None):
        out = self._out(x, out)
        fn = self.lib.qwsg_ddd_in_d if x.dtype == self.torch.float64 else self.lib.qwsg_ddd_in_s
        _check(fn(self.h, _ptr(out), _ptr(x), int(colour)))
        return out

    def ddd_out(self, x, colour, factor, out=None):
        out = self._out(x, out)
        fn = self.lib.qwsg_ddd_out_d if x.dtype == self.torch.float64 else self.lib.qwsg_ddd_out_s
        _check(fn(self.h, _ptr(out), _ptr(x), int(colour), float(factor)))
        return out

    def jinv(self, b, colour, nm, out=None):
        out = self._out(b, out)
        _check(self.lib.qwsg_jinv_s(self.h, _ptr(out), _ptr(b), int(colour), int(nm)))
        return out

    def prec_ddd(self, x, nsap=4, nm=2, out=None):
        out = self._out(x, out)
        _check(self.lib.qwsg_prec_ddd_s(self.h, _ptr(out), _ptr(x), int(nsap), int(nm)))
        return out

    def prec(self, x, nsap=4, nm=2, out=None):
        out = self._out(x, out)
        _check(self.lib.qwsg_prec_s(self.h, _ptr(out), _ptr(x), int(nsap), int(nm)))
        return out

    def bicgstab_precdd(self, b, tol, maxiter, nsap=4, nm=2, out=None):
        out = self._out(b, out)
        it, rel = ctypes.c_int(), ctypes.c_double()
        _check(self.lib.qwsg_bicgstab_precdd_s(self.h, _ptr(out), _ptr(b), float(tol), int(maxiter),
                                               int(nsap), int(nm), ctypes.byref(it),
                                               ctypes.byref(rel)))
        return out, it.value, rel.value

    def bicgstab_dd_mix(self, x, b, tol, maxiter, tol_s, maxiter_s, nsap=4, nm=2):
        """Solve D x = b in place (x holds the initial guess)."""
        st = SolveStats()
        _check(self.lib.qwsg_bicgstab_dd_mix(self.h, _ptr(x), _ptr(b), float(tol), int(maxiter),
                                             float(tol_s), int(maxiter_s), int(nsap), int(nm),
                                             ctypes.byref(st)))
        return st.as_dict()

    # ---- even-odd (site parity) family ---------------------------------------
    def deo(self, x, pe, which=3, dag=0, clov=0, mode=0, factor=0.0, in0=None, out=None):
        """Sites of parity pe receive the hops from the other parity (see
        qwsg_deo_d in include/qwsg.h for which/dag/clov/mode)."""
        out = self._out(x, out)
        fn = self.lib.qwsg_deo_d if x.dtype == self.torch.float64 else self.lib.qwsg_deo_s
        _check(fn(self.h, _ptr(out), _ptr(x), int(pe), int(which), int(dag), int(clov), int(mode),
                  float(factor), _ptr(in0) if in0 is not None else None))
        return out

    def clv(self, x, pe, out=None):
        out = self._out(x, out)
        fn = self.lib.qwsg_clv_d if x.dtype == self.torch.float64 else self.lib.qwsg_clv_s
        _check(fn(self.h, _ptr(out), _ptr(x), int(pe)))
        return out

    def mtilde(self, x, dag=False, out=None):
        out = self._out(x, out)
        if x.dtype == self.torch.float64:
            fn = self.lib.qwsg_mtilde_dag_d if dag else self.lib.qwsg_mtilde_d
        else:
            if dag:
                raise QwsgError("mtilde_dag is FP64 only (as in the reference)")
            fn = self.lib.qwsg_mtilde_s
        _check(fn(self.h, _ptr(out), _ptr(x)))
        return out

    def bicgstab_vm(self, x, b, maxiter=100):
        it = ctypes.c_int()
        _check(self.lib.qwsg_bicgstab_vm(self.h, _ptr(x), _ptr(b), int(maxiter), ctypes.byref(it)))
        return it.value

    def mtdagmt(self, x, out=None):
        out = self._out(x, out)
        _check(self.lib.qwsg_mtdagmt_d(self.h, _ptr(out), _ptr(x)))
        return out

    def cg_vm(self, x, b, maxiter=1000):
        """CG on mtilde^dag mtilde (parity pce), x = initial guess in, solution out."""
        it = ctypes.c_int()
        _check(self.lib.qwsg_cg_vm(self.h, _ptr(x), _ptr(b), int(maxiter), ctypes.byref(it)))
        return it.value

    def mcg_vm(self, b, sigma, maxiter=1000):
        """Multi-shift CG: (mtilde^dag mtilde + sigma_k) x_k = b; returns
        ([x_k device tensors], iterations)."""
        sigma = np.ascontiguousarray(sigma, np.float64)
        n = len(sigma)
        X = self.torch.zeros(n * 24 * self.pad, dtype=self.torch.float64, device="cuda")
        it = ctypes.c_int()
        _check(self.lib.qwsg_mcg_vm(self.h, _ptr(X), _ptr(b), n,
                                    ctypes.c_void_p(sigma.ctypes.data),
                                    int(maxiter), ctypes.byref(it)))
        return [X[k * 24 * self.pad:(k + 1) * 24 * self.pad] for k in range(n)], it.value

    # ---- precision form (FP16-storage SAP) ----------------------------------
    def prec_h(self, x, nsap=4, nm=2, out=None):
        """M_SAP in FP16 storage (nsap-1 sweeps + final stage); FP32 in/out."""
        out = self._out(x, out)
        _check(self.lib.qwsg_prec_s_h(self.h, _ptr(out), _ptr(x), int(nsap), int(nm)))
        return out

    def ddd_in_h(self, x, colour, out=None):
        """D_blk on one colour with the FP16-storage kernel (FP32 in/out)."""
        out = self._out(x, out)
        _check(self.lib.qwsg_ddd_in_h(self.h, _ptr(out), _ptr(x), int(colour)))
        return out

    def jinv_h(self, b, colour, nm, out=None):
        """nm Richardson steps on one colour with the FP16-storage kernel."""
        out = self._out(b, out)
        _check(self.lib.qwsg_jinv_h(self.h, _ptr(out), _ptr(b), int(colour), int(nm)))
        return out

    def store_h(self, x, out=None):
        """x (FP32) as the FP16 kernels store it (per-site scale, FP16
        round-to-nearest-even) and read it back (qwsg_store_h)."""
        out = self._out(x, out)
        _check(self.lib.qwsg_store_h(self.h, _ptr(out), _ptr(x)))
        return out

    def ddd_out_h(self, x, colour, factor, out=None):
        """out += factor A^-1 H_face x on one colour, FP16-storage kernel."""
        out = self._out(x, out)
        _check(self.lib.qwsg_ddd_out_h(self.h, _ptr(out), _ptr(x), int(colour), float(factor)))
        return out

    def sap_update(self, s, a, rhs, colour, half=False):
        """s_c += rhs_c - D_blk a_c in place (FP32 kernel, or FP16 storage)."""
        fn = self.lib.qwsg_sap_update_h if half else self.lib.qwsg_sap_update_s
        _check(fn(self.h, _ptr(s), _ptr(a), _ptr(rhs), int(colour)))
        return s

    def bicgstab_precdd_h(self, b, tol, maxiter, nsap=4, nm=2, out=None):
        out = self._out(b, out)
        it, rel = ctypes.c_int(), ctypes.c_double()
        _check(self.lib.qwsg_bicgstab_precdd_s_h(self.h, _ptr(out), _ptr(b), float(tol),
                                                 int(maxiter), int(nsap), int(nm),
                                                 ctypes.byref(it), ctypes.byref(rel)))
        return out, it.value, rel.value

    def bicgstab_dd_mix2_hf(self, x, b, tol, maxiter, tol_s, maxiter_s, nsap=4, nm=2,
                            reliable=0):
        """FP64 outer / FP16-SAP flexible inner solve of D x = b in place."""
        st = SolveStats()
        _check(self.lib.qwsg_bicgstab_dd_mix2_hf(self.h, _ptr(x), _ptr(b), float(tol), int(maxiter),
                                                 float(tol_s), int(maxiter_s), int(nsap), int(nm),
                                                 int(reliable), ctypes.byref(st)))
        return st.as_dict()

    def true_residual(self, x, b):
        """|b - D x| / |b| (a list with one value per RHS on a multi-RHS handle)."""
        r = (ctypes.c_double * self.nr)()
        _check(self.lib.qwsg_true_residual(self.h, _ptr(x), _ptr(b), r))
        return r[0] if self.nr == 1 else list(r)

    def inject_breakdown(self, outer_iter):
        """Test hook (host side): the outer loop takes <r0, q> as zero at
        outer iteration outer_iter (0: off); qwsg_inject_breakdown."""
        _check(self.lib.qwsg_inject_breakdown(self.h, int(outer_iter)))

    def set_graphs(self, enable=True):
        _check(self.lib.qwsg_set_graphs(self.h, 1 if enable else 0))

    def set_link_compression(self, mode=1):
        """1: FP32 kernels read 12-real links when the links are SU(3); 0: never."""
        _check(self.lib.qwsg_set_link_compression(self.h, int(mode)))

    def link_compression(self):
        """True when the FP32 kernels read the 12-real links."""
        v = ctypes.c_int()
        _check(self.lib.qwsg_link_compression(self.h, ctypes.byref(v)))
        return bool(v.value)

    def set_hop_threads(self, threads):
        """Threads per CTA of the Dirac-operator kernels (64, 128 or 256)."""
        _check(self.lib.qwsg_set_hop_threads(self.h, int(threads)))

    def kernel_timing(self, enable=True):
        _check(self.lib.qwsg_kernel_timing(self.h, 1 if enable else 0))

    def kernel_stats(self):
        """{kernel name: (launches, total device ms, algorithmic bytes)} since enabling."""
        n = ctypes.c_int(32)
        L = (ctypes.c_long * 32)()
        ms = (ctypes.c_double * 32)()
        by = (ctypes.c_double * 32)()
        _check(self.lib.qwsg_kernel_stats(self.h, ctypes.byref(n), L, ms, by))
        return {self.lib.qwsg_kernel_name(k).decode(): (L[k], ms[k], by[k]) for k in range(n.value)
                if L[k] > 0}

    def counters(self):
        v = [ctypes.c_long() for _ in range(5)]
        _check(self.lib.qwsg_counters(self.h, *[ctypes.byref(x) for x in v]))
        return dict(zip(("prec_ddd_s", "prec_s", "jinv", "inner_iters", "ddd_d"), [x.value for x in v]))


class BatchLattice(Lattice):
    """nrhs right-hand sides on the fields and kappa of a parent Lattice
    (qwsg_create_batch): every operator launch serves all RHS.  Device
    buffers hold 24*pad*nrhs reals; host spinors are [nrhs, V, 24]."""

    def __init__(self, parent, nrhs, stream=None):
        import torch
        self.torch = torch
        self.lib = parent.lib
        self.parent = parent  # keeps the fields' owner alive
        self.L, self.NB = parent.L, parent.NB
        h = ctypes.c_void_p()
        _check(self.lib.qwsg_create_batch(ctypes.byref(h), parent.h, int(nrhs)))
        self.h = h
        self.V, self.pad, self.nr = parent.V, parent.pad, int(nrhs)
        self.kappa = parent.kappa
        self.set_stream(stream if stream is not None else torch.cuda.current_stream())

    def set_kappa(self, kappa):
        raise QwsgError("kappa belongs to the parent lattice (or use set_kappas)")

    def set_parent(self, parent):
        """Serve another lattice of the same extents and block grid with this
        handle's buffers (qwsg_batch_set_parent); per-RHS kappas and
        tolerances must be set again."""
        _check(self.lib.qwsg_batch_set_parent(self.h, parent.h))
        self.parent = parent
        self.kappa = parent.kappa
        self.kappas = None
        self.tols = None

    def set_kappas(self, kappas, csw):
        """A kappa per RHS: clover terms of the parent's gauge field built on
        the GPU for each (qwsg_batch_set_kappas)."""
        k = np.ascontiguousarray(kappas, np.float64)
        assert k.size == self.nr
        _check(self.lib.qwsg_batch_set_kappas(self.h, ctypes.c_void_p(k.ctypes.data), float(csw)))
        self.kappas = k.copy()

    def set_tols(self, tols):
        """A stopping tolerance per RHS for the FP64 outer solvers
        (qwsg_batch_set_tols); None: the solver's tol argument for all."""
        if tols is None:
            _check(self.lib.qwsg_batch_set_tols(self.h, None))
            self.tols = None
            return
        t = np.ascontiguousarray(tols, np.float64)
        assert t.size == self.nr
        _check(self.lib.qwsg_batch_set_tols(self.h, ctypes.c_void_p(t.ctypes.data)))
        self.tols = t.copy()

    def load_fields(self, *a, **k):
        raise QwsgError("fields belong to the parent lattice")

    def batch_stats(self):
        """Per-RHS stats of the last DD solve and iteration counts of the last inner solve."""
        st = (SolveStats * self.nr)()
        it = (ctypes.c_int * self.nr)()
        _check(self.lib.qwsg_batch_stats(self.h, st, it))
        return [s.as_dict() for s in st], list(it)
