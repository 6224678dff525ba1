"""Test-side bindings: the CPU oracle (oracle/liboracle.so), the reference
built from its own sources (oracle/_ref/<variant>/libqwsref.so), and numpy
converters between the natural lattice layout and QWS's SIMD-lane layout.

Test infrastructure only; nothing in the product imports this module.

QWS host layout (qws.h:111-192, main.cc:426-429): the local lattice is split
into two x-halves ("domains").  A spinor array is indexed
    [domain][t][z][y][x_half / VLEN]   each element c[3 col][4 spin][2 ri][VLEN]
with lane = x_half % VLEN.  Links: [domain][mu][t][z][y][xv] c[col][row][ri][VLEN]
(column-major SU(3)).  Clover: [domain][t][z][y][xv] c[2][36][VLEN].
Natural layout: site = x + Lx*(y + Ly*(z + Lz*t)); spinor [V][3][4][2],
gauge [4][V][3 row][3 col][2], clover [V][72].
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
ORACLE_DIR = REPO / "oracle"
ORACLE_SO = ORACLE_DIR / "liboracle.so"
REF_DIR = ORACLE_DIR / "_ref"

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_fp)


def iarr(vals):
    return (ctypes.c_int * len(vals))(*vals)


# --------------------------------------------------------------------------
# oracle
# --------------------------------------------------------------------------
_oracle = None


def load_oracle():
    global _oracle
    if _oracle is not None:
        return _oracle
    srcs = [ORACLE_DIR / n for n in ("qws_oracle.cc", "qws_oracle.h", "fields_oracle.cc")]
    if not ORACLE_SO.exists() or any(ORACLE_SO.stat().st_mtime < s.stat().st_mtime
                                     for s in srcs if s.exists()):
        subprocess.run(["make", "-C", str(ORACLE_DIR), "oracle", "CXX=g++"], check=True,
                       stdout=subprocess.DEVNULL)
    lib = ctypes.CDLL(str(ORACLE_SO))
    vp = ctypes.c_void_p
    lib.orc_create.restype = vp
    lib.orc_create.argtypes = [_ip, _ip, ctypes.c_int]
    lib.orc_destroy.argtypes = [vp]
    lib.orc_set_kappa.argtypes = [vp, ctypes.c_double]
    lib.orc_volume.restype = ctypes.c_long
    lib.orc_volume.argtypes = [vp]
    for n in ("orc_set_gauge_d", "orc_set_clover_d"):
        getattr(lib, n).argtypes = [vp, _dp]
    for n in ("orc_set_gauge_s", "orc_set_clover_s"):
        getattr(lib, n).argtypes = [vp, _fp]
    lib.orc_gen_main_fields.argtypes = [_ip, _ip, _dp, _dp, ctypes.c_int, _dp]
    lib.orc_ddd_in_d.argtypes = [vp, _dp, _dp, ctypes.c_int, ctypes.c_int]
    lib.orc_ddd_out_d.argtypes = [vp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_double]
    lib.orc_ddd_d.argtypes = [vp, _dp, _dp]
    lib.orc_ddd_in_s.argtypes = [vp, _fp, _fp, ctypes.c_int, ctypes.c_int]
    lib.orc_ddd_out_s.argtypes = [vp, _fp, _fp, ctypes.c_int, ctypes.c_int, ctypes.c_float]
    lib.orc_ddd_s.argtypes = [vp, _fp, _fp]
    lib.orc_clover_d.argtypes = [vp, _dp]
    lib.orc_clover_s.argtypes = [vp, _fp]
    lib.orc_jinv_s.argtypes = [vp, _fp, _fp, ctypes.c_int, ctypes.c_int]
    lib.orc_prec_ddd_s.argtypes = [vp, _fp, _fp, ctypes.c_int, ctypes.c_int]
    lib.orc_prec_s.argtypes = [vp, _fp, _fp, ctypes.c_int, ctypes.c_int]
    lib.orc_bicgstab_precdd_s.restype = ctypes.c_int
    lib.orc_bicgstab_precdd_s.argtypes = [vp, _fp, _fp, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, _dp]
    lib.orc_bicgstab_dd_mix.argtypes = [vp, _dp, _dp, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, _dp, _dp]
    lib.orc_bicgstab_precdd_s_h.restype = ctypes.c_int
    lib.orc_bicgstab_precdd_s_h.argtypes = [vp, _fp, _fp, ctypes.c_double, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, _dp]
    lib.orc_bicgstab_dd_mix2_hf.argtypes = [vp, _dp, _dp, ctypes.c_double, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, _dp]
    lib.orc_deo_d.argtypes = [vp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, ctypes.c_double, _dp]
    lib.orc_deo_s.argtypes = [vp, _fp, _fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, ctypes.c_float, _fp]
    lib.orc_clv_d.argtypes = [vp, _dp, _dp, ctypes.c_int]
    lib.orc_clv_s.argtypes = [vp, _fp, _fp, ctypes.c_int]
    lib.orc_mtilde_d.argtypes = [vp, _dp, _dp]
    lib.orc_mtilde_dag_d.argtypes = [vp, _dp, _dp]
    lib.orc_bicgstab_vm.restype = ctypes.c_int
    lib.orc_bicgstab_vm.argtypes = [vp, _dp, _dp, ctypes.c_int]
    lib.orc_mtdagmt_d.argtypes = [vp, _dp, _dp]
    lib.orc_cg_vm.restype = ctypes.c_int
    lib.orc_cg_vm.argtypes = [vp, _dp, _dp, ctypes.c_int]
    lib.orc_mcg_vm.restype = ctypes.c_int
    lib.orc_mcg_vm.argtypes = [vp, _dp, _dp, ctypes.c_int, _dp, ctypes.c_int]
    lib.orc_gen_gauge.argtypes = [_dp, _ip, ctypes.c_ulonglong, ctypes.c_int, ctypes.c_double,
                                  _dp]
    lib.orc_plaquette.restype = ctypes.c_double
    lib.orc_plaquette.argtypes = [_dp, _ip]
    lib.orc_gen_clover.restype = ctypes.c_int
    lib.orc_gen_clover.argtypes = [_dp, _dp, _ip, ctypes.c_double, ctypes.c_double]
    lib.orc_gen_source.argtypes = [_dp, _ip, ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int]
    lib.orc_plant_breakdown.argtypes = [ctypes.c_int]
    lib.orc_norm2_d.restype = ctypes.c_double
    lib.orc_norm2_d.argtypes = [_dp, ctypes.c_long]
    lib.orc_norm2_s.restype = ctypes.c_double
    lib.orc_norm2_s.argtypes = [_fp, ctypes.c_long]
    _oracle = lib
    return lib


class Oracle:
    """One lattice in the oracle (global lattice L, block grid NB)."""

    def __init__(self, L, NB, tbc=1, kappa=0.0):
        self.lib = load_oracle()
        self.L = tuple(int(v) for v in L)
        self.NB = tuple(int(v) for v in NB)
        self.V = int(np.prod(self.L))
        self.h = self.lib.orc_create(iarr(self.L), iarr(self.NB), int(tbc))
        self.lib.orc_set_kappa(self.h, float(kappa))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def set_kappa(self, k):
        self.lib.orc_set_kappa(self.h, float(k))

    def set_fields(self, U, C, Us=None, Cs=None):
        U = np.ascontiguousarray(U, dtype=np.float64)
        C = np.ascontiguousarray(C, dtype=np.float64)
        self.lib.orc_set_gauge_d(self.h, dptr(U))
        self.lib.orc_set_clover_d(self.h, dptr(C))
        if Us is not None:
            self.lib.orc_set_gauge_s(self.h, fptr(np.ascontiguousarray(Us, dtype=np.float32)))
        if Cs is not None:
            self.lib.orc_set_clover_s(self.h, fptr(np.ascontiguousarray(Cs, dtype=np.float32)))

    def spinor_d(self):
        return np.zeros((self.V, 24), np.float64)

    def spinor_s(self):
        return np.zeros((self.V, 24), np.float32)

    def ddd_d(self, x):
        out = self.spinor_d()
        self.lib.orc_ddd_d(self.h, dptr(out), dptr(np.ascontiguousarray(x)))
        return out

    def ddd_s(self, x):
        out = self.spinor_s()
        self.lib.orc_ddd_s(self.h, fptr(out), fptr(np.ascontiguousarray(x)))
        return out

    def ddd_in_d(self, x, kind, sel, out=None):
        out = self.spinor_d() if out is None else out
        self.lib.orc_ddd_in_d(self.h, dptr(out), dptr(x), kind, sel)
        return out

    def ddd_out_d(self, x, kind, sel, factor, out=None):
        out = self.spinor_d() if out is None else out
        self.lib.orc_ddd_out_d(self.h, dptr(out), dptr(x), kind, sel, factor)
        return out

    def ddd_in_s(self, x, kind, sel, out=None):
        out = self.spinor_s() if out is None else out
        self.lib.orc_ddd_in_s(self.h, fptr(out), fptr(x), kind, sel)
        return out

    def ddd_out_s(self, x, kind, sel, factor, out=None):
        out = self.spinor_s() if out is None else out
        self.lib.orc_ddd_out_s(self.h, fptr(out), fptr(x), kind, sel, factor)
        return out

    def clover_d(self, x):
        y = np.array(x, np.float64, copy=True)
        self.lib.orc_clover_d(self.h, dptr(y))
        return y

    def clover_s(self, x):
        y = np.array(x, np.float32, copy=True)
        self.lib.orc_clover_s(self.h, fptr(y))
        return y

    def jinv_s(self, b, colour, nm, x=None):
        x = self.spinor_s() if x is None else x
        self.lib.orc_jinv_s(self.h, fptr(x), fptr(b), colour, nm)
        return x

    def prec_ddd_s(self, x, nsap, nm):
        out = self.spinor_s()
        self.lib.orc_prec_ddd_s(self.h, fptr(out), fptr(np.ascontiguousarray(x)), nsap, nm)
        return out

    def prec_s(self, x, nsap, nm):
        out = self.spinor_s()
        self.lib.orc_prec_s(self.h, fptr(out), fptr(np.ascontiguousarray(x)), nsap, nm)
        return out

    def bicgstab_precdd_s(self, b, tol, maxiter, nsap, nm):
        x = self.spinor_s()
        rel = ctypes.c_double(0)
        it = self.lib.orc_bicgstab_precdd_s(self.h, fptr(x), fptr(np.ascontiguousarray(b)), tol,
                                            maxiter, nsap, nm, ctypes.byref(rel))
        return x, it, rel.value

    def bicgstab_precdd_s_h(self, b, tol, maxiter, nsap, nm):
        x = self.spinor_s()
        rel = ctypes.c_double(0)
        it = self.lib.orc_bicgstab_precdd_s_h(self.h, fptr(x), fptr(np.ascontiguousarray(b)), tol,
                                              maxiter, nsap, nm, ctypes.byref(rel))
        return x, it, rel.value

    def bicgstab_dd_mix2_hf(self, b, x0, tol, maxiter, tol_s, maxiter_s, nsap, nm):
        x = np.array(x0, np.float64, copy=True)
        stats = np.zeros(3)
        self.lib.orc_bicgstab_dd_mix2_hf(self.h, dptr(x), dptr(np.ascontiguousarray(b)), tol,
                                         maxiter, tol_s, maxiter_s, nsap, nm, dptr(stats))
        return x, stats

    # ---- even-odd operators ------------------------------------------------
    # deo(x, pe, which, dag, clov, mode, factor, in0): sites of parity pe get
    # the hops from the other parity; which 1 = inside the rank box (deo_in),
    # 2 = across its faces (deo_out), 3 = all; mode 0 store, 1 out += factor*,
    # 2 out = in0 + factor*.
    def deo(self, x, pe, which=3, dag=0, clov=0, mode=0, factor=0.0, in0=None, out=None):
        dbl = np.asarray(x).dtype == np.float64
        out = (self.spinor_d() if dbl else self.spinor_s()) if out is None else out
        if dbl:
            p0 = dptr(in0) if in0 is not None else None
            self.lib.orc_deo_d(self.h, dptr(out), dptr(np.ascontiguousarray(x)), pe, which, dag,
                               clov, mode, factor, p0)
        else:
            p0 = fptr(in0) if in0 is not None else None
            self.lib.orc_deo_s(self.h, fptr(out), fptr(np.ascontiguousarray(x)), pe, which, dag,
                               clov, mode, factor, p0)
        return out

    def clv(self, x, pe, out=None):
        dbl = np.asarray(x).dtype == np.float64
        out = np.array(x, copy=True) if out is None else out
        fn, pp = (self.lib.orc_clv_d, dptr) if dbl else (self.lib.orc_clv_s, fptr)
        fn(self.h, pp(out), pp(np.ascontiguousarray(x)), pe)
        return out

    def mtilde(self, x, dag=False):
        out = self.spinor_d()
        fn = self.lib.orc_mtilde_dag_d if dag else self.lib.orc_mtilde_d
        fn(self.h, dptr(out), dptr(np.ascontiguousarray(x)))
        return out

    def bicgstab_vm(self, b, x0, maxiter):
        x = np.array(x0, np.float64, copy=True)
        it = self.lib.orc_bicgstab_vm(self.h, dptr(x), dptr(np.ascontiguousarray(b)), maxiter)
        return x, it

    def mtdagmt(self, x):
        out = self.spinor_d()
        self.lib.orc_mtdagmt_d(self.h, dptr(out), dptr(np.ascontiguousarray(x)))
        return out

    def cg_vm(self, b, x0, maxiter):
        x = np.array(x0, np.float64, copy=True)
        it = self.lib.orc_cg_vm(self.h, dptr(x), dptr(np.ascontiguousarray(b)), maxiter)
        return x, it

    def mcg_vm(self, b, sigma, maxiter):
        sigma = np.ascontiguousarray(sigma, np.float64)
        X = np.zeros((len(sigma),) + np.shape(b), np.float64)
        it = self.lib.orc_mcg_vm(self.h, dptr(X), dptr(np.ascontiguousarray(b)), len(sigma),
                                 dptr(sigma), maxiter)
        return X, it

    def bicgstab_dd_mix(self, b, x0, tol, maxiter, tol_s, maxiter_s, nsap, nm):
        x = np.array(x0, np.float64, copy=True)
        stats = np.zeros(3)
        hist = np.zeros(2 * maxiter)
        self.lib.orc_bicgstab_dd_mix(self.h, dptr(x), dptr(np.ascontiguousarray(b)), tol, maxiter,
                                     tol_s, maxiter_s, nsap, nm, dptr(stats), dptr(hist))
        return x, stats, hist


def gen_gauge(L, seed=1, n_smear=5, alpha=0.36):
    """The benchmark's seeded SU(3) links after n_smear smoothing steps,
    natural layout [4, V, 18] (fields_oracle.cc); returns (U, plaquette).
    Bit-equal to the product's qws_b200.gen_gauge."""
    lib = load_oracle()
    V = int(np.prod(L))
    U = np.empty((4, V, 18), np.float64)
    p = ctypes.c_double()
    lib.orc_gen_gauge(dptr(U), iarr(L), int(seed), int(n_smear), float(alpha), ctypes.byref(p))
    return U, p.value


def plaquette(U, L):
    return float(load_oracle().orc_plaquette(dptr(np.ascontiguousarray(U, np.float64)), iarr(L)))


def gen_clover(U, L, csw, kappa):
    """Clover-leaf term of U as the packed inverse [V, 72] (fields_oracle.cc)."""
    lib = load_oracle()
    V = int(np.prod(L))
    C = np.empty((V, 72), np.float64)
    bad = lib.orc_gen_clover(dptr(C), dptr(np.ascontiguousarray(U, np.float64)), iarr(L),
                             float(csw), float(kappa))
    if bad:
        raise ValueError(f"{bad} singular clover blocks")
    return C


def gen_source(L, seed=2, kind="gauss", arg=0):
    """Sources [V, 24]: kind gauss | point (arg = 4*colour+spin) | z2 (fields_oracle.cc)."""
    lib = load_oracle()
    V = int(np.prod(L))
    S = np.empty((V, 24), np.float64)
    lib.orc_gen_source(dptr(S), iarr(L), int(seed), {"gauss": 0, "point": 1, "z2": 2}[kind],
                       int(arg))
    return S


def gen_main_fields(Lloc, npe=(1, 1, 1, 1), nsrc=2):
    """main.cc's seeded fields (mt19937(12345)), tiled over the rank grid."""
    lib = load_oracle()
    L = [a * b for a, b in zip(Lloc, npe)]
    V = int(np.prod(L))
    U = np.zeros((4, V, 18), np.float64)
    C = np.zeros((V, 72), np.float64)
    S = np.zeros((max(nsrc, 1), V, 24), np.float64)
    lib.orc_gen_main_fields(iarr(Lloc), iarr(npe), dptr(U), dptr(C), nsrc, dptr(S))
    return U, C, S[:nsrc]


# --------------------------------------------------------------------------
# QWS <-> natural layout
# --------------------------------------------------------------------------
def nat_to_qws_spinor(v, L, vlen):
    """natural [V,24] -> QWS scd_t/scs_t array [(2*vol), 24*vlen] (flattened)."""
    Lx, Ly, Lz, Lt = L
    nxh = Lx // 2
    a = np.asarray(v).reshape(Lt, Lz, Ly, 2, nxh // vlen, vlen, 24)
    a = a.transpose(3, 0, 1, 2, 4, 6, 5)  # dom,t,z,y,xv,comp,lane
    return np.ascontiguousarray(a).reshape(-1)


def qws_to_nat_spinor(q, L, vlen):
    Lx, Ly, Lz, Lt = L
    nxh = Lx // 2
    a = np.asarray(q).reshape(2, Lt, Lz, Ly, nxh // vlen, 24, vlen)
    a = a.transpose(1, 2, 3, 0, 4, 6, 5)  # t,z,y,dom,xv,lane,comp
    return np.ascontiguousarray(a).reshape(-1, 24)


def nat_to_qws_gauge(U, L, vlen):
    """natural [4,V,3row,3col,2] -> QWS glu array [dom][mu][t][z][y][xv] c[col][row][ri][lane]."""
    Lx, Ly, Lz, Lt = L
    nxh = Lx // 2
    a = np.asarray(U).reshape(4, Lt, Lz, Ly, 2, nxh // vlen, vlen, 3, 3, 2)
    a = a.transpose(4, 0, 1, 2, 3, 5, 8, 7, 9, 6)  # dom,mu,t,z,y,xv,col,row,ri,lane
    return np.ascontiguousarray(a).reshape(-1)


def nat_to_qws_clover(C, L, vlen):
    Lx, Ly, Lz, Lt = L
    nxh = Lx // 2
    a = np.asarray(C).reshape(Lt, Lz, Ly, 2, nxh // vlen, vlen, 72)
    a = a.transpose(3, 0, 1, 2, 4, 6, 5)
    return np.ascontiguousarray(a).reshape(-1)


# BQCD host layout (qws_bqcd.cc:66-642): site index i-1 = lex//2 inside its
# parity eo = (x+y+z+t)%2 (the default std_xyzt2i_/e_o_ of this library)
def _bqcd_slots(L):
    lex = np.arange(int(np.prod(L)))
    Lx, Ly, Lz, Lt = L
    x, y = lex % Lx, (lex // Lx) % Ly
    z, t = (lex // (Lx * Ly)) % Lz, lex // (Lx * Ly * Lz)
    return lex // 2, (x + y + z + t) % 2


# BQCD's 36 reals of one chiral block -> QWS packing index (qws_bqcd.cc:301-377)
BQCD_CLV_PERM = np.array([0, 1, 20, 21, 32, 33, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15,
                          16, 17, 18, 19, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 34, 35])


def nat_to_bqcd_gauge(U, L):
    """natural [4,V,(row,col,ri)] -> u[ri + 2 row + 6 col + 18 i + 18 volh eo + 36 volh mu]."""
    V = int(np.prod(L))
    i, eo = _bqcd_slots(L)
    out = np.zeros((4, 2, V // 2, 3, 3, 2))  # mu, eo, i, col, row, ri
    out[:, eo, i] = np.asarray(U).reshape(4, V, 3, 3, 2).transpose(0, 1, 3, 2, 4)
    return out.reshape(-1)


def nat_to_bqcd_clover(C, L):
    """natural [V,72] (QWS packing) -> c[perm[k] + 36 ud + 72 i + 72 volh eo]."""
    V = int(np.prod(L))
    i, eo = _bqcd_slots(L)
    out = np.zeros((2, V // 2, 2, 36))
    Cn = np.asarray(C).reshape(V, 2, 36)
    blk = np.zeros_like(Cn)
    blk[:, :, BQCD_CLV_PERM] = Cn
    out[eo, i] = blk
    return out.reshape(-1)


def nat_to_bqcd_spinor(v, L):
    """natural [V,24] -> (even, odd) arrays in[2 s + 8 c + ri + 24 i]."""
    V = int(np.prod(L))
    i, eo = _bqcd_slots(L)
    out = np.zeros((2, V // 2, 24))
    out[eo, i] = np.asarray(v).reshape(V, 24)
    return out[0].reshape(-1), out[1].reshape(-1)


def bqcd_to_nat_spinor(e, o, L):
    V = int(np.prod(L))
    i, eo = _bqcd_slots(L)
    both = np.stack([np.asarray(e).reshape(V // 2, 24), np.asarray(o).reshape(V // 2, 24)])
    return both[eo, i]


def aligned_empty(n, dtype, align=256):
    dtype = np.dtype(dtype)
    raw = np.empty(n * dtype.itemsize + align, np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off:off + n * dtype.itemsize].view(dtype)


# --------------------------------------------------------------------------
# the reference library (built from its sources)
# --------------------------------------------------------------------------
def ref_variant_path(variant):
    return REF_DIR / variant / "libqwsref.so"


class RefQWS:
    """Drives one process-global instance of the reference library.

    The reference keeps all state in globals (qws.cc:74-127), so one
    RefQWS per variant is alive at a time; lattice = one rank's local volume.
    """

    _loaded = {}

    def __init__(self, variant, L, tbc=-1, vlend=None, vlens=None):
        path = ref_variant_path(variant)
        if not path.exists():
            raise FileNotFoundError(path)
        if variant not in RefQWS._loaded:
            RefQWS._loaded[variant] = ctypes.CDLL(str(path), mode=os.RTLD_LOCAL)
        self.lib = lib = RefQWS._loaded[variant]
        tag = variant.split("_")[0]  # v8s16
        self.vlend = vlend or int(tag[1:tag.index("s")])
        self.vlens = vlens or int(tag[tag.index("s") + 1:])
        self.L = tuple(L)
        Lx, Ly, Lz, Lt = L
        self.V = Lx * Ly * Lz * Lt
        self._npe = iarr([1, 1, 1, 1])
        self._fbc = iarr([1, 1, 1, tbc])
        self._pce = ctypes.c_int(0)
        self._pco = ctypes.c_int(1)
        self._bs = iarr([1, 2, 2, 2])
        args = [ctypes.byref(ctypes.c_int(v)) for v in L]
        lib.qws_init_(*args, self._npe, self._fbc, ctypes.byref(self._pce),
                      ctypes.byref(self._pco), self._bs)
        self.vold = ctypes.c_int.in_dll(lib, "vold").value
        self.vols = ctypes.c_int.in_dll(lib, "vols").value

    def set_kappa(self, k):
        self.lib.ref_set_kappa(ctypes.c_double(k))

    def _global_ptr(self, name):
        return ctypes.c_void_p.in_dll(self.lib, name).value

    def set_fields(self, U, C):
        """U natural double [4,V,18]; C natural double [V,72]; FP32 copies are casts."""
        for name, arr in (("glud", nat_to_qws_gauge(U, self.L, self.vlend)),
                          ("clvd", nat_to_qws_clover(C, self.L, self.vlend))):
            ctypes.memmove(self._global_ptr(name), arr.ctypes.data, arr.nbytes)
        for name, arr in (("glus", nat_to_qws_gauge(U, self.L, self.vlens).astype(np.float32)),
                          ("clvs", nat_to_qws_clover(C, self.L, self.vlens).astype(np.float32))):
            ctypes.memmove(self._global_ptr(name), arr.ctypes.data, arr.nbytes)

    # spinor helpers ---------------------------------------------------------
    def to_d(self, v):
        q = nat_to_qws_spinor(v, self.L, self.vlend)
        buf = aligned_empty(q.size, np.float64)
        buf[:] = q
        return buf

    def to_s(self, v):
        q = nat_to_qws_spinor(np.asarray(v, np.float32), self.L, self.vlens)
        buf = aligned_empty(q.size, np.float32)
        buf[:] = q
        return buf

    def from_d(self, q):
        return qws_to_nat_spinor(q, self.L, self.vlend)

    def from_s(self, q):
        return qws_to_nat_spinor(q, self.L, self.vlens)

    def call(self, name, *args):
        fn = getattr(self.lib, name)
        conv = []
        for a in args:
            if isinstance(a, np.ndarray):
                conv.append(ctypes.c_void_p(a.ctypes.data))
            elif isinstance(a, float):
                conv.append(ctypes.c_float(a))
            else:
                conv.append(a)
        fn(*conv)

    def finalize(self):
        self.lib.qws_finalize_()


def parse_golden(text):
    """check.sh's extraction: lines `name : value` and `name^2 = value`."""
    import re
    out = []
    for line in text.splitlines():
        if "git commit hash" in line:
            continue
        if re.search(r" : +[0-9]|2 += +[0-9]", line):
            parts = line.split()
            out.append((parts[0], float(parts[-1])))
    return out


def check_sh_ok(name, val, ref):
    """check.sh:17-26 tolerances."""
    if name == "rnorm^2":
        return val < 1e-15
    d = abs(val - ref)
    if name.endswith("_s_") or name.endswith("_s"):
        return d / val < 3e-6
    return d / val < 1e-14


# --------------------------------------------------------------------------
# even-odd reading of QWS's arrays
# --------------------------------------------------------------------------
def eo_perm(L):
    """QWS stores even-odd fields in the same array shapes as DD fields
    (deo_in_d.cc:65-86: parity p at the slot of x-half p, compressed index
    x_eo = x // 2 at the slot of x_half).  main.cc fills its arrays with the DD
    generator and then reads them with both operator families, so the field
    an even-odd operator sees at site (x, y, z, t) is the DD field at
    (p*nx/2 + x//2, y, z, t) with p = (x+y+z+t) % 2.  Returns that map as an
    index array over natural site numbers."""
    Lx, Ly, Lz, Lt = L
    t, z, y, x = np.meshgrid(np.arange(Lt), np.arange(Lz), np.arange(Ly), np.arange(Lx),
                             indexing="ij")
    p = (x + y + z + t) % 2
    xd = p * (Lx // 2) + x // 2
    return (xd + Lx * (y + Ly * (z + Lz * t))).reshape(-1)


def eo_partner(L):
    """site of the other parity with the same compressed index: where a
    half-array argument of one parity aliases the other parity's half
    (e.g. in0 = in in main.cc:593-611)."""
    Lx, Ly, Lz, Lt = L
    t, z, y, x = np.meshgrid(np.arange(Lt), np.arange(Lz), np.arange(Ly), np.arange(Lx),
                             indexing="ij")
    p = (x + y + z + t) % 2
    xo = 2 * (x // 2) + (1 - p + y + z + t) % 2
    return (xo + Lx * (y + Ly * (z + Lz * t))).reshape(-1)


def parity_mask(L, p):
    Lx, Ly, Lz, Lt = L
    t, z, y, x = np.meshgrid(np.arange(Lt), np.arange(Lz), np.arange(Ly), np.arange(Lx),
                             indexing="ij")
    return ((x + y + z + t) % 2 == p).reshape(-1)
