"""QWS host layouts (qws.h:111-192) from and to the natural layout, in numpy.

Natural layout: site n = x + Lx*(y + Ly*(z + Lz*t)); spinor [n][24] with the
24 reals ordered [colour][spin][re,im]; gauge [mu][n][row][col][re,im];
clover [n][72] in QWS's packed chiral order.  QWS's arrays (what the
drop-in entry points of include/qws_dropin.h take) split the lattice into
two x-halves ("domains") and store `vlen` consecutive x sites as SIMD lanes
(scd_t: vlen = VLEND, scs_t: vlen = VLENS):

  spinor  [dom][t][z][y][x/vlen][24][lane]
  gauge   [dom][mu][t][z][y][x/vlen][col][row][re,im][lane]
  clover  [dom][t][z][y][x/vlen][72][lane]

These converters are for callers that hold natural-layout fields (tests,
the benchmark); a QWS program already holds its arrays in this layout.
"""
from __future__ import annotations

import numpy as np


def aligned_empty(n, dtype, align=256):
    """n elements of dtype on an `align`-byte boundary (QWS's CLS alignment)."""
    dtype = np.dtype(dtype)
    raw = np.empty(n * dtype.itemsize + align, np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off:off + n * dtype.itemsize].view(dtype)


def _check(L, vlen):
    if L[0] % 2 or (L[0] // 2) % vlen:
        raise ValueError(f"x extent {L[0]} must split into two halves of whole {vlen}-site vectors")


def nat_to_qws_spinor(v, L, vlen, out=None):
    """natural [V, 24] -> flat QWS spinor array (2*vol elements of 24*vlen reals)."""
    _check(L, vlen)
    Lx, Ly, Lz, Lt = L
    a = np.asarray(v).reshape(Lt, Lz, Ly, 2, Lx // 2 // vlen, vlen, 24)
    a = a.transpose(3, 0, 1, 2, 4, 6, 5)
    if out is None:
        return np.ascontiguousarray(a).reshape(-1)
    out.reshape(a.shape)[...] = a
    return out


def qws_to_nat_spinor(q, L, vlen):
    _check(L, vlen)
    Lx, Ly, Lz, Lt = L
    a = np.asarray(q).reshape(2, Lt, Lz, Ly, Lx // 2 // vlen, 24, vlen)
    return np.ascontiguousarray(a.transpose(1, 2, 3, 0, 4, 6, 5)).reshape(-1, 24)


def nat_to_qws_gauge(U, L, vlen):
    """natural [4, V, 3, 3, 2] -> flat QWS gauge array (glud_t / glus_t)."""
    _check(L, vlen)
    Lx, Ly, Lz, Lt = L
    a = np.asarray(U).reshape(4, Lt, Lz, Ly, 2, Lx // 2 // vlen, vlen, 3, 3, 2)
    a = a.transpose(4, 0, 1, 2, 3, 5, 8, 7, 9, 6)
    return np.ascontiguousarray(a).reshape(-1)


def nat_to_qws_clover(C, L, vlen):
    """natural [V, 72] -> flat QWS clover array (clvd_t / clvs_t)."""
    _check(L, vlen)
    Lx, Ly, Lz, Lt = L
    a = np.asarray(C).reshape(Lt, Lz, Ly, 2, Lx // 2 // vlen, vlen, 72)
    return np.ascontiguousarray(a.transpose(3, 0, 1, 2, 4, 6, 5)).reshape(-1)
