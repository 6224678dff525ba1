"""Single applications of every kernel the SAP preconditioner is made of,
in FP32 and in FP16 storage, each against the FP64 oracle with a stated
error bound -- the counterpart of the reference's own per-operator check of
its half-precision kernels (debug_half, prec_ddd_s_h.h:279-387, which
compares the FP16 D_block, A^-1_block and D_eo with FP32 at 1e-5).

Fields: seeded SU(3) links after 2 smoothing steps, clover-leaf clover at
csw 1.7, kappa 0.1365, an 8x8x8x16 lattice cut into SAP blocks of 4x4x4x8
(many faces) and at the reference's one-rank partition (2,1,1,1).

Operators (o = colour of the blocks handled, K = kappa A^-1 H_blk):
  D_blk      out_o = in_o - K in_o                (ddd_in_*, qws.cc / ddd_in_h.h:54)
  J (nm=2)   x_0 = b, x_k = b + K x_{k-1}          (jinv_ddd_in_*, static_solver.cc:65)
  face       out += f A^-1 H_face in, face sites  (ddd_out_pre/pos_*, ddd_out_h.h:57,283)
  SAP update s_o += in_o - D_blk a_o               (qws.cc:815-818, prec_ddd_s_h.h:143-150)

FP16 storage (IO<H16>): a spinor site is stored as FP16 values of v / n with
n = max_i |v_i| (FP32), links and clover as FP16 values of their FP32 copies;
the arithmetic is FP32.  Two checks per operator:

1. The kernel computes the rounded operator: a CPU emulation of the format
   (round-to-nearest-even FP16 of the same FP32 quantities, numpy) run through
   the FP64 oracle must agree with the GPU component by component to one FP16
   ulp of the site's scale, 2^-10 n (a component may round to the other
   neighbour when the FP32 arithmetic moves it across a rounding boundary),
   and to 2^-20 (16 FP32 roundoffs) in norm.

2. The error of the FP16 operator against the exact FP64 one is inside a
   first-order bound in units of u16 = 2^-11, the binary16 unit roundoff:
     - a stored spinor has componentwise relative error <= u16 (FP16 values of
       v/n, |v/n| <= 1; components below 2^-14 n lose relative accuracy but
       carry a negligible share of the norm): ||dv|| <= u16 ||v||;
     - an SU(3) link rounded entrywise has ||dU||_2 <= ||dU||_F <= u16 ||U||_F
       = sqrt(3) u16; a 6x6 clover block rounded entrywise has
       ||dM||_2 <= u16 ||M||_F <= sqrt(6) u16 ||M||_2;
     - ||H|| <= 8 for unitary links (four directions, each a sum of the two
       complementary projections (1 -+ gamma) of norm 2), so with
       a = max ||A^-1||_2 over the lattice, ||K|| <= 8 kappa a and its
       rounding moves it by at most c_K u16 with c_K = 8 kappa a (sqrt(3)+sqrt(6));
     - FP32 arithmetic adds O(2^-24) per operation: 0.02 u16 for the ~30-term
       chains of one site, included as a constant 0.05 u16 ||out||.
   D_blk:  ||d out|| <= u16 [(1 + 8 kappa a + c_K) ||in|| + ||out||]
   face:   ||d out|| <= u16 [||out_0|| + |f| 8 a (1 + sqrt(3) + sqrt(6)) ||in|| + ||out||]
   update: ||d s||   <= u16 [||s_0|| + ||in|| + (1 + 8 kappa a + c_K) ||a|| + ||s||]
   J:      e_0 = u16 ||b||, e_k = u16 ||b|| + 8 kappa a e_{k-1} + c_K u16 ||x_{k-1}||
           + u16 ||x_k|| (each step reads the stored b and x_{k-1} and stores x_k).
   These worst-case bounds are 10-45 u16 relative here (a = max ||A^-1||
   is 2.2 at csw 1.7 on these fields, and every term is taken at its
   maximum).  The typical size is far smaller: a round-to-nearest relative
   error is spread over [-u16, u16] (RMS u16/sqrt(3)) independently per
   component, so the errors add in quadrature and the storage of the input
   and of the output dominate, each ~0.58 u16 of its norm: about 0.8 u16 for
   D_blk, the face and the update, about 1.1 u16 for two Richardson steps
   (three stored fields).  Each FP16 operator is also held to TYPICAL (below)
   -- 1 u16, 1.5 u16 for J -- which the format itself meets at 0.5-0.66 u16
   (test_fp16_format_error_within_bound, CPU).

The FP32 kernels are checked against the FP64 oracle the same way with
u32 = 2^-24: their operands are the FP32 roundings of the FP64 fields and
spinors (same first-order terms as above with u32; an SU(3) link read in its
12-real form has its third row rebuilt, ||dU|| <= 3 sqrt(3) u32), plus 40 u32
for the FP32 arithmetic along a site's chain (projection, 3x3 complex
product, eight-hop sum, 6x6 complex clover product, epilogue), i.e. the FP16
bounds with u16 replaced by u32 and the arithmetic constant 0.05 by 40.
"""
import numpy as np
import pytest

import qws_b200
from qwsref import Oracle

L = (8, 8, 8, 16)
KAPPA, CSW = 0.1365, 1.7
U16, U32 = 2.0 ** -11, 2.0 ** -24
S3, S6 = np.sqrt(3.0), np.sqrt(6.0)
# typical-size bound of each FP16 operator's relative error, in u16 (docstring)
TYPICAL = {"dblk": 1.0, "jinv": 1.5, "face": 1.0, "update": 1.0}


# --------------------------------------------------------------------------
# emulation of the FP16 storage format (IO<H16> in qws_b200/csrc/lattice.cuh)
# --------------------------------------------------------------------------
def store16(v):
    """A spinor field [V, 24] as the FP16 kernels store and read it back (FP32
    values): n = max |v_i| per site, FP16 of v * (1/n) in FP32, times n."""
    v32 = np.asarray(v, np.float32)
    n = np.abs(v32).max(axis=1, keepdims=True)
    keep = n >= np.float32(1e-30)
    inv = np.where(keep, np.float32(1) / np.where(keep, n, 1), np.float32(0)).astype(np.float32)
    h = (v32 * inv).astype(np.float16).astype(np.float32)
    return (h * np.where(keep, n, 0).astype(np.float32)).astype(np.float64)


def field16(a):
    """links / clover: FP16 of the FP32 copy of the FP64 field"""
    return np.asarray(a).astype(np.float32).astype(np.float16).astype(np.float64)


def colour_mask(NB, colour):
    B = [l // n for l, n in zip(L, NB)]
    x, y, z, t = np.meshgrid(*[np.arange(l) for l in L], indexing="ij")
    col = (x // B[0] + y // B[1] + z // B[2] + t // B[3]) % 2
    return col.transpose(3, 2, 1, 0).reshape(-1) == colour


def clover_inverse_norm(C):
    """max over sites and chiral blocks of ||A^-1||_2 = 2 ||M|| (the packed
    block M holds half the inverse: the kernel applies 2 M, see
    qws_b200/csrc/fields.cu)"""
    C = np.asarray(C).reshape(-1, 2, 36)
    M = np.zeros(C.shape[:2] + (6, 6), complex)
    idx = np.arange(6)
    M[..., idx, idx] = C[..., :6]
    n = 0
    for j in range(6):
        for k in range(j + 1, 6):
            M[..., j, k] = C[..., 6 + 2 * n] + 1j * C[..., 7 + 2 * n]
            M[..., k, j] = np.conj(M[..., j, k])
            n += 1
    return 2 * float(np.abs(np.linalg.eigvalsh(M)).max())


@pytest.fixture(scope="module", params=[(2, 2, 2, 2), (2, 1, 1, 1)], ids=["blocks4x4x4x8", "ref"])
def setup(request):
    NB = request.param
    U, _ = qws_b200.gen_gauge(L, seed=21, n_smear=2, alpha=0.36)
    C = qws_b200.gen_clover(U, L, CSW, KAPPA)
    exact = Oracle(L, NB, tbc=-1, kappa=KAPPA)
    exact.set_fields(U, C)
    rounded = Oracle(L, NB, tbc=-1, kappa=KAPPA)  # FP16-rounded fields
    rounded.set_fields(field16(U), field16(C))
    rng = np.random.default_rng(5)
    V = int(np.prod(L))
    vecs = [rng.standard_normal((V, 24)) for _ in range(3)]
    a = clover_inverse_norm(C)
    return dict(NB=NB, U=U, C=C, exact=exact, rounded=rounded, vecs=vecs, a=a)


# --------------------------------------------------------------------------
# the four operators through the oracle (FP64), exact and on the rounded format
# --------------------------------------------------------------------------
def op_dblk(o, x, col, q=lambda v: v):
    out = o.ddd_in_d(q(x), 0, col)
    return q(out)


def op_jinv(o, b, col, nm, q=lambda v: v):
    bq = q(b)
    x = bq
    for _ in range(max(nm, 1)):
        x = q(bq + x - o.ddd_in_d(x, 0, col))
    return x


def op_face(o, x, out0, col, f, q=lambda v: v):
    out = q(out0).copy()
    o.ddd_out_d(q(x), 0, col, f, out=out)
    return q(out)


def op_update(o, s0, a, rhs, col, q=lambda v: v):
    return q(q(s0) + q(rhs) - o.ddd_in_d(q(a), 0, col))


def nrm(v, m):
    return float(np.linalg.norm(np.asarray(v)[m]))


def bounds(S, col, u, arith, c_link=S3):
    """first-order error bounds (absolute, in the norm over colour `col`)
    of the four operators for roundoff u; arith: the arithmetic term's
    factor; c_link: ||dU||_2 / u of one stored link"""
    o, (x, y, z) = S["exact"], S["vecs"]
    m = colour_mask(S["NB"], col)
    kn = 8 * KAPPA * S["a"]
    cK = 8 * KAPPA * S["a"] * (c_link + S6)
    d = op_dblk(o, x, col)
    b_dblk = u * ((1 + kn + cK) * nrm(x, m) + (1 + arith) * nrm(d, m))
    f = KAPPA
    fo = op_face(o, x, y, col, f)
    # the face hops read the other colour's sites
    b_face = u * (nrm(y, m) + abs(f) * 8 * S["a"] * (1 + c_link + S6) * nrm(x, ~m) +
                  (1 + arith) * nrm(fo, m))
    up = op_update(o, y, x, z, col)
    b_up = u * (nrm(y, m) + nrm(z, m) + (1 + kn + cK) * nrm(x, m) + (1 + arith) * nrm(up, m))
    e = u * nrm(x, m)
    xk = x
    for _ in range(2):
        xn = x + xk - o.ddd_in_d(xk, 0, col)
        e = u * nrm(x, m) + kn * e + cK * u * nrm(xk, m) + (1 + arith) * u * nrm(xn, m)
        xk = xn
    return {"dblk": b_dblk, "face": b_face, "update": b_up, "jinv": e}


def exact_results(S, col):
    o, (x, y, z) = S["exact"], S["vecs"]
    return {"dblk": op_dblk(o, x, col), "jinv": op_jinv(o, x, col, 2),
            "face": op_face(o, x, y, col, KAPPA), "update": op_update(o, y, x, z, col)}


def rounded_results(S, col):
    o, (x, y, z) = S["rounded"], S["vecs"]
    q = store16
    return {"dblk": op_dblk(o, x, col, q), "jinv": op_jinv(o, x, col, 2, q),
            "face": op_face(o, x, y, col, KAPPA, q), "update": op_update(o, y, x, z, col, q)}


@pytest.mark.parametrize("col", [0, 1])
def test_fp16_format_error_within_bound(setup, col):
    """CPU only: the emulated FP16 operators against the exact FP64 ones,
    inside the first-order bounds of the module docstring."""
    m = colour_mask(setup["NB"], col)
    ex, rd = exact_results(setup, col), rounded_results(setup, col)
    bd = bounds(setup, col, U16, 0.05)
    for k in ex:
        err = nrm(rd[k] - ex[k], m)
        assert err <= bd[k], (k, err / nrm(ex[k], m) / U16, bd[k] / nrm(ex[k], m) / U16)
        assert err <= TYPICAL[k] * U16 * nrm(ex[k], m), (k, err / nrm(ex[k], m) / U16)
        assert err > 0.05 * U16 * nrm(ex[k], m), k  # the rounding is really there


def gpu_results(S, lat, col, half):
    x, y, z = S["vecs"]
    dev = lambda v: lat.to_device(np.asarray(v, np.float32))
    host = lat.to_host
    if half:
        return {"dblk": host(lat.ddd_in_h(dev(x), col, out=dev(np.zeros_like(x)))),
                "jinv": host(lat.jinv_h(dev(x), col, 2, out=dev(np.zeros_like(x)))),
                "face": host(lat.ddd_out_h(dev(x), col, KAPPA, out=dev(y))),
                "update": host(lat.sap_update(dev(y), dev(x), dev(z), col, half=True))}
    return {"dblk": host(lat.ddd_in(dev(x), col, out=dev(np.zeros_like(x)))),
            "jinv": host(lat.jinv(dev(x), col, 2, out=dev(np.zeros_like(x)))),
            "face": host(lat.ddd_out(dev(x), col, KAPPA, out=dev(y))),
            "update": host(lat.sap_update(dev(y), dev(x), dev(z), col, half=False))}


@pytest.fixture(scope="module")
def lattice(setup):
    lat = qws_b200.Lattice(L, setup["NB"], tbc=-1, kappa=KAPPA)
    lat.load_fields(setup["U"], setup["C"])
    yield lat
    lat.close()


@pytest.mark.gpu
@pytest.mark.parametrize("col", [0, 1])
def test_fp16_kernels_compute_the_rounded_operator(setup, lattice, col):
    m = colour_mask(setup["NB"], col)
    rd = rounded_results(setup, col)
    got = gpu_results(setup, lattice, col, half=True)
    for k in rd:
        g, e = got[k][m], rd[k][m]
        n = np.abs(e).max(axis=1, keepdims=True)
        assert (np.abs(g - e) <= 2.0 ** -10 * n + 1e-6 * np.abs(e)).all(), k
        assert nrm(g - e, slice(None)) <= 2.0 ** -20 * nrm(e, slice(None)) * 64, k


@pytest.mark.gpu
@pytest.mark.parametrize("col", [0, 1])
def test_fp16_kernels_error_in_units_of_u16(setup, lattice, col):
    m = colour_mask(setup["NB"], col)
    ex = exact_results(setup, col)
    got = gpu_results(setup, lattice, col, half=True)
    bd = bounds(setup, col, U16, 0.05)
    for k in ex:
        err = nrm(got[k] - ex[k], m)
        print(f"fp16 {setup['NB']} colour {col} {k}: {err / nrm(ex[k], m) / U16:.3f} u16 "
              f"(bound {bd[k] / nrm(ex[k], m) / U16:.1f}, typical {TYPICAL[k]})")
        assert err <= bd[k], (k, err / nrm(ex[k], m) / U16, bd[k] / nrm(ex[k], m) / U16)
        assert err <= TYPICAL[k] * U16 * nrm(ex[k], m), (k, err / nrm(ex[k], m) / U16)


@pytest.mark.gpu
@pytest.mark.parametrize("col", [0, 1])
def test_fp32_kernels_error_in_units_of_u32(setup, lattice, col):
    """The FP32 block, Richardson, face and SAP-update kernels against the
    FP64 oracle (the face kernel ddd_out_pre/pos_s_ had no test of its own)."""
    m = colour_mask(setup["NB"], col)
    ex = exact_results(setup, col)
    got = gpu_results(setup, lattice, col, half=False)
    # 12-real links (SU(3) fields): the third row is rebuilt from the two
    # stored rounded rows, each of its entries a difference of two products:
    # <= 4 u32 per entry, ||dU||_F <= u32 sqrt(6 + 3 * 16) < 3 sqrt(3) u32
    bd = bounds(setup, col, U32, 40.0, c_link=3 * S3)
    for k in ex:
        err = nrm(got[k] - ex[k], m)
        print(f"fp32 {setup['NB']} colour {col} {k}: {err / nrm(ex[k], m) / U32:.2f} u32 "
              f"(bound {bd[k] / nrm(ex[k], m) / U32:.1f})")
        assert err <= bd[k], (k, err / nrm(ex[k], m) / U32, bd[k] / nrm(ex[k], m) / U32)


@pytest.mark.gpu
def test_fp16_pair_kernels_equal_single_rhs(setup, lattice):
    """Two RHS on one handle run the packed two-RHS kernels (k_hop_pair); each
    RHS is bit-equal to the one-RHS kernel's result."""
    x, y, z = setup["vecs"]
    B = lattice.batch(2)
    try:
        dev2 = lambda a, b: B.to_device(np.stack([a, b]).astype(np.float32))
        for col in (0, 1):
            pairs = {
                "dblk": B.to_host(B.ddd_in_h(dev2(x, y), col, out=dev2(0 * x, 0 * x))),
                "jinv": B.to_host(B.jinv_h(dev2(x, y), col, 2, out=dev2(0 * x, 0 * x))),
                "face": B.to_host(B.ddd_out_h(dev2(x, z), col, KAPPA, out=dev2(y, x))),
                "update": B.to_host(B.sap_update(dev2(y, z), dev2(x, y), dev2(z, x), col,
                                                 half=True)),
            }
            single = gpu_results(setup, lattice, col, half=True)
            for k in pairs:
                np.testing.assert_array_equal(pairs[k][0], single[k], err_msg=k)
    finally:
        B.close()


@pytest.mark.gpu
@pytest.mark.parametrize("nr", [1, 2])
def test_fp16_storage_bit_exact(setup, lattice, nr):
    """The FP16 storage format itself, bit for bit (the counterpart of the
    reference's fp16 conversion dump, testhf.cc): a field stored and read
    back by the device (qwsg_store_h, one and two RHS per handle) equals the
    numpy emulation store16 exactly -- FP32 site maximum, FP32 reciprocal and
    products, round-to-nearest-even FP16.  Site magnitudes span 70 decades;
    one component per site is a million times below the site's maximum
    (FP16 subnormals), one site is zero and one is FP32-denormal (both
    stored as zero)."""
    V = int(np.prod(L))
    rng = np.random.default_rng(9 + nr)
    v = rng.standard_normal((nr, V, 24)) * 10.0 ** rng.uniform(-35, 35, (nr, V, 1))
    v[..., 5] *= 1e-6
    v[:, 0] = 0.0
    v[:, 1] = 1e-40
    v = v.astype(np.float32)
    want = store16(v.reshape(-1, 24)).astype(np.float32).reshape(v.shape)
    assert np.isfinite(want).all()
    h = lattice if nr == 1 else lattice.batch(nr)
    try:
        x = h.to_device(v[0] if nr == 1 else v)
        got = h.to_host(h.store_h(x)).reshape(v.shape)
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
        assert not got[:, :2].any()
    finally:
        if h is not lattice:
            h.close()
