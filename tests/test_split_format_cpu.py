"""The split-precision number format of the tcgen05 chi0 contraction, restated in numpy.

Test infrastructure only: the CUDA kernels (split_quantize_kernel,
split_contract_kernel) are what ships; this file checks the format they
implement, on the CPU.
  * per chunk and operand element the scale 2^(46 - E), E the frexp exponent of
    the chunk's largest |Re|, |Im|; X = rint(x 2^(46 - E)), |X| <= 2^46;
  * six balanced base-256 digits, most significant first: with Y = X +
    0x8080808080 the low five are bytes 0..4 of Y minus 128 and the top one
    is Y >> 40, so X = d0 2^40 + d1 2^32 + d2 2^24 + d3 2^16 + d4 2^8 + d5;
  * the 21 digit products of levels l = i + j <= 5 summed per level in exact
    integers, recombined as sum_l S_l 2^(-12 - 8 l) 2^(E_A + E_B) (the same
    weights as a five-digit 38-bit format: the sixth digit only extends it).
The operands are Green functions of the synthetic sq2 system near the real
axis, in the layout of the contraction (A = w G1, B = G2^T per point), so the
error is that of the realistic sums the format was chosen on.
"""
import numpy as np

from oracle import titan_oracle as O
from titan_b200.host import synthetic
from titan_b200.host.system import initial_state

BITS = 46
NDIG = 6


def digits(X):
    """Balanced base-256 digits of int64 X (|X| <= 2^46), most significant first."""
    Y = X + 0x8080808080
    low = (Y & 0xFFFFFFFF).astype(np.uint32) ^ np.uint32(0x80808080)
    d = [(Y >> 40).astype(np.int64), (((Y >> 32) & 0xFF) ^ 0x80).astype(np.int8).astype(np.int64)]
    for sh in (24, 16, 8, 0):
        d.append(((low >> np.uint32(sh)) & np.uint32(0xFF)).astype(np.int64).astype(np.int8).astype(np.int64))
    return d


def quantise(x):
    """x [points, elements] real -> (digits, E per element) over the chunk (all points)."""
    m = np.max(np.abs(x), axis=0)
    E = np.where(m > 0, np.frexp(m)[1], 0)
    X = np.rint(np.ldexp(x, BITS - E[None, :])).astype(np.int64)
    assert np.max(np.abs(X)) <= 2 ** BITS
    return digits(X), E, X


def split_product(a, b, max_level=5, chunk=None):
    """sum_p a[p, u] b[p, v] for real a, b through the digit format (one scale per element
    and chunk of `chunk` points; None = one chunk)."""
    if chunk is not None and chunk < a.shape[0]:
        return sum(split_product(a[s:s + chunk], b[s:s + chunk], max_level)
                   for s in range(0, a.shape[0], chunk))
    da, Ea, _ = quantise(a)
    db, Eb, _ = quantise(b)
    # the digit products summed over the points stay below 2^14 npts < 2^53: float64 matrix
    # products are exact here and run on BLAS
    da = [x.astype(np.float64) for x in da]
    db = [x.astype(np.float64) for x in db]
    out = np.zeros((a.shape[1], b.shape[1]))
    for lvl in range(max_level + 1):
        S = np.zeros_like(out)
        for i in range(NDIG):
            j = lvl - i
            if 0 <= j < NDIG:
                S += da[i].T @ db[j]
        out += np.ldexp(S, -12 - 8 * lvl)
    return np.ldexp(out, Ea[:, None] + Eb[None, :])


def complex_split(A, B, max_level=5, chunk=None):
    rr = split_product(A.real, B.real, max_level, chunk)
    ii = split_product(A.imag, B.imag, max_level, chunk)
    ri = split_product(A.real, B.imag, max_level, chunk)
    ir = split_product(A.imag, B.real, max_level, chunk)
    return (rr - ii) + 1j * (ri + ir)


def operands(npts=96, y=2e-3):
    s = synthetic.make_system("sq2")
    m = O.Model(s, s.h0(initial_state(s)))
    rng = np.random.default_rng(5)
    k = rng.uniform(-0.5, 0.5, size=(npts, 3))
    k[:, 2] = 0.0
    z = s.Ef + 1j * y
    G2 = m.green(np.full(npts, z), k)
    G1 = m.green(np.full(npts, z + 0.05), k)
    w = rng.uniform(0.5, 1.5, size=npts) / npts
    # one site-pair block (site 0 rows, site 1 columns) of A = w G1 and B = G2^T
    n0 = s.norbs[0]
    r = np.r_[0:n0, n0:2 * n0]
    c = np.r_[2 * n0:2 * n0 + s.norbs[1], 2 * n0 + s.norbs[1]:2 * n0 + 2 * s.norbs[1]]
    A = (w[:, None, None] * G1[:, r][:, :, c]).reshape(npts, -1)
    B = np.transpose(G2, (0, 2, 1))[:, c][:, :, r].reshape(npts, -1)
    return A, B


def test_digits_reconstruct_exactly():
    rng = np.random.default_rng(0)
    X = rng.integers(-2 ** BITS, 2 ** BITS + 1, size=20000, dtype=np.int64)
    X[:4] = [2 ** BITS, -2 ** BITS, 0, -1]
    d = digits(X)
    assert all(np.all(np.abs(di) <= 128) for di in d[1:]) and np.all(np.abs(d[0]) <= 64)
    rec = d[0] * 2 ** 40 + d[1] * 2 ** 32 + d[2] * 2 ** 24 + d[3] * 2 ** 16 + d[4] * 2 ** 8 + d[5]
    assert np.array_equal(rec, X)
    # the level sums stay exact int32: at most six products of |d_i d_j| <= 2^14 per level
    assert 6 * 2 ** 14 * 16384 < 2 ** 31


def test_split_contraction_error_and_dropped_levels():
    A, B = operands()
    ref = A.T @ B
    err = np.linalg.norm(complex_split(A, B) - ref) / np.linalg.norm(ref)
    assert err < 1e-11, err
    # dropping level 5 (the digit products of level L = 7) costs accuracy the format cannot afford
    err6 = np.linalg.norm(complex_split(A, B, max_level=4) - ref) / np.linalg.norm(ref)
    assert err6 > 10 * err, (err, err6)


def test_short_chunks_bound_the_error_of_every_significant_entry():
    """Near the real axis (Im z = 2e-3) |G| varies by orders of magnitude along the k list:
    one scale per element and 128-point chunk keeps every entry holding at least 1e-4 of
    the largest within 1e-9 relative, where one 4096-point chunk does not."""
    A, B = operands(npts=4096)
    ref = A.T @ B
    big = np.abs(ref) >= 1e-4 * np.abs(ref).max()

    def worst(chunk):
        got = complex_split(A, B, chunk=chunk)
        return np.max(np.abs(got - ref)[big] / np.abs(ref)[big])

    short, long_ = worst(128), worst(4096)
    assert short < 1e-9, short
    assert long_ > 2 * short, (short, long_)


def test_exponent_sidecar_gives_the_quantiser_the_same_scale():
    """The spectral G kernel stores per value the exponent field of max(|Re|, |Im|) minus
    1022 (-32768 for zero or subnormal); the row maxima store 2^(E - 1) of the largest.
    That equals frexp's exponent of the true maximum, and 2^(E - 1) gives it back."""
    rng = np.random.default_rng(3)
    x = rng.standard_normal((4000, 2)) * np.exp(rng.uniform(-700, 700, size=(4000, 1)))
    x[:3] = [[0.0, 0.0], [5e-324, 0.0], [1.0, -1.0]]
    m = np.max(np.abs(x), axis=1)
    f = (m.view(np.int64) >> 52) & 0x7FF
    code = np.where(f == 0, -32768, f - 1022)
    normal = f != 0
    assert np.array_equal(code[normal], np.frexp(m[normal])[1])
    for chunk in np.array_split(np.arange(len(m)), 40):
        E = code[chunk].max()
        if E == -32768:
            continue
        stored = np.ldexp(1.0, int(E) - 1)
        assert np.frexp(stored)[1] == np.frexp(m[chunk].max())[1]


def test_error_bound_covers_every_entry():
    """The per-point bound behind tg_chi0_error_bound: rounding to 46 bits of the chunk scale
    plus the dropped digit products of levels i + j >= 6 stay within 6.02 2^(E_A + E_B - 46)
    per point and real product, so every entry of a chunked product lies within the sum of
    the bounds of its chunks (here with margin for the float64 reference's own rounding)."""
    A, B = operands(npts=512)
    chunk = 128
    for a, b in ((A.real, B.real), (A.imag, B.real), (A.real, B.imag), (A.imag, B.imag)):
        got = split_product(a, b, chunk=chunk)
        ref = a.T @ b
        bound = np.zeros_like(ref)
        for s0 in range(0, a.shape[0], chunk):
            _, Ea, _ = quantise(a[s0:s0 + chunk])
            _, Eb, _ = quantise(b[s0:s0 + chunk])
            live = np.outer(np.max(np.abs(a[s0:s0 + chunk]), axis=0) > 0, np.max(np.abs(b[s0:s0 + chunk]), axis=0) > 0)
            bound += np.where(live, chunk * 6.02 * np.ldexp(1.0, Ea[:, None] + Eb[None, :] - 46), 0.0)
        slack = 4e-16 * (np.abs(a).T @ np.abs(b))
        assert np.all(np.abs(got - ref) <= bound + slack)
        # and the bound is not vacuous: within three orders of the largest error
        assert np.max(np.abs(got - ref)) > 1e-3 * np.max(bound)
