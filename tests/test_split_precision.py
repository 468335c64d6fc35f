"""Precision of the z pass's operand splits (CPU model).

The wide z kernel multiplies the fixed-point tile by the z twiddles as f16
head + rounded remainder of both operands (kind::f16 MMAs, FP32 accumulation,
all four products); the other tensor-core passes use 3xTF32 (TF32 head with
the low 13 mantissa bits cleared plus the FP32 remainder, three products).  This
model of one item's GEMM (128 z x 21 kz, sparse tile values around the padding
mean, in the kernel's fixed-point units and 2^-17 scaling) checks that both
stay within 5e-7 of the largest FP64 result and that the f16 form is no less
accurate than 3xTF32; a box-wide model checks the lowest-q amplitude, for which
the mean must be subtracted inside the tile.
"""
import numpy as np


def _tf32(x):
    return (x.view(np.uint32) & np.uint32(0xFFFFE000)).view(np.float32)


def _f32(x):
    return x.astype(np.float32)


def test_f16_split_matches_3xtf32_precision():
    rng = np.random.default_rng(3)
    scale, mean = 2.0 ** 23, 0.03
    v = rng.exponential(0.03, size=(1024, 128)) * (rng.random((1024, 128)) < 0.5)
    i = np.rint(v * scale).astype(np.int64)
    z = np.arange(128)
    kz = np.arange(21)
    tw = np.cos(2 * np.pi * np.outer(z, kz) / 256)
    exact = (i / scale - mean) @ tw

    # f16: (i - mean * scale) * 2^-17, head and rounded remainder of both operands
    a = _f32((i.astype(np.float32) - np.float32(mean * scale)) * np.float32(2.0 ** -17))
    ah = a.astype(np.float16)
    al = (a - ah.astype(np.float32)).astype(np.float16)
    b = _f32(tw)
    bh = b.astype(np.float16)
    bl = (b - bh.astype(np.float32)).astype(np.float16)
    d = (_f32(ah) @ _f32(bh) + _f32(ah) @ _f32(bl)) + (_f32(al) @ _f32(bh) + _f32(al) @ _f32(bl))
    z16 = d.astype(np.float64) * 2.0 ** 17 / scale

    # 3xTF32 on the real-valued tile
    a2 = _f32(i.astype(np.float32) / np.float32(scale) - np.float32(mean))
    a2h = _tf32(a2)
    a2l = _tf32(_f32(a2 - a2h))
    b2h = _tf32(b)
    b2l = _tf32(_f32(b - b2h))
    z32 = (a2h @ b2h + a2h @ b2l + a2l @ b2h).astype(np.float64)

    top = np.abs(exact).max()
    e16 = np.abs(z16 - exact).max() / top
    e32 = np.abs(z32 - exact).max() / top
    assert e16 < 5e-7 and e32 < 5e-7, (e16, e32)
    assert e16 <= 1.2 * e32, (e16, e32)


def _gemm16(a, tw):
    """f16 head + rounded remainder of both operands, four products, FP32."""
    ah = a.astype(np.float16)
    al = (a - ah.astype(np.float32)).astype(np.float16)
    b = _f32(tw)
    bh = b.astype(np.float16)
    bl = (b - bh.astype(np.float32)).astype(np.float16)
    return _f32((_f32(ah) @ _f32(bh) + _f32(ah) @ _f32(bl)) + (_f32(al) @ _f32(bh) + _f32(al) @ _f32(bl)))


def test_mean_inside_the_tile_keeps_lowest_q_amplitude():
    # The lowest-q amplitude sums Z over every column of the box.  With the
    # padding mean subtracted inside the tile (as the wide z kernel does) the FP32
    # accumulation works on rho - mean and its rounding averages out over the
    # columns; subtracting mean * sum_z tw after the transform instead leaves each
    # column's FP32 sum of the positive density ~mean * |sum_z tw| large, and the
    # box-wide sum several times less accurate.  A uniform 64-z system of 4096
    # columns, kz = 1 of a 128 supercell.
    errs_in, errs_after = [], []
    for seed in range(3):
        rng = np.random.default_rng(11 + seed)
        scale, ez, nz = 2.0 ** 23, 64, 128
        rho = rng.poisson(0.11 * 8, size=(4096, ez)) / 8.0
        mean = np.float32(rho.mean())
        i = np.rint(rho * scale).astype(np.int64)
        z = np.arange(ez)
        tw = np.stack([np.cos(2 * np.pi * z / nz), -np.sin(2 * np.pi * z / nz)], axis=1)
        exact = ((i / scale - np.float64(mean)) @ tw).sum(axis=0)
        top = np.abs(exact).max()
        x_in = _f32((i.astype(np.float32) - np.float32(mean * scale)) * np.float32(2.0 ** -17))
        z_in = _gemm16(x_in, tw).astype(np.float64) * 2.0 ** 17 / scale
        x_pos = _f32(i.astype(np.float32) * np.float32(2.0 ** -17))
        z_after = _gemm16(x_pos, tw).astype(np.float64) * 2.0 ** 17 / scale - np.float64(mean) * tw.sum(axis=0)
        errs_in.append(np.abs(z_in.sum(axis=0) - exact).max() / top)
        errs_after.append(np.abs(z_after.sum(axis=0) - exact).max() / top)
    assert max(errs_in) < 2e-6, errs_in
    assert min(e / f for e, f in zip(errs_after, errs_in)) > 3, (errs_after, errs_in)


def _f16_scale(m_t, ez, nx, ny, ey=None):
    """The kernels' power-of-two row scale of an f16 y (ey None) or x pass
    (dtc_f16_scale): bound = M_t + ez * M_t / (nx * ny) + 1, times ey for x."""
    bound = np.float32(m_t + m_t * ez / (nx * ny) + 1.0)
    if ey is not None:
        bound *= np.float32(ey)
    return np.float32(2.0 ** (14 - np.ceil(np.log2(bound))))


def _complex_gemm_operands(rows, extent, nk, nn, rng, amp):
    z = (rng.normal(0, amp, (rows, extent)) + 1j * rng.normal(0, amp, (rows, extent)))
    z[rng.random((rows, extent)) < 0.01] *= 50.0   # a few large columns
    u = np.arange(extent)
    k = np.arange(-(nk // 2), nk // 2 + 1)
    w = np.exp(-2j * np.pi * np.outer(u, k) / nn)
    a = np.stack([z.real, z.imag], axis=2).reshape(rows, 2 * extent)           # [r][2u + c]
    b = np.zeros((2 * extent, 2 * len(k)))                                    # {Wr, Wi; -Wi, Wr}
    b[0::2, 0::2], b[0::2, 1::2] = w.real, w.imag
    b[1::2, 0::2], b[1::2, 1::2] = -w.imag, w.real
    return a, b


def _split16(x):
    h = x.astype(np.float16)
    return h, (x - h.astype(np.float32)).astype(np.float16)


def test_f16_y_and_x_passes_match_3xtf32_precision():
    rng = np.random.default_rng(4)
    m_t = 60_000
    for name, ey, amp in (("y", None, 3.0), ("x", 128, 300.0)):
        a, b = _complex_gemm_operands(128, 128, 41, 256, rng, amp)
        exact = a @ b
        s = _f16_scale(m_t, 128, 128, 128, ey)
        a32 = _f32(a * s)
        assert np.abs(a32).max() < 2.0 ** 14
        ah, al = _split16(a32)
        bh, bl = _split16(_f32(b))
        f = lambda x: _f32(x)  # noqa: E731
        side = (f(ah) @ f(bh) + f(ah) @ f(bl)) + (f(al) @ f(bh) + f(al) @ f(bl))   # [Bh | Bl]
        three = f(al) @ f(bh) + f(ah) @ f(bl) + f(ah) @ f(bh)                   # separate blocks
        d_side = side.astype(np.float64) / s
        d_three = three.astype(np.float64) / s
        a2h = _tf32(_f32(a))
        a2l = _tf32(_f32(_f32(a) - a2h))
        b2h = _tf32(_f32(b))
        b2l = _tf32(_f32(_f32(b) - b2h))
        d32 = (a2h @ b2h + a2h @ b2l + a2l @ b2h).astype(np.float64)
        top = np.abs(exact).max()
        e_side = np.abs(d_side - exact).max() / top
        e_three = np.abs(d_three - exact).max() / top
        e32 = np.abs(d32 - exact).max() / top
        # (K' = 256 terms accumulated in FP32 bound all three forms near 1e-6)
        assert e_side < 2e-6 and e_three < 2e-6, (name, e_side, e_three, e32)
        assert max(e_side, e_three) <= 1.5 * e32 + 1e-8, (name, e_side, e_three, e32)
