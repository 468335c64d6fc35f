"""Precision of the z pass's operand splits (CPU model).

The wide z kernel multiplies the fixed-point tile by the z twiddles as f16
head + rounded remainder of both operands (kind::f16 MMAs, FP32 accumulation,
all four products); the other tensor-core passes use 3xTF32 (TF32 head with
the low 13 mantissa bits cleared plus the FP32 remainder, three products).  This
model of one item's GEMM (128 z x 21 kz, sparse tile values around the padding
mean, in the kernel's fixed-point units and 2^-17 scaling) checks that both
stay within 5e-7 of the largest FP64 result and that the f16 form is no less
accurate than 3xTF32.
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
