"""CPU model of the tensor-core NUDFT's arithmetic (impatient-mri_b200/csrc/nudft_tc.cu):
the TF32 head/tail split of cos, sin and the coil data, the B-operand rows of the
head and tail accumulator columns, and the MMA's truncation of its 32-bit inputs to
TF32.  The products are summed exactly (float64) so that only the split's error is
measured: every product must match the FP64 complex multiply-add
    re = dx cos + dy sin,  im = dy cos - dx sin   (the k_nudft products,
    kernels/ftGpu.cu:306-604 / 756-1013 in the reference)
to the bound the kernel's header states (dropped lo*lo below 2^-22; tails rounded
or truncated to TF32 at most 2^-21 of the value)."""
import numpy as np


def tf32_rna(v):
    """Round float32 values to TF32 (10 mantissa bits), ties away from zero: the
    kernel's (bits + 0x1000) & 0xFFFFE000."""
    b = np.asarray(v, np.float32).view(np.uint32)
    return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def tf32_trunc(v):
    """The MMA's view of a 32-bit operand: the low 13 mantissa bits ignored."""
    b = np.asarray(v, np.float32).view(np.uint32)
    return (b & np.uint32(0xFFFFE000)).view(np.float32)


def split(v):
    v = np.asarray(v, np.float32)
    hi = tf32_rna(v)
    lo = (v - hi).astype(np.float32)  # exact in FP32
    return hi, lo


def tc_products(cs, sn, dx, dy):
    """(re, im) of one pair as the kernel's accumulator columns hold them."""
    ch, cl = split(cs)
    sh, sl = split(sn)
    A = np.stack([ch, sh, cl, sl], -1)  # K = 4 per element
    xh = tf32_rna(dx)
    yh = tf32_rna(dy)
    xl = tf32_rna((np.asarray(dx, np.float32) - xh).astype(np.float32))
    yl = tf32_rna((np.asarray(dy, np.float32) - yh).astype(np.float32))
    z = np.zeros_like(xh)
    rows = {  # B rows of the four columns of one coil
        "re_head": np.stack([xh, yh, xh, yh], -1),
        "im_head": np.stack([yh, -xh, yh, -xh], -1),
        "re_tail": np.stack([xl, yl, z, z], -1),
        "im_tail": np.stack([yl, -xl, z, z], -1),
    }
    At = tf32_trunc(A).astype(np.float64)
    col = {k: (At * tf32_trunc(b).astype(np.float64)).sum(-1) for k, b in rows.items()}
    return col["re_head"] + col["re_tail"], col["im_head"] + col["im_tail"]


def test_head_tail_split_reproduces_the_complex_multiply_add():
    rng = np.random.default_rng(0)
    n = 200000
    ang = rng.uniform(-np.pi, np.pi, n)
    cs = np.cos(ang).astype(np.float32)
    sn = np.sin(ang).astype(np.float32)
    mag = 10.0 ** rng.uniform(-8, 8, n)  # data over sixteen decades
    dx = (mag * rng.standard_normal(n)).astype(np.float32)
    dy = (mag * rng.standard_normal(n)).astype(np.float32)
    re, im = tc_products(cs, sn, dx, dy)
    c64, s64, x64, y64 = (a.astype(np.float64) for a in (cs, sn, dx, dy))
    re_ref = x64 * c64 + y64 * s64
    im_ref = y64 * c64 - x64 * s64
    scale = np.hypot(x64, y64)  # |d| |e|, |e| = 1
    err = np.maximum(np.abs(re - re_ref), np.abs(im - im_ref)) / scale
    assert err.max() < 2.0 ** -21, err.max()  # measured 2^-21.6
    assert np.sqrt(np.mean(err ** 2)) < 2.0 ** -23  # measured 2^-24.0


def test_without_tails_the_error_is_tf32_sized():
    """The tails matter: heads alone (one TF32 MMA) miss the bound by far."""
    rng = np.random.default_rng(1)
    n = 20000
    ang = rng.uniform(-np.pi, np.pi, n)
    cs = np.cos(ang).astype(np.float32)
    sn = np.sin(ang).astype(np.float32)
    dx = rng.standard_normal(n).astype(np.float32)
    dy = rng.standard_normal(n).astype(np.float32)
    re = (tf32_trunc(cs).astype(np.float64) * tf32_trunc(dx) +
          tf32_trunc(sn).astype(np.float64) * tf32_trunc(dy))
    ref = dx.astype(np.float64) * cs + dy.astype(np.float64) * sn
    err = np.abs(re - ref) / np.hypot(dx, dy)
    assert err.max() > 2.0 ** -14


def test_tf32_rounding_matches_the_bit_recipe():
    # ties away from zero on the 10-bit mantissa grid, sign symmetric
    one_plus_half_ulp = np.float32(1.0 + 2.0 ** -11)
    assert tf32_rna(one_plus_half_ulp) == np.float32(1.0 + 2.0 ** -10)
    assert tf32_rna(-one_plus_half_ulp) == -np.float32(1.0 + 2.0 ** -10)
    v = np.float32(1.0 + 2.0 ** -11 - 2.0 ** -23)
    assert tf32_rna(v) == np.float32(1.0)
    assert tf32_trunc(np.float32(1.0 + 2.0 ** -10 + 2.0 ** -12)) == np.float32(1.0 + 2.0 ** -10)
