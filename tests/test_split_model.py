"""Arithmetic of the split used by the tensor-core operator, modelled in
numpy on the CPU: the fixed-point leading parts make every K=32 slice of the
main product an exact FP32 number, and the parts sum back to the value.

The kernels (dage_b200/csrc/op3d_mixed.cu: lead_f32 / lead_f64,
split_lead_*) compute lead = rint(v 2^(7-E)) 2^(E-7) with 2^E >= max |v| of
a 32-run (data) or 1 (matrix rows scaled by a power of two >= their max);
bf16x3 keeps the floating lead bf16(v)."""
import numpy as np


def _bf16(x):
    """Round float32 to the nearest bfloat16 (ties to even), as float32."""
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def _lead(v, m):
    E = np.ceil(np.log2(np.where(m > 0, m, 1.0))).astype(int)
    return np.where(m > 0, np.rint(np.ldexp(v, 7 - E)) * np.ldexp(1.0, E - 7), 0.0)


def _split(v, m, nparts):
    """bf16x6 (3 parts): fixed-point lead; bf16x3 (2 parts): floating lead."""
    lead = _lead(v, m) if nparts > 2 else _bf16(v).astype(np.float64)
    parts = [np.asarray(lead, np.float32)]
    r = (v - lead).astype(np.float32)
    for _ in range(nparts - 1):
        p = _bf16(r)
        parts.append(p)
        r = (r - p).astype(np.float32)
    return parts


def test_lead_is_bf16_and_small_integer():
    rng = np.random.default_rng(0)
    x = (rng.standard_normal((64, 32)) * 10.0 ** rng.uniform(-20, 5, (64, 1))).astype(np.float32)
    m = np.abs(x).max(axis=1, keepdims=True)
    lead = _split(x, m, 3)[0]
    assert np.array_equal(_bf16(lead), lead)
    E = np.ceil(np.log2(m)).astype(int)
    j = np.ldexp(lead.astype(np.float64), 7 - E)
    assert np.array_equal(j, np.rint(j)) and np.abs(j).max() <= 128


def test_main_slice_exact_in_fp32():
    rng = np.random.default_rng(1)
    x = (rng.uniform(-1, 1, (16, 32)) * 10.0 ** rng.uniform(-8, 3, (16, 1))).astype(np.float32)
    t = rng.uniform(-1, 1, (32, 24))
    x0 = _split(x, np.abs(x).max(axis=1, keepdims=True), 3)[0].astype(np.float64)
    t0 = _split(t, np.ones_like(t), 3)[0].astype(np.float64)
    exact = x0 @ t0  # exact in FP64 (integers below 2^19 times one power of two)
    assert np.array_equal(exact.astype(np.float32).astype(np.float64), exact)


def test_parts_reconstruct():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((32, 32)).astype(np.float32)
    m = np.abs(x).max(axis=1, keepdims=True)
    s = sum(p.astype(np.float64) for p in _split(x, m, 3))
    assert np.abs(s - x).max() <= 2.0 ** -24 * m.max()
    s = sum(p.astype(np.float64) for p in _split(x, m, 2))
    assert np.all(np.abs(s - x) <= 2.0 ** -16 * np.abs(x))
