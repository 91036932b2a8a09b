"""CPU checks of the integer bit tricks the pack/unpack kernels use
(begputhinning_b200/csrc/kernels.cu: nz4_to_bits, bytes4_to_bits,
bits4_to_bytes), restated in numpy on 32-bit words."""
import numpy as np

M32 = np.uint64(0xFFFFFFFF)


def bytes4_to_bits(cmp):
    return (((cmp & np.uint64(0x80808080)) * np.uint64(0x00204081)) & M32) >> np.uint64(28)


def nz4_to_bits(c):
    t = ((c & np.uint64(0x7F7F7F7F)) + np.uint64(0x7F7F7F7F)) & M32
    return bytes4_to_bits(t | c)


def bits4_to_bytes(nib):
    return ((nib * np.uint64(0x00204081)) & M32) & np.uint64(0x01010101)


def want_nz(c):
    return sum((((c >> np.uint64(8 * k)) & np.uint64(0xFF)) != 0).astype(np.uint64) << np.uint64(k) for k in range(4))


def test_nz4_every_byte_value_in_every_position():
    rng = np.random.default_rng(5)
    for k in range(4):
        other = rng.integers(0, 2**32, 256 * 64, dtype=np.uint64)
        vals = np.tile(np.arange(256, dtype=np.uint64), 64)
        c = (other & ~(np.uint64(0xFF) << np.uint64(8 * k)) & M32) | (vals << np.uint64(8 * k))
        assert np.array_equal(nz4_to_bits(c), want_nz(c))


def test_nz4_random_and_sparse_words():
    rng = np.random.default_rng(6)
    c = rng.integers(0, 2**32, 1 << 20, dtype=np.uint64)
    sparse = rng.integers(0, 2, (1 << 16, 4), dtype=np.uint64)
    c2 = sum(sparse[:, k] << np.uint64(8 * k) for k in range(4))
    for x in (c, c2):
        assert np.array_equal(nz4_to_bits(x), want_nz(x))


def test_bits4_to_bytes_roundtrip():
    nib = np.arange(16, dtype=np.uint64)
    b = bits4_to_bytes(nib)
    assert np.array_equal(nz4_to_bits(b), nib)
    assert np.all((b & ~np.uint64(0x01010101)) == 0)
