"""hash_any restatements agree: the product's (host build of the device
code), the oracle's, and the producer's (used for inner-relation hashes)."""
import ctypes

import numpy as np

import xb_oracle as O
import xb_producer as P
import xpu_b200


def _lib_hash(data: bytes):
    a = np.frombuffer(data, dtype=np.uint8).copy() if data else np.zeros(1, dtype=np.uint8)
    return xpu_b200.lib().xpuB200HashBytes(ctypes.c_void_p(a.ctypes.data), len(data))


def test_hash_known_lengths():
    r = np.random.default_rng(7)
    for n in list(range(0, 40)) + [63, 64, 100, 127, 255]:
        for _ in range(3):
            d = r.integers(0, 256, n, dtype=np.uint8).tobytes()
            h = P.hash_any(d)
            assert O.hash_bytes(d) == h
            assert _lib_hash(d) == h


def test_hash_vectorised_int_paths():
    v = np.array([0, 1, -1, 2**31 - 1, -2**31, 12345], dtype=np.int64)
    h4 = P.hash_u32_array(v.astype(np.int32), 4)
    h8 = P.hash_u64_array(v)
    for x, a, b in zip(v, h4, h8):
        assert int(a) == P.hash_any(int(x).to_bytes(4, "little", signed=True) if -2**31 <= x < 2**31 else b"")
        assert int(b) == P.hash_any(int(x).to_bytes(8, "little", signed=True))
