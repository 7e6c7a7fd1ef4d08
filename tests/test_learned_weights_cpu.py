"""The learned stage's weight file (include/lmm_learned.h): the format and
its checks, without a GPU (learned.write_weights / read_weights; the
library's lmm_net_save / lmm_net_load are checked against them in
test_learned_gpu.py)."""
from __future__ import annotations

import struct

import numpy as np
import pytest

from lowmachmixtures_b200 import learned


def test_fnv1a64_known_answers():
    # published FNV-1a 64-bit test vectors
    assert learned.fnv1a64(b"") == 0xCBF29CE484222325
    assert learned.fnv1a64(b"a") == 0xAF63DC4C8601EC8C
    assert learned.fnv1a64(b"foobar") == 0x85944171F73967E8


def _params(seed=0):
    return np.random.default_rng(seed).standard_normal(learned.num_params()).astype(np.float32)


def test_round_trip_is_bitwise_and_header_as_documented(tmp_path):
    p = _params()
    path = tmp_path / "w.bin"
    learned.write_weights(str(path), p)
    data = path.read_bytes()
    nl = len(learned.LAYERS)
    assert data[:8] == b"LMMNET01"
    assert struct.unpack_from("<II", data, 8) == (1, nl)
    assert struct.unpack_from("<Q", data, 16 + 8 * nl)[0] == p.size
    assert len(data) == 32 + 8 * nl + 4 * p.size
    q = learned.read_weights(str(path))
    assert q.dtype == np.float32 and np.array_equal(q.view(np.uint32), p.view(np.uint32))


@pytest.mark.parametrize("damage,msg", [
    (lambda d: d[:-1], "size"),                                     # truncated
    (lambda d: d + b"\0", "size"),                                  # trailing bytes
    (lambda d: d[:-5] + bytes([d[-5] ^ 1]) + d[-4:], "checksum"),   # one payload bit
    (lambda d: b"XMMNET01" + d[8:], "magic"),
    (lambda d: d[:8] + struct.pack("<I", 2) + d[12:], "version"),
    (lambda d: d[:16] + struct.pack("<II", 8, 32) + d[24:], "architecture"),
])
def test_damaged_files_are_rejected(tmp_path, damage, msg):
    path = tmp_path / "w.bin"
    learned.write_weights(str(path), _params(1))
    path.write_bytes(damage(path.read_bytes()))
    with pytest.raises(ValueError, match=msg):
        learned.read_weights(str(path))


def test_wrong_parameter_count_is_refused_on_write(tmp_path):
    with pytest.raises(ValueError):
        learned.write_weights(str(tmp_path / "w.bin"), np.zeros(10, np.float32))
