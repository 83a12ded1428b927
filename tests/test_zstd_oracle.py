"""The zstd frame definition of the GPU zstd codec, on the CPU: the oracle's
restatement (oracle/zstd_frame.c) must decode through an independent
decoder, the system's libzstd, for every kind of input the reference's
chunk-parallel zstd path (crates/gpzip-codec-cpu/src/compress.rs:76-126)
feeds it: empty, tiny, ragged, incompressible, runs, text, logs, binary,
and 2 MiB members."""
import numpy as np
import pytest

from gpzip_b200 import workloads as W
from oracle import oracle as O


def cases():
    rng = np.random.default_rng(9)
    return {
        "empty": b"",
        "one": b"a",
        "abc": b"abcabcabcabcabc" * 10,
        "random_5000": rng.integers(0, 256, 5000, dtype=np.uint8).tobytes(),
        "zeros_200k": bytes(200_000),
        "text_300k": W.text(300_000, seed=1).tobytes(),
        "logs_500k": W.logs(500_000, seed=2).tobytes(),
        "binary_400k": W.binary(400_000, seed=3).tobytes(),
        "edge_131073": W.text(131_073, seed=5).tobytes(),
        "edge_4097": rng.integers(0, 3, 4097, dtype=np.uint8).tobytes(),
    }


@pytest.mark.parametrize("name", list(cases()))
def test_frames_decode_with_libzstd(name):
    data = cases()[name]
    f = O.zstd_chunk(data, 131072)
    assert f[:6] == bytes([0x28, 0xB5, 0x2F, 0xFD, 0x00, 0x30])
    assert O.zstd_decompress(f, len(data)) == data


def test_two_mib_members_and_concatenated_frames():
    a = W.logs((2 << 20) + 12_345, seed=6).tobytes()
    b = W.binary(70_001, seed=7).tobytes()
    fa = O.zstd_chunk(a, 2 << 20)
    fb = O.zstd_chunk(b, 131072)
    assert O.zstd_decompress(fa, len(a)) == a
    # frames concatenate into one stream, as the reference's .tar.zst writes them
    assert O.zstd_decompress(fa + fb, len(a) + len(b)) == a + b


def test_ratio_is_in_libzstd_range():
    """Raw literals and the predefined distributions cost ratio against
    libzstd level 3; the frames still compress the log workload."""
    t = W.logs(1 << 20, seed=8).tobytes()
    ours, ref = len(O.zstd_chunk(t, 131072)), len(O.zstd_compress(t, 3))
    assert ours < 0.45 * len(t)
    assert ref < ours < 2.5 * ref
