"""Pipe runner (bridct_b200/bridct_runner): the wire protocol of the reference's test runner
(tests/test_runner.c:19-52).  Malformed requests are rejected before any device work, so those
cases run on CPU; the transform round trips need a GPU."""
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

RUNNER = Path(__file__).resolve().parents[1] / "bridct_b200" / "bridct_runner"
MAGIC = 0x42524443


def run(payload: bytes, timeout=120):
    return subprocess.run([str(RUNNER)], input=payload, capture_output=True, timeout=timeout)


def request(h, w, mode, x=None):
    head = struct.pack("<4I", MAGIC, h, w, mode)
    return head + (b"" if x is None else np.ascontiguousarray(x, np.float32).tobytes())


def test_runner_built():
    assert RUNNER.exists(), "build the package first (python -m bridct_b200.build)"


def test_empty_input_exits_cleanly():
    assert run(b"").returncode == 0


@pytest.mark.parametrize("payload", [
    b"\x00" * 7,                                   # truncated header
    struct.pack("<4I", 0x12345678, 8, 8, 0),       # wrong magic
    struct.pack("<4I", MAGIC, 12, 8, 0),           # unsupported length
    struct.pack("<4I", MAGIC, 8, 2048, 0),         # too long
    struct.pack("<4I", MAGIC, 8, 8, 3),            # unknown mode
])
def test_malformed_requests_exit_2(payload):
    assert run(payload).returncode == 2


@pytest.mark.gpu
def test_runner_transforms_match_oracle():
    from oracle import oracle as O

    rng = np.random.default_rng(17)
    cases = [(8, 16, 0), (64, 64, 1), (256, 128, 2), (64, 64, 0), (1024, 8, 1)]
    xs = [rng.uniform(-1, 1, (h, w)).astype(np.float32) for h, w, _ in cases]
    r = run(b"".join(request(h, w, m, x) for (h, w, m), x in zip(cases, xs)))
    assert r.returncode == 0, r.stderr.decode()
    buf, pos = r.stdout, 0
    for (h, w, m), x in zip(cases, xs):
        magic, status, intact, unchanged = struct.unpack_from("<4I", buf, pos)
        pos += 16
        y = np.frombuffer(buf, np.float32, h * w, pos).reshape(h, w)
        pos += 4 * h * w
        assert (magic, status, intact, unchanged) == (MAGIC, 0, 1, 1)
        assert O.rel_max_error(y[None], O.fp64_apply(x[None], m), x[None], output_scaled=True) <= 2e-6
    assert pos == len(buf)


@pytest.mark.gpu
def test_truncated_payload_exits_4():
    assert run(request(16, 16, 0) + b"\x00" * 100).returncode == 4
