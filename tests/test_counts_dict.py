"""The C builder of simulate_shots' count dictionaries (dqsim/_counts.c)
against the same dictionary built in Python from the C ABI's flat buffers."""

import numpy as np
import pytest

from dqsim import _core


def python_counts(raw, w, counts):
    text = raw.decode("ascii")
    n = len(counts)
    return dict(zip([text[i:i + w] for i in range(0, n * w, w)] if w else [""] * n, counts.tolist()))


@pytest.mark.skipif(_core._counts is None, reason="dqsim._counts not built")
@pytest.mark.parametrize("n,w", [(0, 5), (1, 0), (3, 1), (1000, 30), (20000, 64)])
def test_counts_builder_matches_python(n, w):
    rng = np.random.default_rng(n + w)
    keys = rng.integers(0, 2, size=(n, w)).astype(np.uint8) + ord("0")
    raw = keys.tobytes()
    counts = rng.integers(1, 2**40, size=n, dtype=np.uint64)
    got = _core._counts.build(raw, w, counts.tobytes())
    assert got == python_counts(raw, w, counts)
    assert all(type(k) is str for k in got)


@pytest.mark.skipif(_core._counts is None, reason="dqsim._counts not built")
def test_counts_builder_rejects_short_keys():
    with pytest.raises(ValueError):
        _core._counts.build(b"0101", 3, np.ones(2, dtype=np.uint64).tobytes())
