"""The serving client's host-side pieces, without a GPU."""
import pytest


def test_result_ring_slots(pkg):
    """Result slots are consecutive views of one buffer; a request that does
    not fit the rest of the buffer starts over at its beginning; a request
    larger than the buffer is refused."""
    from importlib import import_module
    serving = import_module("pss_b200.serving")
    ring = serving.ResultRing(10)
    a, b = ring.take(4), ring.take(5)
    assert a.shape == (4,) and b.shape == (5,)
    a[:] = 1
    b[:] = 2
    assert list(ring.buf[:9]) == [1] * 4 + [2] * 5
    c = ring.take(3)  # 9 + 3 > 10: wraps to the start
    c[:] = 3
    assert list(ring.buf[:4]) == [3, 3, 3, 1]
    with pytest.raises(ValueError):
        ring.take(11)
