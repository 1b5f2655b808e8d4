"""Host logic of the serving loop: the request-buffer arena and the request stream."""
import random

from syclfft_b200 import serving


class _Buf:
    def __init__(self, n):
        self.n = n

    def numel(self):
        return self.n


def test_arena_first_fit_never_overlaps_and_coalesces():
    a = serving.Arena(_Buf(1 << 20))
    rng = random.Random(3)
    live = []
    for _ in range(20000):
        if live and rng.random() < 0.5:
            off, n = live.pop(rng.randrange(len(live)))
            a.release(off, n)
        else:
            n = rng.randint(1, 60000)
            off = a.alloc(n)
            if off is not None:
                assert off % serving.Arena.ALIGN == 0
                live.append((off, n))
        spans = sorted([(o, (n + 255) // 256 * 256) for o, n in live] + a.free)
        for (o1, s1), (o2, _) in zip(spans, spans[1:]):
            assert o1 + s1 <= o2
    for off, n in live:
        a.release(off, n)
    assert a.free == [(0, 1 << 20)] and a.used == 0


def test_arena_refuses_what_does_not_fit():
    a = serving.Arena(_Buf(4096))
    x = a.alloc(3000)
    assert x == 0 and a.alloc(2000) is None
    a.release(x, 3000)
    assert a.alloc(4096) == 0


def test_request_stream_shape():
    reqs = serving.make_request_stream(count=3000, rate=50000.0, seed=5)
    assert len(reqs) == 3000
    assert all(reqs[i].arrival <= reqs[i + 1].arrival for i in range(len(reqs) - 1))
    assert 0.7 < sum(not r.double for r in reqs) / len(reqs) < 0.9
    assert all(1 <= r.batch <= 512 and r.direction in (-1, 1) and 0 <= r.normalization <= 3 for r in reqs)
