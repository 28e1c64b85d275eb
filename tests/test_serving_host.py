"""Host logic of the serving loop (no GPU): the pinned output ring never
hands out overlapping or out-of-range runs, reclaims space in FIFO order
whatever order requests complete in, and refuses (admission waits) when
full; latency percentiles."""
import random

from cuda_knn_aggregate.serving import PinnedRing, ServeStats


def test_ring_never_overlaps_and_reclaims():
    for seed in range(8):
        rng = random.Random(seed)
        r = PinnedRing(10240)
        live, granted = [], 0
        for _ in range(5000):
            if live and (rng.random() < 0.5 or len(live) > 20):
                off, _ = live.pop(rng.randrange(len(live)) if seed % 2 else 0)
                r.free(off)
            else:
                n = rng.randint(1, 3000)
                off = r.alloc(n)
                if off is None:
                    continue
                m = (n + 255) // 256 * 256
                assert off % 256 == 0 and off + m <= r.cap
                assert all(off + m <= a or a + b <= off for a, b in live)
                live.append((off, m))
                granted += 1
        assert granted > 1000
        for off, _ in live:
            r.free(off)
        assert r.alloc(10240) == 0  # all space back


def test_ring_full_refuses_until_oldest_freed():
    r = PinnedRing(4096)
    a = r.alloc(2048)
    b = r.alloc(2048)
    assert (a, b) == (0, 2048)
    assert r.alloc(256) is None
    r.free(b)                     # not the oldest: nothing reclaimed yet
    assert r.alloc(256) is None
    r.free(a)
    assert r.alloc(4096) == 0


def test_percentiles():
    st = ServeStats(n_requests=100, queries=1000, seconds=2.0, latencies_ms=[float(i) for i in range(1, 101)])
    assert st.pct(50) == 50.0 and st.pct(99) == 99.0 and st.throughput == 500.0
