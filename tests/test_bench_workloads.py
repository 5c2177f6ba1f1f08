"""The benchmark's synthetic workloads, checked on the CPU: the Poisson query
stream has the configured rate and mix, and the per-source work histogram
adds up."""
import numpy as np

import bench


def test_poisson_stream_rate_mix_and_set_sizes():
    reqs = bench.make_stream(V=50_000, rate=2000.0, duration=10.0, seed=3)
    n = len(reqs)
    assert abs(n - 20_000) < 5 * np.sqrt(20_000)            # Poisson count around rate x duration
    times = np.array([r[0] for r in reqs])
    assert np.all(np.diff(times) >= 0) and times[-1] < 10.0
    kinds = np.array([r[1] for r in reqs])
    assert abs((kinds == 0).mean() - 0.7) < 0.02            # 70 % SSSD
    sizes = np.array([len(r[2]) for r in reqs if r[1] == 1])
    assert sizes.min() >= 1 and sizes.max() <= 1000
    # log-uniform in [1, 1000]: about a third of the sets in each decade
    dec = np.histogram(np.log10(sizes), bins=[0, 1, 2, 3.01])[0] / len(sizes)
    assert np.all(np.abs(dec - 1 / 3) < 0.06)
    for r in reqs[:200]:
        if r[1] == 0:
            assert 0 <= r[2] < 50_000 and 0 <= r[3] < 50_000
        else:
            assert len(np.unique(r[2])) == len(r[2]) and r[2].max() < 50_000
    # the same seed gives the same stream
    again = bench.make_stream(V=50_000, rate=2000.0, duration=10.0, seed=3)
    assert len(again) == n and all(a[0] == b[0] and a[1] == b[1] for a, b in zip(reqs, again))


def test_work_histogram():
    w = np.array([0, 300, 500, 700, 1024, 5000], np.int64)
    h = bench.work_histogram(w)
    assert sum(h["log2_buckets"].values()) == 5              # sources without work are left out
    assert h["min"] == 300 and h["max"] == 5000 and h["median"] == 700
    assert h["log2_buckets"]["[2^8,2^9)"] == 2 and h["log2_buckets"]["[2^10,2^11)"] == 1
    assert abs(h["top1pct_share"] - 5000 / w.sum()) < 1e-12
