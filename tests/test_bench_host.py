"""Host-side helpers of bench.py (CPU): the CPU baseline's core count is read once per process,
so repeated samples (the reference arm's warm-up and timed steps) keep every core even after an
OpenMP region has bound the main thread to one of them."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


@pytest.mark.skipif(not hasattr(os, "sched_setaffinity"), reason="needs sched_setaffinity")
def test_host_cpu_is_read_once():
    import bench
    first = bench.host_cpu()
    before = os.sched_getaffinity(0)
    try:
        os.sched_setaffinity(0, {min(before)})   # what OMP_PROC_BIND does to the main thread
        assert bench.host_cpu() == first
    finally:
        os.sched_setaffinity(0, before)
    assert first[1] >= 1 and first[2] >= first[1]
