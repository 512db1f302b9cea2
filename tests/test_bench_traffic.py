"""bench.py reports the step kernel's DRAM traffic from the committed ncu
summary only for a launch of the shape that summary was captured with."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def captured_shape():
    path = os.path.join(ROOT, "profiles", "flif_gl_step_n20000_l1024.md")
    with open(path) as f:
        for line in f:
            if line.startswith("traffic_launch_shape:"):
                return line.split(":", 1)[1].strip()
    return None


def test_traffic_only_for_the_captured_shape():
    shape = captured_shape()
    assert shape is not None
    t = bench.profile_traffic(shape)
    assert t is not None and t > 0
    # per-launch DRAM bytes below the algorithmic bytes of the 256-step launch
    # means part of the ring comes from the L2; far above them would mean re-reads
    assert t < 1.05 * 42.67e9
    ctas, warps, var, stages, rows, pin = shape.split(":")
    other = ":".join([ctas, warps, var, stages, rows, "0"])
    assert bench.profile_traffic(other) is None
    assert bench.profile_traffic(":".join([ctas, warps, var, "2", "64", pin])) is None
