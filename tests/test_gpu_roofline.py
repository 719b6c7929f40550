"""The per-node timing module runs every node's filter on device buffers with
the 12 MP workload's blobs (at a small size here) and reports positive,
finite bandwidths."""
import math

import pytest

from cpipe_b200.roofline import NODES, node_roofline


@pytest.mark.gpu
def test_node_roofline_small(cuda_device):
    res = node_roofline(512, 384, reps=2, peak_gbs=6500.0)
    assert len(res) == len(NODES)
    for name, v in res.items():
        assert v["device_ms"] > 0.0 and v["call_ms"] > 0.0, name
        assert math.isfinite(v["achieved_gbs"]) and v["achieved_gbs"] > 0.0, name
