"""bench.py's reference arm on the replica sweep: the unmodified reference
(oracle/_ref) run as several processes at once, one replica each, summed into
an all-cores aggregate."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def test_replica_aggregate_two_processes():
    import dpd_oracle
    if not os.path.exists(dpd_oracle.REF_DRIVER):
        pytest.skip("reference driver not built")
    import bench
    r = bench.reference_replica_aggregate(512, 2, seconds=1.0)
    assert r["cores"] == 2 and r["kind"] == "reference"
    assert r["value"] > 0 and r["run_seconds"] > 0
    assert "replicas 0..1 of 512" in r["sample"]
