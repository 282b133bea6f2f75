"""prefixSum and radixSort as pm:: API task flows (unicorn_b200/serve/
scan_sort_tasks) with the B200 GPU callbacks of libpmb_app_prefixSum.so and
libpmb_app_radixSort.so: the prefix sum's two tasks with the host scan of
slice totals between them, and one task per LSD round with ordered
redistribution of the digit buckets.  Results are compared with the oracle
(restatements of serialPrefixSum / serialLsbRadixSort) bit for bit on ragged
sizes; the full configuration (2^28 keys, 2^22 per subtask) checks itself
(consecutive differences / sortedness and permutation)."""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from test_scan_sort_oracle import orc_scan

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "unicorn_b200", "serve", "_build", "scan_sort_tasks")


def run(args, timeout=900):
    p = subprocess.run([BIN, *map(str, args)], capture_output=True, text=True, timeout=timeout)
    assert p.returncode == 0, p.stderr + p.stdout
    rep = json.loads(p.stdout.strip().splitlines()[-1])
    assert rep["check"] is True
    return rep


@pytest.mark.parametrize("n,per", [((1 << 22) + 12345, 1 << 18), (1000, 1000), (4097, 4096)])
def test_prefix_flow_matches_oracle(oracle, tmp_path, n, per):
    prefix = str(tmp_path / "scan")
    run(["prefix", "--n", n, "--per", per, "--steps", 1, "--warmup", 1, "--dump", prefix])
    x = np.fromfile(prefix + ".in", np.uint32)
    y = np.fromfile(prefix + ".out", np.uint64)
    assert np.array_equal(y, orc_scan(oracle, x))


@pytest.mark.parametrize("bits", [8, 4])
@pytest.mark.parametrize("n,per", [((1 << 21) + 77, 1 << 17), (5000, 1024)])
def test_sort_flow_matches_sorted_keys(tmp_path, bits, n, per):
    prefix = str(tmp_path / "sort")
    run(["sort", "--n", n, "--per", per, "--bits", bits, "--steps", 1, "--warmup", 0, "--dump", prefix])
    x = np.fromfile(prefix + ".in", np.uint32)
    y = np.fromfile(prefix + ".out", np.uint32)
    assert np.array_equal(y, np.sort(x))


@pytest.mark.parametrize("flow", ["prefix", "sort"])
def test_full_configuration_flows(flow):
    rep = run([flow, "--n", 1 << 28, "--per", 1 << 22, "--steps", 1, "--warmup", 1])
    assert rep["subtasks"] == 64
