"""The run postings' piece rules checked without a GPU (tests/run_pieces_check.cu):
list and bitmap chunks give the same pieces, each inside one bin, disjoint,
covering the set and maximal, and per-bin overlaps of two rows' pieces sum
to their intersection, for every bin width the planner can choose."""
import pytest

from harness import run_host_check


@pytest.mark.timeout(600)
def test_run_piece_rules(sb):
    assert run_host_check("run_pieces_check").strip().endswith("ok")
