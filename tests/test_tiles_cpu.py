"""Planning of the bitmap x bitmap engine, checked without a GPU
(tests/tiles_check.cu): every tiling covers each pair i <= j exactly once,
the host-output panels partition the tile list, and the copy / upload plan
on them copies every row once, after its tiles, and reads only uploaded
rows."""
import pytest

from harness import run_host_check


@pytest.mark.timeout(600)
def test_tilings_panels_and_host_plan(sb):
    assert run_host_check("tiles_check").strip().endswith("ok")
