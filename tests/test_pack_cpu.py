"""Host packing of STORM_t rows, checked without a GPU: the threaded bulk
packer (ChunkPack::add_rows) must lay out exactly what the row-by-row
packer (ChunkPack::add_row) does (tests/pack_identity.cu)."""
import pytest

from harness import run_host_check


@pytest.mark.timeout(600)
def test_bulk_packer_matches_row_by_row(sb):
    assert run_host_check("pack_identity").strip().endswith("identical")
