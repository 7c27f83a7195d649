"""The split-K autotuner's table on the host (no GPU needed): classes merged
from a saved file, looked up by GEMM shape, written back unchanged, and the
errors for a malformed file and an unknown mode.

A class is (output CTAs, power-of-two bucket of the k tiles): 128 x 128 output
tiles times output batches, and k tiles of 16 over all reduction batches, so a
200 x 300 output (2 x 3 tiles) with k = 1000 (63 k tiles, bucket 5) is class
(6, 5).
"""
import pytest

import libuw12_b200 as L


@pytest.fixture
def clean_table():
    L.autotune_clear()
    L.autotune(L.AUTOTUNE_OFF)
    yield
    L.autotune_clear()
    L.autotune(L.AUTOTUNE_OFF)


def test_table_round_trip_and_lookup(tmp_path, clean_table):
    src = tmp_path / "table.txt"
    src.write_text("# output_ctas k_tile_bucket split ms\n6 5 4 0.125\n148 10 1 2.5\n\n")
    assert L.autotune_size() == 0
    L.autotune(L.AUTOTUNE_USE, str(src))
    assert L.autotune_size() == 2
    assert L.autotune_lookup(200, 300, 1000) == 4
    # same class: k tiles 32..63, reduction batches included
    assert L.autotune_lookup(256, 384, 16 * 21, nbr=3) == 4
    # another bucket, another CTA count
    assert L.autotune_lookup(200, 300, 2000) == 0
    assert L.autotune_lookup(200, 300, 1000, nbo=2) == 0
    assert L.autotune_lookup(37 * 128, 4 * 128, 16 * 1024) == 1
    out = tmp_path / "saved.txt"
    L.autotune_save(str(out))
    L.autotune_clear()
    assert L.autotune_size() == 0
    L.autotune(L.AUTOTUNE_USE, str(out))
    assert L.autotune_size() == 2
    assert L.autotune_lookup(200, 300, 1000) == 4
    # a missing file leaves the table as it is
    L.autotune(L.AUTOTUNE_TUNE, str(tmp_path / "absent.txt"))
    assert L.autotune_size() == 2


@pytest.mark.parametrize("line", ["6 5\n", "6 5 0 1.0\n", "0 5 2 1.0\n", "6 5 65 1.0\n",
                                  "six 5 2 1.0\n"])
def test_malformed_table_is_rejected(tmp_path, clean_table, line):
    bad = tmp_path / "bad.txt"
    bad.write_text("# header\n6 5 4 0.1\n" + line)
    with pytest.raises(L.UW12CudaError, match="malformed line 3"):
        L.autotune(L.AUTOTUNE_USE, str(bad))
    assert L.autotune_size() == 0


def test_unknown_mode_is_rejected(clean_table):
    with pytest.raises(L.UW12CudaError, match="mode"):
        L.autotune(3)
