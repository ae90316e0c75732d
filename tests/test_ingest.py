"""The reference's text dataset format (src/generator.h:43-227), read and
written by the library on the host: round trips, the TPC-H header, the
width -> storage mapping, cardinalities, and the errors."""
import numpy as np
import pytest

from fastmulticolsort_b200 import capi


def _cols(n, widths, seed):
    rng = np.random.default_rng(seed)
    out = []
    for w in widths:
        dt = {2: np.uint16, 4: np.uint32, 8: np.uint64}[capi.storage_bytes(w)]
        hi = (1 << w) - 1
        out.append(rng.integers(0, hi, size=n, dtype=np.uint64, endpoint=True).astype(dt))
    return out


def test_storage_bytes():
    assert [capi.storage_bytes(w) for w in (1, 16, 17, 32, 33, 64)] == [2, 2, 4, 4, 8, 8]
    assert capi.storage_bytes(0) == 0 and capi.storage_bytes(65) == 0


@pytest.mark.parametrize("header", [False, True])
def test_round_trip(tmp_path, header):
    widths = [3, 16, 17, 33, 64]
    cols = _cols(5000, widths, 1)
    p = tmp_path / "d.dat"
    capi.write_columns_text(p, cols, header=header)
    if header:
        assert capi.text_header(p) == (5000, len(widths))
        got, card = capi.read_columns_text(p, widths, header=True)
    else:
        got, card = capi.read_columns_text(p, widths, nrows=5000)
    for a, b in zip(cols, got):
        assert a.dtype == b.dtype and np.array_equal(a, b)
    assert card == [len(np.unique(c)) for c in cols]


def test_reads_files_written_one_value_per_line(tmp_path):
    """The generator's own layout: every value on its own line, column after column."""
    cols = _cols(1000, [12, 40], 2)
    p = tmp_path / "gen.dat"
    with open(p, "w") as f:
        for c in cols:
            f.write("\n".join(str(int(v)) for v in c) + "\n")
    got, _ = capi.read_columns_text(p, [12, 40], nrows=1000)
    assert all(np.array_equal(a, b) for a, b in zip(cols, got))


def test_errors(tmp_path):
    with pytest.raises(capi.FmcsError):
        capi.read_columns_text(tmp_path / "missing.dat", [8], nrows=1)
    bad = tmp_path / "bad.dat"
    bad.write_text("1\n2\nx3\n")
    with pytest.raises(capi.FmcsError):
        capi.read_columns_text(bad, [8], nrows=3)
    big = tmp_path / "big.dat"
    big.write_text("70000\n")   # does not fit a 16-bit column's storage
    with pytest.raises(capi.FmcsError):
        capi.read_columns_text(big, [16], nrows=1)
    short = tmp_path / "short.dat"
    short.write_text("1\n2\n")
    with pytest.raises(capi.FmcsError):
        capi.read_columns_text(short, [8], nrows=3)
    hdr = tmp_path / "hdr.dat"
    hdr.write_text("3\n1\n1\n2\n3\n")
    with pytest.raises(capi.FmcsError):
        capi.read_columns_text(hdr, [8], nrows=4, header=True)   # header says 3 rows
