"""Dataset ingest (hj_import_text / hj_import_binary) against the reference's
importer, restated in the oracle with the same standard-library calls
(getline on ',' and `stringstream >> DTYPE`, import_dataset.cpp:10-40).

The parallel parser must give the same values in the same order, bit for bit,
on the reference generator's own output format (datasets/
dataset_gen_fixed_len_expo_dist.cpp:78-83: "v, v, ..., v" lines at the
stream's default precision), on full-precision files, on a file cut into many
chunks, and on hostile inputs where the stream's grammar decides what counts.
"""
import numpy as np
import pytest

import oracle
from hegjoin_b200 import workloads


def _write_reference_format(path, db, fmt):
    with open(path, "w") as f:
        for row in db:
            f.write(", ".join(fmt % float(v) for v in row) + "\n")


def _check(path, d, dtype):
    import hegjoin_b200 as hj
    flat = oracle.import_text(str(path), dtype)
    got = hj.import_text(str(path), d, dtype)
    keep = (len(flat) // d) * d
    assert got.shape == (len(flat) // d, d)
    assert np.array_equal(got.reshape(-1).view(np.uint8), flat[:keep].view(np.uint8))   # bit for bit
    return got


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reference_generator_format(tmp_path, dtype):
    db = workloads.exp40(90, 3000, 6, dtype)
    p = tmp_path / "ref_format.txt"
    _write_reference_format(p, db, "%g")                    # ostream's default: 6 significant digits
    got = _check(p, 6, dtype)
    assert got.shape == (3000, 6)


@pytest.mark.parametrize("dtype,fmt", [(np.float32, "%.9g"), (np.float64, "%.17g")])
def test_full_precision_round_trip(tmp_path, dtype, fmt):
    db = workloads.exp40(91, 5000, 18, dtype)
    p = tmp_path / "full.txt"
    _write_reference_format(p, db, fmt)                     # max_digits10: parses back to the same values
    got = _check(p, 18, dtype)
    assert np.array_equal(got, db)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_many_chunks(tmp_path, dtype):
    db = workloads.exp40(92, 120_000, 5, dtype)             # several MB: the file is cut into many chunks
    p = tmp_path / "big.txt"
    _write_reference_format(p, db, "%.9g" if dtype == np.float32 else "%.17g")
    got = _check(p, 5, dtype)
    assert np.array_equal(got, db)


HOSTILE = ("1,2,3\n4,5,6\r\n7 , 8,9\n+.5, -0, 1e5, 1E-3, 2.5e+2, 3.e1, .25\n"
           "1.5e, 4, abc, 5,, 6, 1.2.3, 0x10, inf, nan, -.e1, 7e\n"
           "  8 9 10 ,11\t12, 13abc 14, 1e400, -1e400, 1e-40, 1e-320, 00012.50, -00.0e-0,\n"
           "+, -, ., e5, 9\n")


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("d", [1, 3, 4])
def test_hostile_inputs_follow_the_stream_grammar(tmp_path, dtype, d):
    p = tmp_path / "hostile.txt"
    p.write_text(HOSTILE)
    _check(p, d, dtype)


def test_empty_and_short_files(tmp_path):
    import hegjoin_b200 as hj
    p = tmp_path / "empty.txt"
    p.write_text("")
    assert hj.import_text(str(p), 3, np.float32).shape == (0, 3)
    p.write_text("1, 2")                                    # fewer values than one point
    assert hj.import_text(str(p), 3, np.float32).shape == (0, 3)
    with pytest.raises(hj.HJError):
        hj.import_text(str(tmp_path / "missing.txt"), 3, np.float32)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_binary_twin_and_reference_raw_layout(tmp_path, dtype):
    import hegjoin_b200 as hj
    db = workloads.exp40(93, 7777, 7, dtype)
    p = tmp_path / "db.hjds"
    hj.write_binary(str(p), db)
    assert np.array_equal(hj.import_binary(str(p), 7, dtype), db)
    with pytest.raises(hj.HJError):
        hj.import_binary(str(p), 6, dtype)                 # the header's d differs
    raw = tmp_path / "db.raw"                               # importNDDatasetBinary's layout: values only
    db.tofile(raw)
    assert np.array_equal(hj.import_binary(str(raw), 7, dtype), db)
