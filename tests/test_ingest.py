"""Catalogue ingest (hg_read_ascii, hg_read_gadget) against the reference's own readers
(readParticleBOSS, particle.hpp:93-154; readParticlesFromGagdetSnapshot,
particleGadget.hpp:211-298), whose outputs on the same files are the fixture
(tests/golden/make_golden.py --ingest).  Host code only: runs without a GPU."""
import os

import numpy as np
import pytest

from conftest import load_golden


@pytest.fixture(scope="module")
def gold():
    return load_golden("ingest.npz")


def test_ascii_matches_reference_reader(gold, tmp_path):
    from hitomi_b200.ingest import read_ascii
    p = tmp_path / "cat.txt"
    p.write_bytes(gold["ascii_text"].tobytes())
    got = read_ascii(str(p))
    # bit-identical, NaN and inf included; lines that do not give four numbers are skipped
    np.testing.assert_array_equal(got, gold["ascii_ref"])


def test_ascii_thread_split_is_invisible(gold, tmp_path):
    """The file is parsed in byte ranges split at line ends, one per thread: the result does
    not depend on where the ranges fall (a catalogue far larger than one range)."""
    from hitomi_b200.ingest import read_ascii
    body = gold["ascii_text"].tobytes()
    p = tmp_path / "big.txt"
    p.write_bytes(body * 4)
    got = read_ascii(str(p))
    # the text ends without a newline, so the last line of one copy ("9 9 9 9") joins the
    # first of the next ("# x y z w"): that line still reads as 9 9 9 9
    np.testing.assert_array_equal(got, np.tile(gold["ascii_ref"], (4, 1)))


def test_ascii_missing_file():
    from hitomi_b200.api import HitomiError
    from hitomi_b200.ingest import read_ascii
    with pytest.raises(HitomiError, match="Cannot open"):
        read_ascii("/nonexistent/catalogue.txt")


def test_gadget_matches_reference_reader(gold, tmp_path):
    from hitomi_b200.ingest import read_gadget
    base = tmp_path / "snap"
    for i in (0, 1):
        (tmp_path / f"snap.{i}").write_bytes(gold[f"gadget{i}"].tobytes())
    rec, hdr = read_gadget(str(base))
    np.testing.assert_array_equal(rec, gold["gadget_ref"])
    assert hdr.num_files == 2 and hdr.npartTotal[1] == rec.shape[0] and hdr.BoxSize == 1000.0


def test_gadget_missing_second_file(gold, tmp_path):
    from hitomi_b200.api import HitomiError
    from hitomi_b200.ingest import read_gadget
    (tmp_path / "snap.0").write_bytes(gold["gadget0"].tobytes())
    with pytest.raises(HitomiError, match="can not open"):
        read_gadget(str(tmp_path / "snap"))
