"""The numpy restatement of the generators and file writers (oracle/synth.py,
used by the benchmark's reference arm so that it loads no library of this
repository) against the library's own generators and .bel writer."""
import numpy as np
import pytest

import beep_b200 as B
from beep_b200 import patterns as P
from oracle import synth as S


@pytest.mark.parametrize("args", [(9, 8, 0.57, 0.19, 0.19, 6), (12, 8, 0.57, 0.19, 0.19, 1),
                                  (14, 6, 0.57, 0.19, 0.19, 2)])
def test_rmat_identical(built, args):
    a, b = B.gen_rmat(*args), S.rmat(*args)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("args", [(4096, 0.004, 1), (300, 0.05, 5), (60, 0.15, 3), (50, 1.0, 2)])
def test_erdos_renyi_identical(built, args):
    a, b = B.gen_erdos_renyi(*args), S.erdos_renyi(*args)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("args", [(2000, 10.0, 2.1, 4), (1 << 12, 32.0, 2.1, 13001)])
def test_chung_lu_identical(built, args):
    a, b = B.gen_chung_lu(*args), S.chung_lu(*args)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_bel_and_mtx_bytes(built, tmp_path):
    rp, col = B.gen_rmat(9, 8, 0.57, 0.19, 0.19, 6)
    B.write_bel(str(tmp_path / "a.bel"), rp, col)
    S.write_bel(str(tmp_path / "b.bel"), rp, col)
    assert (tmp_path / "a.bel").read_bytes() == (tmp_path / "b.bel").read_bytes()
    B.write_mtx(str(tmp_path / "a.mtx"), P.DIAMOND)
    S.write_mtx(str(tmp_path / "b.mtx"), P.DIAMOND)
    assert (tmp_path / "a.mtx").read_text() == (tmp_path / "b.mtx").read_text()
