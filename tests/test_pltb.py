"""The .pltb output/restart format: the restatement (oracle/pltb.py) against
the reference's own Matrix4D writer and reader (src/Matrix.cpp:5700-5720,
5780-5808), compiled from source in oracle/_ref."""
import numpy as np
import pytest

import oracle as O
import pltb


@pytest.mark.skipif(not O.have_reference(), reason="reference not built here")
def test_restatement_matches_reference_writer_and_reader(tmp_path):
    ref = O.reference(lu_caching=True)
    a = np.random.default_rng(1).standard_normal((3, 4, 5, 6))
    a[0, 0, 0, :2] = [np.inf, -0.0]
    p_ref, p_ours = tmp_path / "ref.pltb", tmp_path / "ours.pltb"
    ref.write_pltb(p_ref, a)
    pltb.write(p_ours, a)
    assert p_ref.read_bytes() == p_ours.read_bytes()
    assert np.array_equal(pltb.read(p_ref), a)
    assert np.array_equal(ref.read_pltb(p_ours, a.shape), a)


def test_lst_line(tmp_path):
    import ctypes

    from verb4d_b200 import _lib as L

    lib = L.load()
    lst = tmp_path / "PSD.lst"
    assert lib.verb_append_lst(str(lst).encode(), ctypes.c_double(1.0 / 24), b"PSD_00001.pltb") == 0
    assert lib.verb_append_lst(str(lst).encode(), ctypes.c_double(2.5), b"PSD_00002.pltb") == 0
    assert lst.read_text() == "0.04167\tPSD_00001.pltb\n2.50000\tPSD_00002.pltb\n"
