"""Asynchronous PSD output and restart through .pltb files on the GPU.

The file a context writes equals, byte for byte, the format restatement
(oracle/pltb.py, pinned against the reference's writer on the CPU); an
asynchronous write captures the field at the call even though the next step
runs while it is written; a context restarted from a written file continues
bit for bit like the one that wrote it.
"""
import numpy as np
import pytest

import pltb
from verb4d_b200 import workload as W

from test_gpu_step import load_ctx, without_conv_loss

pytestmark = pytest.mark.gpu


def test_async_write_and_restart(gpu, tmp_path):
    wl = without_conv_loss(W.make_workload(W.CONFIGS["cfg1"], seed=21))
    c = load_ctx(wl)
    c.step(wl.dt, wl.sub_dt)
    c.sync()
    snap = c.download()
    f1 = tmp_path / "PSD_00001.pltb"
    c.write_pltb(str(f1), wait=False)        # returns at once
    c.step(wl.dt, wl.sub_dt)                 # overwrites the PSD meanwhile
    c.output_wait()
    ref_file = tmp_path / "ref.pltb"
    pltb.write(ref_file, snap)
    assert f1.read_bytes() == ref_file.read_bytes()
    c.step(wl.dt, wl.sub_dt)
    c.sync()
    cont = c.download()
    c.close()

    # restart from the file: two more steps as the original context took
    r = load_ctx(wl)
    r.read_pltb(str(f1))
    r.step(wl.dt, wl.sub_dt)
    r.step(wl.dt, wl.sub_dt)
    r.sync()
    assert np.array_equal(r.download(), cont)
    r.close()


def test_read_rejects_other_dimensions(gpu, tmp_path):
    from verb4d_b200 import _lib as L

    wl = W.make_workload(W.CONFIGS["cfg1"], seed=22)
    c = load_ctx(wl)
    bad = tmp_path / "bad.pltb"
    pltb.write(bad, np.zeros((2, 3, 4, 5)))
    with pytest.raises(L.VerbError):
        c.read_pltb(str(bad))
    c.close()
