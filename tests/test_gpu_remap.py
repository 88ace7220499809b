"""L* remapping on the GPU against the oracle's restatement of the
reference's monotone cubic interpolator (pinned against the interpolator
compiled from source in test_oracle.py): every (P,V,K) line, bit for bit."""
import numpy as np
import pytest

from verb4d_b200 import workload as W

from test_gpu_step import load_ctx

pytestmark = pytest.mark.gpu


def test_remap_matches_oracle(gpu, oracle_lib):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=31)
    f = wl.fields
    P, R, V, K = wl.spec.shape
    psd = f["psd"].copy()
    # some lines monotone in L (the interpolator then adjusts its derivatives)
    psd[:, :, 3, :] = np.linspace(1.0, 2.0, R)[None, :, None]
    psd[:, :, 5, :] = np.linspace(2.0, 1.0, R)[None, :, None] ** 3
    wl.fields["psd"] = psd
    oldL = f["Lg"]
    mlt = np.deg2rad(f["Pg"][:, :1, :1, :1] * 15.0)
    newL = oldL * (1.0 + 0.03 * np.sin(mlt)) + 0.01 * f["Vg"]   # still increasing in R
    c = load_ctx(wl)
    c.remap_L(newL)
    got = c.download()
    gotL = c.download("Lg")
    c.close()
    assert np.array_equal(gotL, newL)
    want = np.empty_like(psd)
    for p in range(P):
        for v in range(V):
            for k in range(K):
                st, want[p, :, v, k] = oracle_lib.monot_cubic(oldL[p, :, v, k], psd[p, :, v, k],
                                                              newL[p, :, v, k])
                assert st == 0
    assert np.array_equal(got, want)
