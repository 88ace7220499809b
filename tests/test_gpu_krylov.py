"""The Krylov form of the local (V,K) solve and its learned warm start.

* The training triples the solver writes (verb_local_triples): features equal
  their CPU definition (learned.features, FP32 arithmetic; log10f may differ
  from numpy's by an ulp), and the target is (x - f) / max|f| with x the LU
  solution, bit for bit.
* The Krylov step (FP64-refined FP32 BiCGSTAB, banded LU for the systems that
  miss the residual tolerance) agrees with the LU step to 1e-8 relative from
  every guess; with no Krylov passes every system takes the LU and the step is
  bit-identical to the LU step.
* The CNN is trained on the GPU by the project's own kernels on 19,200
  triples of the 24 x 25 x 31 x 31 grid (eight seeds, four steps each) and
  its warm start is compared with x0 = f (the state the step starts from:
  the method without the network) and x0 = 0 on a held-out seed.  The test
  asserts that training lowers the loss and that the step from the network's
  guess is as accurate as the others; the gain itself is printed, not
  asserted, because on this workload there is none: the local step is stiff
  (dt D / dalpha^2 spans ~1e-2..1e2 with log-normal coefficients drawn
  independently per grid point), so the increment x - f is a non-local
  function of the coefficients, and a 4-layer 3x3 network sees 9 x 9 points.
  Training lowers the loss by ~10% and the held-out increment error stays
  near that of x0 = f; BiCGSTAB iteration counts are the same for all three
  guesses.
"""
import numpy as np
import pytest

from verb4d_b200 import learned
from verb4d_b200 import workload as W

from test_gpu_step import load_ctx

pytestmark = pytest.mark.gpu
TOL = 1e-8


def split_ctx(wl):
    """A context that has taken the convection and radial parts of a step."""
    c = load_ctx(wl)
    c.step(wl.dt, wl.sub_dt, 1, 1, 0)
    return c


def lu_step(wl):
    c = split_ctx(wl)
    c.local(wl.dt, wl.sub_dt)
    c.sync()
    out = c.download()
    c.close()
    return out


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_triples_match_cpu_definition(gpu):
    import torch

    wl = W.make_workload(W.CONFIGS["cfg1"], seed=21, sources=True, losses=True)
    P, R, V, K = wl.spec.shape
    assert wl.sub_dt >= wl.dt   # one sub-step: the triple starts from `before`
    c = split_ctx(wl)
    before = c.download()
    feat = torch.zeros((P * R, 4, K, V), dtype=torch.float32, device="cuda")
    targ = torch.zeros((P * R, 1, K, V), dtype=torch.float32, device="cuda")
    c.local_triples(wl.dt, wl.sub_dt, feat.data_ptr(), targ.data_ptr())
    c.sync()
    x = c.download()
    c.close()
    f = feat.cpu().numpy()
    t = targ.cpu().numpy()[:, 0]
    fl = wl.fields
    shp = (P * R, V, K)
    ref, scale = learned.features(fl["DVV"].reshape(shp), fl["DKK"].reshape(shp),
                                  fl["DVK"].reshape(shp), before.reshape(shp))
    # log10f may differ from numpy's float32 log10 by an ulp
    np.testing.assert_allclose(f[:, :3], ref[:, :3], rtol=0, atol=2e-6)
    # f / max|f| is one IEEE FP32 division: bit-exact
    assert np.array_equal(f[:, 3], ref[:, 3])
    # target = (x - f) / max|f| in FP64, rounded to FP32: bit-exact
    xt = x.reshape(shp).transpose(0, 2, 1)
    ft = before.reshape(shp).transpose(0, 2, 1)
    want = ((xt - ft) / scale.astype(np.float64)[:, None, None]).astype(np.float32)
    assert np.array_equal(t, want)


@pytest.mark.parametrize("guess", ["zero", "prev"])
def test_krylov_step_matches_lu(gpu, guess):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=22, sources=True, losses=True)
    ref = lu_step(wl)
    c = split_ctx(wl)
    st = c.local_krylov(wl.dt, wl.sub_dt, guess=guess)
    c.sync()
    got = c.download()
    c.close()
    assert st["systems"] == wl.spec.P * wl.spec.R
    assert 0 <= st["fallbacks"] < st["systems"]
    assert st["max_rel_residual"] >= 0
    assert rel(got, ref) < TOL
    print(guess, st)


def test_all_fallback_is_the_lu_step(gpu):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=23, sources=True, losses=True)
    ref = lu_step(wl)
    c = split_ctx(wl)
    st = c.local_krylov(wl.dt, wl.sub_dt, guess="prev", max_outer=0)
    c.sync()
    got = c.download()
    c.close()
    assert st["fallbacks"] == st["systems"] and st["inner_iterations"] == 0
    assert np.array_equal(got, ref)


def test_learned_warm_start(gpu):
    import torch

    spec = W.CONFIGS["cfg1"]
    nsys = spec.P * spec.R
    feat, targ = learned.collect_triples(range(1, 9), 4, spec)   # 19,200 triples
    assert feat.shape[0] == 8 * 4 * nsys
    net = learned.CNN(spec.K, spec.V, nsys, seed=0)
    hist = learned.train(net, feat, targ, epochs=10, batch=256, lr=1e-3)
    print("training loss by epoch", [round(h, 4) for h in hist])
    assert hist[-1] < 0.95 * hist[0]
    # held-out systems: another seed
    hf, ht = learned.collect_triples([100], 1, spec)
    out = torch.empty_like(ht)
    net.forward(hf.data_ptr(), out.data_ptr(), nsys)
    torch.cuda.synchronize()
    err_cnn = ((out - ht).norm() / ht.norm()).item()   # x0 = f has error 1.0 here
    print("held-out increment error: cnn %.3f, x0=f 1.000" % err_cnn)
    assert np.isfinite(err_cnn)
    # the Krylov step from the network's guess is as accurate as any other
    wl = W.make_workload(spec, seed=100, sources=True, losses=True)
    ref = lu_step(wl)
    stats = {}
    for guess in ("zero", "prev", "cnn"):
        c = split_ctx(wl)
        st = c.local_krylov(wl.dt, wl.sub_dt, guess=guess, cnn=net if guess == "cnn" else None)
        c.sync()
        got = c.download()
        c.close()
        assert rel(got, ref) < TOL
        stats[guess] = st
        ns = st["systems"] - st["fallbacks"]
        print(guess, "iterations per Krylov-solved system %.1f" % (st["solved_iterations"] / ns),
              "fallbacks", st["fallbacks"], "guess residual %.3g" % st["guess_rel_residual"])
    net.close()


def test_krylov_mixed_fallback_refined(gpu):
    # with FP32 factors the LU fallback takes the mixed form's FP64 refinement
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=24, sources=True, losses=True)
    ref = lu_step(wl)
    for max_outer in (0, 10):
        c = split_ctx(wl)
        c.set_local_precision("mixed", 10)
        st = c.local_krylov(wl.dt, wl.sub_dt, guess="prev", max_outer=max_outer)
        c.sync()
        got = c.download()
        c.close()
        assert st["fallbacks"] > 0
        assert rel(got, ref) < TOL, max_outer


def test_triples_step_is_the_lu_step(gpu):
    # the state after verb_local_triples is the LU step's, in the FP64 form
    # and in the mixed form with refinement
    import torch

    wl = W.make_workload(W.CONFIGS["cfg1"], seed=25, sources=True, losses=True)
    P, R, V, K = wl.spec.shape
    for form in (("fp64", 0), ("mixed", 10)):
        c = split_ctx(wl)
        c.set_local_precision(*form)
        c.local(wl.dt, wl.sub_dt)
        c.sync()
        want = c.download()
        c.close()
        c = split_ctx(wl)
        c.set_local_precision(*form)
        feat = torch.zeros((P * R, 4, K, V), dtype=torch.float32, device="cuda")
        targ = torch.zeros((P * R, 1, K, V), dtype=torch.float32, device="cuda")
        c.local_triples(wl.dt, wl.sub_dt, feat.data_ptr(), targ.data_ptr())
        c.sync()
        got = c.download()
        c.close()
        assert np.array_equal(got, want), form
