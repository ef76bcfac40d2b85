"""The learned KPP surrogate: GPU gradients against the CPU (numpy FP64)
restatement, features/targets, training gain over the untrained method, and
the in-step gate / sampled check / fallback."""
import numpy as np
import pytest

from tests import _mlp_ref as ref
from tests._cases import columns, hot_cfg, oracle_state, assert_bitwise

pytestmark = pytest.mark.gpu
DT = 3600.0


@pytest.fixture(scope="module")
def L():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200 import learned

    return learned


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def test_gradients_match_cpu(L):
    import torch

    s = L.KPPSurrogate(seed=3)
    for b in s.b:   # non-zero biases
        b.normal_(0.0, 0.1)
    B = 256
    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn(B, L.NINP, device="cuda", generator=g)
    X[:, L.NIN:] = 0
    Xb = X.to(torch.bfloat16).contiguous()
    XT = Xb.T.contiguous()
    T = torch.randn(B, L.NOUTP, device="cuda", generator=g)
    loss, Y, gW, gb = s.gradients(Xb, XT, B, T)
    torch.cuda.synchronize()
    assert int(s.err.item()) == 0
    W = [w.double().cpu().numpy() for w in s.W]
    bias = [b.double().cpu().numpy() for b in s.b]
    r_loss, r_Y, r_gW, r_gb = ref.forward_backward(Xb.float().double().cpu().numpy(), W, bias,
                                                   T.double().cpu().numpy(), s.loss_w.double().cpu().numpy())
    assert rel(Y.cpu().numpy(), r_Y) < 5e-3
    assert abs(float(loss.item()) - r_loss) <= 5e-3 * abs(r_loss)
    for k in range(3):
        assert rel(gW[k].cpu().numpy(), r_gW[k]) < 2e-2, f"dW{k + 1}"
        assert rel(gb[k].cpu().numpy(), r_gb[k]) < 2e-2, f"db{k + 1}"
    # padding stays inert: no gradient into the 6 padded inputs or the 3 padded outputs
    assert float(gW[0][:, L.NIN:].abs().max()) == 0.0
    assert float(gW[2][L.NOUT:, :].abs().max()) == 0.0


def test_features_and_targets(L):
    import ctypes

    import torch

    from roundabout_b200 import _ffi
    from roundabout_b200.column import VerticalPhysics

    cols = columns(nx=40, ny=24, nz=30, seed=41, ntr=2)
    vp = VerticalPhysics(cols.nx, cols.ny, cols.nz, 2, hot_cfg(ntr=2))
    vp.load_columns(cols)
    n = cols.nx * cols.ny
    raw = torch.empty(n, L.NIN, device="cuda")
    T = torch.empty(n, L.NOUTP, device="cuda")
    colH = torch.empty(n, device="cuda")
    vp.eos()
    _ffi.check(vp.lib.vphys_kpp_features(vp.handle, None, None, ctypes.c_float(1e30), L._p(raw), None, None, 0, None,
                                         L._p(colH)), "features")
    vp.assemble()
    _ffi.check(vp.lib.vphys_kpp_targets(vp.handle, L._p(T)), "targets")
    torch.cuda.synchronize()
    assert torch.isfinite(raw).all() and torch.isfinite(T).all()
    bl = np.asarray(vp.get("bl_depth")).ravel(order="F")
    hb_from_t = 10.0 * np.exp(T[:, 0].double().cpu().numpy())
    wet = colH.cpu().numpy() > 0
    live = bl > 0.1
    assert np.allclose(hb_from_t[wet & live], bl[wet & live], rtol=1e-5)
    depth = colH.cpu().numpy()[wet]
    assert np.allclose(raw[:, 3].cpu().numpy()[wet], depth / 1000.0, rtol=1e-6)
    # the shape outputs are the reference's G(sigma) * 27/4: within [0, 1]
    G = T[:, 2:L.NOUT].cpu().numpy()
    assert G.min() >= 0.0 and G.max() <= 1.0 + 1e-6
    vp.close()


@pytest.fixture(scope="module")
def trained(L):
    import torch

    raw, T = L.collect(64, 256, 30, domains=2, snapshots=[0, 5, 23], seed=7)
    s = L.KPPSurrogate(seed=7)
    s.fit_standardisation(raw, T)
    n = raw.shape[0]
    ntest = 8192
    X, XT, Ts = s.standardise(raw[:-ntest].contiguous(), T[:-ntest].contiguous())
    Xte, _, _ = s.standardise(raw[-ntest:].contiguous(), T[-ntest:].contiguous())
    hb_te = 10.0 * torch.exp(T[-ntest:, 0])
    untrained = s.predict_hb(Xte)
    hist = s.train(X, XT, Ts, epochs=6, batch=4096, lr=2e-3)
    return s, hist, Xte, hb_te, untrained, n


def rms_rel(pred, want):
    import torch

    return float(torch.sqrt(torch.mean(((pred - want) / torch.clamp(want, min=1.0)) ** 2)))


def test_training_gains_over_untrained(L, trained):
    s, hist, Xte, hb_te, untrained, n = trained
    e_train = rms_rel(s.predict_hb(Xte), hb_te)
    e_untrained = rms_rel(untrained, hb_te)
    print(f"held-out OBL depth RMS rel error: trained {e_train:.3f}, untrained {e_untrained:.3f}; n_train {n}")
    assert hist[-1] < hist[0]
    assert e_train < 0.5 * e_untrained
    assert e_train < 0.5


def test_learned_step_gate_falls_back_bitwise(L, trained, oracle):
    """Every column gated: the learned step is the plain step, bit for bit."""
    from roundabout_b200.column import VerticalPhysics

    s = trained[0]
    cols = columns(nx=40, ny=24, nz=30, seed=42, ntr=4)
    cfg = hot_cfg(ntr=4)
    st = oracle_state(oracle, cols, cfg)
    vp = VerticalPhysics(cols.nx, cols.ny, cols.nz, 4, hot_cfg(ntr=4, learned_kpp=1))
    vp.load_columns(cols)
    s.attach(vp, gate_limit=1e-9)
    assert st.call("vpo_step", cfg, DT, 3) == 0
    vp.step(DT, 3)
    for n in ("kv", "kt", "bl_depth", "u"):
        assert_bitwise(n, vp.get(n), getattr(st, n))
    stats = L.kpp_stats(vp)
    assert stats["gated"] > 0 and stats["gemm_err"] == 0
    vp.close()


def test_learned_step_check_and_fallback(L, trained):
    from roundabout_b200.column import VerticalPhysics

    s = trained[0]
    cols = columns(nx=64, ny=48, nz=30, seed=43, ntr=2, land_frac=0.2)
    vp = VerticalPhysics(cols.nx, cols.ny, cols.nz, 2, hot_cfg(ntr=2, learned_kpp=1))
    vp.load_columns(cols)
    plain = VerticalPhysics(cols.nx, cols.ny, cols.nz, 2, hot_cfg(ntr=2))
    plain.load_columns(cols)
    s.attach(vp, check_fraction=0.05, check_tolerance=0.25, fail_fraction=0.5)
    vp.step(DT, 4)
    plain.step(DT, 4)
    st = L.kpp_stats(vp)
    assert st["checked"] > 0 and st["steps"] == 4 and st["gemm_err"] == 0
    bl, blp = np.asarray(vp.get("bl_depth")), np.asarray(plain.get("bl_depth"))
    wet = blp > 0
    e = np.sqrt(np.mean(((bl - blp) / np.maximum(blp, 1.0))[wet] ** 2))
    print(f"4-step OBL RMS rel error vs plain: {e:.3f}; stats {st}")
    assert np.isfinite(bl).all()
    # a zero tolerance fails every check: the next step runs the plain KPP everywhere
    s.attach(vp, check_fraction=0.05, check_tolerance=0.0, fail_fraction=0.0)
    vp.step(DT, 3)
    st = L.kpp_stats(vp)
    assert st["fallback_steps"] >= 1
    vp.close()
    plain.close()
