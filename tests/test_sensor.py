"""Learned troubled-face sensor: BF16 tensor-core kernels against the numpy
restatement (oracle/sensor_mlp.py), harvested features/labels against the CPU
oracle's face fluxes, training, and what the trained network gains over the
component-wise method on a shock problem."""
import importlib
import json
import math

import numpy as np
import pytest

from conftest import interior, rel_l2
from oracle import sensor_mlp as SM

pkg = importlib.import_module("3dnssolver_b200")
wl = importlib.import_module("3dnssolver_b200.workloads")
P, N = pkg.BC_PERIODIC, pkg.BC_NEUMANN


def test_init_layout_cpu():
    w = pkg.sensor_init(7)
    assert w.shape == (SM.NP,)
    W1 = w[:1024].reshape(32, 32)
    assert np.all(W1[:, SM.NF:] == 0) and np.abs(W1[:, :SM.NF]).max() > 0
    assert np.all(w[SM.OFF_B1:SM.OFF_W2] == 0) and np.all(w[SM.OFF_B2:SM.OFF_W3] == 0)
    assert w[SM.OFF_B3] == 0
    np.testing.assert_array_equal(w, pkg.sensor_init(7))


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.gpu
def test_gradients_match_numpy():
    rng = np.random.default_rng(0)
    n = 1000
    X = (rng.standard_normal((n, SM.NF)) * 0.7).astype(np.float32)
    y = (rng.random(n) < 0.25).astype(np.float32)
    w = pkg.sensor_init(3)
    w[SM.OFF_B1:SM.OFF_W2] = 0.1 * rng.standard_normal(32)
    w[SM.OFF_B3] = -0.3
    dX, dy = _dev(X), _dev(y)
    g, loss = pkg.sensor_gradients(dX.data_ptr(), dy.data_ptr(), n, w, pos_weight=3.0)
    loss_ref, g_ref = SM.loss_and_grad(X, y, w, 3.0)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    # BF16 operands, FP32 accumulation: a few 1e-3 per element, 1e-2 on the whole
    rel = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    cos = g @ g_ref / (np.linalg.norm(g) * np.linalg.norm(g_ref))
    assert rel < 3e-2 and cos > 0.999, (rel, cos)
    for name, a, b in [("W1", 0, 1024), ("b1", 1024, 1056), ("W2", 1056, 2080), ("b2", 2080, 2112),
                       ("w3", 2112, 2144), ("b3", 2144, 2145)]:
        e = np.linalg.norm(g[a:b] - g_ref[a:b]) / (np.linalg.norm(g_ref[a:b]) + 1e-12)
        assert e < 5e-2, (name, e)


@pytest.mark.gpu
def test_logits_match_numpy():
    import torch
    rng = np.random.default_rng(1)
    n = 777
    X = (rng.standard_normal((n, SM.NF)) * 0.7).astype(np.float32)
    w = pkg.sensor_init(4)
    dX = _dev(X)
    out = torch.zeros(n, dtype=torch.float32, device="cuda")
    pkg.sensor_predict(dX.data_ptr(), n, w, out.data_ptr())
    ref, _ = SM.forward(X, w)
    err = np.abs(out.cpu().numpy() - ref)
    assert (err <= 2e-2 * (1 + np.abs(ref))).all(), err.max()


@pytest.mark.gpu
def test_harvest_features_and_labels_match_oracle(oracle):
    import torch
    p = pkg.make_params(12, 10, 8, convection=pkg.CONV_WENO5_CHAR, bc=(N, P, P), mu=0.01)
    W0 = wl.random_field(p, seed=31, smooth=False)
    with pkg.Solver(p) as s:
        s.upload_primitive(W0)
        cap = s.faces()
        feat = torch.zeros((cap, SM.NF), dtype=torch.float32, device="cuda")
        lab = torch.zeros(cap, dtype=torch.float32, device="cuda")
        n = s.sensor_harvest(feat.data_ptr(), lab.data_ptr(), cap, 1e-3)
    assert n == cap
    feat, lab = feat.cpu().numpy(), lab.cpu().numpy()
    W, U = oracle.prologue(p, W0)
    pc = pkg.make_params(12, 10, 8, convection=pkg.CONV_WENO5, bc=(N, P, P), mu=0.01)
    rows_f, rows_l = [], []
    nx, ny, nz = 12, 10, 8
    for d in range(3):
        fx = oracle.face_flux(p, d, W, U)
        fc = oracle.face_flux(pc, d, W, U)
        sl = [slice(3, 3 + nx), slice(3, 3 + ny), slice(3, 3 + nz)]
        sl[d] = slice(2, 3 + [nx, ny, nz][d])
        a, b = fx[tuple(sl)].reshape(-1, 5), fc[tuple(sl)].reshape(-1, 5)
        rows_l.append(np.linalg.norm(a - b, axis=1) > 1e-3 * (np.linalg.norm(a, axis=1) + 1e-12))
        rows_f.append(SM.features(*SM.stencils(W, d), p.gamma))
    ref_l = np.concatenate(rows_l).astype(np.float32)
    ref_f = np.concatenate(rows_f)
    assert (lab != ref_l).mean() <= 1e-3
    assert 0.02 < ref_l.mean() < 0.98  # the field mixes troubled and smooth faces
    np.testing.assert_allclose(feat, ref_f, atol=2e-4, rtol=1e-3)


def _sod_params(nx, ny, nz, **kw):
    args = dict(L=(1.0, 1.0, 1.0), mu=1e-4, Pr=0.72, cfl=0.4, convection=pkg.CONV_WENO5_CHAR,
                diffusion_order=2, bc=(N, P, P))
    args.update(kw)
    return pkg.make_params(nx, ny, nz, **args)


def _harvest_run(p, W0, snapshots, every):
    """Device features/labels of several snapshots of an FP64 characteristic run."""
    import torch
    feats, labs = [], []
    with pkg.Solver(p) as s:
        s.upload_primitive(W0)
        cap = s.faces()
        for k in range(snapshots):
            f = torch.zeros((cap, SM.NF), dtype=torch.float32, device="cuda")
            l = torch.zeros(cap, dtype=torch.float32, device="cuda")
            s.sensor_harvest(f.data_ptr(), l.data_ptr(), cap, 1e-3)
            feats.append(f)
            labs.append(l)
            s.advance(every)
    return torch.cat(feats), torch.cat(labs)


@pytest.mark.gpu
def test_training_learns_the_labels():
    import torch
    p = _sod_params(64, 12, 12)
    X, y = _harvest_run(p, wl.sod(p, seed=3), snapshots=3, every=15)
    n = X.shape[0]
    npos = float(y.sum().item())
    assert 0 < npos < n
    pw = min((n - npos) / npos, 20.0)
    w0 = pkg.sensor_init(11)
    w, losses = pkg.sensor_train(X.data_ptr(), y.data_ptr(), n, w0, epochs=6, batch=2048, lr=3e-3,
                                 pos_weight=pw, seed=5)
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.6 * losses[0], losses
    lg = torch.zeros(n, dtype=torch.float32, device="cuda")
    pkg.sensor_predict(X.data_ptr(), n, w, lg.data_ptr())
    pred = (lg > 0).float()
    recall = float((pred * y).sum() / y.sum())
    assert recall > 0.8, recall


@pytest.mark.gpu
def test_gated_form_gains_over_component_wise(tmp_path):
    """Train on a Sod run at one resolution, gate the FP32 characteristic scheme on
    another; errors in rho and rhoE against the FP64 characteristic run."""
    import torch
    ptrain = _sod_params(96, 12, 12)
    X, y = _harvest_run(ptrain, wl.sod(ptrain, seed=3), snapshots=4, every=20)
    n = X.shape[0]
    npos = float(y.sum().item())
    w, losses = pkg.sensor_train(X.data_ptr(), y.data_ptr(), n, pkg.sensor_init(2), epochs=5,
                                 batch=4096, lr=3e-3, pos_weight=min((n - npos) / npos, 20.0), seed=9)
    nx, ny, nz, steps = 128, 16, 16, 60
    p64 = _sod_params(nx, ny, nz)
    W0 = wl.sod(p64, seed=4, amp=0.02)

    def run(**kw):
        pr = _sod_params(nx, ny, nz, **kw)
        with pkg.Solver(pr) as s:
            if kw.get("sensor"):
                s.set_sensor_weights(w)
            s.upload_primitive(W0)
            s.advance(steps)
            d = s.diagnostics()
            return s.download_conservative(), d

    U64, _ = run()
    res = {}
    for name, kw in {"fp32_comp": dict(precision=pkg.PREC_FP32, convection=pkg.CONV_WENO5),
                     "fp32_gated": dict(precision=pkg.PREC_FP32, sensor=1),
                     "fp32_char": dict(precision=pkg.PREC_FP32)}.items():
        U, d = run(**kw)
        e = rel_l2(interior(U), interior(U64))
        res[name] = {"rel_l2_rho": float(e[0]), "rel_l2_rhoE": float(e[1]),
                     "sensor_fraction": d["sensor_fraction"]}
    res["train"] = {"faces": n, "positive_fraction": npos / n, "epoch_loss": [float(x) for x in losses]}
    print(json.dumps(res))
    (tmp_path / "sensor_gain.json").write_text(json.dumps(res, indent=1))
    g, c, x = res["fp32_gated"], res["fp32_comp"], res["fp32_char"]
    assert 0.0 < g["sensor_fraction"] < 1.0
    assert g["rel_l2_rho"] < c["rel_l2_rho"] and g["rel_l2_rhoE"] < c["rel_l2_rhoE"], res


@pytest.mark.gpu
@pytest.mark.parametrize("order,weights,bc", [(2, 0, (N, P, P)), (4, 1, (P, N, P)), (6, 0, (N, N, N))])
def test_gate_extremes_equal_the_ungated_forms(order, weights, bc):
    """A network whose only nonzero parameter is the output bias flags every face
    (b3 > 0) or none (b3 < 0).  None: the gated step is the component-wise stage
    alone, bit for bit.  Every face: component-wise stages corrected by the
    characteristic-wise minus component-wise flux of every face, which is FP32
    characteristic-wise up to the FP32 rounding of that difference: as close to
    the FP64 characteristic-wise run as ungated FP32 characteristic-wise is (to
    10 %), and within 5e-6 of it (measured 1.4e-6 in rhoW, 2e-7 in rho)."""
    shape = (20, 12, 10)
    kw = dict(convection=pkg.CONV_WENO5_CHAR, diffusion_order=order, weights=weights, bc=bc, mu=0.02,
              cfl=0.3, precision=pkg.PREC_FP32)
    p = pkg.make_params(*shape, **kw)
    W0 = wl.random_field(p, seed=31, smooth=False)

    def run(b3=None, **extra):
        q = pkg.make_params(*shape, **dict(kw, **extra))
        with pkg.Solver(q) as s:
            if b3 is not None:
                w = np.zeros(pkg.SENSOR_NPARAMS, dtype=np.float32)
                w[-1] = b3
                s.set_sensor_weights(w)
            s.upload_primitive(W0)
            s.advance(3)
            return s.download_conservative(), s.diagnostics()["sensor_fraction"]

    U_64, _ = run(precision=pkg.PREC_FP64)
    U_char, _ = run()
    U_comp, _ = run(convection=pkg.CONV_WENO5)
    U_all, f_all = run(sensor=1, b3=10.0)
    U_none, f_none = run(sensor=1, b3=-10.0)
    assert f_all == 1.0 and f_none == 0.0
    np.testing.assert_array_equal(interior(U_none), interior(U_comp))
    e_all = rel_l2(interior(U_all), interior(U_char))
    assert (e_all <= 5e-6).all(), f"all flagged vs characteristic-wise: {e_all}"
    acc_all = rel_l2(interior(U_all), interior(U_64))
    acc_char = rel_l2(interior(U_char), interior(U_64))
    assert (acc_all <= 1.1 * acc_char).all(), (acc_all, acc_char)


@pytest.mark.gpu
def test_step_flags_agree_with_the_predict_path():
    """The per-step flags (the network on the tcgen05 tensor cores, from the step's
    FP32 primitive planes) flag the same faces, up to the last BF16 rounding, as
    ns_sensor_predict (mma.sync) on the features harvested from the same state."""
    import torch
    sensor_mod = importlib.import_module("3dnssolver_b200.sensor")
    X, y = sensor_mod.default_training_set()
    w, _ = sensor_mod.train(X, y, seed=3)
    p32 = _sod_params(96, 12, 12, precision=pkg.PREC_FP32, sensor=1)
    W0 = wl.sod(p32, seed=3)
    with pkg.Solver(p32) as s:
        s.set_sensor_weights(w)
        s.upload_primitive(W0)
        s.advance(1)
        frac_step = s.diagnostics()["sensor_fraction"]
    p64 = _sod_params(96, 12, 12)
    with pkg.Solver(p64) as s:
        s.upload_primitive(W0)
        cap = s.faces()
        f = torch.empty((cap, pkg.SENSOR_FEATURES), dtype=torch.float32, device="cuda")
        lab = torch.empty(cap, dtype=torch.float32, device="cuda")
        n = s.sensor_harvest(f.data_ptr(), lab.data_ptr(), cap)
    lg = torch.empty(n, dtype=torch.float32, device="cuda")
    pkg.sensor_predict(f.data_ptr(), n, w, lg.data_ptr())
    frac_pred = float((lg > 0).float().mean().item())
    assert frac_pred > 0.01
    assert abs(frac_step - frac_pred) <= 0.005 + 0.02 * frac_pred, (frac_step, frac_pred)
