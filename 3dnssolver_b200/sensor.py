"""Training of the learned troubled-face sensor on the GPU.

Faces are harvested from FP64 runs (features + labels, see ns_sensor_harvest)
and the network is trained by the library's own BF16 tensor-core kernels
(ns_sensor_train).  Device buffers are torch tensors.

The training recipe: about 50 M faces harvested from seeded runs of the
component-wise 64^3 shear layer (100 steps) and the 512x128x128 Sod shock tube,
a seeded 90/10 split into training and held-out faces, Adam at lr 1e-3 for 5
epochs, and the held-out precision and recall of the trained network.
"""
import importlib
import math
import time

import numpy as np

_pkg = importlib.import_module(__package__)
_wl = importlib.import_module(__package__ + ".workloads")


def harvest(params, W0, snapshots, every, rel_threshold=1e-3, start=0):
    """Features/labels of `snapshots` states of an FP64 run of params from W0: the
    state after `start` steps, then every `every` steps."""
    import torch
    feats, labs = [], []
    with _pkg.Solver(params) as s:
        s.upload_primitive(W0)
        if start:
            s.advance(start)
        cap = s.faces()
        for k in range(snapshots):
            f = torch.empty((cap, _pkg.SENSOR_FEATURES), dtype=torch.float32, device="cuda")
            l = torch.empty(cap, dtype=torch.float32, device="cuda")
            s.sensor_harvest(f.data_ptr(), l.data_ptr(), cap, rel_threshold)
            feats.append(f)
            labs.append(l)
            if k + 1 < snapshots:
                s.advance(every)
    return torch.cat(feats), torch.cat(labs)


def sod_params(nx, ny, nz, **kw):
    """3D Sod problem along x (Neumann x, periodic y/z) on the unit box."""
    args = dict(L=(1.0, 1.0, 1.0), mu=1e-4, Pr=0.72, cfl=0.4, convection=_pkg.CONV_WENO5_CHAR,
                diffusion_order=2, bc=(_pkg.BC_NEUMANN, _pkg.BC_PERIODIC, _pkg.BC_PERIODIC))
    args.update(kw)
    return _pkg.make_params(nx, ny, nz, **args)


def shear_params(n, **kw):
    L = 2 * math.pi
    args = dict(L=(L, L, L), mu=2.0 * 0.05 * 2 * math.pi / 1000.0, Pr=0.72, cfl=0.5,
                convection=_pkg.CONV_WENO5_CHAR, diffusion_order=2)
    args.update(kw)
    return _pkg.make_params(n, n, n, **args)


def default_training_set():
    """A small set for tests: seeded runs of a Sod-type shock tube and the shear layer."""
    import torch
    ps = sod_params(96, 12, 12)
    Xs, ys = harvest(ps, _wl.sod(ps, seed=3), snapshots=4, every=20)
    ph = shear_params(48)
    Xh, yh = harvest(ph, _wl.shear_layer(ph, seed=1), snapshots=3, every=10)
    return torch.cat([Xs, Xh]), torch.cat([ys, yh])


def sod_cfl(semantics):
    """CFL of the 512x128x128 Sod run: the reference semantics' characteristic-wise run turns
    non-finite within 40 steps at CFL 0.4 (its min-over-axes dt and eigenvector terms) and
    stays finite to t = 0.2 at CFL 0.2; the physical semantics run at CFL 0.4."""
    return 0.4 if semantics == _pkg.SEM_PHYSICAL else 0.2


def recipe_training_set(semantics=0, shear_snapshots=31, sod_start=150, sod_shape=(512, 128, 128)):
    """The recipe's faces: the 64^3 component-wise shear layer (states every 3 steps over
    its first 93 steps, 0.8 M faces each) and the Sod shock tube 512x128x128 with Ly = Lz = 1
    after `sod_start` steps (25.3 M faces), labels from the FP64 fluxes of `semantics`."""
    import torch
    p1 = shear_params(64, convection=_pkg.CONV_WENO5, semantics=semantics)
    X1, y1 = harvest(p1, _wl.shear_layer(p1, seed=1), snapshots=shear_snapshots, every=3)
    p3 = sod_params(*sod_shape, semantics=semantics, cfl=sod_cfl(semantics))
    X3, y3 = harvest(p3, _wl.sod(p3, seed=3), snapshots=1, every=1, start=sod_start)
    X, y = torch.cat([X1, X3]), torch.cat([y1, y3])
    del X1, X3
    return X, y, {"shear_faces": int(y1.numel()), "sod_faces": int(y3.numel())}


def train(X, y, *, epochs=5, batch=4096, lr=1e-3, seed=0, max_pos_weight=20.0):
    """Trains a fresh network on device samples; returns (weights, info)."""
    import torch
    n = int(X.shape[0])
    npos = float(y.sum().item())
    pw = min((n - npos) / max(npos, 1.0), max_pos_weight)
    t0 = time.perf_counter()
    w, losses = _pkg.sensor_train(X.data_ptr(), y.data_ptr(), n, _pkg.sensor_init(seed), epochs=epochs,
                                  batch=batch, lr=lr, pos_weight=pw, seed=seed + 1)
    torch.cuda.synchronize()
    info = {"faces": n, "positive_fraction": npos / n, "pos_weight": pw, "epochs": epochs, "lr": lr,
            "batch": batch, "epoch_loss": [float(x) for x in losses],
            "seconds": time.perf_counter() - t0}
    return w, info


def evaluate(X, y, w, threshold=0.5):
    """Precision, recall and accuracy of the network's flags (sigmoid > threshold) on device samples."""
    import torch
    n = int(X.shape[0])
    lg = torch.empty(n, dtype=torch.float32, device=X.device)
    _pkg.sensor_predict(X.data_ptr(), n, w, lg.data_ptr())
    pred = lg > math.log(threshold / (1.0 - threshold))
    lab = y > 0.5
    tp = float((pred & lab).sum().item())
    fp = float((pred & ~lab).sum().item())
    fn = float((~pred & lab).sum().item())
    return {"faces": n, "positive_fraction": float(lab.float().mean().item()),
            "flagged_fraction": float(pred.float().mean().item()),
            "precision": tp / max(tp + fp, 1.0), "recall": tp / max(tp + fn, 1.0),
            "accuracy": float((pred == lab).float().mean().item())}


def train_recipe(semantics=0, seed=0, holdout=0.1, **set_kw):
    """The full recipe: harvest, seeded 90/10 split, Adam lr 1e-3 for 5 epochs, held-out metrics."""
    import torch
    t0 = time.perf_counter()
    X, y, src = recipe_training_set(semantics, **set_kw)
    n = int(y.numel())
    g = torch.Generator(device="cuda")
    g.manual_seed(1000 + seed)
    perm = torch.randperm(n, device="cuda", generator=g)
    nh = int(round(holdout * n))
    hold, tr = perm[:nh], perm[nh:]
    Xh, yh = X[hold].contiguous(), y[hold].contiguous()
    Xt, yt = X[tr].contiguous(), y[tr].contiguous()
    del X, y, perm
    harvest_s = time.perf_counter() - t0
    w, info = train(Xt, yt, epochs=5, lr=1e-3, seed=seed)
    info["held_out"] = evaluate(Xh, yh, w)
    info["train_set"] = evaluate(Xt, yt, w)
    info.update(src)
    info["harvest_seconds"] = harvest_s
    info["semantics"] = "physical" if semantics else "reference"
    del Xt, yt, Xh, yh
    torch.cuda.empty_cache()
    return w, info
