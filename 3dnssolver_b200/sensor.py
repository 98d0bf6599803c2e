"""Training of the learned troubled-face sensor on the GPU.

Faces are harvested from FP64 characteristic-wise runs (features + labels, see
ns_sensor_harvest) and the network is trained by the library's own BF16
tensor-core kernels (ns_sensor_train).  Device buffers are torch tensors.
"""
import importlib
import math
import time

import numpy as np

_pkg = importlib.import_module(__package__)
_wl = importlib.import_module(__package__ + ".workloads")


def harvest(params, W0, snapshots, every, rel_threshold=1e-3):
    """Features/labels of `snapshots` states of an FP64 run of params from W0, `every` steps apart."""
    import torch
    feats, labs = [], []
    with _pkg.Solver(params) as s:
        s.upload_primitive(W0)
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
    """Seeded runs of the two workload families: a Sod-type shock tube and the shear layer."""
    import torch
    ps = sod_params(96, 12, 12)
    Xs, ys = harvest(ps, _wl.sod(ps, seed=3), snapshots=4, every=20)
    ph = shear_params(48)
    Xh, yh = harvest(ph, _wl.shear_layer(ph, seed=1), snapshots=3, every=10)
    return torch.cat([Xs, Xh]), torch.cat([ys, yh])


def train(X, y, *, epochs=5, batch=4096, lr=3e-3, seed=0, max_pos_weight=20.0):
    """Trains a fresh network on device samples; returns (weights, info)."""
    import torch
    n = int(X.shape[0])
    npos = float(y.sum().item())
    pw = min((n - npos) / max(npos, 1.0), max_pos_weight)
    t0 = time.perf_counter()
    w, losses = _pkg.sensor_train(X.data_ptr(), y.data_ptr(), n, _pkg.sensor_init(seed), epochs=epochs,
                                  batch=batch, lr=lr, pos_weight=pw, seed=seed + 1)
    torch.cuda.synchronize()
    info = {"faces": n, "positive_fraction": npos / n, "pos_weight": pw, "epochs": epochs,
            "epoch_loss": [float(x) for x in losses], "seconds": time.perf_counter() - t0}
    return w, info
