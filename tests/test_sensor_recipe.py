"""The learned sensor's training recipe at full size, on the GPU: about 50 M faces
harvested from the 64^3 component-wise shear layer and the 512x128x128 Sod shock
tube, a seeded 90/10 split, Adam at lr 1e-3 for 5 epochs on the library's own
BF16 tensor-core kernels, and the network judged on the held-out tenth.

Bounds (physical semantics, the headline workload's): held-out recall of the
faces whose characteristic-wise and component-wise fluxes differ by more than
1e-3 relative >= 0.9 (measured 0.98 on B200), precision >= 0.4 (measured 0.58):
the gate must find nearly every such face, and a false alarm only costs a
characteristic-wise face where a component-wise one would have done."""
import importlib
import math

import pytest

pkg = importlib.import_module("3dnssolver_b200")
sensor = importlib.import_module("3dnssolver_b200.sensor")

pytestmark = pytest.mark.gpu


def test_recipe_held_out_recall_and_precision():
    w, info = sensor.train_recipe(semantics=pkg.SEM_PHYSICAL, seed=0)
    assert 45e6 <= info["faces"] + info["held_out"]["faces"] <= 55e6  # about 50 M faces
    assert info["held_out"]["faces"] == pytest.approx(0.1 * (info["faces"] + info["held_out"]["faces"]), rel=1e-3)
    loss = info["epoch_loss"]
    assert all(math.isfinite(x) for x in loss) and loss[-1] < loss[0], loss
    h = info["held_out"]
    assert h["recall"] >= 0.9, h
    assert h["precision"] >= 0.4, h
