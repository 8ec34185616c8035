"""The trained plan model that ships with the package, evaluated on its own
held-out tensors (measured sweep times of every candidate plan): its choice
against the analytic model's, by regret against exhaustive timing. CPU only
(FP64 numpy forward of the committed parameters)."""
import json
import os

import numpy as np

from _mlp_ref import forward
from conftest import ROOT

DATA = os.path.join(ROOT, "adatm_b200", "planner_data")


def load():
    """The model, and the union of the data sets it was trained on (tensor
    ids offset per set) with its held-out mask per tensor."""
    m = np.load(os.path.join(DATA, "plan_model.npz"))
    rep = json.loads(str(m["report"]))
    names = rep.get("data", ["plan_data.npz"])
    X, y, t, c, a = [], [], [], [], []
    off = 0
    for n in names:
        d = np.load(os.path.join(DATA, n))
        X.append(d["X"])
        y.append(d["y"])
        t.append(d["tensor"] + off)
        c.append(d["cand"])
        a.append(d["analytic"])
        off += len(d["analytic"])
    data = {"X": np.concatenate(X), "y": np.concatenate(y), "tensor": np.concatenate(t),
            "cand": np.concatenate(c), "analytic": np.concatenate(a)}
    if "held" in m.files:
        held = np.asarray(m["held"], dtype=bool)
    else:
        held = np.arange(off) >= int(m["split"])
    return m, rep, data, held


def regrets(m, d, ids):
    X = (d["X"] - m["mean"]) / m["std"]
    pred, _, _ = forward(m["params"], [int(w) for w in m["widths"]], X)
    y, tensor, cand, analytic = d["y"], d["tensor"], d["cand"], d["analytic"]
    learned, anal = [], []
    for k in ids:
        sel = tensor == k
        if not sel.any():
            continue
        ms = 10.0 ** y[sel].astype(np.float64)
        learned.append(ms[np.argmin(pred[sel])] / ms.min() - 1)
        a = np.where(cand[sel] == analytic[k])[0]
        anal.append(ms[a[0]] / ms.min() - 1 if len(a) else ms.max() / ms.min() - 1)
    return np.array(learned), np.array(anal)


def test_model_shape_and_features():
    m, rep, d, held = load()
    widths = [int(w) for w in m["widths"]]
    assert widths[0] == 16 and widths[-1] == 1
    assert d["X"].shape[1] == 16 and np.all(np.isfinite(d["X"]))
    assert len(held) == len(d["analytic"]) == int(d["tensor"].max()) + 1


def test_learned_choice_beats_the_analytic_model_on_held_out_tensors():
    m, rep, d, held = load()
    ids = np.nonzero(held)[0]
    learned, anal = regrets(m, d, ids)
    assert len(learned) >= 100
    assert learned.mean() < 0.03
    assert learned.mean() < 0.25 * anal.mean()
    # the same choices the GPU forward made when the report was written
    assert abs(learned.mean() - rep["held_out"]["learned"]["mean"]) < 2e-3
    assert abs(anal.mean() - rep["held_out"]["analytic"]["mean"]) < 1e-6
