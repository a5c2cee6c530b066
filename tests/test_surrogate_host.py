"""Surrogate scoring on the CPU: CSI = H / (H + F + M) over flooded cells
(FloodCA prep/floodca_prep/validation_metrics.py:84-106, 0 when nothing is
flooded in either map) and the RMSE of peak depth."""
import numpy as np
import pytest
import torch

from floodca_b200.surrogate import metrics


def test_csi_and_rmse_by_hand():
    truth = torch.tensor([[0.0, 0.2, 0.5], [0.05, 0.3, 0.0]])
    pred = torch.tensor([[0.15, 0.25, 0.05], [0.0, 0.4, 0.0]])
    m = metrics(pred, truth, thr=0.1)
    # flooded truth: (0,1) (0,2) (1,1); flooded prediction: (0,0) (0,1) (1,1)
    assert (m["hits"], m["false_alarms"], m["misses"]) == (2, 1, 1)
    assert m["csi_0p1"] == pytest.approx(2 / 4)
    e = (pred - truth).double().numpy()
    assert m["rmse_m"] == pytest.approx(float(np.sqrt((e ** 2).mean())))


def test_csi_empty_maps_is_zero():
    z = torch.zeros(4, 4)
    assert metrics(z, z)["csi_0p1"] == 0.0
