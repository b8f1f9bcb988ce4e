"""Host-side checks of the backend-table adapter and its harness (no GPU).

The adapter library (fluidity_b200/_lib/libfluidity_b200_backend.so, built
against the reference's headers) exports B200LiquidBackend3D; the harness
(oracle/_ref/libfluidity_backend_check.so) loads it beside the reference's CPU
table. Without a B200 the B200 table cannot be made and says so
(FailedPrecondition); the CPU table runs the bounded tank dam break on the host.
"""

import subprocess

import numpy as np
import pytest

import backend_tables as bt
from fluidity_b200 import build as cuda_build

pytestmark = pytest.mark.skipif(not bt.available(), reason="backend harness not built")


def test_adapter_exports_the_backend():
    out = subprocess.run(["nm", "-DC", "--defined-only", str(cuda_build.BACKEND)], capture_output=True, text=True,
                         check=True).stdout
    assert "fluidity::B200LiquidBackend3D::Create()" in out
    assert "fluidity::B200LiquidBackend3D::operations()" in out


def test_b200_table_refuses_without_a_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    code, _ = bt.filled(bt.B200)
    assert code == 9  # FailedPrecondition, as the reference's CUDA operators without a device
    assert bt.deposit(bt.B200, bt.Scene())[0] == 9


def test_cpu_table_runs_the_bounded_dam_break():
    code, mask = bt.filled(bt.CPU)
    assert code == 0 and mask == 0x7FF
    s = bt.Scene(mixed_sides=False)
    code, q, st = bt.deposit(bt.CPU, s)
    assert code == 0
    assert q["stress"].max() == 0 and q["mass"].min() >= 0
    # every particle's compatible weights sum to one per component
    w = np.where(st["compatible"] == 1, st["weight"], 0.0).sum(axis=2)
    assert np.abs(w - 1.0).max() < 1e-12
    code, m, v, val = bt.normalize(bt.CPU, q, 0.1 * float(s.particles["mass"][0]))
    assert code == 0 and {0, 1, 3} <= set(np.unique(val).tolist())
    code, g, counts = bt.gather(bt.CPU, s, (v, val), (v, val))
    assert code == 0 and counts[0] == counts[1] > 0


def test_cpu_table_assembles_the_links_of_the_frozen_pool():
    s = bt.LinkScene()
    code, cells, faces, lower = bt.links(bt.CPU, s)
    assert code == 0 and lower > 0
    assert np.array_equal(np.bincount(faces[:, 0].astype(int), minlength=3) > 0, [True, True, True])
