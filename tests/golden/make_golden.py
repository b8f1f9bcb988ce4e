"""Regenerate the golden vectors under tests/golden/ from the FluidiTy Python
reference (reference/src/fluidity_reference in the FluidiTy tree).

    FLUIDITY_REFERENCE=/path/to/FluidiTy python tests/golden/make_golden.py

Writes:
* transfer_3d.json -- uniform_mac_transfer_3d_fixture(): exact-rational P2G
  weights, offsets, gradients, masses and pure momenta of one particle across
  a block corner (transfer_3d_fixtures.py:23-111).
* pressure_3d.json -- uniform_mac_pressure_3d_fixture(): the seven dense
  manufactured pressure cases solved in FP64 (pressure_3d_fixtures.py:197-327).
* transport_3d.json -- sample_mac_transport(..., reconstruction="quadratic") on
  a seeded quadratic face field at seeded positions (mac_transport_3d.py:73-132):
  interpolated velocity and true gradient, the G2P oracle.

The reference is only needed to regenerate these files; tests read the JSON.
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _tolist(v):
    if isinstance(v, np.ndarray):
        return v.tolist()
    if isinstance(v, (list, tuple)):
        return [_tolist(x) for x in v]
    if isinstance(v, (np.integer,)):
        return int(v)
    if isinstance(v, (np.floating,)):
        return float(v)
    return v


def main():
    # the FluidiTy sources: $FLUIDITY_REFERENCE, else a checkout beside this repository
    root = Path(os.environ.get("FLUIDITY_REFERENCE", str(HERE.parent.parent.parent / "reference")))
    sys.path.insert(0, str(root / "reference" / "src"))
    from fluidity_reference import mac_transport_3d, pressure_3d_fixtures, transfer_3d_fixtures

    arrays, meta = transfer_3d_fixtures.uniform_mac_transfer_3d_fixture()
    (HERE / "transfer_3d.json").write_text(json.dumps({"arrays": _tolist(arrays), "metadata": meta}, indent=1))

    arrays, meta = pressure_3d_fixtures.uniform_mac_pressure_3d_fixture()
    (HERE / "pressure_3d.json").write_text(
        json.dumps({"arrays": {k: _tolist(v) for k, v in arrays.items()}, "metadata": meta}, indent=1))

    # Seeded quadratic-in-space face field: u_a(X) = c0 + g.X + X^T Q X on each axis.
    rng = np.random.default_rng(0)
    h = 0.25
    coeffs = [(rng.normal(), rng.normal(size=3), rng.normal(size=(3, 3))) for _ in range(3)]

    def field(axis, index):
        anchor = np.array(index, dtype=np.float64) + np.where(np.arange(3) == axis, 0.0, 0.5)
        c0, g, q = coeffs[axis]
        xw = anchor * h
        return float(c0 + g @ xw + xw @ q @ xw)

    positions = rng.uniform(1.0, 3.0, size=(16, 3))
    velocity, gradient = [], []
    for p in positions:
        v, gr = mac_transport_3d.sample_mac_transport(p, h, field, reconstruction="quadratic")
        velocity.append(v.tolist())
        gradient.append(gr.tolist())
    (HERE / "transport_3d.json").write_text(json.dumps({
        "h": h,
        "coefficients": [[float(c0), g.tolist(), q.tolist()] for c0, g, q in coeffs],
        "positions": positions.tolist(),
        "velocity": velocity,
        "gradient": gradient,
        "provenance": "fluidity_reference.mac_transport_3d.sample_mac_transport, reconstruction='quadratic'",
    }, indent=1))


if __name__ == "__main__":
    main()
