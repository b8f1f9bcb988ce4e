"""The C-ABI library builds, loads and exports every declared entry point; with
no usable B200 the compute path refuses loudly (no CPU fallback). CPU only."""

import ctypes
import re
from pathlib import Path

import pytest

import fluidity_b200 as fb

HEADER = Path(__file__).resolve().parent.parent / "include" / "fluidity_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^(?:int|int64_t)\s+(fl_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_hot_path():
    names = declared_symbols()
    for required in ("fl_sort_particles_by_block", "fl_p2g", "fl_pressure_project", "fl_g2p", "fl_step",
                     "fl_deposit_mac_3d", "fl_deposit_mac_quanta_3d", "fl_gather_mac_3d"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = fb.library()
    for name in declared_symbols():
        assert hasattr(lib, name), name
        assert isinstance(getattr(lib, name), ctypes._CFuncPtr)


def test_no_cpu_fallback_without_a_b200():
    info = fb.runtime_info()
    assert info["compiled_architecture"] == 1000
    if info["device_count"] > 0 and info["major"] == 10:
        pytest.skip("a B200 is present")
    with pytest.raises(fb.FluidityError) as e:
        fb.LiquidContext(32, capacity=16)
    assert e.value.code == fb.FAILED_PRECONDITION
    with pytest.raises(fb.FluidityError) as e:
        fb.deposit_mac_3d([0, 0, 0], 1.0, [[0, 0, 0]], [[1.5] * 6 + [1.0] + [0.0] * 12])
    assert e.value.code == fb.FAILED_PRECONDITION
    # the allocation-free P2G refuses too (its pointers are never dereferenced on the host)
    import ctypes

    grid = fb.StaticGrid()
    grid.h, grid.block_count = 1.0, 1
    grid.block_coords = grid.neighbors = grid.cell_start = 16
    parts = fb.Particles()
    for d in range(3):
        parts.x[d] = parts.v[d] = 16
    for d in range(9):
        parts.c[d] = 16
    parts.count = 1
    outs = (ctypes.c_void_p * 3)(16, 16, 16)
    tp = fb.transfer_params(1e-3, 1.0)
    assert fb.library().fl_p2g_static_scratch(ctypes.byref(grid), ctypes.byref(parts), ctypes.byref(tp), 0, outs,
                                              outs, None, None) == fb.FAILED_PRECONDITION
