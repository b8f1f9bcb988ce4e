"""The allocation-free P2G entry point (fl_p2g_static_scratch) against the
context P2G (fl_p2g) through the C-ABI.

It exists for callers that cannot call cudaMalloc where they deposit (an
engine that owns all device memory through its own pool, or a substep that
must not allocate once started): its tile scratch is a static device array.
The test runs it twice in a row on the same inputs -- the second call sees
the first call's leftover scratch -- and requires both results to equal
fl_p2g's bit for bit, in both P2G modes (the same kernels in the same cell
order), with the device's free memory unchanged across the second call. A
malformed layout is refused before any output is written. It lives in its
own file, collected last, and needs a GPU."""

import ctypes

import numpy as np
import pytest

import fluidity_b200 as fb
from fluidity_b200 import scenes

pytestmark = pytest.mark.gpu


def _neighbors(blocks, bdim):
    table = -np.ones(tuple(bdim[::-1]), np.int32)
    table[blocks[:, 2], blocks[:, 1], blocks[:, 0]] = np.arange(len(blocks), dtype=np.int32)
    out = np.zeros((len(blocks), 27), np.int32)
    for n in range(27):
        dx, dy, dz = n % 3 - 1, (n // 3) % 3 - 1, n // 9 - 1
        x, y, z = blocks[:, 0] + dx, blocks[:, 1] + dy, blocks[:, 2] + dz
        inside = (x >= 0) & (y >= 0) & (z >= 0) & (x < bdim[0]) & (y < bdim[1]) & (z < bdim[2])
        out[:, n] = -2
        out[inside, n] = table[z[inside], y[inside], x[inside]]
    return out


def _particles(tensors, count):
    p = fb.Particles()
    for d in range(3):
        p.x[d] = tensors[d].data_ptr()
        p.v[d] = tensors[3 + d].data_ptr()
    for d in range(9):
        p.c[d] = tensors[6 + d].data_ptr()
    p.mass = None
    p.count = count
    return p


def test_static_scratch_p2g_matches_context_p2g_twice():
    import torch

    lib = fb.library()
    StaticGrid = fb.StaticGrid
    n = 64
    soa, mass = scenes.dam_break(n)
    count = soa.shape[1]
    ctx = fb.LiquidContext(n, capacity=count)
    src = [torch.from_numpy(np.ascontiguousarray(soa[k])).cuda() for k in range(15)]
    dst = [torch.empty_like(t) for t in src]
    pin, pout = _particles(src, count), _particles(dst, count)
    rep = fb.Report()
    assert lib.fl_topology_from_particles(ctx.handle, ctypes.byref(pin), None, ctypes.byref(rep)) == fb.OK
    assert lib.fl_sort_particles_by_block(ctx.handle, ctypes.byref(pin), ctypes.byref(pout), None,
                                          ctypes.byref(rep)) == fb.OK
    blocks = ctx.active_blocks()
    nb = len(blocks)
    assert 0 < nb <= 512
    f = ctx.fields()
    coords = torch.from_numpy(np.ascontiguousarray(blocks.astype(np.int32))).cuda()
    nbrs = torch.from_numpy(_neighbors(blocks, [n // 8] * 3)).cuda()
    grid = StaticGrid()
    grid.origin[:] = [0.0, 0.0, 0.0]
    grid.h = 1.0 / n
    grid.solid_lo[:] = [1, 1, 1]
    grid.solid_hi[:] = [n - 2] * 3
    grid.block_coords, grid.neighbors = coords.data_ptr(), nbrs.data_ptr()
    grid.cell_start, grid.block_count = f["cell_start"], nb
    tp = fb.transfer_params(scenes.DT, mass)
    arr = lambda ts: (ctypes.c_void_p * 3)(*[t.data_ptr() for t in ts])
    for mode in (0, 1):
        ref = [torch.zeros(nb * 512, device="cuda") for _ in range(6)]
        assert lib.fl_p2g(ctx.handle, ctypes.byref(pout), ctypes.byref(tp), mode, arr(ref[:3]), arr(ref[3:]), None,
                          ctypes.byref(rep)) == fb.OK
        for call in range(2):
            got = [torch.full((nb * 512,), float("nan"), device="cuda") for _ in range(6)]
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            code = lib.fl_p2g_static_scratch(ctypes.byref(grid), ctypes.byref(pout), ctypes.byref(tp), mode,
                                             arr(got[:3]), arr(got[3:]), None, ctypes.byref(rep))
            torch.cuda.synchronize()
            free_after = torch.cuda.mem_get_info()[0]
            assert code == fb.OK and rep.error == 0 and rep.compiled_architecture == 1000
            if call == 1:  # the first call on the device may load the module; later ones allocate nothing
                assert free_after == free_before
            for a in range(6):
                assert torch.equal(got[a], ref[a]), (mode, call, a)
    # a neighbour ordinal past the block count: refused, nothing written
    bad = nbrs.clone()
    bad[0, 13 + 1] = nb + 5
    malformed = StaticGrid.from_buffer_copy(grid)
    malformed.neighbors = bad.data_ptr()
    got = [torch.full((nb * 512,), 7.0, device="cuda") for _ in range(6)]
    code = lib.fl_p2g_static_scratch(ctypes.byref(malformed), ctypes.byref(pout), ctypes.byref(tp), 0,
                                     arr(got[:3]), arr(got[3:]), None, ctypes.byref(rep))
    assert code == fb.INVALID_ARGUMENT and rep.error == fb.INVALID_ARGUMENT
    assert rep.first_bad_index == nb * 512 + 1 + 14
    assert all(bool((t == 7.0).all()) for t in got)
    # a particle range past the particle count: refused as well
    host_cs = np.zeros(nb * 512 + 1, np.int32)
    assert lib.fl_copy_to_host(host_cs.ctypes.data, ctypes.c_void_p(f["cell_start"]), host_cs.nbytes) == fb.OK
    assert host_cs[-1] == count
    host_cs[-1] = count + 1000
    cs = torch.from_numpy(host_cs).cuda()
    malformed = StaticGrid.from_buffer_copy(grid)
    malformed.cell_start = cs.data_ptr()
    code = lib.fl_p2g_static_scratch(ctypes.byref(malformed), ctypes.byref(pout), ctypes.byref(tp), 0,
                                     arr(got[:3]), arr(got[3:]), None, ctypes.byref(rep))
    assert code == fb.INVALID_ARGUMENT and rep.first_bad_index == nb * 512
    assert all(bool((t == 7.0).all()) for t in got)
    too_many = StaticGrid.from_buffer_copy(grid)
    too_many.block_count = 513
    out = [torch.zeros(16, device="cuda") for _ in range(6)]
    code = lib.fl_p2g_static_scratch(ctypes.byref(too_many), ctypes.byref(pout), ctypes.byref(tp), 0,
                                     (ctypes.c_void_p * 3)(*[t.data_ptr() for t in out[:3]]),
                                     (ctypes.c_void_p * 3)(*[t.data_ptr() for t in out[3:]]), None, None)
    assert code == fb.RESOURCE_EXHAUSTED
    ctx.close()
