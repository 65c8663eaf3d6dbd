"""Host-side layout of a batched ensemble (dclaw_batch_layout): pure host
code in the C library, so it runs without a GPU."""
import ctypes

import numpy as np
import pytest

from dclaw_b200 import _lib
from dclaw_b200.params import CBatch, CMember

NREC = 14
TPB = 256


def _layout(mx, my, shape=0, dx=None):
    lib = _lib.load()
    n = len(mx)
    mx = np.asarray(mx, dtype=np.int32)
    my = np.asarray(my, dtype=np.int32)
    dxs = np.full(n, 0.05) if dx is None else np.asarray(dx, dtype=np.float64)
    cm = (CMember * n)()
    cb = CBatch()
    rc = lib.dclaw_batch_layout(n, mx.ctypes.data, my.ctypes.data, dxs.ctypes.data, dxs.ctypes.data, shape, cm,
                                ctypes.byref(cb))
    return rc, list(cm), cb


def test_struct_sizes():
    assert ctypes.sizeof(CMember) == 88
    assert ctypes.sizeof(CBatch) == 56


@pytest.mark.parametrize("shape", [0, 1, 2])
def test_layout_covers_every_member(shape):
    lib = _lib.load()
    tx = (ctypes.c_int32 * 8)()
    ty = (ctypes.c_int32 * 8)()
    nshape = lib.dclaw_batch_tile_shapes(tx, ty, 8)
    assert nshape == 3
    TX, TY = tx[shape], ty[shape]
    rng = np.random.default_rng(shape)
    mx = rng.integers(2, 300, size=17)
    my = rng.integers(2, 90, size=17)
    rc, cm, cb = _layout(mx, my, shape)
    assert rc == 0
    assert cb.nmembers == 17 and cb.tile_shape == shape
    q = b = w = tiles = rch = sch = 0
    for k, M in enumerate(cm):
        assert (M.mx, M.my) == (mx[k], my[k])
        assert M.q_off == q and M.b_off == b and M.tile0 == tiles and M.rchunk0 == rch and M.schunk0 == sch
        cells, npad = int(mx[k]) * int(my[k]), (int(mx[k]) + 4) * (int(my[k]) + 4)
        assert M.rec_off == w and M.rec_off % 32 == 0          # 256-byte aligned member block
        assert M.qs_off == w + NREC * npad
        assert M.ntiles_x == -(-int(mx[k]) // TX)
        assert M.ntiles == M.ntiles_x * -(-int(my[k]) // TY)
        assert M.nrchunks == -(-npad // TPB) and M.nschunks == -(-cells // TPB)
        q += 5 * cells
        b += cells
        w = -(-(M.qs_off + 5 * cells) // 32) * 32
        tiles += M.ntiles
        rch += M.nrchunks
        sch += M.nschunks
    assert (cb.q_doubles, cb.b_doubles, cb.ntiles, cb.nrchunks, cb.nschunks) == (q, b, tiles, rch, sch)
    # + two tile lists (active tiles, tiles whose records are built) and one
    # 32-bit activity flag per tile, each 256-byte aligned, then the counters
    assert cb.work_bytes == 8 * w + 3 * (-(-4 * tiles // 256) * 256) + 256


def test_layout_rejects_bad_members():
    assert _layout([10, 1], [10, 10])[0] == 1          # mx < 2
    assert _layout([10], [10], shape=3)[0] == 1         # no such tile shape
    assert _layout([10], [10], dx=[0.0])[0] == 1        # dx <= 0
    assert _layout([10], [10], dx=[float("nan")])[0] == 1
