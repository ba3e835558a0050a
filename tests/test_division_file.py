"""SHOCK's .sddc division files (src/Load.c:191-250): rows written by
cases.write_division in the layout loadDivision reads, read back by the
library's shock_read_division, including the Transform sign SHOCK derives
from the point ranges (check_TransformationMatrix, src/Functions.c:3902-4005),
the byte-swapped form (SwapDivFile) and a wrong rank count."""
import struct

import numpy as np
import pytest

import shock_b200
from shock_b200 import cases


def _division(rotated):
    c = cases.taylor_green(12, order=5)
    d = cases.split(c, (2, 2, 2))
    if rotated:
        d = cases.rotate_block(d, 3, (1, 0, 2), (True, False, False))
        d = cases.rotate_block(d, 6, (0, 2, 1), (False, False, True))
    return d


@pytest.mark.parametrize("rotated", [False, True])
def test_division_file_round_trip(tmp_path, rotated):
    d = _division(rotated)
    path = tmp_path / "div.sddc"
    cases.write_division(d, str(path))
    nb, tr, tf, co, sz = shock_b200.read_division(path, 3, len(d.blocks))
    assert np.array_equal(nb, d.neighbour)
    assert np.array_equal(tr, d.translation)
    want = np.where(d.neighbour[..., None] >= 0, d.transform, 0)
    assert np.array_equal(tf, want)
    for b, bl in enumerate(d.blocks):
        assert tuple(sz[b]) == (bl.ni, bl.nj, bl.nk)
    # the division read back sets up the same geometry, bit for bit
    back = cases.Division(case=d.case, parts=d.parts, blocks=d.blocks, neighbour=nb, translation=tr, lo=d.lo,
                          transform=tf, axes=d.axes, flips=d.flips)
    # (blocks with permuted axes take the full metric)
    g0 = shock_b200.host_multi_geometry(d, full_metric=rotated)
    g1 = shock_b200.host_multi_geometry(back, full_metric=rotated)
    assert all(np.array_equal(a, b) for a, b in zip(g0, g1))


def test_transform_sign_from_ranges(tmp_path):
    """A row whose face-axis Transform entry has the wrong sign (as grid tools
    write it) is read with the sign the point ranges give."""
    d = _division(True)
    path = tmp_path / "div.sddc"
    cases.write_division(d, str(path))
    raw = bytearray(path.read_bytes())
    row = len(raw) // len(d.blocks)
    ifblock = 4 + 3 * 4 + 2 * 6 * 8 + 9 * 4
    flipped = 0
    for b in range(len(d.blocks)):
        for f in range(6):
            off = b * row + 32 + 6 * 8 + f * ifblock + 4 + 4 * (f // 2)
            (v,) = struct.unpack_from("<i", raw, off)
            if v:
                struct.pack_into("<i", raw, off, -v)
                flipped += 1
    assert flipped == 48
    path.write_bytes(bytes(raw))
    _, _, tf, _, _ = shock_b200.read_division(path, 3, len(d.blocks))
    assert np.array_equal(tf, np.where(d.neighbour[..., None] >= 0, d.transform, 0))


def test_byte_swapped_division_file(tmp_path):
    d = _division(True)
    path = tmp_path / "div.sddc"
    cases.write_division(d, str(path))
    raw = path.read_bytes()
    row = len(raw) // len(d.blocks)
    ifblock = 4 + 3 * 4 + 2 * 6 * 8 + 9 * 4
    out = bytearray()
    for b in range(len(d.blocks)):
        r = raw[b * row:(b + 1) * row]
        out += r[:32]
        out += b"".join(r[32 + 8 * i:40 + 8 * i][::-1] for i in range(6))
        for f in range(6):
            blk = r[32 + 48 + f * ifblock:32 + 48 + (f + 1) * ifblock]
            sizes = [4] * 4 + [8] * 12 + [4] * 9
            pos = 0
            for s in sizes:
                out += blk[pos:pos + s][::-1]
                pos += s
    path.write_bytes(bytes(out))
    nb, tr, tf, _, _ = shock_b200.read_division(path, 3, len(d.blocks), swap=True)
    assert np.array_equal(nb, d.neighbour) and np.array_equal(tr, d.translation)
    assert np.array_equal(tf, np.where(d.neighbour[..., None] >= 0, d.transform, 0))


def test_division_file_size_checked(tmp_path):
    d = _division(False)
    path = tmp_path / "div.sddc"
    cases.write_division(d, str(path))
    with pytest.raises(shock_b200.ShockError):
        shock_b200.read_division(path, 3, len(d.blocks) + 1)
