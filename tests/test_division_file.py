"""SHOCK's .sddc division files (src/Load.c:191-250): rows written by
cases.write_division in the layout loadDivision reads, read back by the
library's shock_read_division, including the Transform sign SHOCK derives
from the point ranges (check_TransformationMatrix, src/Functions.c:3902-4005),
the byte-swapped form (SwapDivFile) and a wrong rank count; and the same
files read by SHOCK itself: its ranks load their rows with its own
loadDivision, take them in as loadFile does and set up their geometry, bit
for bit the geometry the library sets up from its reading of the file."""
import os
import struct

import numpy as np
import pytest

import shock_b200
from refbind import generator_path, load_division_row, multirank_available, run_multirank
from shock_b200 import cases
from test_multiblock_host import CGRIDS, DIVISIONS, cgrid_division, division as named_division


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


def _read_back(d, path, swap=False):
    nb, tr, tf, _, _ = shock_b200.read_division(path, d.case.dim, len(d.blocks), swap=swap)
    return cases.Division(case=d.case, parts=d.parts, blocks=d.blocks, neighbour=nb, translation=tr, lo=d.lo,
                          transform=tf, axes=d.axes, flips=d.flips)


def _flip_face_axis_entries(d, path):
    """Negate every interface's Transform entry of its own face axis in the
    file, as grid tools write it; returns how many were negated."""
    dim = d.case.dim
    raw = bytearray(path.read_bytes())
    row = len(raw) // len(d.blocks)
    ifblock = 4 + dim * 4 + 4 * dim * 8 + 9 * 4
    flipped = 0
    for b in range(len(d.blocks)):
        for f in range(2 * dim):
            off = b * row + 32 + 2 * dim * 8 + f * ifblock + 4 + 4 * (f // 2)
            (v,) = struct.unpack_from("<i", raw, off)
            if v:
                struct.pack_into("<i", raw, off, -v)
                flipped += 1
    path.write_bytes(bytes(raw))
    return flipped


def _swap_file(d, path):
    """The file with every number byte-swapped (a big-endian writer)."""
    dim = d.case.dim
    raw = path.read_bytes()
    row = len(raw) // len(d.blocks)
    sizes = [4] * (1 + dim) + [8] * (4 * dim) + [4] * 9
    out = bytearray()
    for b in range(len(d.blocks)):
        r = raw[b * row:(b + 1) * row]
        out += r[:32]
        out += b"".join(r[32 + 8 * i:40 + 8 * i][::-1] for i in range(2 * dim))
        pos = 32 + 16 * dim
        for f in range(2 * dim):
            for sz in sizes:
                out += r[pos:pos + sz][::-1]
                pos += sz
    path.write_bytes(bytes(out))


@pytest.mark.parametrize("form", ["as_written", "face_axis_signs_flipped", "byte_swapped"])
@pytest.mark.parametrize("name", sorted(DIVISIONS))
def test_shock_reads_the_same_division(tmp_path, name, form):
    case, d, full = named_division(name)
    if not multirank_available(case.order, case.dim, full=full):
        pytest.skip("multi-rank reference build absent (make -C oracle with the reference sources)")
    if form != "as_written" and "rotated" not in name:
        pytest.skip("the altered forms run on the rotated divisions")
    path = tmp_path / "div.sddc"
    cases.write_division(d, str(path))
    swap = False
    if form == "face_axis_signs_flipped":
        assert _flip_face_axis_entries(d, path) == int((d.neighbour[:, :2 * case.dim] >= 0).sum())
    elif form == "byte_swapped":
        _swap_file(d, path)
        swap = True
    got = shock_b200.host_multi_geometry(_read_back(d, path, swap), full_metric=full)
    # SHOCK's SwapDivFile: 2 swaps always, 0 decides by the host's byte order
    ref = run_multirank(d, 0, full=full, division_file=path, swap=2 if swap else 0)
    for b in range(len(d.blocks)):
        assert np.array_equal(got[b], ref[b]["geometry"]), (name, form, b)


# the division files SHOCK ships with its test cases, in the reference tree
# beside this repository (the same place oracle/Makefile compiles from)
SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "reference", "testcases")


# SHOCK's cube test cases: 2D divided 2x2, 3D 2x4x1 (16x16x16) and 2x2x2
SHIPPED_FILES = ("2d_cube_16x16.sddc", "2d_cube_32x32.sddc", "2d_cube_64x64.sddc", "3d_cube_16x16x16.sddc",
                 "3d_cube_32x32x32.sddc", "3d_cube_64x64x64.sddc")


@pytest.mark.parametrize("name", SHIPPED_FILES)
def test_shipped_division_files(name):
    """SHOCK's own division files (2D 2x2, 3D 2x4x1 and 2x2x2 divisions of
    its cube test cases) read by the library as SHOCK's loadDivision reads them:
    every rank's corners, neighbours, Transforms (with the face-axis sign
    check_TransformationMatrix takes from the point ranges) and
    Translations."""
    if not os.path.exists(os.path.join(SHIPPED, name)):
        pytest.skip("SHOCK's test cases are not beside this repository")
    if not multirank_available(5, 2) or not multirank_available(5, 3):
        pytest.skip("multi-rank reference build absent (make -C oracle with the reference sources)")
    dim = 2 if name.startswith("2d") else 3
    path = os.path.join(SHIPPED, name)
    row = 32 + 16 * dim + 2 * dim * (4 + 4 * dim + 32 * dim + 36)
    size = os.path.getsize(path)
    assert size % row == 0
    nranks = size // row
    nb, tr, tf, co, sz = shock_b200.read_division(path, dim, nranks)
    interfaces = 0
    for r in range(nranks):
        corners, faces = load_division_row(path, dim, r, nranks)
        assert np.array_equal(co[r], corners)
        assert np.array_equal(sz[r][:dim], corners[3:3 + dim] - corners[:dim] + 1)
        for f, (n, t, rng, drng, trans) in enumerate(faces):
            assert nb[r, f] == (n - 1 if n else -1)
            if not n:
                continue
            interfaces += 1
            a = f // 2
            me = next(x for x in range(dim) if rng[x] == rng[dim + x])
            do = next(x for x in range(dim) if drng[x] == drng[dim + x])
            want = t[:dim].copy()
            want[a] = (1 if rng[me] != 1 else -1) * (1 if drng[do] == 1 else -1) * abs(t[a])
            assert np.array_equal(tf[r, f, :dim], want)
            assert np.array_equal(tr[r, f], trans)
            # every neighbour names this rank back across its matching face
            assert nb[n - 1, f ^ 1] == r
    assert interfaces == {2: 8, 3: 20 if "16x16x16" in name else 24}[dim]


def _check_rows_as_shock_reads_them(path, dim, nranks):
    """Every rank's row of a division file: the library's reading against
    SHOCK's loadDivision with the face-axis sign of
    check_TransformationMatrix; returns the library's tables."""
    nb, tr, tf, co, sz = shock_b200.read_division(path, dim, nranks)
    for r in range(nranks):
        corners, faces = load_division_row(path, dim, r, nranks)
        assert np.array_equal(co[r], corners), r
        for f, (n, t, rng, drng, trans) in enumerate(faces):
            assert nb[r, f] == (n - 1 if n else -1), (r, f)
            if not n:
                continue
            a = f // 2
            me = next(x for x in range(dim) if rng[x] == rng[dim + x])
            do = next(x for x in range(dim) if drng[x] == drng[dim + x])
            want = t[:dim].copy()
            want[a] = (1 if rng[me] != 1 else -1) * (1 if drng[do] == 1 else -1) * abs(t[a])
            assert np.array_equal(tf[r, f, :dim], want), (r, f)
            assert np.array_equal(tr[r, f], trans), (r, f)
    return nb, tr, tf, co, sz


def test_generated_cgrid_division(tmp_path):
    """The division SHOCK's own generator writes (TOOLS/generatedivfile/
    generatedivfile_3.c, run unmodified: a 2048x256x256 C-grid in 4096
    blocks of 32^3, the wake cut joining mirrored blocks bottom to bottom
    with Transform (-1,-2,3), a periodic span with a float32 Translation)
    read by the library as SHOCK reads it, every rank; and every interface
    named back from the other side with the inverse Transform, which is what
    the library's division set-up requires."""
    import subprocess
    gen = generator_path()
    if gen is None or not multirank_available(5, 3):
        pytest.skip("SHOCK's generator or the multi-rank reference build absent (make -C oracle)")
    subprocess.run([gen], cwd=tmp_path, check=True, capture_output=True)
    (path,) = list(tmp_path.glob("*.sddc"))
    nb, tr, tf, co, sz = _check_rows_as_shock_reads_them(path, 3, 4096)
    assert (sz == 32).all()
    wake = 0
    for r in range(4096):
        for f in range(6):
            n = nb[r, f]
            if n < 0:
                continue
            t = tf[r, f]
            a, hi = f // 2, f % 2
            fd = 2 * (abs(t[a]) - 1) + (hi ^ int(t[a] > 0))
            assert nb[n, fd] == r, (r, f)
            back = tf[n, fd]
            for ax in range(3):
                assert back[abs(t[ax]) - 1] == np.sign(t[ax]) * (ax + 1), (r, f)
            assert np.array_equal(tr[n, fd], -tr[r, f]), (r, f)
            wake += fd == f
    # the wake cut: 8 blocks at each end of the 64 along i, 8 spans in k
    assert wake == 2 * 8 * 8


def _zone_case(name, dim, size):
    """A zone of the shipped division's size with a face type on every outer
    face (the cube's CGNS grid is not readable here): walls, stretched grid."""
    if dim == 2:
        return cases.channel(2, 5, (size[0], size[1], 1), walls_i=True, stretch=1.2)
    c = cases.smooth_random(3, 5, tuple(size), seed=9, stretch=0.05, inviscid=True)
    return c.replace(periodic=(False, False, False), bc=(cases.BC_NAMES["wall_inviscid"],) * 6)


@pytest.mark.parametrize("name", SHIPPED_FILES)
def test_shipped_division_geometry(name):
    """A grid divided by SHOCK's own division file: the library's division
    (cases.load_division over its reader) sets up, on every ghosted point of
    every block, the geometry SHOCK's ranks set up reading the same file with
    loadDivision and exchanging their mesh halos."""
    if not os.path.exists(os.path.join(SHIPPED, name)):
        pytest.skip("SHOCK's test cases are not beside this repository")
    dim = 2 if name.startswith("2d") else 3
    if not multirank_available(5, dim):
        pytest.skip("multi-rank reference build absent (make -C oracle with the reference sources)")
    path = os.path.join(SHIPPED, name)
    nranks = 4 if dim == 2 else 8
    _, _, _, co, _ = shock_b200.read_division(path, dim, nranks)
    size = [int(co[:, 3 + a].max()) for a in range(dim)]
    case = _zone_case(name, dim, size + [1] * (3 - dim))
    d = cases.load_division(case, path, nranks)
    assert sum(b.real_points for b in d.blocks) == case.real_points
    got = shock_b200.host_multi_geometry(d)
    ref = run_multirank(d, 0, division_file=path)
    for b in range(nranks):
        assert np.array_equal(got[b], ref[b]["geometry"]), (name, b)


@pytest.mark.parametrize("name", sorted(CGRIDS))
def test_shock_reads_the_same_cgrid_division(tmp_path, name):
    """A C-grid's division with its wake cut (bottom-to-bottom interfaces,
    Transform (-1,-2,3)) written as a .sddc file: SHOCK's ranks read it with
    loadDivision and set up, bit for bit, the geometry the library sets up
    from its own reading of the file."""
    case, d, full = cgrid_division(name)
    if not multirank_available(case.order, case.dim, full=full):
        pytest.skip("multi-rank reference build absent (make -C oracle with the reference sources)")
    path = tmp_path / "cgrid.sddc"
    cases.write_division(d, str(path))
    _check_rows_as_shock_reads_them(path, case.dim, len(d.blocks))
    got = shock_b200.host_multi_geometry(_read_back(d, path), full_metric=full)
    ref = run_multirank(d, 0, full=full, division_file=path)
    for b in range(len(d.blocks)):
        assert np.array_equal(got[b], ref[b]["geometry"]), (name, b)


def test_load_division(tmp_path):
    """cases.load_division gives back the division a file was written from
    (blocks, neighbours, Translations, face types), and refuses a file whose
    blocks are meshed in other orientations than the zone."""
    c = cases.channel(3, 5, (16, 14, 12))
    d = cases.split(c, (2, 2, 1))
    path = tmp_path / "div.sddc"
    cases.write_division(d, str(path))
    e = cases.load_division(c, str(path), len(d.blocks))
    assert np.array_equal(e.neighbour, d.neighbour) and np.array_equal(e.translation, d.translation)
    assert np.array_equal(e.lo, d.lo) and tuple(e.parts) == tuple(d.parts)
    for a, b in zip(d.blocks, e.blocks):
        assert (a.ni, a.nj, a.nk, a.bc) == (b.ni, b.nj, b.nk, b.bc)
        assert np.array_equal(a.x, b.x) and np.array_equal(a.p, b.p)
    cases.write_division(_division(True), str(path))
    with pytest.raises(ValueError):
        cases.load_division(cases.taylor_green(12, order=5), str(path), 8)


def test_division_file_size_checked(tmp_path):
    d = _division(False)
    path = tmp_path / "div.sddc"
    cases.write_division(d, str(path))
    with pytest.raises(shock_b200.ShockError):
        shock_b200.read_division(path, 3, len(d.blocks) + 1)
