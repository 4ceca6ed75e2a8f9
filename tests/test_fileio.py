"""Restart and field files in the reference's formats (suli-openmp_b200/fileio.py).

CPU tests use the oracle, which has the solver's upload/download surface; the GPU test writes
from a device context and reads into the oracle and back."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from helpers import STATE_FIELDS, pkg, small_params

fileio = pkg.fileio


def stepped_oracle(orc, steps=2):
    p, init = pkg.cases.dam_break(nx=12, ny=6, nz=10, dx=0.04, cg_tol=1e-10)
    o = orc.Oracle(p)
    init(o)
    for it in range(1, steps + 1):
        assert o.step(it)["status"] == 0
    return p, o


RESTART_ARRAYS = [n for n in fileio.RESTART_ORDER if n not in fileio.MASKS + fileio.RESTART_SCALARS]


def test_restart_round_trip_continues_identically(orc, tmp_path):
    """restart_salva -> restart_ini: every array and scalar back bit for bit, and the next
    step of the restarted state equals the next step of the original."""
    p, o = stepped_oracle(orc)
    f = tmp_path / "dados" / "arquivorestart"
    fileio.write_restart(o, f)
    assert len(f.read_text().split()) == fileio.restart_count(p)
    r = orc.Oracle(p)
    extra = fileio.read_restart(r, f)
    assert extra == {"d_max": 0.0, "d_min": 0.0, "ls_m": 0.0}
    for n in RESTART_ARRAYS:
        assert np.array_equal(r.download(n), o.download(n)), n
    for s in ("vol_ini", "vol_ins"):
        assert r.get_scalar(s) == o.get_scalar(s)
    assert r.ntt == o.ntt and r.a_dt == o.a_dt
    so, sr = o.step(3), r.step(3)
    assert so["cg_iters"] == sr["cg_iters"]
    for n in ("u", "v", "w", "ls", "prd1"):
        assert np.array_equal(r.download(n), o.download(n)), n


def fortran_list_directed(values, ints=()):
    """Text in the style of a Fortran list-directed WRITE: blanks, records of a few values,
    E and D exponents, and r*c repeat counts for runs of equal values."""
    out, i, n = [], 0, len(values)
    while i < n:
        j = i
        while j + 1 < n and values[j + 1] == values[i]:
            j += 1
        v = values[i]
        tok = (f"{int(v)}" if i in ints else
               (f"{v:.16E}".replace("E", "D") if i % 3 == 0 else f"{v:.17G}"))
        out.append(f"{j - i + 1}*{tok}" if j > i else tok)
        i = j + 1
    lines = [" ".join(out[k:k + 4]) for k in range(0, len(out), 4)]
    return ("\n".join(lines) + "\n").encode()


def test_restart_reads_list_directed_forms(orc, tmp_path):
    """A restart file written with repeat counts, D exponents and several values per record
    (all legal list-directed input) loads the same values."""
    p = small_params(nx=5, ny=4, nz=4)
    rng = np.random.default_rng(3)
    vals, ints, pos = [], set(), 0
    ref = {}
    for n in fileio.RESTART_ORDER:
        m = int(np.prod(fileio.restart_shape(p, n)))
        if n in fileio.MASKS:
            chunk = np.zeros(m)
            ints.update(range(pos, pos + m))
        elif n in fileio.RESTART_SCALARS:
            chunk = np.array([0.0 if n in ("d_max", "d_min", "ls_m") else rng.uniform(0.1, 1.0)])
        else:
            chunk = rng.standard_normal(m) * 10.0 ** rng.integers(-8, 8)
            if n.startswith("tf_"):
                chunk[:] = 0.0                      # long runs: repeat counts
        ref[n] = chunk
        vals.extend(chunk.tolist())
        pos += m
    f = tmp_path / "arquivorestart"
    f.write_bytes(fortran_list_directed(vals, ints))
    o = orc.Oracle(p)
    fileio.read_restart(o, f)
    for n in RESTART_ARRAYS:
        got = np.ravel(o.download(n), order="F")
        assert np.array_equal(got, ref[n]), n
    assert o.get_scalar("vol_ins") == ref["vol_ins"][0]


def test_restart_refuses_other_grids_and_unexpected_obstacles(orc, tmp_path):
    """A file of another grid is refused, and so is one with obstacle masks for a model run
    without obstacles (obst_t = 0)."""
    p, o = stepped_oracle(orc, steps=1)
    f = tmp_path / "arquivorestart"
    fileio.write_restart(o, f)
    q = p.copy()
    q.nx += 1
    with pytest.raises(ValueError, match="values"):
        fileio.read_restart(orc.Oracle(q), f)
    # a mask value (ku starts after u, v, w) marks an obstacle
    lines = f.read_text().split("\n")
    k = sum(int(np.prod(fileio.restart_shape(p, n))) for n in ("u", "v", "w"))
    lines[k] = "3"
    f.write_text("\n".join(lines))
    with pytest.raises(ValueError, match="obst_t = 0"):
        fileio.read_restart(orc.Oracle(p), f)


@pytest.mark.parametrize("t_plot", [0, 1])
def test_campos_record_and_visu(orc, tmp_path, t_plot):
    """The campos record (4_plot.f90:255-340) against the formulas at sample points, and
    every Seek of visu.xdmf pointing at the array it names."""
    p, o = stepped_oracle(orc)
    wr = fileio.FieldWriter(tmp_path, p, t_plot=t_plot, dt_frame=0.5)
    first = wr.snapshot(o)
    st = {f: o.download(f) for f in ("u", "v", "w", "ls", "prd1", "nut")}   # the state written
    assert o.step(3)["status"] == 0                                       # steps on meanwhile
    wr.snapshot(o)
    wr.close()
    assert first.name == "campos_00010" and (tmp_path / "campos_00011").exists()
    raw = first.read_bytes()
    n = int(np.frombuffer(raw[:4], "<i4")[0])
    assert len(raw) == n + 8 and int(np.frombuffer(raw[-4:], "<i4")[0]) == n
    arrs = fileio.read_campos(first, p, t_plot)
    x, y, z, ua, va, wa, ls, kaux = arrs[:8]
    nx, ny, nz = p.nx, p.ny, p.nz
    u, v, w = st["u"], st["v"], st["w"]
    # x1(0) = -dx, x1(i) = x1(i-1) + dx, summed in order
    xs, acc = [], -p.dx
    for _ in range(nx + 1):
        acc = acc + p.dx
        xs.append(acc)
    assert np.array_equal(x[:, 2, 3], np.array(xs, np.float32))
    for (i, j, k) in [(1, 1, 1), (nx + 1, ny + 1, nz + 1), (3, 2, 5)]:
        assert ua[i - 1, j - 1, k - 1] == np.float32((u[i, j, k] + u[i, j - 1, k] + u[i, j, k - 1] + u[i, j - 1, k - 1]) * 0.25)
        assert va[i - 1, j - 1, k - 1] == np.float32((v[i, j, k] + v[i - 1, j, k] + v[i, j, k - 1] + v[i - 1, j, k - 1]) * 0.25)
        assert wa[i - 1, j - 1, k - 1] == np.float32((w[i, j, k] + w[i, j - 1, k] + w[i - 1, j, k] + w[i - 1, j - 1, k]) * 0.25)
    assert np.array_equal(ls, st["ls"].astype(np.float32)) and not kaux.any()
    if t_plot == 1:
        prd, vi, vj, vk, xn, yn, zn = arrs[8:]
        i, j, k = 2, 3, 4
        dwdy = (w[i, j + 1, k] - w[i, j, k]) / p.dy
        dvdz = (v[i, j, k + 1] - v[i, j, k]) / p.dz
        assert vi[i - 1, j - 1, k - 1] == np.float32(dwdy - dvdz)
        nut = st["nut"]
        assert xn[0, 0, 0] == xn[1, 0, 0] == np.float32((nut[1, 0, 0] + nut[0, 0, 0]) * 0.5)
        assert zn[0, 0, nz] == np.float32((nut[0, 0, nz - 1] + nut[0, 0, nz - 2]) * 0.5)
        assert np.array_equal(prd, st["prd1"][1:nx + 1, 1:ny + 1, 1:nz + 1].astype(np.float32))
    # visu.xdmf: every binary DataItem reads back the array it describes
    tree = ET.parse(tmp_path / "visu.xdmf")
    grids = tree.getroot().findall(".//Grid[@GridType='Uniform']")
    assert [g.get("Name") for g in grids] == ["campos_00010", "campos_00011"]
    items = [d for d in grids[0].iter("DataItem") if d.get("Seek")]
    expect = [x, y, z, ua, va, wa, ls, kaux] + (arrs[8:12] if t_plot == 1 else [])
    order = [0, 1, 2, 3, 4, 5, 6, 7] + ([8, 9, 10, 11] if t_plot == 1 else [])
    assert len(items) == len(order)
    for d, m in zip(items, order):
        dims = [int(s) for s in d.get("Dimensions").split()][:3]
        seek = int(d.get("Seek"))
        cnt = int(np.prod(dims))
        data = np.frombuffer(raw[seek:seek + 4 * cnt], "<f4").reshape(dims)   # (z, y, x) C order
        assert np.array_equal(data, np.transpose(expect[m], (2, 1, 0))), (d.get("Seek"), m)


def test_campos_refuses_oversized_record(tmp_path):
    big = [np.broadcast_to(np.float32(0), ((1 << 29) + 1,))]
    with pytest.raises(ValueError, match="record"):
        fileio.write_campos(tmp_path / "x", big)


@pytest.mark.gpu
def test_restart_between_device_and_oracle(orc, tmp_path):
    """A restart written from a GPU context loads into the oracle bit for bit, and one
    written by the oracle loads into a GPU context bit for bit."""
    p, o = stepped_oracle(orc)
    g = pkg.Solver(p)
    f1 = tmp_path / "from_oracle"
    fileio.write_restart(o, f1)
    fileio.read_restart(g, f1)
    f2 = tmp_path / "from_gpu"
    fileio.write_restart(g, f2)
    assert f2.read_bytes() == f1.read_bytes()
    for n in RESTART_ARRAYS:
        assert np.array_equal(g.download(n), o.download(n)), n
    g.close()
