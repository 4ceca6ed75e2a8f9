"""Checkpoint/restart and field output in the reference's file formats.

* Restart (11_diversos.f90:232-330): `restart_salva` writes, and `restart_ini` reads, one
  list-directed text file `dados/arquivorestart` holding the module arrays and scalars of
  RESTART_ORDER in that order, each array in Fortran (column-major) order.  `write_restart`
  writes a file that list-directed READ accepts (one value per line, 17 significant digits, so
  every FP64 value reads back exactly); `read_restart` reads that and any whitespace- or
  comma-separated list-directed file, with `r*c` repeat counts and `D` exponents.
* Fields (4_plot.f90:239-345, t_plot 0 and 1): `arquivos/campos_NNNNN` is one Fortran
  unformatted sequential record (4-byte little-endian length markers before and after) of the
  float32 arrays x, y, z, u, v, w at the cell corners (nx+1, ny+1, nz+1), then ls and the
  obstacle mask at the cells, and with t_plot = 1 the pressure, the three vorticity components
  and the face viscosities face(nut).  `visu` (12_paraview_3D.f90:1-181) writes
  `arquivos/visu.xdmf`, the ParaView index of those files.
* `FieldWriter` downloads a snapshot and hands the arithmetic and the file writing to a
  background thread, so that the device goes on stepping meanwhile.

Every function takes any object with the solver's surface (`params`, `shape`, `download`,
`upload`, `get_scalar`, `set_scalar`): `Solver` on the GPU or the CPU restatement used by
the tests.  The obstacle masks ku, kv, kw are those the model was given by `set_obstacle`
(its `obstacle` attribute; zeros without obstacles).
"""
from __future__ import annotations

import pathlib
import queue
import re
import threading
import warnings

import numpy as np

from ._abi import field_shape

# restart_salva's list (11_diversos.f90:322-326); "ku", "kv", "kw" are integer masks and
# "d_max", "d_min", "ls_m", "vol_ini", "vol_ins" scalars
RESTART_ORDER = [
    "u", "v", "w", "ku", "kv", "kw", "prd0", "prd1", "prd", "rho", "ls_nu", "ls", "mod_ls",
    "bxx0", "bxx1", "bxy0", "bxz0", "bxxf", "bxxf1", "bxyf", "bxzf",
    "byx0", "byy0", "byy1", "byz0", "byxf", "byyf", "byyf1", "byzf",
    "bzx0", "bzy0", "bzz0", "bzz1", "bzxf", "bzyf", "bzzf", "bzzf1",
    "ub", "vb", "wb", "d_max", "d_min", "ls_m",
    "hsx", "hsy", "hsz", "hs", "kurv", "xnut", "ynut", "znut", "tf_u", "tf_v", "tf_w", "vol_ini", "vol_ins",
]
MASKS = ("ku", "kv", "kw")
RESTART_SCALARS = ("d_max", "d_min", "ls_m", "vol_ini", "vol_ins")


def mask_shape(p, name: str):
    """ku(0:nx1+1, 0:ny+1), kv(0:nx+1, 0:ny1+1), kw(0:nx+1, 0:ny+1) (0_modules.f90:76-79)."""
    return {"ku": (p.nx + 3, p.ny + 2), "kv": (p.nx + 2, p.ny + 3), "kw": (p.nx + 2, p.ny + 2)}[name]


def restart_shape(p, name: str):
    if name in MASKS:
        return mask_shape(p, name)
    if name in RESTART_SCALARS:
        return ()
    s = field_shape(p, name)
    return s[:2] if name.startswith("b") else s   # boundary planes are 2-D


def restart_count(p) -> int:
    """Values in a restart file of this grid."""
    return sum(int(np.prod(restart_shape(p, n))) for n in RESTART_ORDER)


# ---------------------------------------------------------------------------------- restart
def write_restart(model, path, *, d_max: float = 0.0, d_min: float = 0.0, ls_m: float | None = None) -> None:
    """restart_salva (11_diversos.f90:314-330): the state of `model` as a list-directed file.

    d_max and d_min (0_modules.f90:124) are set to zero by `iniciais` (2_iniciais.f90:45-46)
    and written nowhere else; ls_m (14_level_set.f90:46-51) is zero for t_hs = 0 and
    0.481803535 max(dx, dy, dz) alpha1 for t_hs = 1."""
    p = model.params
    if ls_m is None:
        ls_m = 0.0 if p.t_hs == 0 else 0.481803535 * max(p.dx, p.dy, p.dz) * p.alpha1
    scal = {"d_max": d_max, "d_min": d_min, "ls_m": ls_m,
            "vol_ini": model.get_scalar("vol_ini"), "vol_ins": model.get_scalar("vol_ins")}
    path = pathlib.Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as f:
        for name in RESTART_ORDER:
            if name in MASKS:
                masks = getattr(model, "obstacle", None)
                m = masks[MASKS.index(name)] if masks is not None else np.zeros(mask_shape(p, name), np.int64)
                np.ravel(np.asarray(m, np.int64), order="F").tofile(f, sep="\n", format="%d")
            elif name in RESTART_SCALARS:
                np.array([scal[name]]).tofile(f, sep="\n", format="%.17g")
            else:
                a = model.download(name)
                np.ravel(a, order="F").tofile(f, sep="\n", format="%.17g")
            f.write("\n")


_REPEAT = re.compile(rb"[*]")


def _parse_list_directed(data: bytes) -> np.ndarray:
    """Values of a list-directed file: separators are blanks, newlines and commas; `r*c` is
    r copies of c; D or Q exponents are E exponents."""
    data = data.replace(b",", b" ").translate(bytes.maketrans(b"DdQq", b"EeEe"))
    if not _REPEAT.search(data):
        with warnings.catch_warnings():
            # numpy warns and stops at a token it cannot read; make that an error
            warnings.simplefilter("error", DeprecationWarning)
            return np.fromstring(data.decode("ascii"), dtype=np.float64, sep=" ")
    out = []
    for tok in data.split():
        if b"*" in tok:
            r, c = tok.split(b"*", 1)
            out.extend([float(c)] * int(r))
        else:
            out.append(float(tok))
    return np.array(out, dtype=np.float64)


def read_restart(model, path) -> dict:
    """restart_ini (11_diversos.f90:232-312): load a restart file into `model`.

    Uploads every array, sets vol_ini and vol_ins, and sets the time-step table from t_tempo
    with t = 0, as restart_ini does.  Non-zero obstacle masks are passed to
    `model.set_obstacle` (the model's obst_t must be non-zero).  Returns the scalars d_max,
    d_min, ls_m.  Refuses a file whose length does not match this grid."""
    p = model.params
    vals = _parse_list_directed(pathlib.Path(path).read_bytes())
    want = restart_count(p)
    if vals.size != want:
        raise ValueError(f"restart file holds {vals.size} values, a {p.nx}x{p.ny}x{p.nz} grid needs {want}")
    pos, scal, masks = 0, {}, {}
    for name in RESTART_ORDER:
        shape = restart_shape(p, name)
        n = int(np.prod(shape))
        chunk = vals[pos:pos + n]
        pos += n
        if name in MASKS:
            masks[name] = chunk.reshape(shape, order="F").astype(np.int32)
        elif name in RESTART_SCALARS:
            scal[name] = float(chunk[0])
        else:
            model.upload(name, chunk.reshape(field_shape(p, name), order="F"))
    if any(m.any() for m in masks.values()):
        if p.obst_t == 0:
            raise ValueError("restart file has obstacle masks; the model has obst_t = 0")
        model.set_obstacle(*(masks[n] for n in MASKS))
    model.set_scalar("vol_ini", scal["vol_ini"])
    model.set_scalar("vol_ins", scal["vol_ins"])
    # time-step table of restart_ini (:252-270); the time restarts at zero
    dt = p.dt
    table = {0: (1, dt, dt, dt), 3: (1, dt, dt, dt), 1: (2, 0.5 * dt, dt, dt), 2: (3, 0.5 * dt, dt, dt)}
    ntt, a1, a2, a3 = table[p.t_tempo]
    model.set_scalar("ntt", ntt)
    model.set_scalar("a_dt1", a1)
    model.set_scalar("a_dt2", a2)
    model.set_scalar("a_dt3", a3)
    model.set_scalar("dt", dt)
    model.set_scalar("t", 0.0)
    return {k: scal[k] for k in ("d_max", "d_min", "ls_m")}


# ----------------------------------------------------------------------------- field output
def _interp_cf(a: np.ndarray, axis: int) -> np.ndarray:
    """interp?_cf (8_derivadas.f90:304-434): centre -> face average, end faces copied."""
    n = a.shape[axis]
    inner = (np.take(a, range(1, n), axis=axis) + np.take(a, range(0, n - 1), axis=axis)) * 0.5
    first = np.take(inner, [0], axis=axis)
    last = np.take(inner, [n - 2], axis=axis)
    return np.concatenate([first, inner, last], axis=axis)


def campos_arrays(p, fields: dict, t_plot: int = 1, kw=None) -> list:
    """The arrays of one campos file (4_plot.f90:255-340), in FP64 before the float32 store.

    `fields` holds u, v, w, ls (and prd1, nut for t_plot = 1) as downloaded (Fortran extents
    with halos, 0-based numpy indices); `kw` is the w obstacle mask, if any."""
    nx, ny, nz = p.nx, p.ny, p.nz
    u, v, w = fields["u"], fields["v"], fields["w"]
    # corner coordinates: x1(0) = -dx, x1(i) = x1(i-1) + dx summed in order (:252-264)
    cx = np.add.accumulate(np.concatenate([[-p.dx], np.full(nx + 1, p.dx)]))[1:]
    cy = np.add.accumulate(np.concatenate([[-p.dy], np.full(ny + 1, p.dy)]))[1:]
    cz = np.add.accumulate(np.concatenate([[-p.dz], np.full(nz + 1, p.dz)]))[1:]
    sh = (nx + 1, ny + 1, nz + 1)
    x11 = np.broadcast_to(cx[:, None, None], sh)
    y11 = np.broadcast_to(cy[None, :, None], sh)
    z11 = np.broadcast_to(cz[None, None, :], sh)
    I, J, K = slice(1, nx + 2), slice(1, ny + 2), slice(1, nz + 2)
    Im, Jm, Km = slice(0, nx + 1), slice(0, ny + 1), slice(0, nz + 1)
    # velocities averaged to the cell corners (:266-268)
    uaux = (u[I, J, K] + u[I, Jm, K] + u[I, J, Km] + u[I, Jm, Km]) * 0.25
    vaux = (v[I, J, K] + v[Im, J, K] + v[I, J, Km] + v[Im, J, Km]) * 0.25
    waux = (w[I, J, K] + w[I, Jm, K] + w[Im, J, K] + w[Im, Jm, K]) * 0.25
    # obstacle cells: kaux(i,j,k) = 1 for k = 1 .. kw(i,j)-1 (:285-296)
    kaux = np.zeros((nx, ny, nz))
    if kw is not None:
        kk = np.arange(1, nz + 1)[None, None, :]
        kaux[kk < np.asarray(kw)[1:nx + 1, 1:ny + 1, None]] = 1.
    out = [x11, y11, z11, uaux, vaux, waux, fields["ls"], kaux]
    if t_plot == 1:
        c = (slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1))
        prdaux = fields["prd1"][c]
        # forward differences of the staggered components at the cells (:320-333)
        dudy = (u[1:nx + 1, 2:ny + 2, 1:nz + 1] - u[c]) / p.dy
        dudz = (u[1:nx + 1, 1:ny + 1, 2:nz + 2] - u[c]) / p.dz
        dvdx = (v[2:nx + 2, 1:ny + 1, 1:nz + 1] - v[c]) / p.dx
        dvdz = (v[1:nx + 1, 1:ny + 1, 2:nz + 2] - v[c]) / p.dz
        dwdx = (w[2:nx + 2, 1:ny + 1, 1:nz + 1] - w[c]) / p.dx
        dwdy = (w[1:nx + 1, 2:ny + 2, 1:nz + 1] - w[c]) / p.dy
        nut = fields["nut"]
        out += [prdaux, dwdy - dvdz, dudz - dwdx, dvdx - dudy,
                _interp_cf(nut, 0), _interp_cf(nut, 1), _interp_cf(nut, 2)]
    return out


CAMPOS_FIELDS = {0: ("u", "v", "w", "ls"), 1: ("u", "v", "w", "ls", "prd1", "nut")}
_MAX_RECORD = (1 << 31) - 1


def write_campos(path, arrays: list) -> int:
    """One Fortran unformatted sequential record of the arrays as float32 (real(x, 4)),
    column-major, between two 4-byte little-endian length markers.  Returns the bytes
    written.  Records longer than 2^31 - 1 bytes are refused (a 4-byte marker cannot hold
    them)."""
    n = sum(int(np.prod(a.shape)) for a in arrays) * 4
    if n > _MAX_RECORD:
        raise ValueError(f"campos record of {n} bytes exceeds the 4-byte record marker")
    path = pathlib.Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    marker = np.array([n], dtype="<i4").tobytes()
    with open(path, "wb") as f:
        f.write(marker)
        for a in arrays:
            f.write(np.asarray(a, dtype="<f4").tobytes(order="F"))
        f.write(marker)
    return n + 8


def read_campos(path, p, t_plot: int = 1) -> list:
    """The float32 arrays of a campos file, in write order, shaped as written."""
    raw = pathlib.Path(path).read_bytes()
    n = int(np.frombuffer(raw[:4], "<i4")[0])
    if len(raw) != n + 8 or int(np.frombuffer(raw[-4:], "<i4")[0]) != n:
        raise ValueError("not a single Fortran unformatted record")
    data = np.frombuffer(raw[4:4 + n], "<f4")
    nx, ny, nz = p.nx, p.ny, p.nz
    shapes = [(nx + 1, ny + 1, nz + 1)] * 6 + [(nx, ny, nz)] * 2
    if t_plot == 1:
        shapes += [(nx, ny, nz)] * 4 + [(nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)]
    out, pos = [], 0
    for s in shapes:
        m = int(np.prod(s))
        out.append(data[pos:pos + m].reshape(s, order="F"))
        pos += m
    if pos != data.size:
        raise ValueError(f"campos record holds {data.size} values, t_plot={t_plot} needs {pos}")
    return out


def campos_name(index: int) -> str:
    """campos_NNNNN: the file counter in five digits (4_plot.f90:297-303)."""
    return f"campos_{index:05d}"


def write_visu(path, p, first: int, last: int, dt_frame: float, t_plot: int = 1) -> None:
    """arquivos/visu.xdmf (12_paraview_3D.f90:1-181): a temporal collection of the campos
    files first..last, each a 3DSMesh of the corner coordinates with the corner velocity,
    and the level set and obstacle mask (and, with t_plot = 1, pressure and vorticity) at
    the cells, read from the record at its byte offsets.  The reference also lists the face
    viscosities as cell arrays, at offsets that assume cell-sized arrays; they are
    face-sized, so that attribute is left out here."""
    nx, ny, nz = p.nx, p.ny, p.nz
    N1, N = (nx + 1) * (ny + 1) * (nz + 1) * 4, nx * ny * nz * 4
    d1, d0 = f"{nz + 1} {ny + 1} {nx + 1}", f"{nz} {ny} {nx}"

    def item(seek, dims, name, extra=""):
        return (f'<DataItem{extra} Format="Binary" DataType="Float" Precision="4" Endian="little" '
                f'Seek="{seek}" Dimensions="{dims}">{name}</DataItem>')

    lines = ['<?xml version="1.0" ?>', '<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>',
             '<Xdmf xmlns:xi="http://www.w3.org/2001/XInclude" Version="2.0">', "<Domain>",
             '<Grid Name="TimeSeries" GridType="Collection" CollectionType="Temporal">',
             '<Time TimeType="HyperSlab">',
             f'<DataItem Format="XML" NumberType="Float" Dimensions="3">0.0 {dt_frame!r} {last - first + 1}</DataItem>',
             "</Time>"]
    for ifile in range(first, last + 1):
        name = campos_name(ifile)
        lines += [f'<Grid Name="{name}" GridType="Uniform">',
                  f'<Topology name="topo" TopologyType="3DSMesh" Dimensions="{d1}"/>',
                  '<Geometry name="geo" Type="X_Y_Z">']
        lines += [item(N1 * m + 4, d1, name, f' Name="{c}"') for m, c in enumerate("XYZ")]
        lines += ["</Geometry>",
                  '<Attribute Name="V" AttributeType="Vector" Center="Node">',
                  f'<DataItem Dimensions="{d1} 3" Function="JOIN($0, $1, $2)" ItemType="Function">']
        lines += [item(N1 * m + 4, d1 + " 1", name) for m in (3, 4, 5)]
        lines += ["</DataItem>", "</Attribute>"]
        cells = [("level_set", 0), ("obstaculo", 1)] + ([("pressure", 2)] if t_plot == 1 else [])
        for attr, m in cells:
            lines += [f'<Attribute Name="{attr}" Center="Cell">', item(N1 * 6 + N * m + 4, d0, name), "</Attribute>"]
        if t_plot == 1:
            lines += ['<Attribute Name="vorticity" AttributeType="Vector" Center="Cell">',
                      f'<DataItem Dimensions="{d0} 3" Function="JOIN($0, $1, $2)" ItemType="Function">']
            lines += [item(N1 * 6 + N * m + 4, d0 + " 1", name) for m in (3, 4, 5)]
            lines += ["</DataItem>", "</Attribute>"]
        lines.append("</Grid>")
    lines += ["</Grid>", "</Domain>", "</Xdmf>"]
    path = pathlib.Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text("\n".join(lines) + "\n")


class FieldWriter:
    """Writes campos files in a background thread (plot_i / plot_f, 4_plot.f90:12-345).

    `snapshot(model)` downloads the fields the record needs (this waits for the device work
    already queued) and returns; the corner averages, vorticity, float32 conversion and the
    file write run in the thread while the caller goes on stepping.  The first file is
    campos_00010, as the reference numbers them.  `close()` waits for the queued files and
    writes visu.xdmf."""

    def __init__(self, directory, params, *, t_plot: int = 1, dt_frame: float = 1.0, first: int = 10,
                 max_pending: int = 2):
        self.dir = pathlib.Path(directory)
        self.p = params.copy()
        self.t_plot = t_plot
        self.dt_frame = dt_frame
        self.first = first
        self.next = first
        self.q: queue.Queue = queue.Queue(maxsize=max_pending)
        self.error: BaseException | None = None
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        while True:
            job = self.q.get()
            if job is None:
                return
            path, fields, kw = job
            try:
                write_campos(path, campos_arrays(self.p, fields, self.t_plot, kw))
            except BaseException as e:   # reported by the next snapshot() or close()
                self.error = e

    def _raise(self):
        if self.error is not None:
            e, self.error = self.error, None
            raise RuntimeError("campos writer failed") from e

    def snapshot(self, model) -> pathlib.Path:
        self._raise()
        fields = {n: model.download(n) for n in CAMPOS_FIELDS[self.t_plot]}
        masks = getattr(model, "obstacle", None)
        path = self.dir / campos_name(self.next)
        self.next += 1
        self.q.put((path, fields, None if masks is None else masks[2]))
        return path

    def close(self) -> None:
        if self.thread.is_alive():
            self.q.put(None)
            self.thread.join()
        self._raise()
        if self.next > self.first:
            write_visu(self.dir / "visu.xdmf", self.p, self.first, self.next - 1, self.dt_frame, self.t_plot)
