"""History and restart files (moist_history_*, moist_restart_read): init_history /
output_history (moist.jl:1686-1891) and the restart of run_sim (moist.jl:1905-1919).

The library writes the NetCDF classic format with 64-bit offsets itself. scipy's NetCDF reader
(an independent implementation of the same published format) reads the files back: dimensions,
variable order, dimensions per variable, units, element type and every value are checked
against the reference's init_history / output_history. The restart reader is checked on the
library's own files and on files written by scipy. All of it runs on the host; the last test
writes a record from a device State."""

import numpy as np
import pytest
from scipy.io import netcdf_file

from moist2d_b200 import model
from moist2d_b200.params import STATE_FIELDS

from states import bubble_case

HVARS = [("x", ("x",), "m"), ("z", ("z",), "m"), ("zf", ("z",), "m"), ("time", ("time",), "s"),
         ("rho", "3", "kg/m^3"), ("rhou", "3", "kg/m^2/s"), ("rhow", "3", "kg/m^2/s"), ("u", "3", "m/s"),
         ("w", "3", "m/s"), ("theta", "3", "K"), ("qv", "3", "kg/kg"), ("qc", "3", "kg/kg"),
         ("qr", "3", "kg/kg"), ("RH", "3", "%"), ("temp", "3", "K"), ("pres", "3", "hPa"),
         ("thetae", "3", "K"), ("prec", "2", "kg/m^2"), ("mflux", "2", "kg/m/s^2"),
         ("shflux", "2", "W/m^2"), ("lhflux", "2", "W/m^2"), ("d_rho_theta_mp", "3", "kg K/m^3/s"),
         ("d_rho_qv_mp", "3", "kg/m^3/s"), ("d_rho_qc_mp", "3", "kg/m^3/s"),
         ("d_rho_qr_mp", "3", "kg/m^3/s"), ("d_rho_qr_sed", "3", "kg/m^3/s"),
         ("d_rho_u_sf", "2", "kg/m^2/s^2"), ("d_rho_theta_sf", "2", "kg K/m^3/s"),
         ("d_rho_qv_sf", "2", "kg/kg/m^3/s"), ("d_rho_theta_rd", "3", "kg K/m^3/s")]
STATE_OF = {"rho": "rho", "rhou": "rho_u", "rhow": "rho_w", "prec": "prec", "mflux": "mflux",
            "shflux": "shflux", "lhflux": "lhflux", "d_rho_theta_mp": "d_rho_theta_mp",
            "d_rho_qv_mp": "d_rho_qv_mp", "d_rho_qc_mp": "d_rho_qc_mp", "d_rho_qr_mp": "d_rho_qr_mp",
            "d_rho_qr_sed": "d_rho_qr_sed", "d_rho_u_sf": "d_rho_u_sf", "d_rho_theta_sf": "d_rho_theta_sf",
            "d_rho_qv_sf": "d_rho_qv_sf", "d_rho_theta_rd": "d_rho_theta_rd"}
DIAG = model.History.FIELDS


def random_state(p, s, rng):
    a = s.copy()
    for f in STATE_FIELDS:
        x = getattr(a, f)
        x[...] = (rng.standard_normal(x.shape) * 10.0 + 50.0).astype(p.T)
    return a


def random_diag(p, rng):
    return {f: np.asfortranarray((rng.standard_normal((p.Nz, p.Nx)) * 100.0 + 1e5).astype(p.T)) for f in DIAG}


def read(path):
    with netcdf_file(path, "r", mmap=False, maskandscale=False) as f:
        return {"version": f.version_byte, "dims": dict(f.dimensions),
                "vars": [(n, v.dimensions, v.units.decode(), v.data.dtype.str, np.array(v.data))
                         for n, v in f.variables.items()]}


def write(path, p, records):
    with model.History(path, p) as h:
        for t, s, d in records:
            h.append_host(t, s, d)


@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_history_file_against_init_history(tmp_path, T):
    p, s = bubble_case(T, nx=12, nz=7)
    rng = np.random.default_rng(1)
    recs = [(t, random_state(p, s, rng), random_diag(p, rng)) for t in (0.0, 10.5, 21.0)]
    path = tmp_path / "hist.nc"
    write(path, p, recs)
    f = read(path)
    assert f["version"] == 2
    assert f["dims"] == {"x": p.Nx, "z": p.Nz, "time": None}
    assert [v[0] for v in f["vars"]] == [h[0] for h in HVARS]
    c = slice(p.is_ - 1, p.ie)
    be = ">f8" if T is np.float64 else ">f4"
    for (name, dims, units, dt, data), (_, kind, hunits) in zip(f["vars"], HVARS):
        assert units == hunits, name
        assert dt == be, name
        exp_dims = {"3": ("time", "z", "x"), "2": ("time", "x")}.get(kind, kind)
        assert dims == exp_dims, name
        if name == "x":
            expect = (np.arange(p.Nx).astype(T) + T(0.5)) * T(p.dx)
        elif name in ("z", "zf"):
            expect = getattr(p, name)
        elif name == "time":
            expect = np.array([r[0] for r in recs], dtype=T)
        elif name in STATE_OF:
            fld = STATE_OF[name]
            expect = np.stack([getattr(r[1], fld)[..., c] for r in recs])
        elif name == "pres":
            expect = np.stack([r[2]["pres"] / T(100.0) for r in recs])  # Pa -> hPa in T
        else:
            expect = np.stack([r[2][name] for r in recs])
        assert np.array_equal(data, np.asarray(expect, dtype=T)), name


def test_history_records_are_readable_while_open(tmp_path):
    p, s = bubble_case(np.float32, nx=8, nz=5)
    rng = np.random.default_rng(2)
    path = tmp_path / "hist.nc"
    with model.History(path, p) as h:
        for n in range(3):
            h.append_host(float(n), random_state(p, s, rng), random_diag(p, rng))
            with netcdf_file(path, "r", mmap=False) as f:
                assert f.variables["time"].shape == (n + 1,)
                assert f.variables["rho"].shape == (n + 1, p.Nz, p.Nx)


def test_history_replaces_an_existing_file(tmp_path):
    p, s = bubble_case(np.float64, nx=8, nz=5)
    path = tmp_path / "hist.nc"
    path.write_bytes(b"x" * 100000)
    write(path, p, [(1.0, s, random_diag(p, np.random.default_rng(3)))])
    assert read(path)["dims"]["x"] == p.Nx


@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_restart_reads_the_last_record(tmp_path, T):
    p, s = bubble_case(T, nx=12, nz=7)
    rng = np.random.default_rng(4)
    recs = [(t, random_state(p, s, rng), random_diag(p, rng)) for t in (0.0, 5.0)]
    path = tmp_path / "hist.nc"
    write(path, p, recs)
    r = model.restart_read(path, p)
    _, last, d = recs[-1]
    c = slice(p.is_ - 1, p.ie)
    for f in ("rho", "rho_u", "rho_w"):
        assert np.array_equal(getattr(r, f)[:, c], getattr(last, f)[:, c]), f
    for f, q in (("rho_theta", "theta"), ("rho_qv", "qv"), ("rho_qc", "qc"), ("rho_qr", "qr")):
        assert np.array_equal(getattr(r, f)[:, c], (d[q] * last.rho[:, c]).astype(T)), f
    assert np.array_equal(r.prec[c], last.prec[c])
    # halo columns: periodic copies (exchange_halo!); prec halo untouched
    for f in ("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr"):
        a = getattr(r, f)
        assert np.array_equal(a[:, :p.halo], a[:, p.Nx:p.Nx + p.halo]), f
        assert np.array_equal(a[:, p.halo + p.Nx:], a[:, p.halo:2 * p.halo]), f
    assert np.all(r.prec[:p.halo] == 0) and np.all(r.prec[p.halo + p.Nx:] == 0)
    # rho_qr comes from "qr", not from "qc" as in the reference (moist.jl:1917)
    assert not np.array_equal(r.rho_qr, r.rho_qc)


def scipy_history(path, p, nrec, dtype, rng, extra=True):
    """A history file written by scipy: the restart's variables with the reference's dimension
    order, plus (extra) an unrelated variable, global attributes and attributes of other types."""
    vals = []
    with netcdf_file(path, "w", version=2) as f:
        if extra:
            f.title = "written by scipy"
            f.step_count = np.int32(7)
        f.createDimension("time", None)  # scipy wants the record dimension first: other dimension ids
        f.createDimension("x", p.Nx)
        f.createDimension("z", p.Nz)
        if extra:
            f.createDimension("pair", 2)
            v = f.createVariable("unrelated", "i4", ("pair",))
            v[:] = [1, 2]
            v.scale = np.float64(0.5)
        t = f.createVariable("time", dtype, ("time",))
        vs = {n: f.createVariable(n, dtype, ("time", "z", "x")) for n in ("rho", "rhou", "rhow", "theta", "qv", "qc", "qr")}
        vs["prec"] = f.createVariable("prec", dtype, ("time", "x"))
        if extra:
            vs["rho"].units = "kg/m^3"
            vs["rho"].valid_range = np.array([0.0, 2.0], dtype=np.float32)
        for r in range(nrec):
            t[r] = r
            rec = {}
            for n, v in vs.items():
                shape = (p.Nz, p.Nx) if n != "prec" else (p.Nx,)
                base = 1.0 if n == "rho" else (300.0 if n == "theta" else 1e-3)
                rec[n] = (base * (1.0 + 0.1 * rng.standard_normal(shape))).astype(dtype)
                v[r] = rec[n]
            vals.append(rec)
    return vals


@pytest.mark.parametrize("T,file_dtype", [(np.float64, "f8"), (np.float32, "f4"), (np.float64, "f4")],
                         ids=["f64-file-f64", "f32-file-f32", "f32-file-f64"])
def test_restart_reads_an_independent_writers_file(tmp_path, T, file_dtype):
    p, _ = bubble_case(T, nx=10, nz=6)
    path = tmp_path / "other.nc"
    vals = scipy_history(path, p, 3, file_dtype, np.random.default_rng(5))[-1]
    r = model.restart_read(path, p)
    c = slice(p.is_ - 1, p.ie)
    F = np.float64 if file_dtype == "f8" else np.float32
    assert np.array_equal(r.rho[:, c], vals["rho"].astype(T))
    assert np.array_equal(r.rho_u[:, c], vals["rhou"].astype(T))
    assert np.array_equal(r.rho_w[:, c], vals["rhow"].astype(T))
    for f, q in (("rho_theta", "theta"), ("rho_qv", "qv"), ("rho_qc", "qc"), ("rho_qr", "qr")):
        # product in the file's type, then rounded to T (theta' .* rho, moist.jl:1914)
        prod = (vals[q].astype(F) * vals["rho"].astype(F)).astype(T)
        assert np.array_equal(getattr(r, f)[:, c], prod), f
    assert np.array_equal(r.prec[c], vals["prec"].astype(T))


def test_restart_errors(tmp_path):
    p, s = bubble_case(np.float64, nx=10, nz=6)
    with pytest.raises(OSError, match="cannot open"):
        model.restart_read(tmp_path / "missing.nc", p)
    junk = tmp_path / "junk.nc"
    junk.write_bytes(b"HDF\x89 not classic")
    with pytest.raises(OSError, match="not a NetCDF classic"):
        model.restart_read(junk, p)
    empty = tmp_path / "empty.nc"
    with model.History(empty, p):
        pass
    with pytest.raises(OSError, match="no record"):
        model.restart_read(empty, p)
    good = tmp_path / "good.nc"
    write(good, p, [(0.0, s, random_diag(p, np.random.default_rng(6)))])
    q, _ = bubble_case(np.float64, nx=12, nz=6)
    with pytest.raises(OSError, match="dimension lengths"):
        model.restart_read(good, q)
    partial = tmp_path / "partial.nc"
    with netcdf_file(partial, "w", version=2) as f:
        f.createDimension("time", None)
        f.createDimension("x", p.Nx)
        f.createDimension("z", p.Nz)
        f.createVariable("rho", "f8", ("time", "z", "x"))[0] = np.ones((p.Nz, p.Nx))
    with pytest.raises(OSError, match='no variable "rhou"'):
        model.restart_read(partial, p)
    with pytest.raises(OSError, match="cannot create"):
        model.History(tmp_path / "no" / "such" / "dir.nc", p)


@pytest.mark.gpu
@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_history_record_from_the_device(tmp_path, T):
    """moist_history_append from a context after a few steps: the record holds the downloaded
    State and the device diagnostics (pres in hPa), and a restart from it gives back the State's
    rho, rho_u, rho_w and prec."""
    p, s = bubble_case(T, nx=24, nz=16)
    path = tmp_path / "dev.nc"
    with model.Model(p) as m, model.History(path, p) as h:
        m.upload(s)
        m.step(3)
        h.append(6.0, m)
        fin = s.copy()
        m.download(fin)
        d = m.history()
    f = {v[0]: v[4] for v in read(path)["vars"]}
    c = slice(p.is_ - 1, p.ie)
    assert np.array_equal(f["time"], np.array([6.0], dtype=T))
    assert np.array_equal(f["rho"][0], fin.rho[:, c])
    assert np.array_equal(f["rhou"][0], fin.rho_u[:, c])
    assert np.array_equal(f["d_rho_qr_sed"][0], fin.d_rho_qr_sed[:, c])
    assert np.array_equal(f["prec"][0], fin.prec[c])
    for q in DIAG:
        expect = d[q] / T(100.0) if q == "pres" else d[q]
        assert np.array_equal(f[q][0], expect), q
    r = model.restart_read(path, p)
    for fld in ("rho", "rho_u", "rho_w"):
        assert np.array_equal(getattr(r, fld)[:, c], getattr(fin, fld)[:, c]), fld


def test_history_rejects_records_beyond_the_format(tmp_path):
    """A CDF-2 variable's per-record size is a 32-bit field: 2^17 x 2^13 Float32 cells (4 GiB
    per record of a (time, z, x) variable) are refused before anything is written."""
    from moist2d_b200.params import Params
    p = Params(np.float32, Nx=1 << 17, Nz=1 << 13, H=100.0 * (1 << 13), dz0=100.0, z_fact=1.0,
               Lx=100.0 * (1 << 17))
    with pytest.raises(ValueError):
        model.History(tmp_path / "big.nc", p)
    assert not (tmp_path / "big.nc").exists()


@pytest.mark.gpu
def test_history_record_of_an_ensemble_member(tmp_path):
    """A record from member 1 of a two-member Ensemble after batch steps: the member's State as
    moist_batch_download returns it."""
    p0, s0 = bubble_case(np.float32, nx=24, nz=16)
    p1, s1 = bubble_case(np.float32, seed=9, nx=32, nz=12)
    path = tmp_path / "member.nc"
    with model.Ensemble([p0, p1]) as e, model.History(path, p1) as h:
        e.upload(0, s0)
        e.upload(1, s1)
        e.step(3)
        h.append_member(6.0, e, 1)
        fin = e.download(1, s1.copy())
    f = {v[0]: v[4] for v in read(path)["vars"]}
    c = slice(p1.is_ - 1, p1.ie)
    for name, fld in (("rho", "rho"), ("rhou", "rho_u"), ("rhow", "rho_w")):
        assert np.array_equal(f[name][0], getattr(fin, fld)[:, c]), name
    assert np.array_equal(f["prec"][0], fin.prec[c])


@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_history_record_of_the_oracle_run_and_restart_continuation(tmp_path, T):
    """The oracle's own run: a record written from its State and its output_history diagnostics
    holds them as output_history would (pres in hPa); restarting from it and stepping on gives
    the uninterrupted run's State to within the rounding of the restart's theta * rho and
    q * rho products, as the reference's restart does."""
    from oracle import bind
    p, s = bubble_case(T, nx=24, nz=16)
    bind.rk3_step(s, p, 4, tri64=True)
    d = bind.history_diag(s, p)
    path = tmp_path / "oracle.nc"
    write(path, p, [(8.0, s, {f: d[f] for f in DIAG})])
    f = {v[0]: v[4] for v in read(path)["vars"]}
    c = slice(p.is_ - 1, p.ie)
    assert np.array_equal(f["pres"][0], d["pres"] / T(100.0))
    assert np.array_equal(f["theta"][0], d["theta"]) and np.array_equal(f["rho"][0], s.rho[:, c])
    r = model.restart_read(path, p)
    # interiors as stored; the halos are the restart's exchange, not the step's last one
    assert np.array_equal(r.rho[:, c], s.rho[:, c]) and np.array_equal(r.rho_u[:, c], s.rho_u[:, c])
    direct = s.copy()
    bind.rk3_step(direct, p, 3, tri64=True)
    bind.rk3_step(r, p, 3, tri64=True)
    tol = 1e-4 if T is np.float32 else 1e-12
    for fld in ("rho", "rho_u", "rho_w", "rho_theta", "rho_qv"):
        x, y = getattr(r, fld)[:, c].astype(np.float64), getattr(direct, fld)[:, c].astype(np.float64)
        assert np.linalg.norm(x - y) <= tol * np.linalg.norm(y), fld
