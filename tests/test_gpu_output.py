"""GPU checks of the output writer (dcm_output_*, the reference's output
routine driver_code.f90:725-1145): the file is read back with scipy's
netCDF classic reader, an implementation independent of the writer.

Each record must hold the resident state at the time of its write as FP32
(round to nearest, as netCDF converts double to float), in the reference's
variables and layout; writing must not change the state or the steps that
follow it.
"""
import numpy as np
import pytest

from helpers import cases, small_bubble

pytestmark = pytest.mark.gpu

FIELDS = ("th", "u", "v", "w", "p", "div")
UNITS = {"time": b"seconds", "x": b"m", "y": b"m", "z": b"m", "rhoa": b"kg/m3", "thetan": b"K",
         "trefn": b"K", "th": b"K", "u": b"m/s", "v": b"m/s", "w": b"m/s", "p": b"pa",
         "div": b"m/s**2"}


def _f32(a):
    """interior of a Fortran field a(0:kp+1, 0:jp+1, 0:ip+1) in the file's
    (ip, jp, kp) order, as FP32"""
    return np.ascontiguousarray(a[1:-1, 1:-1, 1:-1].transpose(2, 1, 0)).astype(np.float32)


def _read(path):
    from scipy.io import netcdf_file
    with netcdf_file(str(path), "r", mmap=False) as f:
        dims = dict(f.dimensions)
        vars_ = {n: (v.data.copy(), v.dimensions, getattr(v, "units", None))
                 for n, v in f.variables.items()}
        order = list(f.variables.keys())
        version = f.version_byte
    return dims, vars_, order, version


def _run(dcm, c, tmp_path, precision=0, nrec=3, every=2, **kw):
    core = dcm.DynamicalCore(c.grid)
    core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                      precision=precision, **kw)
    core.driver_start()
    trefn = np.linspace(300.0, 250.0, c.grid.kp + 2)
    path = tmp_path / "out.nc"
    out = dcm.Output(core, path, trefn=trefn)
    states, times = [], []
    for n in range(nrec):
        t = n * every * c.dt
        out.write(t)
        states.append(core.download_state())
        times.append(t)
        core.step(every)
    out.close()
    core.close()
    return path, states, times, trefn


@pytest.mark.parametrize("precision", [0, 1])
def test_records_hold_the_state(dcm, tmp_path, precision):
    c = small_bubble(ip=20, jp=14, kp=12)
    g = c.grid
    path, states, times, trefn = _run(dcm, c, tmp_path, precision)
    dims, v, order, version = _read(path)
    assert version == 1
    assert dims == {"times": None, "ip": g.ip, "jp": g.jp, "kp": g.kp}
    assert order == ["time", "x", "y", "z", "rhoa", "thetan", "trefn"] + list(FIELDS)
    for n, (data, d, units) in v.items():
        assert data.dtype == np.dtype(">f4"), n
        assert units == UNITS[n], n
    assert v["th"][1] == ("times", "ip", "jp", "kp")
    assert np.array_equal(v["time"][0], np.float32(times))
    for n, ref in (("x", g.x), ("y", g.y), ("z", g.z), ("rhoa", g.rhoa), ("thetan", g.thetan),
                   ("trefn", trefn)):
        assert np.array_equal(v[n][0], ref[1:-1].astype(np.float32)), n
    for r, st in enumerate(states):
        for n in FIELDS:
            assert np.array_equal(v[n][0][r], _f32(st[n])), (r, n)


def test_tracers_in_the_reference_layout(dcm, tmp_path):
    c = cases.sheared_convection(ip=16, jp=12, kp=12, ntracers=3)
    g = c.grid
    path, states, times, _ = _run(dcm, c, tmp_path, nrec=2, nq=c.nq, c_s=c.c_s, c_e=c.c_e)
    dims, v, order, version = _read(path)
    assert dims == {"times": None, "ip": g.ip, "jp": g.jp, "kp": g.kp, "nq": 3, "nprec": 1,
                    "l_q_names": 20}
    assert order[-3:] == ["q_names", "q", "precip"]
    assert v["q"][1] == ("times", "ip", "jp", "kp", "nq")
    names = [b"".join(row).decode() for row in v["q_names"][0]]
    assert names == ["q1".ljust(20), "q2".ljust(20), "q3".ljust(20)]
    assert v["q"][2] == b"kg or number per kg"
    for r, st in enumerate(states):
        for m in range(3):
            assert np.array_equal(v["q"][0][r][..., m], _f32(st["q"][m])), (r, m)
    assert v["precip"][0].shape == (2, g.ip, g.jp, g.kp, 1)
    assert not np.any(v["precip"][0])


def test_writing_leaves_the_steps_unchanged(dcm, tmp_path):
    """Writes queued back to back (more than the two records in flight) and
    between steps: the state after the steps is bit-identical to a run
    without output, and every record is complete."""
    c = small_bubble(ip=20, jp=14, kp=12)
    runs = []
    for with_output in (True, False):
        core = dcm.DynamicalCore(c.grid)
        core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                          precision=1)
        core.driver_start()
        out = dcm.Output(core, tmp_path / "b.nc") if with_output else None
        for n in range(4):
            if out:
                for _ in range(3):
                    out.write(float(n))
            core.step(1)
        if out:
            out.close()
        runs.append(core.download_state())
        core.close()
    for n in ("u", "v", "w", "th", "p"):
        assert np.array_equal(runs[0][n], runs[1][n]), n
    dims, v, _, _ = _read(tmp_path / "b.nc")
    assert v["time"][0].tolist() == [float(n) for n in range(4) for _ in range(3)]


def test_open_reports_an_unwritable_path(dcm, tmp_path):
    c = small_bubble(ip=8, jp=8, kp=6)
    core = dcm.DynamicalCore(c.grid)
    core.upload_state(c.state, c.dt)
    with pytest.raises(dcm.DCMError) as e:
        dcm.Output(core, tmp_path / "missing" / "out.nc")
    assert e.value.status == dcm.DCM_E_IO
    core.close()
