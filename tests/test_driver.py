"""The C++ driver (quill_b200/qp_driver) reads QUILL's parse.py record
stream and writes QUILL's output files.  The stream is produced here the way
parse.py produces it (name / value / units / "$"); the outputs are read back
the way python/resread.py reads them (log name/value pairs, t_data rows,
density slices of nx*ny + nx*nz + ny*nz values)."""
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import gpu_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "quill_b200", "qp_driver")

CONF = [  # (key, value, units) as parse.py emits them: plain numbers get '#' units
    ("dx", "0.0625", "#"), ("dy", "0.0625", "#"), ("dz", "0.0625", "#"), ("dt", "0.03125", "#"),
    ("lambda", "1", "um"), ("ne", "0.1", "ncr"),
    ("xlength", "2", "lambda"), ("ylength", "1.5", "lambda"), ("zlength", "1.5", "lambda"),
    ("t_end", "0.5", "lambda"), ("output_period", "0.25", "lambda"),
    ("a0", "5", "#"), ("xsigma", "0.5", "lambda"), ("ysigma", "0.4", "lambda"), ("zsigma", "0.4", "lambda"),
    ("x0", "-0.5", "lambda"),
    ("solver", "#", "fdtd"), ("pusher", "#", "boris"), ("qed", "#", "off"), ("mwindow", "#", "off"),
    ("film", "#", "on"), ("x0film", "1", "lambda"), ("filmwidth", "0.5", "lambda"), ("gradwidth", "0.1", "lambda"),
    ("nfilm", "0.1", "ncr"), ("Tfilm", "0.01", "#"), ("xnpic_film", "2", "#"), ("ynpic_film", "1", "#"),
    ("znpic_film", "1", "#"),
    ("e_components_for_output", "#", "xyz"), ("b_components_for_output", "#", "z"),
    ("particles_for_output", "#", "e"), ("seed", "3", "#"),
]


def stream(conf, folder):
    lines = []
    for k, v, u in conf + [("data_folder", "#", folder)]:
        lines += [k, v, u, "$"]
    lines.append("$")
    return "\n".join(lines) + "\n"


def read_log(path):
    d = {}
    with open(path) as f:
        it = iter(f)
        for line in it:
            line = line.strip()
            if line in ("nx", "ny", "nz"):
                d[line] = int(next(it))
            elif line in ("dx", "dy", "dz", "dt", "t_end", "output_period"):
                d[line] = float(next(it))
    return d


@pytest.mark.gpu
def test_driver_runs_conf_stream_and_writes_reference_formats(tmp_path):
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200 import build
    build.build()
    folder = str(tmp_path / "results")
    r = subprocess.run([DRIVER], input=stream(CONF, folder), text=True, capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr
    log = read_log(os.path.join(folder, "log"))
    nx, ny, nz = log["nx"], log["ny"], log["nz"]
    assert (nx, ny, nz) == (32, 24, 24)
    # N and energy: one tab-separated row per step, 0..last iteration (t_end / dt = 16)
    for name, cols in (("N", 3), ("energy", 4)):
        rows = [ln.split("\t") for ln in open(os.path.join(folder, name)).read().strip().splitlines()]
        assert len(rows) == 17 and all(len(x) == cols for x in rows)
    e = np.array([[float(v) for v in ln.split("\t")] for ln in open(os.path.join(folder, "energy"))])
    assert e[0, 0] > 0 and e[:, 1].max() > 0
    n = np.array([[float(v) for v in ln.split("\t")] for ln in open(os.path.join(folder, "N"))])
    assert n[0, 0] > 0
    # field and density slices at t = 0, 0.25, 0.5 lambda
    for t in ("0", "0.25", "0.5"):
        for name in ("ex", "ey", "ez", "bz", "rho"):
            vals = np.loadtxt(os.path.join(folder, name + t))
            assert vals.size == nx * ny + nx * nz + ny * nz
        ps = open(os.path.join(folder, "phasespace" + t)).read().split()
        assert len(ps) % 9 == 0 and len(ps) > 0
    # the laser is in the box and the plasma moved: fields and density differ over time
    ey0, ey1 = np.loadtxt(os.path.join(folder, "ey0")), np.loadtxt(os.path.join(folder, "ey0.5"))
    assert np.abs(ey0).max() > 1 and not np.allclose(ey0, ey1)


def _run_driver(conf, folder, timeout=300):
    from quill_b200 import build
    build.build()
    r = subprocess.run([DRIVER], input=stream(conf, folder), text=True, capture_output=True, timeout=timeout)
    assert r.returncode == 0, r.stderr
    return r


def _rows(path):
    return np.array([[float(v) for v in ln.split("\t")] for ln in open(path).read().strip().splitlines()])


def test_driver_record_stream_reads_arrays_and_float_values(tmp_path):
    """The record reader takes values with float precision, as var::read's
    stof does, and arrays "[a;b;c]" (low-level.cpp:376-451): unsorted
    profile coordinates are rejected before a device is touched."""
    from quill_b200 import build
    build.build()
    conf = CONF + [("ne_profile_r_coords", "[1;0.5]", "lambda"), ("ne_profile_r_values", "[1;0]", "#")]
    r = subprocess.run([DRIVER], input=stream(conf, str(tmp_path / "r")), text=True, capture_output=True, timeout=60)
    assert r.returncode != 0 and "not sorted" in r.stderr
    conf = CONF + [("ne_profile_r_coords", "[0;0.5;1]", "lambda"), ("ne_profile_r_values", "[1;0]", "#")]
    r = subprocess.run([DRIVER], input=stream(conf, str(tmp_path / "r2")), text=True, capture_output=True, timeout=60)
    assert r.returncode != 0 and "differ in length" in r.stderr


@pytest.mark.gpu
def test_driver_automatic_window(tmp_path):
    """mwindow = auto (main.cpp:1961-1975): the window stands until the
    laser's max E^2 + B^2 in the front slice [nx-6, nx-4) exceeds mwtolerance
    times the box's, then moves one cell per step while it does."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    folder = str(tmp_path / "results")
    conf = [c for c in CONF if c[0] not in ("mwindow", "t_end", "output_period")] + [
        ("mwindow", "#", "auto"), ("mwtolerance", "1e-4", "#"), ("t_end", "1.25", "lambda"),
        ("output_period", "1.25", "lambda")]
    _run_driver(conf, folder)
    mw = np.loadtxt(os.path.join(folder, "mwcoordinate"))
    assert mw.size == 41 and np.all(np.diff(mw) >= 0)
    assert mw[0] == 0 and mw[-1] > 0             # stood first, then moved
    steps = np.diff(mw) / 0.0625
    assert np.all((np.abs(steps) < 1e-9) | (np.abs(steps - 1) < 1e-9))   # zero or one cell per step


@pytest.mark.gpu
def test_driver_neutral_flow(tmp_path):
    """A neutral flow from the left (add_neutral_flow_particles,
    main.cpp:1837-1880): a layer of plasma enters at i = 2..3 each time the
    flow has advanced a cell, i.e. every dx / (v dt) = 4 steps at v = 0.5;
    the moving window is switched off."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    # a cold film and no laser: only the flow changes the electron charge
    base = [c for c in CONF if c[0] not in ("mwindow", "a0", "Tfilm")] + [("a0", "0", "#")]
    flow = base + [("nelflow", "1", "#"), ("vlflow", "0.5", "#"), ("Tlflow", "0", "#"), ("mcrlflow", "1", "#")]
    b = str(tmp_path / "flow")
    _run_driver(flow, b)
    assert "mwindow\noff\n" in open(os.path.join(b, "log")).read()
    assert not os.path.exists(os.path.join(b, "mwcoordinate"))
    ne = _rows(os.path.join(b, "N"))[:, 0]
    inc = np.diff(ne)
    jumps = np.nonzero(inc > 1e-6 * ne[0])[0] + 1
    assert len(jumps) >= 4 and jumps[0] == 1 and np.all(np.isin(np.diff(jumps), (4, 5)))
    quiet = np.setdiff1d(np.arange(1, ne.size), jumps)
    assert np.all(np.abs(inc[quiet - 1]) <= 1e-9 * ne[0])
    # every entering layer carries the same charge
    np.testing.assert_allclose(inc[jumps - 1], inc[jumps[0] - 1], rtol=1e-9)


@pytest.mark.gpu
def test_driver_film_density_across_y(tmp_path):
    """nfilm_y0 / nfilm_y1 (film, init.cpp:579-583): the film density grows
    linearly from y0film to y1film; the electron density at t = 0 shows it."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    folder = str(tmp_path / "results")
    conf = [c for c in CONF if c[0] not in ("nfilm", "mwindow", "a0", "Tfilm")] + [
        ("mwindow", "#", "off"), ("nfilm_y0", "0.05", "ncr"), ("nfilm_y1", "0.2", "ncr"), ("a0", "0", "#")]
    _run_driver(conf, folder)
    log = read_log(os.path.join(folder, "log"))
    nx, ny, nz = log["nx"], log["ny"], log["nz"]
    rho = np.loadtxt(os.path.join(folder, "rho0"))
    xy = np.abs(rho[:nx * (ny + nz)].reshape(nx, ny + nz)[:, :ny])   # per i: the xy line, then the xz line
    col = xy[20, 2:ny - 3]                  # inside the film (x = 1.25 lambda), across y
    assert np.all(np.diff(col) > 0)
    assert col[-1] / col[0] > 3


@pytest.mark.gpu
def test_driver_moving_window(tmp_path):
    """Without mwindow the reference's default, on, applies: the window moves
    one cell whenever (l + 1) dt mwspeed passes nmw dx (main.cpp:1953-1959),
    the mwcoordinate file follows it, and the exposed front layer is seeded
    with the uniform plasma ne (add_moving_window_particles)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200 import build
    build.build()
    folder = str(tmp_path / "results")
    conf = [c for c in CONF if c[0] != "mwindow"]
    r = subprocess.run([DRIVER], input=stream(conf, folder), text=True, capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "mwindow\non\n" in open(os.path.join(folder, "log")).read()
    mw = np.loadtxt(os.path.join(folder, "mwcoordinate"))
    assert mw.size == 17 and np.all(np.diff(mw) >= 0)
    np.testing.assert_allclose(mw[-1], 8 * 0.0625, rtol=1e-12)   # 8 shifts of dx = lambda/16
    n = np.array([[float(v) for v in ln.split("\t")] for ln in open(os.path.join(folder, "N"))])
    assert n[-1, 0] > 1.05 * n[0, 0]   # new plasma entered at the front


@pytest.mark.gpu
def test_driver_particle_merging(tmp_path):
    """pmerging = ti with a low crpc: the driver merges before the steps that
    follow an over-full one (main.cpp:1691-1748, 2321-2322).  Merging keeps
    the charge (the weighted count N_e agrees with a run without merging:
    exactly while no particle has left the box, within a few per cent after)
    and thins the macro-particles."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200 import build
    build.build()
    out = {}
    for name, extra in (("plain", []), ("merged", [("pmerging", "#", "ti"), ("crpc", "0.05", "#")])):
        folder = str(tmp_path / name)
        r = subprocess.run([DRIVER], input=stream(CONF + extra, folder), text=True, capture_output=True, timeout=300)
        assert r.returncode == 0, r.stderr
        n = np.array([[float(v) for v in ln.split("\t")] for ln in open(os.path.join(folder, "N"))])
        ps = len(open(os.path.join(folder, "phasespace0.5")).read().split()) // 9
        out[name] = (n, ps, open(os.path.join(folder, "log")).read())
    (n0, ps0, _), (n1, ps1, log1) = out["plain"], out["merged"]
    assert "pmerging\nti\n" in log1 and "crpc\n0.05\n" in log1
    lossless = n0[:, 0] == n0[0, 0]
    assert lossless[:3].all()
    np.testing.assert_allclose(n1[lossless, 0], n0[lossless, 0], rtol=1e-9)
    np.testing.assert_allclose(n1[:, 0], n0[:, 0], rtol=0.05)
    assert ps1 < 0.5 * ps0


@pytest.mark.gpu
def test_driver_catching(tmp_path):
    """catching = on: energy_deleted gets one row per step with the
    cumulative energy of the erased particles per class (e, p, ph), and the
    deleted<t> files carry 9 values per written particle, positioned outside
    the region (main.cpp:189-367)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200 import build
    build.build()
    folder = str(tmp_path / "results")
    conf = CONF + [("catching", "#", "on")]
    r = subprocess.run([DRIVER], input=stream(conf, folder), text=True, capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr
    ed = np.loadtxt(os.path.join(folder, "energy_deleted"))
    assert ed.shape == (17, 3)
    assert np.all(np.diff(ed[:, 0]) >= 0) and ed[-1, 0] > 0     # electrons leave and are counted
    log = read_log(os.path.join(folder, "log"))
    total = 0
    for t in ("0", "0.25", "0.5"):
        vals = open(os.path.join(folder, "deleted" + t)).read().split()
        assert len(vals) % 9 == 0
        rec = np.array(vals, dtype=float).reshape(-1, 9)
        total += rec.shape[0]
        # positions in lambda: outside the inner cells [1, n-3] on some axis
        cells = np.floor(rec[:, 1:4] / np.array([log["dx"], log["dy"], log["dz"]])).astype(int)
        n = np.array([log["nx"], log["ny"], log["nz"]])
        assert np.all(((cells <= 0) | (cells >= n - 2)).any(axis=1))
    assert total > 0


@pytest.mark.gpu
def test_driver_tracks(tmp_path):
    """n_tracks electrons along a line through the film are tracked from
    tr_start on (start_tracking, main.cpp:1516-1612); each gets a file
    track_-1_<n> with 9 values per step while it stays in [nm, nx - nm)
    (fout_tracks, fout.cpp:706-734)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200 import build
    build.build()
    folder = str(tmp_path / "results")
    conf = CONF + [("n_tracks", "4", "#"), ("particles_to_track", "#", "e"), ("tr_start", "0", "lambda"),
                   ("xtr1", "1.1", "lambda"), ("ytr1", "0.75", "lambda"), ("ztr1", "0.75", "lambda"),
                   ("xtr2", "1.4", "lambda"), ("ytr2", "0.75", "lambda"), ("ztr2", "0.75", "lambda")]
    r = subprocess.run([DRIVER], input=stream(conf, folder), text=True, capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr
    files = sorted(f for f in os.listdir(folder) if f.startswith("track_-1_"))
    assert [f for f in files] == [f"track_-1_{i}" for i in range(1, 5)]
    for f in files:
        rec = np.array(open(os.path.join(folder, f)).read().split(), dtype=float).reshape(-1, 9)
        assert 1 <= rec.shape[0] <= 16
        assert np.all(rec[:, 0] < 0)                     # electrons
        assert np.all((rec[:, 1] > 1.0) & (rec[:, 1] < 1.6))  # near the film, in lambda
        # continuous trajectories: at most half a cell per step in x
        assert np.all(np.abs(np.diff(rec[:, 1])) <= 0.5 * 0.0625 + 1e-12)


@pytest.mark.gpu
def test_driver_tracks_in_a_volume(tmp_path):
    """tr_init = volume (start_tracking, main.cpp:1612-1690): n_tracks cells
    drawn uniformly in the box [xtr1, xtr2] x [ytr1, ytr2] x [ztr1, ztr2];
    the first electron of each gets the next track number (a cell drawn
    twice renumbers it)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    folder = str(tmp_path / "results")
    conf = CONF + [("n_tracks", "12", "#"), ("particles_to_track", "#", "e"), ("tr_start", "0", "lambda"),
                   ("tr_init", "#", "volume"),
                   ("xtr1", "1.1", "lambda"), ("ytr1", "0.5", "lambda"), ("ztr1", "0.5", "lambda"),
                   ("xtr2", "1.4", "lambda"), ("ytr2", "1.0", "lambda"), ("ztr2", "1.0", "lambda")]
    _run_driver(conf, folder)
    files = sorted((f for f in os.listdir(folder) if f.startswith("track_-1_")), key=lambda f: int(f.split("_")[-1]))
    nums = [int(f.split("_")[-1]) for f in files]
    assert 6 <= len(nums) <= 12 and all(1 <= n_ <= 12 for n_ in nums) and len(set(nums)) == len(nums)
    for f in files:
        rec = np.array(open(os.path.join(folder, f)).read().split(), dtype=float).reshape(-1, 9)
        assert np.all(rec[:, 0] < 0)
        assert np.all((rec[:, 1] > 1.0) & (rec[:, 1] < 1.6))
        assert np.all((rec[:, 2] > 0.4) & (rec[:, 2] < 1.1)) and np.all((rec[:, 3] > 0.4) & (rec[:, 3] < 1.1))


def _slices(folder, name, t, nx, ny, nz):
    """The xy line at k = nz/2 and the xz line at j = ny/2 per i, then the
    yz plane (the field and density slice layout)."""
    a = np.loadtxt(os.path.join(folder, name + t))
    lines = a[:nx * (ny + nz)].reshape(nx, ny + nz)
    return lines[:, :ny], lines[:, ny:], a[nx * (ny + nz):].reshape(ny, nz)


@pytest.mark.gpu
def test_driver_laser_envelopes_and_uniform_b(tmp_path):
    """f_envelope = sscos / pearl / tophat (f_init_cos's sscos 1-3,
    init.cpp:122-166) give a pulse with the requested transverse shape (pearl
    and tophat without E_x); uniformB (init.cpp:387-400) sets B_y, B_z to a0y,
    a0z everywhere."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    base = [c for c in CONF if c[0] not in ("mwindow", "t_end", "output_period", "film")] + [
        ("mwindow", "#", "off"), ("t_end", "0.0625", "lambda"), ("output_period", "0.0625", "lambda")]
    maps = {}
    for env in ("cos", "sscos", "pearl", "tophat"):
        f = str(tmp_path / env)
        _run_driver(base + [("f_envelope", "#", env)], f)
        log = read_log(os.path.join(f, "log"))
        nx, ny, nz = log["nx"], log["ny"], log["nz"]
        ey = _slices(f, "ey", "0", nx, ny, nz)[0]   # (x, y) at z = the centre
        assert 1 < np.abs(ey).max() < 1.5 * 5   # a0 = 5 is the vector potential; E has its derivative terms too
        maps[env] = ey
    envs = list(maps)
    for a in range(len(envs)):
        for b in range(a + 1, len(envs)):
            assert not np.allclose(maps[envs[a]], maps[envs[b]], rtol=1e-3, atol=1e-3), (envs[a], envs[b])
    # across y at the pulse's peak: the top hat is flat over most of its
    # radius, the cos pulse is not
    c, th = np.abs(maps["cos"]), np.abs(maps["tophat"])
    i0 = int(np.argmax(c.max(axis=1)))
    jc = ny // 2
    assert th[i0, jc + 3] / th[i0, jc] > c[i0, jc + 3] / c[i0, jc]
    f = str(tmp_path / "ub")
    ub = [c for c in base if c[0] != "b_components_for_output"] + [("b_components_for_output", "#", "xyz")]
    _run_driver(ub + [("f_envelope", "#", "uniformB"), ("a0y", "2", "#"), ("a0z", "3", "#")], f)
    log = read_log(os.path.join(f, "log"))
    nx, ny, nz = log["nx"], log["ny"], log["nz"]
    by, bz = _slices(f, "by", "0", nx, ny, nz)[0], _slices(f, "bz", "0", nx, ny, nz)[0]
    assert np.abs(_slices(f, "ey", "0", nx, ny, nz)[0]).max() == 0
    np.testing.assert_allclose(by[2:-2, 2:-2], 2.0, rtol=1e-12)
    np.testing.assert_allclose(bz[2:-2, 2:-2], 3.0, rtol=1e-12)


def _split3(s):
    p = ["", "", ""]
    k = 0
    for ch in s:
        if ch == "&":
            k += 1
            if k == 3:
                break
        else:
            p[k] += ch
    return p


def _reference_initial_fields(q, shape):
    """init_fields (main.cpp:1041-1229) for one region (x0_sr = 0), calling
    the reference's own f_init_cos / f_init_focused; q holds the parameters
    in c/omega units after main.cpp's input handling (the focused waist and
    amplitude of main.cpp:2906-2925 included)."""
    from oracle import oracle
    nx, ny, nz = shape
    reg = oracle.Region(nx, ny, nz, q["dx"], q["dy"], q["dz"], q["dt"], kind="ref")
    A, Z, x0, y0, z0 = q["a0y"], q["a0z"], q["x0"], q["y0"], q["z0"]
    xl = q["xlength"] / 2
    tg = (q["xt"], q["yt"], q["zt"])
    lp, fr = _split3(q["lp"]), _split3(q["fr"])
    sy = lambda m: (1 - 2 * (fr[m] == "y")) * A
    sz = lambda m: (1 - 2 * (fr[m] == "z")) * Z
    if q["focused"]:
        def P(ay, az, xc, x1, yy, zz, append, phi, phase=q["phase"], K=1):
            reg.f_init_focused(ay, az, q["xsigma"], q["sigma0"], xc, x1, q["b_sign"], phase, yy, zz, append, phi,
                               q["sscos"], K, *tg)
    else:
        def P(ay, az, xc, x1, yy, zz, append, phi):
            reg.f_init_cos(ay, az, q["xsigma"], q["ysigma"], q["zsigma"], xc, q["sscos"], q["b_sign"], x1,
                           q["phase"], yy, zz, append, phi, *tg)
    if not q["focused"] and q["phi_rotate"] != 0:
        P(A, Z, xl + x0, x0, y0, z0, 1, q["phi_rotate"])
    else:
        if q["focused"] and q["sh"] != 0:
            al, be = np.sqrt(1 - q["sh"]), np.sqrt(q["sh"])
            P(A * al, Z * al, xl + x0, x0, y0, z0, 0, 0)
            P(A * be, Z * be, xl + x0, x0, y0, z0, 1, 0, phase=q["shphase"], K=2)
        else:
            P(A, Z, xl + x0, x0, y0, z0, 0 if q["focused"] else 1, 0)
        if q["phi"] != 0:
            P(A, Z, xl - x0, -x0, -y0, -z0, 1, q["phi"])
        elif lp[0] == "xy":
            P(sy(0), sz(0), xl + x0, x0, y0, -z0, 1, 0)
            if lp[1] == "xz":
                P(sy(1), sz(1), xl + x0, x0, -y0, z0, 1, 0)
                P(sy(1), sz(1), xl + x0, x0, -y0, -z0, 1, 0)
                if lp[2] == "yz":
                    for yy, zz in ((y0, z0), (y0, -z0), (-y0, z0), (-y0, -z0)):
                        P(sy(2), sz(1), xl - x0, -x0, yy, zz, 1, 0)
            elif lp[1] == "yz":
                P(sy(1), sz(1), xl - x0, -x0, y0, z0, 1, 0)
                P(sy(1), sz(1), xl - x0, -x0, y0, -z0, 1, 0)
                if lp[2] == "xz":
                    P(sy(2), sz(1), xl - x0, -x0, -y0, z0, 1, 0)
                    P(sy(2), sz(1), xl + x0, x0, -y0, z0, 1, 0)
                    P(sy(2), sz(1), xl - x0, -x0, -y0, -z0, 1, 0)
                    P(sy(2), sz(1), xl + x0, x0, -y0, -z0, 1, 0)
        elif lp[0] == "xz":
            P(sy(0), sz(0), xl + x0, x0, -y0, z0, 1, 0)
            if lp[1] == "yz":
                P(sy(1), sz(1), xl - x0, -x0, -y0, z0, 1, 0)
                P(sy(1), sz(1), xl - x0, -x0, y0, z0, 1, 0)
        elif lp[0] == "yz":
            P(sy(0), sz(0), xl - x0, -x0, y0, z0, 1, 0)
    out = reg.get_fields()[:6].reshape(6, nx, ny, nz)
    reg.close()
    return out


_PULSES = {  # extra records over CONF (lengths in lambda, as the records give them)
    "cos": [],
    "sscos": [("f_envelope", "#", "sscos")],
    "pearl": [("f_envelope", "#", "pearl")],
    "tophat": [("f_envelope", "#", "tophat")],
    "cos_oblique_circular_phi": [("polarization", "#", "circular"), ("y0", "0.15", "lambda"),
                                 ("z0", "-0.1", "lambda"), ("phi", "0.25", "pi"), ("phase", "0.3", "pi")],
    "cos_reflections": [("y0", "0.15", "lambda"), ("z0", "0.1", "lambda"), ("lp_reflection", "#", "xy&xz&yz"),
                        ("f_reflection", "#", "y&z&y")],
    "cos_rotated_target": [("phi_rotate", "0.25", "pi"), ("xtarget", "0.1", "lambda"),
                           ("ytarget", "-0.05", "lambda"), ("b_sign", "-1", "#")],
    "focused": [("f_envelope", "#", "focused")],
    "focussedSSC": [("f_envelope", "#", "focussedSSC")],
    "focused_second_harmonic": [("f_envelope", "#", "focused"), ("shenergy", "0.2", "#"),
                                ("shphase", "0.5", "pi"), ("a0z", "2", "#"), ("a0y", "4", "#")],
    "focused_oblique_reflections": [("f_envelope", "#", "focused"), ("y0", "0.2", "lambda"),
                                    ("z0", "-0.1", "lambda"), ("lp_reflection", "#", "xy&yz&xz"),
                                    ("f_reflection", "#", "z&y&z")],
    "focused_phi_target": [("f_envelope", "#", "focused"), ("phi", "0.5", "pi"), ("ztarget", "0.05", "lambda"),
                           ("polarization", "#", "circular")],
}


@pytest.mark.parametrize("name", list(_PULSES))
def test_driver_initial_pulses_match_reference(tmp_path, name):
    """The driver's initial fields (qp_driver --initial-fields, no GPU
    needed) equal the reference's own f_init_cos / f_init_focused, called in
    init_fields' order, for every envelope, oblique incidence, the
    counter-propagating copy, mirror images, rotation, targets and the
    second harmonic."""
    from oracle import oracle
    if not oracle.available("ref"):
        pytest.skip("reference library not built (make -C oracle ref)")
    from quill_b200 import build
    build.build()
    extra = _PULSES[name]
    keys = {k for k, _, _ in extra}
    conf = [c for c in CONF if c[0] not in keys] + extra
    out = str(tmp_path / "fields.bin")
    r = subprocess.run([DRIVER, "--initial-fields", out], input=stream(conf, str(tmp_path / "res")), text=True,
                       capture_output=True, timeout=120)
    assert r.returncode == 0, r.stderr
    shape = (32, 24, 24)
    drv = np.fromfile(out).reshape((6,) + shape)
    # values are read in float precision, as the reference's stof does (low-level.cpp:414)
    rec = {k: (float(np.float32(v)) if v != "#" else 0.0, u) for k, v, u in conf}
    L = lambda k: rec[k][0] * 2 * np.pi if k in rec else 0.0
    ang = lambda k: (rec[k][0] * (np.pi if rec[k][1] == "pi" else 1.0)) if k in rec else 0.0
    env = rec.get("f_envelope", (0.0, ""))[1]
    a0y = rec["a0y"][0] if "a0y" in rec else rec["a0"][0]
    a0z = rec["a0z"][0] if "a0z" in rec else (a0y if rec.get("polarization", (0.0, ""))[1] == "circular" else 0.0)
    q = dict(dx=L("dx"), dy=L("dy"), dz=L("dz"), dt=L("dt"),
             xlength=L("xlength"), xsigma=L("xsigma"), ysigma=L("ysigma"), zsigma=L("zsigma"),
             x0=L("x0"), y0=L("y0"), z0=L("z0"), xt=L("xtarget"), yt=L("ytarget"), zt=L("ztarget"),
             a0y=a0y, a0z=a0z, phase=ang("phase"), phi=ang("phi"), phi_rotate=ang("phi_rotate"),
             b_sign=0 if rec.get("b_sign", (0.0,))[0] == -1 else 1,
             lp=rec.get("lp_reflection", (0.0, "off"))[1], fr=rec.get("f_reflection", (0.0, "off"))[1],
             focused=env in ("focused", "focussedSSC"),
             sscos={"sscos": 1, "pearl": 2, "tophat": 3, "focussedSSC": 1}.get(env, 0),
             sh=rec["shenergy"][0] if "shenergy" in rec else 0.0, shphase=ang("shphase"))
    if q["focused"]:
        x00 = np.sqrt(q["x0"] ** 2 + q["y0"] ** 2 + q["z0"] ** 2)
        q["sigma0"] = 0.5 * (q["ysigma"] + q["zsigma"])
        sigma = np.sqrt(q["sigma0"] ** 2 + 4 * x00 * x00 / q["sigma0"] ** 2)
        q["a0y"] *= q["sigma0"] / sigma
        q["a0z"] *= q["sigma0"] / sigma
    ref = _reference_initial_fields(q, shape)
    assert np.abs(ref).max() > 0.1
    np.testing.assert_allclose(drv, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


@pytest.mark.gpu
def test_driver_reflected_pulses(tmp_path):
    """lp_reflection = xy (init_fields, main.cpp:1153-1229) adds the pulse's
    mirror image at -z0.  In vacuum the field step is linear, so the run
    equals the sum of a run with the pulse at z0 and one with it at -z0."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    base = [c for c in CONF if c[0] not in ("mwindow", "t_end", "output_period", "film", "zsigma")] + [
        ("mwindow", "#", "off"), ("t_end", "0.0625", "lambda"), ("output_period", "0.0625", "lambda"),
        ("zsigma", "0.2", "lambda")]
    f1, f2, f3 = str(tmp_path / "up"), str(tmp_path / "both"), str(tmp_path / "down")
    _run_driver(base + [("z0", "0.1", "lambda")], f1)
    _run_driver(base + [("z0", "0.1", "lambda"), ("lp_reflection", "#", "xy")], f2)
    _run_driver(base + [("z0", "-0.1", "lambda")], f3)
    log = read_log(os.path.join(f1, "log"))
    nx, ny, nz = log["nx"], log["ny"], log["nz"]
    for name in ("ex", "ey", "ez", "bz"):
        a, b, c = (np.loadtxt(os.path.join(f, name + "0")) for f in (f1, f2, f3))
        assert np.abs(a).max() > 0
        # (to 1e-4 of the peak: the text files carry 6 significant digits and
        # cells at the envelope's edge enter with rounding-level differences)
        np.testing.assert_allclose(b, a + c, rtol=0, atol=1e-4 * np.abs(b).max(), err_msg=name)


@pytest.mark.gpu
def test_driver_particle_beam(tmp_path):
    """beam = on (init_beam / add_beam, main.cpp:1230-1239, init.cpp:480-535):
    electrons with the parabolic profile moving along phib, and the beam's
    own fields; the beam is the only charge of the run."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    f = str(tmp_path / "beam")
    conf = [c for c in CONF if c[0] not in ("mwindow", "film", "a0", "t_end", "output_period")] + [
        ("mwindow", "#", "off"), ("a0", "0", "#"), ("t_end", "0.0625", "lambda"), ("output_period", "0.0625", "lambda"),
        ("beam", "#", "on"), ("Nb", "1e9", "#"), ("epsb", "100", "MeV"), ("xb", "0.3", "lambda"),
        ("rb", "0.3", "lambda"), ("x0b", "1", "lambda"), ("y0b", "0", "lambda"), ("phib", "0", "deg")]
    _run_driver(conf, f)
    n = _rows(os.path.join(f, "N"))
    assert n[0, 0] > 0 and n[0, 1] == 0
    log = read_log(os.path.join(f, "log"))
    nx, ny, nz = log["nx"], log["ny"], log["nz"]
    ey = _slices(f, "ey", "0", nx, ny, nz)[0]
    assert np.abs(ey).max() > 0
    ps = np.array(open(os.path.join(f, "phasespace0")).read().split(), dtype=float).reshape(-1, 9)
    # q x y z ux uy uz g chi: every beam electron moves along +x with gamma = 100 / 0.511
    assert ps.shape[0] > 0
    # (after one step in the beam's own fields, which nearly cancel)
    assert np.all(ps[:, 4] > 0)
    assert np.abs(ps[:, 5]).max() < 1e-2 * ps[:, 4].min() and np.abs(ps[:, 6]).max() < 1e-2 * ps[:, 4].min()
    np.testing.assert_allclose(ps[:, 7], 100 / 0.511, rtol=1e-3)
