"""The FDTD job reader: a 3D job of rects on a stack of fixed indices, read as the reference's
Setup::new reads it (src/job/fdtd.rs:414-712), its permittivity the reference's closure
(src/job/fdtd.rs:1344-1425), its stop rule the runner's (src/job/fdtd.rs:2700-2850).

CPU: the reading, the refusals, the permittivity at points on every face, the pulse's spectrum
against the oracle's, and the stop rule run in runs of steps against the same rule applied step
by step to one long probe series (both on the oracle). GPU: the job on the engine in f64 gives
the oracle's bits: the step it stops at, every flux, every spectrum, every transform.
"""
import math

import numpy as np
import pytest

from photonoxide_b200 import job as J
from photonoxide_b200.types import Axis, Field, Periodic, Pml

import pyoracle

JOB = """
name = "strip-3d-dipole"
[task]
kind = "fdtd"
wavelength_um = 1.55
layer = "core"
dimensions = 3
x_um = [-0.6, 0.6]
y_um = [-0.6, 0.6]
z_um = [-0.5, 0.72]
step_nm = 50.0
pml_cells = 5
spectrum = { from_um = 1.5, to_um = 1.6, points = 5 }

[task.stack]
substrate = 1.44
cladding = 1.0
[[task.stack.layer]]
name = "core"
thickness_um = 0.22
material = 3.48
background = 1.44

[[task.rect]]
layer = "core"
center_um = [0.0, 0.0]
size_um = [2.0, 0.45]

[[task.source]]
type = "dipole"
position_um = [-0.1, 0.02, 0.11]
component = "Ey"

[[task.monitor]]
type = "flux"
name = "out"
normal = "x"
at_um = 0.3
y_um = [-0.3, 0.3]
z_um = [-0.2, 0.45]

[[task.monitor]]
type = "flux_box"
name = "box"
x_um = [-0.3, 0.25]
y_um = [-0.25, 0.3]
z_um = [-0.15, 0.4]

[[task.monitor]]
type = "field"

[task.stop]
until = "decay"
fraction = 1e-3
limit_um = 400.0
"""


def test_reads_the_window_grid_and_pulse():
    job = J.load(JOB)
    g = job.grid
    assert (g.nx, g.ny, g.nz) == (24, 24, 24)  # round(1.2 / 0.05), round(1.22 / 0.05)
    assert g.dx == 1.2 / 24 and g.dz == 1.22 / 24 and g.z0 == -0.5
    assert job.boundaries.x == Pml(5, 5) and job.boundaries.z == Pml(5, 5)
    assert job.wavelengths_um == [1.5 + (1.6 - 1.5) * float(k) / 4.0 for k in range(5)]
    carrier = 1.0 / 1.55
    reach = max(abs(1.0 / w - carrier) for w in job.wavelengths_um)
    assert job.bandwidth == max(2.0 * reach, 0.05 * carrier)
    w = job.waveform()
    width = math.sqrt(2.0 * math.log(2.0)) / (math.pi * job.bandwidth)
    assert w.params == (carrier, width, 6.0 * width)
    d = job.dipoles[0]
    assert (d.field, d.component, d.position, d.amplitude) == (Field.E, Axis.Y,
                                                               (-0.1, 0.02, 0.11), 1.0)
    assert job.until == ("decay", 1e-3, 400.0)


def test_places_flux_planes_on_half_planes():
    job = J.load(JOB)
    out, box, field = job.monitors
    plane, sign = out.faces[0]
    # round((0.3 + 0.6)/0.05 - 0.5) = round(17.5) = 18 (away from zero; Python's round gives 18
    # too, but 0.5 cases below it would not)
    assert (plane.axis, plane.plane, sign) == (Axis.X, 18, 1.0)
    assert plane.window == ((J._half_plane(job, 1, -0.3, ""), J._half_plane(job, 1, 0.3, "")),
                            (J._half_plane(job, 2, -0.2, ""), J._half_plane(job, 2, 0.45, "")))
    assert len(box.faces) == 6 and [s for _, s in box.faces] == [-1.0, 1.0] * 3
    assert [f.axis for f, _ in box.faces] == [Axis.X, Axis.X, Axis.Y, Axis.Y, Axis.Z, Axis.Z]
    planes = [(J._half_plane(job, 0, -0.3, ""), J._half_plane(job, 0, 0.25, "")),
              (J._half_plane(job, 1, -0.25, ""), J._half_plane(job, 1, 0.3, "")),
              (J._half_plane(job, 2, -0.15, ""), J._half_plane(job, 2, 0.4, ""))]
    for q, (f, _) in enumerate(box.faces):
        b, c = f.axis.others()
        assert f.plane == planes[int(f.axis)][q % 2]
        assert f.window == (planes[int(b)], planes[int(c)])
    assert field.kind == "field" and field.wavelengths_um == [1.55]
    # the view's plane: floor((0.11 - (-0.5)) / dz), the layer's middle
    assert field.k == math.floor((0.11 + 0.5) / job.grid.dz)
    pts = job.probe_points()
    assert len(pts) == 7  # the flux plane's middle, then each face's
    assert pts[0] == (18, (plane.window[0][0] + plane.window[0][1]) // 2,
                      (plane.window[1][0] + plane.window[1][1]) // 2)


def reference_eps(x, y, z, layers, substrate, cladding, rects):
    """The reference's 3D closure for a plain stack (src/job/fdtd.rs:1396-1425), literally."""
    if z < 0.0:
        return substrate * substrate
    tops, t = [], 0.0
    for l in layers:
        t += l["thickness_um"]
        tops.append(t)
    for i, top in enumerate(tops):
        if z < top:
            inside = any(r["layer"] == layers[i]["name"]
                         and r["center_um"][0] - r["size_um"][0] / 2.0 <= x
                         <= r["center_um"][0] + r["size_um"][0] / 2.0
                         and r["center_um"][1] - r["size_um"][1] / 2.0 <= y
                         <= r["center_um"][1] + r["size_um"][1] / 2.0 for r in rects)
            n = layers[i]["material"] if inside else layers[i]["background"]
            return n * n
    return cladding * cladding


def test_permittivity_is_the_reference_closure_on_every_face():
    import tomllib
    task = tomllib.loads(JOB)["task"]
    task["stack"]["layer"].append({"name": "cap", "thickness_um": 0.13, "material": 2.0,
                                   "background": 1.5})
    task["rect"].append({"layer": "cap", "center_um": [0.1, -0.05], "size_um": [0.3, 0.25]})
    job = J.load({"task": task})
    layers, rects = task["stack"]["layer"], task["rect"]
    xs = [-0.4, -0.225, 0.0, 0.225, 0.4, -0.05, 0.25, -1.0, 1.0]
    ys = [-0.3, -0.225, 0.0, 0.225, 0.3, -0.175, 0.075]
    zs = [-0.1, -0.0, 0.0, 0.11, 0.22, 0.22 + 0.13, 0.5, 0.2199999999999999,
          math.nextafter(0.0, -1.0)]
    rng = np.random.default_rng(5)
    pts = [(x, y, z) for x in xs for y in ys for z in zs]
    pts += [tuple(p) for p in rng.uniform([-0.6, -0.6, -0.5], [0.6, 0.6, 0.72], (2000, 3))]
    for x, y, z in pts:
        want = reference_eps(x, y, z, layers, 1.44, 1.0, rects)
        assert job.geometry(x, y, z) == want, (x, y, z)


def test_rust_round_takes_halves_away_from_zero():
    assert [J.rust_round(v) for v in (0.5, 1.5, 2.5, -0.5, -2.5, 0.49999999999999994, 17.5)] == \
        [1.0, 2.0, 3.0, -1.0, -3.0, 0.0, 18.0]


@pytest.mark.parametrize("change, words", [
    (("dimensions = 3", "dimensions = 2"), "effective index"),
    (("material = 3.48", 'material = "si"'), "fixed refractive index"),
    (("material = 3.48", "material = 0.9"), "at least 1"),
    (('type = "dipole"', 'type = "mode"'), "beyond this reader's subset"),
    (('type = "field"', 'type = "resonance"'), "beyond this reader's subset"),
    (('type = "field"', 'type = "flux"\nname = "out"\nnormal = "y"\nat_um = 0.0'),
     'two monitors are named "out"'),
    (("at_um = 0.3", "at_um = 0.58"), "inside its CPMLs"),
    (("fraction = 1e-3", "fraction = 1.5"), "between 0 and 1"),
    (('until = "decay"', 'until = "time"'), "fraction and limit_um are for"),
    (("step_nm = 50.0", "step_nm = 0.05"), "more than 10000"),
    (("pml_cells = 5", "pml_cells = 11"), "leave nothing"),
    (("size_um = [2.0, 0.45]", "size_um = [2.0, 0.45]\netch = { depth_um = 0.1 }"), "etched"),
    (('component = "Ey"', 'component = "Ew"'), 'unknown component "Ew"'),
    (("position_um = [-0.1, 0.02, 0.11]", "position_um = [-0.1, 0.02]"), "[x, y], z"),
    (("position_um = [-0.1, 0.02, 0.11]", "position_um = [-0.1, 0.02, 0.9]"), "outside the window"),
    (('layer = "core"\ndimensions', 'layer = "clad"\ndimensions'), "no layer clad"),
])
def test_refuses_what_the_reference_or_the_subset_refuses(change, words):
    text = JOB.replace(*change)
    assert text != JOB
    with pytest.raises(J.JobError) as e:
        J.load(text)
    assert words in str(e.value)


def test_refuses_a_named_stack_and_a_device():
    import tomllib
    doc = tomllib.loads(JOB)
    doc["task"]["stack"] = "soi_220"
    with pytest.raises(J.JobError, match="named stack"):
        J.load(doc)
    doc = tomllib.loads(JOB)
    doc["device"] = {"kind": "waveguide"}
    with pytest.raises(J.JobError, match="device"):
        J.load(doc)


def test_yaml_and_a_path_read_the_same(tmp_path):
    import tomllib
    import yaml
    doc = tomllib.loads(JOB)
    p = tmp_path / "job.yaml"
    p.write_text(yaml.safe_dump(doc))
    a, b = J.load(JOB), J.load(str(p))
    assert a.grid == b.grid and a.geometry.boxes == b.geometry.boxes
    assert [m.faces for m in a.monitors] == [m.faces for m in b.monitors]


def test_the_pulse_spectrum_is_the_oracles_to_the_bit():
    """The engine's host-side Waveform::spectrum (the reference's exp and sin/cos) against the
    oracle's restatement: the divisor of a dipole run's spectra."""
    from photonoxide_b200.fdtd import waveform_spectrum
    job = J.load(JOB)
    w = job.waveform()
    for field in (Field.E, Field.H):
        a = waveform_spectrum(w, field, 0.026, 4000, job.frequencies())
        b = pyoracle.waveform_spectrum(w, field, 0.026, 4000, job.frequencies())
        assert np.array_equal(a.view(np.float64), b.view(np.float64))
    assert np.all(np.abs(a) > 0)


def literal_stop(job, series, dt):
    """The runner's loop (src/job/fdtd.rs:2746-2790) applied one step at a time to a precomputed
    series of (Ex, Ey, Ez) at each probe point: the step it stops at and how."""
    w = job.waveform()
    pulse_end = w.params[2] + 6.0 * w.params[1]
    check = 10.0 * (1.0 / job.carrier)
    limit = job.until[2] if job.until[0] == "decay" else job.until[1]
    npts = len(series)
    peaks, block = [0.0] * npts, [0.0] * npts
    block_end = pulse_end + check
    growth = J._Growth.after(pulse_end, check)
    for n in range(len(series[0][0])):
        t = float(n + 1) * dt
        for k in range(npts):
            v = sum(float(series[k][c][n]) ** 2 for c in range(3))
            peaks[k] = max(peaks[k], v)
            if t > pulse_end:
                block[k] = max(block[k], v)
        decayed = grew = False
        if t >= block_end:
            worst = max([b / p if p > 0 else 0.0 for p, b in zip(peaks, block)] + [0.0])
            decayed = job.until[0] == "decay" and worst <= job.until[1] and max(peaks) > 0
            grew = growth.check(max(block + [0.0])) is not None
            block = [0.0] * npts
            block_end += check
        if decayed or grew or t >= limit:
            return n + 1, "decayed" if decayed else "grew" if grew else "limit"
    return None, None


WALLS = JOB.replace("pml_cells = 5", 'pml_cells = 5\nboundaries = { x = "wall", y = "wall", '
                    'z = "wall" }').replace("limit_um = 400.0", "limit_um = 250.0")


@pytest.mark.parametrize("text, how", [(JOB, "decayed"), (WALLS, "limit")])
def test_the_stop_rule_in_runs_of_steps_is_the_rule_step_by_step(text, how):
    """A run that decays at its first check, and one between walls that never decays, checked
    at each of its checks until the limit."""
    job = J.load(text)
    out = job.run(cls=pyoracle.OracleSimulation, precision=64,
                  spectrum=pyoracle.waveform_spectrum)
    assert out["stopped"] == how and out["steps"] > 0
    # one long run with the same probes, and the rule applied to it step by step
    s, _ = job.simulation(cls=pyoracle.OracleSimulation, precision=64)
    probes = [[s.add_probe(Field.E, c, p) for c in J.ALL3] for p in job.probe_points()]
    s.run(out["steps"] + 50)
    series = [[s.probe(q) for q in pr] for pr in probes]
    steps, how = literal_stop(job, series, s.dt)
    assert (steps, how) == (out["steps"], out["stopped"])
    # the flux box's spectrum: each face's flux with its sign, over |W|^2 of the pulse
    assert set(out["spectra"]) == {"out", "box"}
    assert np.all(np.isfinite(out["spectra"]["box"])) and np.all(out["incident"] > 0)


@pytest.mark.gpu
def test_a_job_on_the_engine_is_the_oracles_bits():
    """The job through the reader on the B200 in f64 against the same job on the oracle: the
    same stop step, fluxes, spectra and transforms, bit for bit; in f32 the same stop rule's
    outcome and spectra within 1e-3 of the largest."""
    job = J.load(JOB)
    ref = job.run(cls=pyoracle.OracleSimulation, precision=64, spectrum=pyoracle.waveform_spectrum)
    got = job.run(precision=64)
    assert (got["steps"], got["stopped"]) == (ref["steps"], ref["stopped"])
    for name in ref["fluxes"]:
        assert np.array_equal(got["fluxes"][name], ref["fluxes"][name]), name
        assert np.array_equal(got["spectra"][name], ref["spectra"][name]), name
    assert np.array_equal(got["incident"], ref["incident"])
    assert np.array_equal(got["transforms"], ref["transforms"])
    f32 = job.run(precision=32)
    assert f32["stopped"] == ref["stopped"] and abs(f32["steps"] - ref["steps"]) <= 1000
    for name in ref["spectra"]:
        a, b = f32["spectra"][name], ref["spectra"][name]
        assert np.max(np.abs(a - b)) <= 1e-3 * np.max(np.abs(b)), name
