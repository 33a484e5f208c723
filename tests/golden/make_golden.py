"""Generate the golden fixtures in this directory by running the UNMODIFIED
rave-sim big-wave FP64 path (``big-wave/*.py`` of the reference checkout).

This script is the only place that touches the reference; it runs in the
development container, never on a GPU host, and its outputs (``*.npz``) are
committed so that the tests and the oracle can be pinned without the
reference present.

big-wave imports a few packages that are not installed here. They are
replaced by minimal stand-ins registered in ``sys.modules`` before the
reference modules are imported:

* ``ruamel.yaml``   -> PyYAML-backed ``YAML`` with ``load``/``dump``/``indent``
  (used by ``big-wave/config.py:191-200``), ``comments.CommentedMap = dict``.
* ``bfpy``          -> a namespace with a ``ChunkedEditor`` attribute (only the
  type annotation at ``big-wave/vector.py:227`` needs it; DiskVector is unused).
* ``freezegun``, ``h5py`` -> no-op modules (imported by ``test.py`` /
  ``multisim.py``; not on the path exercised here).
* ``nist_lookup.xraydb`` -> an ``xrayDB`` over the reference's own
  ``xrayref.db`` read with ``sqlite3`` instead of SQLAlchemy, implementing the
  three lookups ``xraydb_plugin.xray_delta_beta`` uses
  (``nist_lookup/nist_lookup/xraydb.py:219-250`` and ``:371-403``: a
  smoothing spline through an 11-point energy window for f1, log-log linear
  interpolation for the other columns). The real ``xraydb_plugin.py`` and
  ``chemparser.py`` are used unchanged.

Usage:  python tests/golden/make_golden.py [/path/to/reference]
"""

from __future__ import annotations

import json
import os
import sqlite3
import sys
import tempfile
import types
from pathlib import Path

import numpy as np
import yaml

HERE = Path(__file__).resolve().parent


# --------------------------------------------------------------------------
# import stand-ins
# --------------------------------------------------------------------------
def _install_stubs(ref: Path) -> None:
    class _YAML:
        def __init__(self, typ="rt", **kw):
            self._indent = {}

        def load(self, path):
            with open(path) as f:
                return yaml.safe_load(f)

        def indent(self, **kw):
            self._indent = kw

        def dump(self, data, f):
            def plain(o):
                if isinstance(o, dict):
                    return {k: plain(v) for k, v in o.items()}
                if isinstance(o, (list, tuple)):
                    return [plain(v) for v in o]
                if isinstance(o, np.generic):
                    return o.item()
                return o

            yaml.safe_dump(plain(data), f, sort_keys=False)

    ruamel = types.ModuleType("ruamel")
    ruamel_yaml = types.ModuleType("ruamel.yaml")
    comments = types.ModuleType("ruamel.yaml.comments")
    comments.CommentedMap = dict
    ruamel_yaml.YAML = _YAML
    ruamel_yaml.comments = comments
    ruamel.yaml = ruamel_yaml
    sys.modules.update(
        {"ruamel": ruamel, "ruamel.yaml": ruamel_yaml, "ruamel.yaml.comments": comments}
    )

    bfpy = types.ModuleType("bfpy")
    bfpy.ChunkedEditor = object
    sys.modules["bfpy"] = bfpy

    fg = types.ModuleType("freezegun")
    fg.freeze_time = lambda *a, **k: (lambda f: f)
    sys.modules["freezegun"] = fg
    sys.modules["h5py"] = types.ModuleType("h5py")

    db_path = ref / "nist_lookup" / "nist_lookup" / "xrayref.db"

    class xrayDB:  # noqa: N801 - mirrors the reference class name
        def __init__(self, dbname="xrayref.db", read_only=True):
            self.conn = sqlite3.connect(f"file:{db_path}?mode=ro", uri=True)

        def _elem(self, element):
            row = self.conn.execute(
                "select atomic_number, molar_mass from elements where element=?",
                (element.title(),),
            ).fetchone()
            assert row is not None, element
            return row

        def atomic_number(self, element):
            return int(self._elem(element)[0])

        def atomic_mass(self, element):
            return self._elem(element)[1]

        def chantler_data(self, element, energy, column, **kws):
            from scipy.interpolate import UnivariateSpline

            row = self.conn.execute(
                f"select energy, {column} from Chantler where element=?",
                (element.title(),),
            ).fetchone()
            te = np.array(json.loads(row[0]))
            ty_all = np.array(json.loads(row[1]))
            energy = np.asarray([energy]) if np.isscalar(energy) else np.asarray(energy)
            emin, emax = min(energy), max(energy)
            lo = max(0, -5 + max(np.where(te <= emin)[0]))
            hi = min(len(te), 6 + max(np.where(te <= emax)[0]))
            te = te[lo:hi]
            ty = ty_all[lo:hi]
            if column == "f1":
                out = UnivariateSpline(te, ty, s=1)(energy)
            else:
                out = np.exp(np.interp(np.log(energy), np.log(te), np.log(ty)))
            if isinstance(out, np.ndarray) and len(out) == 1:
                return out[0]
            return out

    sys.path.insert(0, str(ref / "nist_lookup"))
    import nist_lookup  # noqa: F401  (the reference's empty package __init__)

    xmod = types.ModuleType("nist_lookup.xraydb")
    xmod.xrayDB = xrayDB
    sys.modules["nist_lookup.xraydb"] = xmod
    sys.path.insert(0, str(ref / "big-wave"))


# --------------------------------------------------------------------------
# cases
# --------------------------------------------------------------------------
def _grating(z_start, pitch, thickness, nr_steps, x_positions, mat_a, mat_b,
             substrate_thickness=0.0, mat_substrate=None, dc=(0.5, 0.5)):
    return {
        "type": "grating", "pitch": pitch, "dc": list(dc), "z_start": z_start,
        "thickness": thickness, "nr_steps": nr_steps,
        "x_positions": list(x_positions),
        "substrate_thickness": substrate_thickness, "mat_a": mat_a,
        "mat_b": mat_b, "mat_substrate": mat_substrate,
    }


SI = ["Si", 2.34]
AU = ["Au", 19.32]
AL = ["Al", 2.70]


def _cases():
    """Small end-to-end cases run through ``wavesim.run_simulation``.

    Each case is (name, config dict in the reference config.yaml schema,
    per-source dict, sample grids, extra element objects).
    """
    cases = []

    # 1. plane wave through one pi-phase Si grating, then a gap (config-1 shape,
    #    reduced N); no frequency cutoff (angles pi/2).
    N = 1 << 14
    dx = 2e-9
    p = 4.2e-6
    cases.append(dict(
        name="plane_grating",
        sim_params=dict(N=N, dx=dx, z_detector=0.0818 + 60e-6 + 0.01,
                        detector_size=N * dx * 0.9, detector_pixel_size_x=1e-6 / 8,
                        detector_pixel_size_y=1.0, chunk_size=N),
        elements=[_grating(0.01, p, 59.37e-6, 5, [0.0], SI, None)],
        source=dict(type="plane", z=0.01), energy=46000.0,
        db=[[SI, [2.27e-7, 1e-10]]], cutoff_angles=[np.pi / 2] * 2,
        save_u=True,
    ))

    # 2. same with a chunk size that does not divide N (per-chunk linspace
    #    coordinates of the grating mask, big-wave/optical_element.py:341-357).
    c2 = dict(cases[-1])
    c2 = json.loads(json.dumps(c2))
    c2["name"] = "plane_grating_chunked"
    c2["sim_params"]["chunk_size"] = 3001
    c2["elements"][0]["x_positions"] = [0.37e-6]
    c2["elements"][0]["dc"] = [0.4, 0.6]
    cases.append(c2)

    # 3. point source, three-grating Talbot-Lau with substrates, active
    #    frequency cutoffs and 4 phase steps of G2.
    N = 1 << 15
    dx = 5e-10
    cases.append(dict(
        name="tl3g_point_phase",
        sim_params=dict(N=N, dx=dx, z_detector=0.30, detector_size=12e-6,
                        detector_pixel_size_x=0.5e-6, detector_pixel_size_y=1e-6,
                        chunk_size=N),
        elements=[
            _grating(0.05, p, 40e-6, 3, [0.0], AU, None, 100e-6, SI),
            _grating(0.15, p, 30e-6, 2, [0.0], SI, None, 50e-6, SI),
            _grating(0.25, p, 40e-6, 3, [k * p / 4 for k in range(4)], AU, SI, 80e-6, SI),
        ],
        source=dict(type="point", x=0.2e-6, z=0.0), energy=46500.0,
        db=[[SI, [2.2888e-7, 2.5847e-10]], [AU, [1.4981e-6, 3.6174e-8]]],
        cutoff_angles=[4e-5, 5e-5, 6e-5, 7e-5],
        save_u=False,
    ))

    # 4. DBA grating (two superposed pitches), multi-chunk, cutoff on.
    N = 1 << 14
    dx = 1e-9
    cases.append(dict(
        name="dba_grating",
        sim_params=dict(N=N, dx=dx, z_detector=0.2, detector_size=14e-6,
                        detector_pixel_size_x=0.7e-6, detector_pixel_size_y=1.0,
                        chunk_size=N // 4),
        elements=[{
            "type": "dba_grating", "pitch0": 1.3e-6, "pitch1": 3.9e-6,
            "dc0": [0.5, 0.45], "dc1": [0.6, 0.6], "z_start": 0.1,
            "thickness": 20e-6, "nr_steps": 3,
            "x_positions": [0.0, 0.4e-6, 0.8e-6],
            "substrate_thickness": 30e-6, "mat_a": AU, "mat_b": None,
            "mat_substrate": SI,
        }],
        source=dict(type="plane", z=0.1), energy=40000.0,
        db=[[SI, [3.0e-7, 2e-10]], [AU, [1.9e-6, 5e-8]]],
        cutoff_angles=[1e-4, 1e-4],
        save_u=True,
    ))

    # 5. grating, then a pixelised int8 sample (3 materials + vacuum), then an
    #    analyser grating with 3 phase steps.
    N = 1 << 14
    dx = 1e-9
    rng = np.random.default_rng(7)
    grid = rng.integers(0, 4, size=(6, 37)).astype(np.int8)
    cases.append(dict(
        name="sample_tl",
        sim_params=dict(N=N, dx=dx, z_detector=0.2, detector_size=14e-6,
                        detector_pixel_size_x=1e-6, detector_pixel_size_y=1.0,
                        chunk_size=N),
        elements=[
            _grating(0.02, 2e-6, 20e-6, 2, [0.0], SI, None),
            {"type": "sample", "z_start": 0.05, "pixel_size_x": 0.3e-6,
             "pixel_size_z": 5e-6, "grid_path": "grid.npy",
             "materials": [AL, SI, AU], "x_positions": [0.0]},
            _grating(0.15, 2e-6, 30e-6, 2, [0.0, 0.5e-6, 1.0e-6], AU, None),
        ],
        grid=grid,
        source=dict(type="plane", z=0.02), energy=30000.0,
        db=[[AL, [6.0e-7, 3e-9]], [SI, [5.4e-7, 1.2e-9]], [AU, [3.5e-6, 1.5e-7]]],
        cutoff_angles=[np.pi / 2] * 4,
        save_u=False,
    ))

    # 6. phase stepping by moving the sample itself (x_positions on a sample),
    #    point source, cutoff on, odd chunking.
    c6 = json.loads(json.dumps({k: v for k, v in cases[-1].items() if k != "grid"}))
    c6["name"] = "sample_stepped"
    c6["grid"] = grid
    c6["elements"][1]["x_positions"] = [0.0, 0.13e-6, -0.41e-6]
    c6["elements"][2]["x_positions"] = [0.0]
    c6["source"] = dict(type="point", x=-0.1e-6, z=0.0)
    c6["cutoff_angles"] = [3e-5, 3e-5, 4e-5, 4e-5]
    c6["sim_params"]["chunk_size"] = 5000
    c6["keypoints"] = True  # big-wave/wavesim.py:35-55: u before / after each element
    cases.append(c6)

    # 7./8. history recording (big-wave/history.py:43-135): a point source
    #    through the three-grating interferometer (analytic source history,
    #    gaps re-propagated from their start, grating sub-steps), and the
    #    sample case (pushes before every sample row).
    c7 = json.loads(json.dumps(cases[2]))
    c7["name"] = "hist_point_tl"
    c7["history_dz"] = 0.02
    cases.append(c7)
    c8 = json.loads(json.dumps({k: v for k, v in cases[4].items() if k != "grid"}))
    c8["name"] = "hist_sample"
    c8["grid"] = grid
    c8["history_dz"] = 0.013
    c8["keypoints"] = True
    cases.append(c8)

    # 9. big-wave's own test_stepping setup (big-wave/test.py:251-300): N = 6,
    #    a point source, two vacuum gratings (the second phase-stepped),
    #    cutoff angles 0.1 / 0.2 / 0.3, history every 0.1 m.
    def _vacuum_grating(z, xs):
        return {"type": "grating", "pitch": 4.2e-6, "dc": [0.5, 0.5], "z_start": z, "thickness": 100e-6,
                "nr_steps": 1, "x_positions": xs, "substrate_thickness": 0.0, "mat_a": None, "mat_b": None,
                "mat_substrate": None}
    cases.append(dict(
        name="stepping_n6",
        sim_params=dict(N=6, dx=10e-9, z_detector=1.0, detector_size=40e-9, detector_pixel_size_x=20e-9,
                        detector_pixel_size_y=1.0, chunk_size=3),
        elements=[_vacuum_grating(0.1, [0.0]), _vacuum_grating(0.2, [0.0, 1.6e-6, 3.1e-6])],
        source=dict(type="point", x=0.0, z=0.0), energy=46000.0, db=[],
        cutoff_angles=[0.1, 0.2, 0.3], history_dz=0.1, save_u=False, keypoints=True,
    ))

    # 10. an odd length (3^8): point source off axis, a chunked grating, a
    #     pixelised sample, active cutoffs (the reference's N / 2 and N // 2
    #     conventions differ for odd N).
    N = 3 ** 8
    grid10 = np.random.default_rng(11).integers(0, 3, size=(5, 29)).astype(np.int8)
    cases.append(dict(
        name="odd_point_sample",
        sim_params=dict(N=N, dx=2e-9, z_detector=0.12, detector_size=10e-6, detector_pixel_size_x=0.5e-6,
                        detector_pixel_size_y=1.0, chunk_size=1000),
        elements=[
            _grating(0.02, 1.9e-6, 20e-6, 2, [0.0], SI, None),
            {"type": "sample", "z_start": 0.05, "pixel_size_x": 0.35e-6, "pixel_size_z": 4e-6,
             "grid_path": "grid.npy", "materials": [AL, SI], "x_positions": [0.0]},
        ],
        grid=grid10,
        source=dict(type="point", x=0.05e-6, z=0.0), energy=35000.0,
        db=[[AL, [4.4e-7, 2e-9]], [SI, [4.0e-7, 1e-9]]],
        cutoff_angles=[5e-5, 6e-5, 7e-5],
        save_u=False, keypoints=True,
    ))

    # 11. an even length that is not a power of two: plane wave, a grating
    #     stepped over 3 positions, then a gap.
    N = 12000
    cases.append(dict(
        name="nonpow2_plane",
        sim_params=dict(N=N, dx=1e-9, z_detector=0.08, detector_size=10e-6, detector_pixel_size_x=1e-6,
                        detector_pixel_size_y=1.0, chunk_size=N),
        elements=[_grating(0.02, 2e-6, 30e-6, 3, [0.0, 0.5e-6, 1.0e-6], SI, None)],
        source=dict(type="plane", z=0.02), energy=46000.0,
        db=[[SI, [2.27e-7, 1e-10]]], cutoff_angles=[np.pi / 2] * 2,
        save_u=True,
    ))

    return cases


def _run_case(case, mods, tmp: Path):
    config, optical_element, propagation, source, vector, wavesim = mods
    sp = dict(case["sim_params"])
    params = propagation.SimParams(
        N=sp["N"], dx=sp["dx"], z_detector=sp["z_detector"],
        detector_size=sp["detector_size"],
        detector_pixel_size_x=sp["detector_pixel_size_x"],
        detector_pixel_size_y=sp["detector_pixel_size_y"],
        wl=propagation.convert_energy_wavelength(case["energy"]),
        chunk_size=sp["chunk_size"],
    )
    if "grid" in case:
        np.save(tmp / "grid.npy", case["grid"])
    elements = []
    for el in case["elements"]:
        if el["type"] == "dba_grating":
            # config.parse_optical_element names a class that does not exist for
            # dba gratings (big-wave/config.py:104), so the element is built
            # directly with the fields that parser reads.
            elements.append(optical_element.DBAGrating(
                pitch0=el["pitch0"], pitch1=el["pitch1"],
                dc0=tuple(el["dc0"]), dc1=tuple(el["dc1"]),
                z_start=el["z_start"], thickness=el["thickness"],
                nr_steps=el["nr_steps"], x_positions=np.array(el["x_positions"]),
                substrate_thickness=el["substrate_thickness"],
                mat_a=config.parse_optional_material(el, "mat_a"),
                mat_b=config.parse_optional_material(el, "mat_b"),
                mat_substrate=config.parse_optional_material(el, "mat_substrate"),
            ))
        else:
            elements.append(config.parse_optical_element(el, tmp))
    src = case["source"]
    N = sp["N"]
    if src["type"] == "point":
        s = source.PointSource(x=src["x"], z=src["z"])
    else:
        s = source.VectorSource(input=vector.NumpyVector(np.ones(N, np.complex128)),
                                z=src["z"])
    db_table = [(config.parse_material(m), complex(v[0], v[1])) for m, v in case["db"]]
    u = vector.NumpyVector(np.zeros(N, np.complex128))
    U = vector.NumpyVector(np.zeros(N, np.complex128))
    sub = tmp / "sub"
    sub.mkdir(exist_ok=True)
    hist = None
    if case.get("history_dz"):
        import history as bw_history
        hist = (bw_history.History(), float(case["history_dz"]))
    kp_dir = None
    if case.get("keypoints"):
        kp_dir = tmp / "keypoints"
        kp_dir.mkdir(exist_ok=True)
    det = wavesim.run_simulation(
        params, s, elements, list(case["cutoff_angles"]), u, U, db_table,
        sub, sub, bool(case.get("save_u", False)), history=hist,
        save_keypoints_path=kp_dir,
    )
    out = {"detected": np.array(det)}
    if kp_dir is not None:
        # keypoint_{element:02}_{0 before | 1 after}.npy, in element order;
        # every s-th sample (s = N // 1024 at most) plus full-vector sums
        kps = np.stack([np.load(kp_dir / f"keypoint_{i:02}_{k}.npy")
                        for i in range(len(elements)) for k in (0, 1)])
        stride = max(1, N // 1024)
        out["keypoints_stride"] = np.int64(stride)
        out["keypoints_sub"] = kps[:, ::stride]
        out["keypoints_sum"] = kps.sum(axis=1)
        out["keypoints_norm2"] = (np.abs(kps) ** 2).sum(axis=1)
    if hist is not None:
        out["history"] = hist[0].get_history()
        out["history_z"] = np.array(hist[0].get_z(), dtype=np.float64)
    if case.get("save_u"):
        us = sorted(sub.glob("u_*.npy"))
        # phase step 0 only, to keep the fixture small
        out["u_final"] = np.load(us[0])
    return out


def main():
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    _install_stubs(ref)
    import config  # noqa: F401  (first: breaks the propagation<->config import cycle)
    import optical_element
    import propagation
    import source
    import vector
    import wavesim
    import multisim
    import util
    import test as bw_test

    mods = (config, optical_element, propagation, source, vector, wavesim)
    cwd = os.getcwd()

    # ---- unit goldens taken from the reference's own tests -------------------
    units = {}
    # big-wave/test.py:209-225
    vec = vector.NumpyVector(np.arange(8, dtype=np.complex128))
    sp = propagation.SimParams(N=8, dx=0.5, z_detector=1.0, detector_size=3.0,
                               detector_pixel_size_x=1.0, detector_pixel_size_y=1.0,
                               wl=1.0, chunk_size=3)
    units["sqd_out"] = np.array(propagation.square_and_downsample(vec, sp, 1.0))
    # fast-wave/test/fwtest.cu:111-127 (np.fft.fft of this 8-vector)
    fft_in = np.array([0, 0, 1, 2 + 1j, 3 + 2j, 2, 1, 0], dtype=np.complex128)
    units["fft2_in"] = fft_in
    units["fft2_out"] = np.fft.fft(fft_in)
    # grating masks (big-wave/test.py:121-158 shape): a few parameter sets
    masks = []
    mask_params = []
    for (pitch, dx, dc, xpos, start, count) in [
        (4.0, 0.5, (0.25, 0.5), 0.01, -8, 16),
        (4.0, 0.5, (0.25, 0.5), 1.51, 3, 11),
        (4.2e-6, 1e-6, (0.25, 0.5), 2.1e-6, 123, 16),
        (4.2e-6, 2e-9, (0.5, 0.5), 0.0, -(1 << 13), 1 << 14),
        (1.3e-6, 1e-9, (0.45, 0.55), 0.33e-6, -4096, 3001),
    ]:
        for zf in (0.0, 0.5, 1.0):
            g = optical_element.Grating(
                pitch=pitch, dc=dc, z_start=0, thickness=1, nr_steps=1,
                x_positions=np.array([xpos]), substrate_thickness=0.0,
                mat_a=None, mat_b=None, mat_substrate=None)
            masks.append(optical_element.generate_grating_chunk(dx, start, count, g, zf, 0))
            mask_params.append([pitch, dx, dc[0], dc[1], xpos, start, count, zf])
    units["mask_params"] = np.array(mask_params, dtype=np.float64)
    units["mask_concat"] = np.concatenate(masks).astype(np.uint8)
    units["mask_lengths"] = np.array([len(m) for m in masks])
    # frequency cutoff (big-wave/test.py:187-199 parameter grid)
    cut = []
    for dx in [0.5, 1.0, 2.3]:
        for n in [3, 4, 5, 6, 7, 8, 1024]:
            for freq in [0.0, 0.1, 0.4, 1.2, 3.5, 100000.0, 0.43478260869565216]:
                v = vector.NumpyVector(np.ones(n, dtype=np.complex128))
                propagation.apply_frequency_cutoff(v, freq, dx, 3)
                cut.append((dx, n, freq, np.flatnonzero(v.vec == 0)))
    units["cut_params"] = np.array([(a, b, c) for a, b, c, _ in cut])
    units["cut_zero_counts"] = np.array([len(z) for *_, z in cut])
    units["cut_zero_first"] = np.array([z[0] if len(z) else -1 for *_, z in cut])
    np.savez_compressed(HERE / "units.npz", **units)

    # ---- Al attenuation for the bremsstrahlung spectrum weights ------------
    # mu_Al(E) = 1/atlen from the reference's material lookup
    # (nist_lookup/nist_lookup/xraydb_plugin.py:134-181), density 2.70 g/cm^3
    energies = np.arange(10000.0, 80001.0, 500.0)
    mu = np.array([1.0 / optical_element.xray_delta_beta("Al", 2.70, float(e))[2] for e in energies])
    np.savez_compressed(HERE / "al_attenuation.npz", energy_ev=energies, mu_per_cm=mu)

    # ---- TestSnapshot (big-wave/test.py:853-960) --------------------------
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        os.chdir(td)
        sim_dir = multisim.setup_simulation(bw_test.TestSnapshot.known_config, td, td)
        multisim.run_single_simulation(sim_dir, 0, sim_dir)
        wf = util.load_wavefronts_filtered(sim_dir)[0][0]
        cfg_txt = (sim_dir / "config.yaml").read_text()
        comp_txt = (sim_dir / "computed.yaml").read_text()
        sub_txt = (sim_dir / "00000000" / "subconfig.yaml").read_text()
        os.chdir(cwd)
    np.savez_compressed(
        HERE / "snapshot.npz",
        detected=np.asarray(wf),
        known_data=bw_test.TestSnapshot.known_data,
        config_yaml=np.array(cfg_txt), computed_yaml=np.array(comp_txt),
        subconfig_yaml=np.array(sub_txt),
    )
    err = np.abs(np.asarray(wf)[0] - bw_test.TestSnapshot.known_data).max()
    print(f"snapshot: max-abs vs known_data {err:.3e}")

    # ---- small end-to-end cases ---------------------------------------------
    for case in _cases():
        with tempfile.TemporaryDirectory() as td:
            td = Path(td)
            os.chdir(td)
            out = _run_case(case, mods, td)
            os.chdir(cwd)
        desc = {k: v for k, v in case.items() if k not in ("grid", "name")}
        arrays = dict(out)
        arrays["case_json"] = np.array(json.dumps(desc))
        if "grid" in case:
            arrays["grid"] = case["grid"]
        np.savez_compressed(HERE / f"case_{case['name']}.npz", **arrays)
        print(f"{case['name']}: detected {out['detected'].shape}")


if __name__ == "__main__":
    main()
