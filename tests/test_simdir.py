"""Simulation-directory drop-in (big-wave/multisim.py:50-150 run_single_simulation,
fast-wave/main.cpp:18-57 ``fastwave <sim_dir> -s <idx>``).

The directories are written here the way ``multisim.setup_simulation`` lays
them out: config.yaml, computed.yaml, grid .npy files beside them, and
NNNNNNNN/subconfig.yaml per source. The snapshot directory holds the YAML
files of the reference's own snapshot test verbatim; its detected.npy must
match the reference's recorded output. The sample directory turns a golden
plane-wave case into a vector source of ones (the sim-dir format has no plane
source), which must reproduce that case's golden detector.
"""

import json

import numpy as np
import pytest
import yaml

from conftest import GOLDEN, load_case, load_snapshot_case, rel_l2
from rave_sim_b200 import simdir


def _write_snapshot_dir(root, save_u=False):
    d = np.load(GOLDEN / "snapshot.npz")
    cfg = yaml.safe_load(str(d["config_yaml"]))
    cfg["save_final_u_vectors"] = bool(save_u)
    (root / "config.yaml").write_text(yaml.safe_dump(cfg))
    (root / "computed.yaml").write_text(str(d["computed_yaml"]))
    sub = root / "00000000"
    sub.mkdir()
    (sub / "subconfig.yaml").write_text(str(d["subconfig_yaml"]))
    return d


def _write_sample_dir(root, dtype="c16"):
    case, grids, d = load_case("sample_tl")
    cfg = {
        "sim_params": case["sim_params"],
        "use_disk_vector": False,
        "save_final_u_vectors": False,
        "dtype": dtype,
        "elements": case["elements"],
    }
    for i, g in grids.items():
        np.save(root / case["elements"][i]["grid_path"], g)
    (root / "config.yaml").write_text(yaml.safe_dump(cfg))
    (root / "computed.yaml").write_text(yaml.safe_dump({"cutoff_angles": case["cutoff_angles"]}))
    src = root / "ones.npy"
    np.save(src, np.ones(case["sim_params"]["N"], dtype=np.complex128))
    sub = root / "00000000"
    sub.mkdir()
    (sub / "subconfig.yaml").write_text(yaml.safe_dump({
        "source": {"type": "vector", "z": case["source"]["z"], "input_path": str(src)},
        "energy": case["energy"],
        "deltabeta_table": case["db"],
    }))
    return case, d


# ------------------------------------------------------------------ host side
def test_load_source_matches_oracle_parser(tmp_path):
    _write_snapshot_dir(tmp_path)
    got = simdir.load_source(tmp_path, 0)
    want, _ = load_snapshot_case()
    assert got["dtype"] == "c16"
    assert got["energy"] == want["energy"]
    assert got["cutoff_angles"] == want["cutoff_angles"]
    assert got["source"] == {"type": "point", "x": want["source"]["x"], "z": want["source"]["z"]}
    assert got["sim_params"] == want["sim_params"]
    assert [e["type"] for e in got["elements"]] == ["grating"] * 3
    assert [m[0] for m, _ in got["db"]] == ["Si", "Au"]


def test_load_source_reads_grids_and_vector_source(tmp_path):
    case, _ = _write_sample_dir(tmp_path)
    got = simdir.load_source(tmp_path, 0)
    assert set(got["grids"]) == {1}
    assert got["grids"][1].dtype == np.int8
    assert got["source"]["type"] == "vector"
    assert got["source"]["z"] == case["source"]["z"]


def test_rejects_bad_dtype_and_sources(tmp_path):
    _write_snapshot_dir(tmp_path)
    cfg = yaml.safe_load((tmp_path / "config.yaml").read_text())
    cfg["dtype"] = "c32"
    (tmp_path / "config.yaml").write_text(yaml.safe_dump(cfg))
    with pytest.raises(ValueError, match="Unknown dtype"):
        simdir.load_source(tmp_path, 0)
    cfg["dtype"] = "c8"
    (tmp_path / "config.yaml").write_text(yaml.safe_dump(cfg))
    sub = yaml.safe_load((tmp_path / "00000000" / "subconfig.yaml").read_text())
    sub["source"] = {"type": "plane", "z": 0.0}
    (tmp_path / "00000000" / "subconfig.yaml").write_text(yaml.safe_dump(sub))
    with pytest.raises(ValueError, match="Unknown source type"):
        simdir.load_source(tmp_path, 0)


def test_cli_reports_errors_without_traceback(tmp_path, capsys):
    assert simdir.main([str(tmp_path / "missing"), "-s", "0"]) == 1
    assert "error:" in capsys.readouterr().err


def test_parse_source_indices():
    assert simdir.parse_indices("7") == [7]
    assert simdir.parse_indices("0-3") == [0, 1, 2, 3]
    assert simdir.parse_indices("0,4,9-11") == [0, 4, 9, 10, 11]
    for bad in ("", "3-1", "-2", "a"):
        with pytest.raises(ValueError):
            simdir.parse_indices(bad)


def test_cli_several_sources_reject_history(tmp_path, capsys):
    _write_snapshot_dir(tmp_path)
    assert simdir.main([str(tmp_path), "-s", "0-1", "--history_dz", "0.1"]) == 1
    assert "single source index" in capsys.readouterr().err


def test_detector_x_vector_matches_reference_formula():
    # util.detector_x_vector (big-wave/util.py:78-82)
    x = simdir.detector_x_vector(2.5e-05, 1.0e-06)
    n = 2.5e-05 // 1.0e-06
    assert np.array_equal(x, (np.arange(n) - n // 2) * 1.0e-06)


# ------------------------------------------------------------------ on the GPU
gpu = pytest.mark.gpu


def _need_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


@gpu
def test_cli_snapshot_dir_matches_reference_output(tmp_path):
    _need_cuda()
    d = _write_snapshot_dir(tmp_path)
    assert simdir.main([str(tmp_path), "-s", "0"]) == 0
    det = np.load(tmp_path / "00000000" / "detected.npy")
    assert det.dtype == np.float64 and det.shape == d["detected"].shape
    np.testing.assert_allclose(det, d["detected"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(det[0], d["known_data"], rtol=0, atol=1e-14)


@gpu
def test_save_final_u_vector(tmp_path):
    _need_cuda()
    from oracle import bigwave_np as bw

    d = _write_snapshot_dir(tmp_path, save_u=True)
    det = simdir.run_single_simulation(tmp_path, 0)
    u = np.load(tmp_path / "00000000" / "u_0000.npy")
    case, _ = load_snapshot_case()
    sim = bw.make_sim(case)
    assert u.shape == (sim.N,) and u.dtype == np.complex128
    again = bw.square_and_downsample(u, sim, sim.z_detector)
    assert rel_l2(again, det[0]) < 1e-13
    assert rel_l2(det, d["detected"]) < 1e-12


@gpu
@pytest.mark.parametrize("dtype,tol", [("c16", 1e-10), ("c8", 1e-5)])
def test_sample_dir_vector_source(tmp_path, dtype, tol):
    _need_cuda()
    case, d = _write_sample_dir(tmp_path, dtype)
    det = simdir.run_single_simulation(tmp_path, 0)
    assert det.shape == d["detected"].shape
    assert rel_l2(det, d["detected"]) < tol
    assert np.array_equal(np.load(tmp_path / "00000000" / "detected.npy"), det)


@gpu
def test_cli_history(tmp_path):
    _need_cuda()
    from oracle import bigwave_np as bw

    _write_snapshot_dir(tmp_path)
    assert simdir.main([str(tmp_path), "-s", "0", "--history_dz", "0.05"]) == 0
    sub = tmp_path / "00000000"
    h, z, x = (np.load(sub / f) for f in ("history.npy", "history_z.npy", "history_x.npy"))
    case, _ = load_snapshot_case()
    det, h_ref, z_ref = bw.run_simulation(case, history_dz=0.05)
    assert np.array_equal(z, z_ref)
    assert h.shape == h_ref.shape
    assert rel_l2(h, h_ref) < 1e-10
    assert x.shape == (h.shape[0],)


def _add_sources(root, energies, x=None):
    """Further subconfigs beside 00000000: the same point source (or one at
    x), other energies, deltabeta scaled by (E0 / E)^2."""
    sub0 = yaml.safe_load((root / "00000000" / "subconfig.yaml").read_text())
    e0 = float(sub0["energy"])
    ks = []
    for i, e in enumerate(energies, start=1):
        sub = dict(sub0, energy=float(e))
        r = (e0 / e) ** 2
        sub["deltabeta_table"] = [[m, [v[0] * r, v[1] * r * r]] for m, v in sub0["deltabeta_table"]]
        if x is not None and i == len(energies):
            sub["source"] = dict(sub0["source"], x=float(x))
        d = root / f"{i:08}"
        d.mkdir()
        (d / "subconfig.yaml").write_text(yaml.safe_dump(sub))
        ks.append(i)
    return [0] + ks


@gpu
def test_several_sources_match_one_by_one(tmp_path):
    # sources 0-3 share the point source and run as one batch, source 4 has
    # its own; every detected.npy equals that source's own run
    _need_cuda()
    _write_snapshot_dir(tmp_path)
    ks = _add_sources(tmp_path, [40000.0, 52000.0, 58000.0, 44000.0], x=-2e-7)
    assert simdir.main([str(tmp_path), "-s", f"0-{ks[-1]}"]) == 0
    batched = {k: np.load(tmp_path / f"{k:08}" / "detected.npy") for k in ks}
    for k in ks:
        one = simdir.run_single_simulation(tmp_path, k)
        assert batched[k].shape == one.shape and batched[k].dtype == np.float64
        assert rel_l2(batched[k], one) < 1e-12, k
    assert rel_l2(batched[0], batched[1]) > 1e-3  # the energies differ
