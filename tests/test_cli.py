"""The ms3gpu.mp processor executable: the MountainLab protocol surface that
needs no GPU (spec, requirements, unknown names, argument parsing)."""
import json
import os
import subprocess

import numpy as np
import pytest

from mountainsort_b200 import mdaio

EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mountainsort_b200", "ms3gpu.mp")


def run(*args, env=None):
    e = dict(os.environ)
    if env:
        e.update(env)
    return subprocess.run([EXE, *args], capture_output=True, text=True, env=e, timeout=60)


def test_spec_lists_the_processors():
    r = run("spec")
    assert r.returncode == 0
    spec = json.loads(r.stdout)
    by = {p["name"]: p for p in spec["processors"]}
    assert set(by) == {"ms3.bandpass_filter", "ms3.whiten", "ms3.compute_whitening_matrix",
                       "ms3.whiten_clips", "ms3.apply_whitening_matrix", "ms3.mask_out_artifacts"}
    bp = by["ms3.bandpass_filter"]
    assert bp["version"] == "0.20"
    params = {p["name"]: p for p in bp["parameters"]}
    assert [n for n in params if not params[n]["optional"]] == ["samplerate", "freq_min", "freq_max"]
    assert params["freq_wid"]["default_value"] == 1000
    assert params["quantization_unit"]["default_value"] == 0
    assert params["subsample_factor"]["default_value"] == 1
    assert bp["inputs"][0]["name"] == "timeseries" and bp["outputs"][0]["name"] == "timeseries_out"
    assert bp["exe_command"].endswith("ms3.bandpass_filter $(arguments)")
    assert bp["requirements_command"].endswith("requirements ms3.bandpass_filter $(arguments)")
    assert by["ms3.whiten"]["version"] == "0.1"


def test_spec_of_the_whitening_matrix_processors():
    # mountainsort3_main.cpp:166-189: versions, inputs/outputs, no requirements command
    by = {p["name"]: p for p in json.loads(run("spec").stdout)["processors"]}
    cw = by["ms3.compute_whitening_matrix"]
    assert cw["version"] == "0.11"
    assert [i["name"] for i in cw["inputs"]] == ["timeseries_list"]
    assert [o["name"] for o in cw["outputs"]] == ["whitening_matrix_out"]
    assert cw["parameters"] == [{"description": "", "name": "channels", "optional": True}]
    wc = by["ms3.whiten_clips"]
    assert wc["version"] == "0.1" and [i["name"] for i in wc["inputs"]] == ["clips", "whitening_matrix"]
    aw = by["ms3.apply_whitening_matrix"]
    assert aw["version"] == "0.1" and [i["name"] for i in aw["inputs"]] == ["timeseries", "whitening_matrix"]
    for p in (cw, wc, aw):
        assert "requirements_command" not in p
    for p in (wc, aw):
        assert p["parameters"][0]["name"] == "quantization_unit" and p["parameters"][0]["default_value"] == 0


def test_timeseries_list_collects_repeated_arguments(tmp_path):
    # a repeated name is a list (clparams.cpp:55-68); recordings must agree in M
    a, b = str(tmp_path / "a.mda"), str(tmp_path / "b.mda")
    mdaio.writemda(np.zeros((4, 50), np.float32), a)
    mdaio.writemda(np.zeros((5, 50), np.float32), b)
    out = str(tmp_path / "w.mda")
    r = run("ms3.compute_whitening_matrix", f"--timeseries_list={a}", f"--timeseries_list={b}",
            f"--whitening_matrix_out={out}")
    assert r.returncode == 255 and "channel count" in r.stderr and not os.path.exists(out)
    # channel numbers are 1-based; 0 (or a non-number) is rejected before any device work
    r = run("ms3.compute_whitening_matrix", f"--timeseries_list={a}", "--channels=1,0",
            f"--whitening_matrix_out={out}")
    assert r.returncode == 255 and "outside 1..4" in r.stderr and not os.path.exists(out)


def test_spec_single_and_unknown():
    r = run("spec", "ms3.whiten")
    assert r.returncode == 0 and json.loads(r.stdout)["name"] == "ms3.whiten"
    r = run("spec", "ms3.nope")
    assert r.returncode == 255 and r.stdout.strip() == "{}"
    assert run("ms3.nope").returncode == 255


def test_requirements(tmp_path, ref32):
    p = str(tmp_path / "raw.mda")
    mdaio.writemda(np.zeros((32, 100), np.float32), p)
    r = run("requirements", "ms3.bandpass_filter", f"--timeseries={p}", "--timeseries_out=x.mda",
            "--samplerate=30000", "--freq_min=300", "--freq_max=6000", "--_request_num_threads=16")
    assert r.returncode == 0, r.stderr
    assert json.loads(r.stdout)["peak_ram_mb"] == pytest.approx(ref32.lib().ref32_bandpass_peak_ram_mb(32, 16))
    # without _request_num_threads, T comes from OMP_NUM_THREADS like omp_get_max_threads()
    r = run("requirements", "ms3.bandpass_filter", "--timeseries", p, "--samplerate", "30000", "--freq_min=300",
            "--freq_max=6000", env={"OMP_NUM_THREADS": "4"})
    assert json.loads(r.stdout)["peak_ram_mb"] == pytest.approx(ref32.lib().ref32_bandpass_peak_ram_mb(32, 4))
    r = run("requirements", "ms3.whiten", f"--timeseries={p}", "--timeseries_out=y.mda")
    assert json.loads(r.stdout)["peak_ram_mb"] == pytest.approx(ref32.lib().ref32_whiten_peak_ram_mb(32))


def test_missing_or_corrupt_input_fails_without_output(tmp_path):
    out = str(tmp_path / "o.mda")
    r = run("ms3.whiten", f"--timeseries={tmp_path / 'missing.mda'}", f"--timeseries_out={out}")
    assert r.returncode == 255 and not os.path.exists(out)
    bad = tmp_path / "bad.mda"
    bad.write_bytes(b"\x00\x01")
    r = run("ms3.bandpass_filter", f"--timeseries={bad}", f"--timeseries_out={out}", "--samplerate=30000",
            "--freq_min=300", "--freq_max=6000")
    assert r.returncode == 255 and not os.path.exists(out)
    d = tmp_path / "dir_input"
    d.mkdir()
    r = run("ms3.whiten", f"--timeseries={d}", f"--timeseries_out={out}")
    assert r.returncode == 255 and "directory" in r.stderr


def test_freq_max_zero_copies_file(tmp_path):
    src = str(tmp_path / "raw.mda")
    mdaio.writemda(np.arange(12, dtype=np.float32).reshape(3, 4), src)
    out = str(tmp_path / "o.mda")
    r = run("ms3.bandpass_filter", f"--timeseries={src}", f"--timeseries_out={out}", "--samplerate=30000",
            "--freq_min=300", "--freq_max=0")
    assert r.returncode == 0
    assert open(out, "rb").read() == open(src, "rb").read()
    # QFile::copy semantics: an existing destination is not overwritten
    r = run("ms3.bandpass_filter", f"--timeseries={src}", f"--timeseries_out={out}", "--freq_max=0")
    assert r.returncode == 255


def test_directory_input_is_concatenated_like_diskreadmda32(tmp_path, ref32):
    # mda/diskreadmda32.cpp:283-288, 896-913: the directory's .mda files sorted by
    # name; subdirectories are looked up as <dir>/dirname (kept as the reference has it)
    d = tmp_path / "rec"
    d.mkdir()
    mdaio.writemda(np.zeros((4, 30), np.float32), str(d / "b.mda"))
    mdaio.writemda(np.zeros((4, 20), np.float32), str(d / "a.mda"))
    (d / "notes.txt").write_text("not an mda")
    sub = d / "sub"
    sub.mkdir()
    mdaio.writemda(np.zeros((5, 10), np.float32), str(sub / "c.mda"))  # skipped: not <dir>/dirname
    r = run("requirements", "ms3.whiten", f"--timeseries={d}", "--timeseries_out=o.mda")
    assert r.returncode == 0, r.stderr
    assert json.loads(r.stdout)["peak_ram_mb"] == pytest.approx(ref32.lib().ref32_whiten_peak_ram_mb(4))
    # a subdirectory literally named "dirname" is read, once per subdirectory
    dn = d / "dirname"
    dn.mkdir()
    mdaio.writemda(np.zeros((6, 10), np.float32), str(dn / "x.mda"))
    r = run("requirements", "ms3.whiten", f"--timeseries={d}", "--timeseries_out=o.mda")
    assert r.returncode == 255 and "differ in channel count" in r.stderr
    # freq_max = 0 copies with QFile::copy, which cannot copy a directory
    out = str(tmp_path / "copy.mda")
    r = run("ms3.bandpass_filter", f"--timeseries={d}", f"--timeseries_out={out}", "--samplerate=30000",
            "--freq_min=300", "--freq_max=0")
    assert r.returncode == 255 and not os.path.exists(out)


def test_mask_out_artifacts_spec_and_parameter_check(tmp_path):
    # mountainsort3_main.cpp:343-350; zero threshold / interval refused (p_mask_out_artifacts.cpp:26-29)
    ma = {p["name"]: p for p in json.loads(run("spec").stdout)["processors"]}["ms3.mask_out_artifacts"]
    assert ma["version"] == "0.1" and "requirements_command" not in ma
    params = {p["name"]: p for p in ma["parameters"]}
    assert params["threshold"]["default_value"] == 6 and params["interval_size"]["default_value"] == 2000
    p = str(tmp_path / "x.mda")
    mdaio.writemda(np.zeros((4, 100), np.float32), p)
    out = str(tmp_path / "o.mda")
    r = run("ms3.mask_out_artifacts", f"--timeseries={p}", f"--timeseries_out={out}", "--threshold=0")
    assert r.returncode == 255 and "zero" in r.stdout and not os.path.exists(out)


def test_python_processor_mirror_matches_the_executable_spec(tmp_path):
    # processors.py mirrors every processor of ms3gpu.mp with the same
    # version, inputs, outputs and parameter defaults
    from mountainsort_b200 import processors

    exe = {p["name"]: p for p in json.loads(run("spec").stdout)["processors"]}
    assert set(processors.SPEC) == set(exe) == set(processors.PROCESSORS)
    for name, spec in processors.SPEC.items():
        e = exe[name]
        assert spec["version"] == e["version"], name
        assert spec["inputs"] == [i["name"] for i in e["inputs"]], name
        assert spec["outputs"] == [o["name"] for o in e["outputs"]], name
        for pname, optional, default in spec["parameters"]:
            ep = {p["name"]: p for p in e["parameters"]}[pname]
            assert ep["optional"] == optional, (name, pname)
            if default is not None:
                assert ep["default_value"] == default, (name, pname)
    # zero threshold / interval are refused before any file is touched
    out = str(tmp_path / "o.mda")
    assert processors.run("ms3.mask_out_artifacts", timeseries="missing.mda", timeseries_out=out, threshold=0) is False
    assert not os.path.exists(out)
