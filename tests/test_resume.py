"""The step log behind --resume / --stop-after of the two front ends
(hpm_mvs and hpm_mvs.py), without a GPU: a run stopped before its first step
writes the log's settings line; resuming with the same settings keeps the
logged steps, with other settings fails, and a fresh run starts an empty
log.  Both front ends write the same log."""
import os
import subprocess
import sys

import pytest

from conftest import PKG

import hpm_mvs
import synthetic as syn


def _folder(tmp_path, name):
    sc = syn.make_scene(3, 64, 48, 3, n_planes=3)
    f = str(tmp_path / name)
    syn.write_dense_folder(sc, f)
    return f


def test_python_progress_log(tmp_path):
    f = str(tmp_path / "d")
    os.makedirs(f)
    p = hpm_mvs.Progress(f, "seed=1", resume=False)
    p.mark("A 0")
    p.mark("A 1")
    q = hpm_mvs.Progress(f, "seed=1", resume=True)
    assert q.done("A 0") and q.done("A 1") and not q.done("G0 0")
    with pytest.raises(Exception, match="cannot resume"):
        hpm_mvs.Progress(f, "seed=2", resume=True)
    r = hpm_mvs.Progress(f, "seed=2", resume=False)
    assert not r.done("A 0")
    assert open(os.path.join(f, "HPM", "progress.txt")).read() == "settings seed=2\n"


@pytest.mark.parametrize("front_end", ["cpp", "py"])
def test_front_end_stops_before_any_work_and_refuses_other_settings(tmp_path, front_end):
    exe = [os.path.join(PKG, "hpm_mvs")] if front_end == "cpp" else [sys.executable, os.path.join(PKG, "hpm_mvs.py")]
    if front_end == "cpp" and not os.path.exists(exe[0]):
        pytest.skip("make -C hpm-mvs_b200 builds hpm_mvs")
    f = _folder(tmp_path, front_end)
    r = subprocess.run(exe + [f, "--seed", "4", "--per-problem", "--stop-after", "0"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and "Stopped after 0 steps" in r.stdout, r.stdout + r.stderr
    log = open(os.path.join(f, "HPM", "progress.txt")).read()
    assert log == "settings seed=4 levels=-1 prior=1 geom_iterations=2 form=per-problem\n"
    r = subprocess.run(exe + [f, "--seed", "5", "--per-problem", "--resume", "--stop-after", "0"], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode != 0 and "cannot resume" in (r.stdout + r.stderr)
    r = subprocess.run(exe + [f, "--seed", "4", "--per-problem", "--resume", "--stop-after", "0"], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0 and open(os.path.join(f, "HPM", "progress.txt")).read() == log


@pytest.mark.parametrize("front_end", ["cpp", "py"])
@pytest.mark.parametrize("fault", ["missing camera", "truncated camera", "truncated pair"])
def test_front_end_reports_a_broken_dense_folder(tmp_path, front_end, fault):
    """A missing or truncated input file ends the run with status 1 and a
    message naming the file (the reference prints and carries on, or
    dereferences NULL: HPM.cpp:273-304); the cameras are read before any
    device work, so this runs without a GPU."""
    exe = [os.path.join(PKG, "hpm_mvs")] if front_end == "cpp" else [sys.executable, os.path.join(PKG, "hpm_mvs.py")]
    if front_end == "cpp" and not os.path.exists(exe[0]):
        pytest.skip("make -C hpm-mvs_b200 builds hpm_mvs")
    f = _folder(tmp_path, front_end)
    cam = os.path.join(f, "cams", "00000001_cam.txt")
    if fault == "missing camera":
        os.remove(cam)
        name = "00000001_cam.txt"
    elif fault == "truncated camera":
        with open(cam) as fh:
            text = fh.read()
        with open(cam, "w") as fh:
            fh.write(text[: len(text) // 3])
        name = "00000001_cam.txt"
    else:
        with open(os.path.join(f, "pair.txt"), "w") as fh:
            fh.write("3\n0\n2 1")
        name = "pair.txt"
    r = subprocess.run(exe + [f, "--no-fusion"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1, (r.returncode, r.stdout[-1000:], r.stderr[-1000:])
    assert name in r.stderr, r.stderr[-1000:]
