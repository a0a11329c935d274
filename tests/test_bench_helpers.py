"""Host-side helpers of the bench and the training script, without a GPU:
the prior-net schedule syntax and the workload names of the bench
configurations."""
import os
import subprocess
import sys

import pytest

from conftest import PKG, ROOT

sys.path.insert(0, PKG)
import priornet  # noqa: E402


@pytest.mark.parametrize("text,want", [("0:2", (0, 2, 1, 3, 3)), ("1:1:2", (1, 1, 2, 3, 3)),
                                       ("0:2:2:2", (0, 2, 2, 2, 2)), ("0:2:2:3:1", (0, 2, 2, 3, 1))])
def test_schedule_syntax(text, want):
    assert priornet.parse_schedule(text) == want


@pytest.mark.parametrize("text", ["0", "0:1:2:3:4:5", "a:b"])
def test_schedule_syntax_errors(text):
    with pytest.raises(ValueError):
        priornet.parse_schedule(text)


@pytest.mark.parametrize("config,parts", [
    ("plain-hpm", ["11 views of 1600x1200", "10 sources", "3-level pyramid"]),
    ("stress", ["20 views of 3200x2133", "10 sources", "3-level pyramid"]),
    ("batched", ["24 views (8 of 1920x1080, 8 of 1600x1200, 8 of 960x540)", "10 sources",
                 "the reference's rule per view size"]),
])
def test_workload_names(config, parts):
    code = ("import sys; sys.argv = ['bench.py', '--config', %r]; import bench; bench.parse_args(); "
            "print(bench.workload_name())" % config)
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    for p in parts:
        assert p in out.stdout, out.stdout
