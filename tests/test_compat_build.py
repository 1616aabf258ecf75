"""The reference's application sources compile unchanged against the drop-in
header gswitch_b200/compat/gswitch.h (where the reference tree is mounted);
the GPU side of the same binaries is tests/test_gpu_compat.py."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from gswitch_b200.compat import reference_tree

REF_APPS = os.path.join(reference_tree(), "application")


@pytest.mark.skipif(not os.path.isdir(REF_APPS), reason="reference tree not mounted")
@pytest.mark.parametrize("app", ["bfs", "cc"])
def test_reference_app_compiles_unchanged(app):
    from gswitch_b200.compat.build_apps import FLAGS, NVCC

    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, app)
        r = subprocess.run([NVCC, *FLAGS, "-o", exe, os.path.join(REF_APPS, app + ".cu")], capture_output=True,
                           text=True)
        assert r.returncode == 0, r.stderr[-2000:]
        assert os.path.getsize(exe) > 0
