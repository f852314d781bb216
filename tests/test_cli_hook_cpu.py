"""The CLI edits of the integration notes, applied to the reference's own fastcw.py.

Runs where the reference's modules are available: FCW_REFERENCE_DIR names the folder that
holds them (skipped otherwise). The test copies fastcw.py to a temporary folder, applies
the three edits the integration notes give (fastcw.py:466-472 choices, :489 metavar,
:644-649 the diffusion length for both heat engines), and checks that the parser lists and
accepts `--engine b200` and still rejects an unknown engine, as
test_engine_cli_parsing.py checks the stock choices. The reference's sources stay outside the
repository: the patched copy lives only in the test's temporary folder."""
import os
import shutil
import subprocess
import sys

import pytest

REF = os.environ.get("FCW_REFERENCE_DIR", "")
pytestmark = pytest.mark.skipif(not os.path.isfile(os.path.join(REF, "fastcw.py")),
                                reason="FCW_REFERENCE_DIR does not name the reference's modules")

EDITS = [
    ('valid = {"potpourri", "potpourri_fmm", "pycortex", "pygeodesic"}',
     'valid = {"potpourri", "potpourri_fmm", "pycortex", "pygeodesic", "b200"}'),
    ('visible = "potpourri, potpourri_fmm, pycortex, pygeodesic"',
     'visible = "potpourri, potpourri_fmm, pycortex, pygeodesic, b200"'),
    ('metavar="{potpourri,potpourri_fmm,pycortex,pygeodesic}"',
     'metavar="{potpourri,potpourri_fmm,pycortex,pygeodesic,b200}"'),
    ('if args.engine == "potpourri":\n        if ("diffusion_length_mm" in engine_kwargs',
     'if args.engine in ("potpourri", "b200"):\n        if ("diffusion_length_mm" in engine_kwargs'),
]


def _patched(tmp_path):
    src = open(os.path.join(REF, "fastcw.py")).read()
    for old, new in EDITS:
        assert src.count(old) == 1, f"the edit target moved: {old[:50]}"
        src = src.replace(old, new)
    path = tmp_path / "fastcw.py"
    path.write_text(src)
    return str(path)


def _run(script, *args):
    env = dict(os.environ, PYTHONPATH=REF + os.pathsep + os.environ.get("PYTHONPATH", ""))
    return subprocess.run([sys.executable, script, *args], capture_output=True, text=True, env=env, timeout=300)


def test_patched_cli_lists_and_accepts_b200(tmp_path):
    script = _patched(tmp_path)
    proc = _run(script, "--help")
    assert proc.returncode == 0, proc.stderr
    text = proc.stdout + proc.stderr
    assert "--engine {potpourri,potpourri_fmm,pycortex,pygeodesic,b200}" in text
    assert _run(script, "--engine", "b200", "--help").returncode == 0
    bad = _run(script, "--engine", "batch_heat", "--output-label", "x", "subjects_dir", "subject_id")
    assert bad.returncode != 0 and "invalid choice" in bad.stdout + bad.stderr
