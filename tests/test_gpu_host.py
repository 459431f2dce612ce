"""The bgk_thermal host program (STEP_7/main.f90 on top of the C ABI)
against the oracle's STEP_7 program: same input.dat, same output files.
Both use the portable tanh, so every field is bit-identical and the printed
values agree exactly, except field_check's means, whose device reduction
adds in a different order (compared to 1e-7 relative, below the 8 printed
digits)."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, small_params

pytestmark = pytest.mark.gpu

NUM = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[EeDd][-+]?\d+|[-+]\d{3})?")


def numbers(path: Path) -> np.ndarray:
    out = []
    for tok in NUM.findall(path.read_text()):
        t = tok.replace("D", "E").replace("d", "e")
        m = re.fullmatch(r"([-+]?\d*\.\d*)([-+]\d{3})", t)
        if m:
            t = m.group(1) + "E" + m.group(2)
        out.append(float(t))
    return np.array(out)


@pytest.fixture(scope="module")
def runs(tmp_path_factory, oracle_mod, lib):
    from bgk_pcm_b200 import build, inputs
    build.build()
    p = small_params(64, 48)
    p.update(iter=3000, noutput=3)
    dirs = {}
    for who in ("oracle", "gpu"):
        d = tmp_path_factory.mktemp(who)
        inputs.write(d / "input.dat", p)
        dirs[who] = d
    oracle_mod.run_main(dirs["oracle"], threads=4, tanh_mode=1)
    r = subprocess.run([str(ROOT / "bgk_pcm_b200" / "bgk_thermal"), str(dirs["gpu"]), "--tanh", "portable"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "Mlups" in r.stdout
    return dirs


FILES = ["fort.666", "fort.667", "fort.668", "non-dim_bulk_numbers.dat", "fort.69", "log.dat",
         "Output_00000000.vtk", "Output_00001000.vtk", "Output_00002000.vtk", "Output_00003000.vtk"]


@pytest.mark.parametrize("name", FILES)
def test_output_file_matches(runs, name):
    a, b = runs["oracle"] / name, runs["gpu"] / name
    assert b.exists(), name
    na, nb = numbers(a), numbers(b)
    assert na.shape == nb.shape
    np.testing.assert_array_equal(nb, na)


def test_field_check_means(runs):
    na, nb = numbers(runs["oracle"] / "fort.64"), numbers(runs["gpu"] / "fort.64")
    assert na.shape == nb.shape
    np.testing.assert_allclose(nb, na, rtol=1e-7)


def test_text_restart_continues_bit_for_bit(tmp_path, lib):
    """dump_out at step 1000 (dumpFile.dat in the reference's record layout,
    phi in dumpPhi.dat), then a run with dump = 1 to step 2000, gives the same
    final VTK file as one uninterrupted run to step 2000: 17 significant
    digits carry every double exactly."""
    from bgk_pcm_b200 import inputs
    exe = str(ROOT / "bgk_pcm_b200" / "bgk_thermal")
    p = small_params(40, 30)
    full, part = tmp_path / "full", tmp_path / "part"
    full.mkdir(); part.mkdir()
    inputs.write(full / "input.dat", dict(p, iter=2000, noutput=2))
    inputs.write(part / "input.dat", dict(p, iter=1000, noutput=1))
    for d, extra in ((full, []), (part, ["--dump-out"])):
        r = subprocess.run([exe, str(d), "--tanh", "portable"] + extra, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    head = (part / "dumpFile.dat").read_text().splitlines()
    nodes = (p["Nx"] + 2) * (p["Ny"] + 2)
    assert int(head[0]) == 1000 and len(head) == 1 + 2 * nodes
    assert len(head[1].split()) == 12 and len(head[2].split()) == 10
    inputs.write(part / "input.dat", dict(p, iter=2000, noutput=2, dump=1))
    r = subprocess.run([exe, str(part), "--tanh", "portable"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert (part / "Output_00002000.vtk").read_text() == (full / "Output_00002000.vtk").read_text()
