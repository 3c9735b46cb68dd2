"""The drop-in, compiled and run: the reference's own matchSeries program
(match-series_b200/adapter: the reference's matchSeries<>() driver and
SeriesMatching built from its sources) run from a parameter file, once with
the reference's CPU registration (deformationModel 22) and once with the GPU
registration plugged into the same RegistrationType slot (deformationModel
23).  With the reference's sum order the level solves are the reference's bit
for bit, so every file the series matching writes -- the displacements of
every template and level, the accumulated and refined ones, the per-level
energy logs, the energies, the deformation norms and the average -- is
byte-identical between the two runs.
(The reference without libpng stops with its PNG exception after writing the
average; both runs stop at the same point.)"""
import filecmp
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "match-series_b200", "adapter", "_build", "match_series_gpu")

PARAMS = """templateNamePattern {frames}/frame_%02d.dat.bz2
templateNumOffset 0
templateNumStep 1
numTemplates {F}
numExtraStages 0
extraStagesLambdaFactor 0.1
saveDirectory {out}/
dontNormalizeInputImages 0
enhanceContrastSaturationPercentage 0.15
normalizeMinToZero 1
lambda 0.1
lambdaFactor 1
maxGDIterations {iters}
stopEpsilon 0
startLevel {start}
stopLevel {level}
precisionLevel {level}
refineStartLevel {refine}
refineStopLevel {level}
checkboxWidth 8
onlySaveDisplacement 1
deformationModel {model}
"""


def _run(tmp, model, frames_dir, F, level, iters):
    out = os.path.join(tmp, f"out{model}")
    par = os.path.join(tmp, f"p{model}.par")
    with open(par, "w") as f:
        f.write(PARAMS.format(frames=frames_dir, F=F, out=out, iters=iters, start=level - 3, level=level,
                              refine=level - 1, model=model))
    r = subprocess.run([BIN, par], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return out, r.stdout + r.stderr


def _files(root):
    got = []
    for d, _, fs in os.walk(root):
        for f in fs:
            got.append(os.path.relpath(os.path.join(d, f), root))
    return sorted(got)


@pytest.mark.parametrize("level,F,seed", [(6, 4, 6601), (7, 5, 6602)])
def test_reference_program_with_gpu_registration_writes_the_reference_files(tmp_path, level, F, seed):
    import msgpu
    from msgpu import synthetic as syn
    assert os.path.exists(BIN), "match_series_gpu is not built (make -f match-series_b200/adapter/Makefile REF=...)"
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, F, syn.SQUARE_257, seed=seed)
    frames_dir = os.path.join(str(tmp_path), "frames")
    os.makedirs(frames_dir)
    for i in range(F):
        msgpu.write_array(os.path.join(frames_dir, f"frame_{i:02d}.dat.bz2"), fr[i], 9)
    ref_out, ref_log = _run(str(tmp_path), 22, frames_dir, F, level, 15)
    gpu_out, gpu_log = _run(str(tmp_path), 23, frames_dir, F, level, 15)
    # every result file of the series matching, the per-level energy logs
    # included, exists in both runs (the logs of the program differ: paths)
    skip = ("log.txt", "parameter-dump.txt")
    ref_files = [f for f in _files(ref_out) if os.path.basename(f) not in skip]
    gpu_files = [f for f in _files(gpu_out) if os.path.basename(f) not in skip]
    assert ref_files == gpu_files, (ref_files, gpu_files)
    defs = [f for f in ref_files if os.path.basename(f).startswith("deformation_")]
    assert len(defs) >= 2 * 3 * (F - 1)   # per template: 3 levels, 2 components
    assert "stage1/average.q2bz" in ref_files and "stage1/energies.txt" in ref_files
    assert any(os.path.basename(f).startswith("energy_") for f in ref_files)
    for f in ref_files:
        a, b = os.path.join(ref_out, f), os.path.join(gpu_out, f)
        if not filecmp.cmp(a, b, shallow=False):
            if f.endswith(".txt"):
                import difflib
                diff = "".join(list(difflib.unified_diff(open(a).readlines(), open(b).readlines()))[:20])
            else:
                diff = ""
            raise AssertionError(f"{f} differs\n{diff}")
    # the displacements are not trivial
    phi = msgpu.read_displacement(os.path.join(gpu_out, "stage1", "1", f"deformation_{level:02d}_%d.dat.bz2"), n)
    assert np.abs(phi).max() * (n - 1) > 0.05
