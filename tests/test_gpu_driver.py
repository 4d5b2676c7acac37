"""The driver program (lbm_main) on the GPU: force.dat carries the force rows
of lbm_run in format (1000f15.8), byte for byte; F<n>.dat and the restart
files appear on their steps; a run restarted from the reference-layout file
writes the remaining rows exactly as the run that never stopped; the residual
lines are those of erranalysis at the start of their steps."""
import subprocess

import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import Lbm, build, cases, io_formats

pytestmark = pytest.mark.gpu


def case_files(tmp_path, case):
    io_formats.write_boundary(tmp_path / "boundary.dat", *case.contours[0])
    io_formats.write_motion(tmp_path / "motion_params.dat", case.table)


def params_args(p):
    a = ["--nx", p.nx, "--ny", p.ny, "--wing-count", p.wing_count, "--points-per-wing", p.points_per_wing,
         "--scale", repr(p.scale), "--ox", repr(p.ox), "--oy", repr(p.oy), "--uu", repr(p.uu), "--re", repr(p.re),
         "--xc", 0, "--yc", 0, "--xp", 0, "--yp", 0, "--mesh-max-scale", repr(p.mesh_max_scale),
         "--delta", "peskin4" if p.delta_kernel == 0 else "smooth",
         "--precision", {0: "fp32", 1: "fp64", 2: "fp16", 3: "bf16"}[p.precision]]
    for k in range(9):
        a += [f"--s{k + 1}", repr(p.s[k])]
    return [str(x) for x in a]


def run_driver(tmp_path, case, out, *extra):
    out.mkdir(exist_ok=True)
    cmd = [build.build_driver(), *params_args(case.params), "--boundary-dir", str(tmp_path),
           "--motion", str(tmp_path / "motion_params.dat"), "--out", str(out), *map(str, extra)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout


def test_driver_rows_outputs_and_restart(gpu_lib, tmp_path):
    case = cases.small_case(precision="fp32", n_steps=400, amp=0.0)   # the reference's init: no perturbation
    case_files(tmp_path, case)
    out1 = tmp_path / "run1"
    log = run_driver(tmp_path, case, out1, "--steps", 250, "--chunk", 64, "--output-every", 100,
                     "--save-every", 200, "--residual-every", 100)
    ref = Lbm.from_case(case, gpu_lib)
    rows = ref.run(99)
    res99 = ref.erranalysis()                     # erranalysis at the start of step 100
    rows = np.concatenate([rows, ref.run(100)])
    res199 = ref.erranalysis()
    rows = np.concatenate([rows, ref.run(51)])
    want = "".join(io_formats.format_force_row(r) + "\n" for r in rows)
    assert (out1 / "force.dat").read_text() == want
    motion = (out1 / "airfoil_motion.dat").read_text().splitlines()
    assert len(motion) == 250 and motion[-1] == io_formats.format_force_row(
        io_formats.airfoil_motion_row(rows[-1, 0], 1))
    assert (out1 / "F100.dat").exists() and (out1 / "F200.dat").exists() and not (out1 / "F250.dat").exists()
    assert (out1 / "saved_flow_feild.dat").exists() and (out1 / "saved_flow_feild_copy.dat").exists()
    lines = [l for l in log.splitlines() if l.startswith("iteration")]
    assert lines == [f"iteration 100, residual {res99:.10e}", f"iteration 200, residual {res199:.10e}"]
    # restart from step 200: the old force.dat has 250 rows, so rows 251.. follow
    out2 = tmp_path / "run2"
    log2 = run_driver(tmp_path, case, out2, "--restart", out1, "--steps", 300, "--save-every", 0,
                      "--residual-every", 0)
    assert "restarted from step 200" in log2 and (out2 / "F200.dat").exists()
    more = ref.run(50)
    assert (out2 / "force.dat").read_text() == "".join(io_formats.format_force_row(r) + "\n" for r in more)
