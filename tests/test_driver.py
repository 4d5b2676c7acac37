"""The driver program (lbm_main, main.f90's loop over the C ABI) on the CPU:
it builds with the host compiler against the library and handles its
options; running it needs a GPU (test_gpu_driver.py)."""
import subprocess

from fortran_loadfile_mitiwing_b200 import build


def test_driver_builds_and_parses_options():
    exe = build.build_driver()
    r = subprocess.run([exe, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "--restart DIR" in r.stdout
    for bad in (["--bogus", "1"], ["--nx"], ["--precision", "fp8"], ["--chunk", "1"], ["--output-window", "5:2"],
                ["--nx", "many"]):
        r = subprocess.run([exe, *bad], capture_output=True, text=True, timeout=60)
        assert r.returncode == 2 and "usage" in r.stderr, (bad, r.returncode, r.stderr)
