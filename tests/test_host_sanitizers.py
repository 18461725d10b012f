"""The host-side C/C++ (set-up library, dump/restart IO, CPU oracle) built with
AddressSanitizer and UndefinedBehaviorSanitizer and driven through the calls
the binding makes: a rotating MHD and a hydro case, three oracle steps,
FLUXES, the CFL reduction, the profiles, BCON, and a dump written and read
back (tests/sanitize/host_driver.cpp)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_host_code_under_asan_and_ubsan(tmp_path):
    if not shutil.which("g++") or not shutil.which("gcc"):
        pytest.skip("no host compiler")
    san = ["-fsanitize=address,undefined", "-fno-sanitize-recover=undefined", "-fno-omit-frame-pointer", "-g", "-O1"]
    inc = ["-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "oracle")]
    obj = str(tmp_path / "oracle.o")
    subprocess.run(["gcc", "-std=c11", "-ffp-contract=off", *san, *inc, "-c", "-o", obj,
                    os.path.join(ROOT, "oracle", "oracle3dmhd.c")], check=True)
    exe = str(tmp_path / "host_driver")
    subprocess.run(["g++", "-std=c++17", "-ffp-contract=off", *san, *inc, "-o", exe,
                    os.path.join(ROOT, "tests", "sanitize", "host_driver.cpp"),
                    os.path.join(ROOT, "rast-3dmhd_b200", "host", "host3dmhd.cpp"),
                    os.path.join(ROOT, "rast-3dmhd_b200", "host", "dumpio.cpp"), obj, "-lm"], check=True)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0", UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "host driver ok" in r.stdout
    assert "runtime error" not in r.stderr, r.stderr
