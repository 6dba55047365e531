"""The host entropy stage (riv2_b200/csrc/riv_entropy.cpp) built with the compiler's
sanitizers and driven by tests/host_sanitize_driver.cpp on CPU: AddressSanitizer with
UndefinedBehaviorSanitizer (out-of-bounds accesses, use after free, bad shifts) and
ThreadSanitizer (data races in the pooled, parallel and handed-off coefficient coders, and in
the MV coder's pipeline: symbol listing and modelling of consecutive frames on two threads at
once, every rANS batch on a pool, as the encoder runs them).  The oracle, the
checker of every parity test, runs small clips under AddressSanitizer and
UndefinedBehaviorSanitizer too (tests/oracle_sanitize_driver.cpp).  The device code cannot run
under a sanitizer here; its kernels bound their own indexes and waits."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "riv2_b200", "csrc")
DRIVER = os.path.join(ROOT, "tests", "host_sanitize_driver.cpp")
ORACLE = os.path.join(ROOT, "oracle")


@pytest.mark.parametrize("sanitizers", ["address,undefined", "thread"])
def test_host_entropy_under_sanitizers(sanitizers, tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "driver")
    cmd = [gxx, "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-fwrapv", f"-fsanitize={sanitizers}",
           "-fno-sanitize-recover=all", "-I", CSRC, DRIVER, os.path.join(CSRC, "riv_entropy.cpp"), "-o", exe,
           "-lpthread"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=1", UBSAN_OPTIONS="print_stacktrace=1",
               TSAN_OPTIONS="halt_on_error=1")
    r = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-4000:]
    assert "ok" in r.stdout


def test_oracle_under_address_and_undefined_sanitizers(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "oracle_driver")
    cmd = [gxx, "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-fwrapv", "-ffp-contract=off",
           "-fno-fast-math", "-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-I", ORACLE,
           os.path.join(ROOT, "tests", "oracle_sanitize_driver.cpp"), os.path.join(ORACLE, "riv_oracle.cpp"), "-o", exe,
           "-lm"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=1", UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-4000:]
    assert "ok" in r.stdout
