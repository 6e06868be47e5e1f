"""The host C library (kd_api.c) under sanitizers, on the CPU.

tests/host/fake_device.c stands in for the device layer (an exhaustive CPU
count over the stored points); tests/host/api_driver.c drives the real C
ABI: counts against an independent brute force, eight threads building,
counting and destroying trees at once and three callers of the threaded
RA/DEC conversion under ThreadSanitizer, and argument
errors, injected device-layer failures, every allocation failing in turn and
4,000 calls with random (valid and invalid) arguments under AddressSanitizer +
UndefinedBehaviorSanitizer (leaks included)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SRC = os.path.join(HERE, "host")


def _build(tmp_path, sanitize, tag):
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    inc = ["-I" + os.path.join(REPO, "include"), "-I" + os.path.join(REPO, "corruscant_b200", "csrc")]
    flags = ["-g", "-O1", "-fno-omit-frame-pointer", "-fsanitize=" + sanitize]
    obj = str(tmp_path / f"api_{tag}.o")
    exe = str(tmp_path / f"driver_{tag}")
    cmds = [
        ["gcc", *flags, *inc, "-include", os.path.join(SRC, "fake_alloc.h"), "-c",
         os.path.join(REPO, "corruscant_b200", "csrc", "kd_api.c"), "-o", obj],
        ["gcc", *flags, *inc, os.path.join(SRC, "fake_device.c"), os.path.join(SRC, "api_driver.c"),
         os.path.join(REPO, "corruscant_b200", "csrc", "coords_api.c"), obj, "-o", exe,
         "-lpthread", "-lm"],
    ]
    for c in cmds:
        r = subprocess.run(c, capture_output=True, text=True)
        if r.returncode != 0:
            if "sanitize" in r.stderr or "tsan" in r.stderr or "asan" in r.stderr:
                pytest.skip(f"{sanitize} sanitizer not usable: {r.stderr[-300:]}")
            raise AssertionError(r.stderr)
    return exe


def _run(exe, *scenarios, env=None):
    r = subprocess.run([exe, *scenarios], capture_output=True, text=True, timeout=300,
                       env={**os.environ, **(env or {})})
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "0 failures" in r.stdout, r.stdout
    return r.stdout


def test_host_library_under_thread_sanitizer(tmp_path):
    exe = _build(tmp_path, "thread", "tsan")
    out = _run(exe, "threads", "count", "coords", env={"TSAN_OPTIONS": "halt_on_error=1"})
    assert "PASS threads" in out and "PASS count" in out and "PASS coords" in out


def test_host_library_under_address_sanitizer(tmp_path):
    exe = _build(tmp_path, "address,undefined", "asan")
    out = _run(exe, "count", "faults", "fuzz",
               env={"ASAN_OPTIONS": "detect_leaks=1:halt_on_error=1",
                    "UBSAN_OPTIONS": "halt_on_error=1:print_stacktrace=1"})
    assert "PASS count" in out and "PASS faults" in out and "PASS fuzz" in out
