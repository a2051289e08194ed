"""The serving and batch admission scheduler (spades-rs_b200/csrc/spk_sched.h)
on the CPU: admission by budget and slots, error messages of failed jobs, a
waiter that outlives stop() and the owner's release, and the results of
uncollected tickets freed at stop.  Built with AddressSanitizer where gcc
supports it, so a use after free fails the run."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _build(tmp_path, sanitize):
    exe = str(tmp_path / ("sched_test_asan" if sanitize else "sched_test"))
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-pthread", os.path.join(HERE, "sched_test.cpp"), "-o", exe]
    if sanitize:
        cmd[1:1] = ["-fsanitize=address", "-fno-omit-frame-pointer"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return exe if r.returncode == 0 else None


def test_scheduler(tmp_path):
    exe = _build(tmp_path, True) or _build(tmp_path, False)
    assert exe, "g++ failed to build tests/sched_test.cpp"
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=1"))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "sched ok" in r.stdout
