"""The GPU replays the reference's std::priority_queue on ties with the
functions of falconnpp_b200/csrc/fpp_heap.h; compile that header for the host
and check it against libstdc++'s own priority_queue, operation by operation,
on tie-heavy random sequences (push, pop, bounded top-p offers, full drains)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_heap_emulation_matches_libstdcxx(tmp_path):
    exe = tmp_path / "heap_check"
    src = os.path.join(ROOT, "tests", "native", "heap_check.cpp")
    inc = os.path.join(ROOT, "falconnpp_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{inc}", src, "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok")
