"""The ring protocol of the overflow queue and the recycled-id pool, on the CPU.

tests/ring_model.cpp replays the protocol (reservation by an add on the
producer cursor, lap-tagged slot writes, consumers that poll their slot's tag,
launch resets that move the consumer cursor to the producer cursor) with the
encoding functions the device compiles (gtap_b200/csrc/gtap_ring.h).  It covers
fresh rings, stale laps, the 2^32 wrap of the cursors, a slot left over from
65,536 launches earlier (where the former 16-bit launch epoch repeated) and
randomised interleavings with aborted launches.
"""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_ring_protocol_model(tmp_path):
    exe = tmp_path / "ring_model"
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Werror", "-o", str(exe),
                    os.path.join(ROOT, "tests", "ring_model.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-4000:]
    assert "all checks passed" in out.stdout
