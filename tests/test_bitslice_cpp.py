"""The coefficient records of the multiply-accumulate kernel, both table
forms (8 + 8 planes and the small-output 6 + 5 + 5), checked on the host by
tests/cpp/test_bitslice.cpp: tables built from random symbols' bit planes,
the record's rows followed in the kernel's lookup order, the result compared
with c * symbol in GF(2^16)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "cpp", "_build", "test_bitslice")


def test_records_reproduce_gf_multiplication():
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "cpp")], check=True)
    r = subprocess.run([BIN], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok 8000")
