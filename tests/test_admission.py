"""The server's memory-budget admission policy (csrc/admission.h), host logic
only: built with g++ and run on the CPU."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "turbo-octo-spice_b200", "csrc")


def test_admission_policy(tmp_path):
    exe = str(tmp_path / "admission_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", f"-I{CSRC}",
                    os.path.join(HERE, "serving", "admission_test.cc"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert "admission: ok" in out.stdout
