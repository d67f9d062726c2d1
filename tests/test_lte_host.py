"""CPU: the library's LTE Helmholtz arithmetic, compiled for the host from the
same header the kernels use, equals the oracle bit for bit (temperature
recovery, LTEEC volume and face fluxes on 20,000 seeded pairs)."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_lte_device_math_equals_oracle_on_host():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "lte_host_check")
        subprocess.check_call(
            ["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2", "-Xcompiler", "-ffp-contract=off",
             "-I", os.path.join(ROOT, "theseus_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
             "-I", os.path.join(ROOT, "oracle"), "-x", "cu",
             os.path.join(ROOT, "tests", "cpp", "lte_host_check.cu"),
             os.path.join(ROOT, "theseus_b200", "csrc", "thx_lte_host.cpp"), "-o", exe],
            stderr=subprocess.DEVNULL)
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout
