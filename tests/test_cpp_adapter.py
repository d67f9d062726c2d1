"""The C++ host adapter (include/theseus_b200/RHSOperator.hpp) compiles against
the C ABI, links the library, fails loudly without a GPU, and on a GPU gives
the oracle's right-hand side.  Its MFEM front end (MFEMRHSOperator, an
mfem::TimeDependentOperator) compiles against a test-only MFEM stand-in
(tests/cpp/mfem_stub) and, driven by that stand-in's SSP-RK3 solver, gives
the oracle's trajectory."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O
import theseus_b200 as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build(tmp, name="adapter_rhs", extra=()):
    exe = os.path.join(tmp, name)
    cuda = "/usr/local/cuda"
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
                           *extra, "-I", f"{cuda}/include", os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
                           "-L", os.path.join(ROOT, "theseus_b200"), "-ltheseus_b200",
                           f"-Wl,-rpath,{os.path.join(ROOT, 'theseus_b200')}",
                           "-L", f"{cuda}/lib64", "-lcudart", f"-Wl,-rpath,{cuda}/lib64", "-o", exe])
    return exe


def test_cpp_adapter_builds_and_refuses_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present; covered by the gpu test")
    with tempfile.TemporaryDirectory() as d:
        exe = build(d)
        r = subprocess.run([exe, os.path.join(d, "out.bin")], capture_output=True, text=True)
        assert r.returncode == 3 and "no CUDA device" in r.stderr


@pytest.mark.gpu
def test_cpp_adapter_matches_oracle(cuda):
    with tempfile.TemporaryDirectory() as d:
        exe = build(d)
        out = os.path.join(d, "out.bin")
        r = subprocess.run([exe, out], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        data = np.fromfile(out, dtype=np.float64)
    m = T.periodic_box(3, 4, (3, 3, 3), [0.0] * 3, [2 * np.pi] * 3)
    u, du = data[: data.size // 2].reshape(m.state_shape()), data[data.size // 2:].reshape(m.state_shape())
    om = O.Mesh(m.dim, m.order, m.jac, m.metric, m.face_elem, m.face_lface, m.face_normal,
                m.face_wminus, m.face_wplus)
    cfg = T.make_config(flow="ns", volume_flux="ranocha", surface_flux="hll", mu=1.0 / 1600, Pr=0.71)
    ref = O.rhs(om, cfg, u, nthreads=4)
    err = np.sqrt(((du - ref) ** 2).sum(axis=(1, 2)) / (ref ** 2).sum(axis=(1, 2)))
    assert err.max() <= 1e-12


MFEM_STUB = ("-I", os.path.join(ROOT, "tests", "cpp", "mfem_stub"))


def test_mfem_adapter_builds_and_refuses_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present; covered by the gpu test")
    with tempfile.TemporaryDirectory() as d:
        exe = build(d, "mfem_adapter", MFEM_STUB)
        r = subprocess.run([exe, os.path.join(d, "out.bin")], capture_output=True, text=True)
        assert r.returncode == 3 and "no CUDA device" in r.stderr


@pytest.mark.gpu
def test_mfem_adapter_rk3_matches_oracle(cuda):
    """Two SSP-RK3 steps of dt = 1e-3 through MFEMRHSOperator::Mult, driven by
    the stand-in RK3SSPSolver, against the oracle's SSP-RK3 (1e-12), and the
    stability rates of the initial state against the oracle's (1e-13)."""
    with tempfile.TemporaryDirectory() as d:
        exe = build(d, "mfem_adapter", MFEM_STUB)
        out = os.path.join(d, "out.bin")
        r = subprocess.run([exe, out], capture_output=True, text=True)
        assert r.returncode == 0, (r.returncode, r.stderr)
        data = np.fromfile(out, dtype=np.float64)
    m = T.periodic_box(3, 4, (3, 3, 3), [0.0] * 3, [2 * np.pi] * 3)
    n = 5 * m.num_nodes
    u0, u1, rates = data[:n].reshape(m.state_shape()), data[n:2 * n].reshape(m.state_shape()), data[2 * n:]
    om = O.Mesh(m.dim, m.order, m.jac, m.metric, m.face_elem, m.face_lface, m.face_normal,
                m.face_wminus, m.face_wplus)
    cfg = T.make_config(flow="ns", volume_flux="ranocha", surface_flux="hll", mu=1.0 / 1600, Pr=0.71)
    ref = O.rk3_steps(om, cfg, u0, 1e-3, 2, nthreads=4)
    err = np.sqrt(((u1 - ref) ** 2).sum(axis=(1, 2)) / (ref ** 2).sum(axis=(1, 2)))
    assert err.max() <= 1e-12, err
    _, ref_rates = O.estimate_dt(om, cfg, u0, 1.0)
    assert np.allclose(rates, ref_rates, rtol=1e-13, atol=0.0), (rates, ref_rates)
