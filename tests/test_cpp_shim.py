"""The C++ face of the library (include/xca_b200.hpp): it compiles against the header and links against
libxca_b200.so; without a GPU every construction throws std::runtime_error (the status mapping); on a
GPU its results agree with the oracle and failing calls throw the reference's exception types."""

import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "shim_check.cpp")


def _build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "shim_check")
    libdir = os.path.join(ROOT, "xca_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe, "-L", libdir,
                    "-l:libxca_b200.so", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def test_shim_builds_and_maps_errors_without_gpu(tmp_path):
    import torch
    exe = _build(tmp_path)
    if torch.cuda.is_available():
        pytest.skip("a GPU is present (covered by the GPU test)")
    p = subprocess.run([exe], capture_output=True, text=True)
    assert p.returncode == 3, p.stdout + p.stderr
    assert p.stdout.startswith("runtime_error:")


@pytest.mark.gpu
@pytest.mark.parametrize("pole", [0.0, 0.7])
def test_shim_vs_oracle(tmp_path, pole):
    from oracle import oracle as O
    exe = _build(tmp_path)
    p = subprocess.run([exe, repr(pole)], capture_output=True, text=True, check=True)
    lines = {ln.split()[0]: ln for ln in p.stdout.splitlines()}
    r = int(lines["rank"].split()[1])
    from xca_b200.pycppdlr import ImTimeOps, build_dlr_rf
    beta, lam, eps = 2.0, 20.0, 1e-10
    rf = build_dlr_rf(lam, eps)
    it = ImTimeOps(lam, rf).get_itnodes()
    d = O.Dlr(lam, eps, rf=rf, it=it)
    assert d.r == r
    F_index = np.array([[-1, 0]], np.int32)
    Fd_index = np.array([[1, -1]], np.int32)
    ones = np.ones((1, 1, 1), np.complex128)
    ev = O.Evaluator(d, beta, np.array([pole]), np.ones((1, 1, 1), np.complex128), np.array([1, 1]), np.array([0]),
                     F_index, [[None, ones]], Fd_index, [[ones, None]])
    G = [np.full((r, 1, 1), -0.5, np.complex128)] * 2
    for key, topo in (("sigma1", [[0, 1]]), ("sigma2", [[0, 2], [1, 3]])):
        got = np.array([float(x) for x in lines[key].split()[1:]])
        ref = np.concatenate([s.real.ravel() for s in ev.compute_self_energy(G, np.array(topo, np.int32))])
        assert np.max(np.abs(got - ref)) <= 1e-12 * max(np.max(np.abs(ref)), 1e-300)
    got = np.array([float(x) for x in lines["spgf1"].split()[1:]])
    ref = ev.compute_single_ptcle_gf(G, np.array([[0, 1]], np.int32)).real.ravel()
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert "bad topology: invalid_argument" in p.stdout
    assert "f_ix out of range: runtime_error" in p.stdout
