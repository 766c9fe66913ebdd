"""The C++ classes of include/azeban_b200.hpp, compiled with g++ and run as a
C++ caller of the library would (tests/cpp/adapter_main.cpp): the boundary a
maintainer binds azeban to.

The CPU test compiles and links the program against libazeban_b200.so; the
GPU tests run it on seeded fields and compare its dudt, dt, SSP-RK3 step and
simulate_until with the oracle (IncompressibleEuler::dudt,
include/azeban/equations/incompressible_euler.hpp:103-124; SSP_RK3::integrate,
include/azeban/evolution/ssp_rk3.hpp:48-64; Simulation::simulate_until,
src/azeban/simulation.cpp:89-102).  Tolerances: FP64 1e-12 (1e-9 after
simulate_until), FP32 bulk 1e-5.
"""

import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import euler_oracle as ora
from tests.gpu_helpers import VISC_CFGS, random_field_hat, rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(out_dir):
    exe = os.path.join(out_dir, "adapter_main")
    lib_dir = os.path.join(ROOT, "azeban_b200")
    cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-Wall", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "adapter_main.cpp"),
           "-L", lib_dir, "-lazeban_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}", "-o", exe]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


@pytest.mark.skipif(shutil.which(os.environ.get("CXX", "g++")) is None, reason="no C++ compiler")
def test_cpp_classes_compile_and_link(tmp_path):
    exe = build(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,N,prec", [(3, 16, "f64"), (2, 32, "f64"), (3, 32, "f32"), (2, 64, "f32")])
def test_cpp_caller_matches_oracle(tmp_path, dim, N, prec):
    exe = build(str(tmp_path))
    u = random_field_hat(dim, N, seed=4242 + N)
    inp = os.path.join(str(tmp_path), "u.bin")
    u.astype(np.complex128).tofile(inp)
    out = os.path.join(str(tmp_path), "out")
    res = subprocess.run([exe, str(dim), str(N), prec, "0.05", inp, out], capture_output=True, text=True,
                         timeout=300)
    assert res.returncode == 0, res.stderr
    tol, tol_sim = (1e-12, 1e-9) if prec == "f64" else (1e-5, 1e-5)
    og = ora.Grid(dim, N)
    eq = ora.IncompressibleEuler(og, ora.make_viscosity(VISC_CFGS["smooth"], og))
    u_in = u.astype(np.complex64).astype(np.complex128) if prec == "f32" else u
    ref = eq.dudt(u_in)
    got = np.fromfile(out + "_dudt.bin", dtype=np.complex128).reshape(u.shape)
    assert rel_l2(got, ref) <= tol
    dt = float(open(out + "_dt.txt").read())
    assert abs(dt - eq.dt(0.2)) <= (1e-13 if prec == "f64" else 1e-5) * eq.dt(0.2)
    step = u_in.copy()
    dt_ref = ora.SSP_RK3(eq).integrate(0.0, 1.0, 0.2, step)
    got = np.fromfile(out + "_step.bin", dtype=np.complex128).reshape(u.shape)
    assert rel_l2(got, step) <= tol
    assert abs(float(open(out + "_step.txt").read()) - dt_ref) <= (1e-13 if prec == "f64" else 1e-5) * dt_ref
    sim = ora.Simulation(og, 0.2, ora.SSP_RK3(eq), u_in)
    nsteps = sim.simulate_until(0.01)
    got = np.fromfile(out + "_sim.bin", dtype=np.complex128).reshape(u.shape)
    assert rel_l2(got, sim.u_) <= tol_sim
    t, n = open(out + "_sim.txt").read().split()
    assert float(t) == 0.01 and int(n) == nsteps
