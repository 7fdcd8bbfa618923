"""include/wcsph_fdps.hpp as a drop-in: a C++ program built from the
reference's own plugin types (src/class.h) calls GPU_WC::HydrDispatchKernel /
GPU_WC::HydrRetrieveKernel and checks them against the reference's own
STD::CalcHydroForce (src/force.h:31-60) on FDPS-style superset walks."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "fdps_shim_check")


def test_shim_built_against_reference_types(oracle_lib, native):
    if not oracle_lib.ref_available():
        pytest.skip("reference sources absent: oracle/_ref not built")
    oracle_lib.build()
    assert os.path.exists(BIN), "oracle/Makefile did not build the FDPS shim check"


@pytest.mark.gpu
def test_shim_matches_reference_functor(native):
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/fdps_shim_check was not built (reference sources absent at build time)")
    r = subprocess.run([BIN, "12"], capture_output=True, text=True, timeout=300)
    print(r.stdout, r.stderr)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "acc_rel_l2" in r.stdout
