import os
import subprocess
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))
GOLDEN = os.path.join(REPO, "tests", "golden")
BUILD = os.path.join(REPO, "tests", "_build")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


@pytest.fixture(scope="session")
def devmath_host():
    """Host build of the device math headers (Faddeeva, QPGF, element rules) for CPU checks."""
    import ctypes as C
    os.makedirs(BUILD, exist_ok=True)
    so = os.path.join(BUILD, "libdevmath_host.so")
    src = os.path.join(REPO, "tests", "native", "devmath_host.cpp")
    hdr = os.path.join(REPO, "bem3_emf_qd2_b200", "csrc")
    newest = max(os.path.getmtime(os.path.join(hdr, f)) for f in os.listdir(hdr))
    if not os.path.exists(so) or os.path.getmtime(so) < max(newest, os.path.getmtime(src)):
        subprocess.run(["g++", "-O2", "-fPIC", "-fopenmp", "-shared", "-x", "c++", "-I" + hdr, src, "-o", so],
                       check=True)
    lib = C.CDLL(so)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    lib.hm_faddeeva.argtypes = [i, vp, vp]
    lib.hm_erfcx.argtypes = [i, vp, vp]
    lib.hm_faddeeva_fast.argtypes = [i, vp, vp]
    lib.hm_qpgf.argtypes = [i, vp, vp, i, vp, vp]
    lib.hm_qpgf2.argtypes = [i, vp, vp, vp, vp]
    lib.hm_pair_regular.argtypes = [vp, i, i, i, i, d, d, vp, i, vp, vp, vp]
    lib.hm_pair_regular.restype = i
    lib.hm_self_interior.argtypes = [vp, i, i, d, d, vp, vp, vp, vp, vp]
    lib.hm_self_periodic.argtypes = [vp, i, i, vp, vp, vp, vp, vp, vp]
    lib.hm_field_coef.argtypes = [vp, i, vp, i, d, d, i, vp, vp, vp]
    lib.hm_field_grad_coef.argtypes = [vp, i, vp, i, d, d, i, vp, vp, vp]
    lib.hm_solid_angle.argtypes = [vp, vp, i, i, vp, vp]
    lib.hm_solid_angle.restype = d
    lib.hm_self_periodic.restype = i
    return lib


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda_lib_host():
    """The CUDA library loaded without a GPU, for its entry points that touch no device."""
    import bem3_emf_qd2_b200 as B
    return B.lib()


@pytest.fixture(scope="session")
def cuda_lib():
    import bem3_emf_qd2_b200 as B
    if not gpu_available():
        pytest.fail("no CUDA device: -m gpu tests need a B200")
    return B
