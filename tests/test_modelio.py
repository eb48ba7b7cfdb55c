"""Model and gradient files (ifos_b200/modelio.py) byte for byte against the
reference's own writers (src/writemod.c, src/mergemod.c,
src/matrix_operations.c:24-50 write_matrix_disk, src/writedsk.c), compiled
in place into oracle/_ref/libifoswriters.so, on a plane with zeros,
negative, tiny and large values, in the binary and the ASCII format."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from ifos_b200 import modelio

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libifoswriters.so")
FPP = C.POINTER(C.POINTER(C.c_float))
NX, NY = 9, 7


def _lib():
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libifoswriters.so is not built (make -C oracle driver)")
    # its own definitions first: the reference oracle library (loaded globally by other tests) defines the
    # same globals and stubs the file merging out
    lib = C.CDLL(LIB, mode=os.RTLD_LOCAL | os.RTLD_DEEPBIND)
    lib.matrix.restype = FPP
    lib.matrix.argtypes = [C.c_int] * 4
    lib.writemod.argtypes = [C.c_char_p, FPP, C.c_int]
    lib.mergemod.argtypes = [C.c_char_p, C.c_int]
    lib.write_matrix_disk.argtypes = [FPP, C.c_char_p]
    lib.orc_writer_globals(NX, NY)
    return lib


def _plane():
    rng = np.random.default_rng(3)
    a = (rng.standard_normal((NY, NX)) * 1e3).astype(np.float32)
    a[0, 0], a[1, 2], a[2, 3], a[3, 4] = 0.0, -1.5e-30, 3.4e37, -0.0
    return a


def _ref_matrix(lib, a):
    m = lib.matrix(1, NY, 1, NX)
    for j in range(NY):
        for i in range(NX):
            m[j + 1][i + 1] = float(a[j, i])
    return m


@pytest.mark.parametrize("fmt", [3, 2])
def test_model_file_matches_writemod_and_mergemod(fmt):
    lib = _lib()
    a = _plane()
    d = tempfile.mkdtemp(prefix="mio", dir="/tmp")
    ref = os.path.join(d, "ref_vp")
    lib.writemod(ref.encode(), _ref_matrix(lib, a), fmt)
    lib.mergemod(ref.encode(), fmt)
    ours = os.path.join(d, "our_vp")
    modelio.write_model_file(ours, a, fmt)
    for suffix in ("", ".0.0"):
        assert open(ref + suffix, "rb").read() == open(ours + suffix, "rb").read(), suffix


def test_gradient_file_matches_write_matrix_disk():
    lib = _lib()
    a = _plane()
    d = tempfile.mkdtemp(prefix="mio", dir="/tmp")
    ref = os.path.join(d, "ref_jac")
    lib.write_matrix_disk(_ref_matrix(lib, a), ref.encode())
    ours = modelio.write_matrix_disk(a, os.path.join(d, "our_jac"))
    assert sorted(os.listdir(d)) == ["our_jac.bin", "ref_jac.bin"]  # the rank file is merged and removed
    assert open(ref + ".bin", "rb").read() == open(ours, "rb").read()
    assert np.array_equal(np.fromfile(ours, np.float32).reshape(NX, NY).T, a)


def test_mergemod_joins_rank_files_in_the_reference_order():
    """Two x ranks by two y ranks of 3 x 2 cells each: the merged file is,
    for each x rank and each of its columns, the y ranks' columns in order."""
    d = tempfile.mkdtemp(prefix="mio", dir="/tmp")
    name = os.path.join(d, "m")
    blocks = {}
    for ip in range(2):
        for jp in range(2):
            blocks[(ip, jp)] = (np.arange(6, dtype=np.float32) + 10 * (2 * ip + jp)).reshape(2, 3)  # ny=2, nx=3
            modelio.writemod(name, blocks[(ip, jp)], pos=(ip, jp))
    modelio.mergemod(name, nx=3, ny=2, nprocx=2, nprocy=2)
    got = np.fromfile(name, np.float32)
    want = np.concatenate([blocks[(ip, jp)].T[i] for ip in range(2) for i in range(3) for jp in range(2)])
    assert np.array_equal(got, want)
