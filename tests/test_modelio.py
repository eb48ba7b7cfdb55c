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


@pytest.mark.parametrize("sws,stage,trim", [(2, None, 0), (3, None, 0), (4, None, 5), (3, 2, 0), (4, 7, 0)])
def test_taper_file_reader_matches_taper_grad_shot(sws, stage, trim):
    """The per-shot taper files of src/taper_grad_shot.c (sws 2, 3, 4 ->
    .vp, .vs, .rho) read as the reference reads them: x outer, the workflow
    file (stage 2 here) before the plain one, the plain one when the workflow
    file is missing (stage 7), and a file short by `trim` values whose last
    cells keep the last value read.  The reference multiplies a plane of
    ones by what it read, so the plane it returns is its coefficient plane."""
    from tests import compat_harness as H
    ref, _ = H.libs()
    nx, ny, ishot = 11, 8, 3
    rng = np.random.default_rng(sws + (stage or 0))
    kind = modelio.TAPER_KINDS[sws]
    d = tempfile.mkdtemp(prefix="tp", dir="/tmp")  # TAPER_FILE_NAME holds 74 characters
    base = os.path.join(d, "taper")
    rng.uniform(0.0, 1.0, nx * ny - trim).astype(np.float32).tofile(f"{base}.shot{ishot}.{kind}")
    if stage == 2:
        rng.uniform(2.0, 3.0, nx * ny).astype(np.float32).tofile(f"{base}.shot{ishot}_{stage}.{kind}")
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    C.c_void_p.in_dll(ref, "FP").value = libc.fopen(os.devnull.encode(), b"w")
    for name, v in (("NX", nx), ("NY", ny), ("NXG", nx), ("NYG", ny), ("NPROCX", 1), ("NPROCY", 1), ("MYID", 0),
                    ("VERBOSE", 0), ("USE_WORKFLOW", int(stage is not None)), ("WORKFLOW_STAGE", stage or 0)):
        C.c_int.in_dll(ref, name).value = v
    pos = (C.c_int * 3).in_dll(ref, "POS")
    pos[0] = pos[1] = pos[2] = 0
    (C.c_char * 74).in_dll(ref, "TAPER_FILE_NAME").value = base.encode()
    W = ref.matrix(1, ny, 1, nx)
    for j in range(ny):
        for i in range(nx):
            W[j + 1][i + 1] = 1.0
    T = ref.matrix(1, ny, 1, nx)
    f = ref.taper_grad_shot
    f.restype = None
    f.argtypes = [H.FPP, H.FPP, H.FPP, C.c_int, H.IPP, C.c_int, C.c_int, C.c_int]
    f(W, T, None, 0, None, 0, ishot, sws)
    want = np.array([[W[j + 1][i + 1] for i in range(nx)] for j in range(ny)], np.float32)
    got = modelio.read_taper_file(base, ishot, sws, nx, ny, workflow_stage=stage)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))
    if stage == 2:
        assert got.min() >= 2.0  # the workflow file was read
    with pytest.raises(FileNotFoundError):
        modelio.read_taper_file(base, ishot + 1, sws, nx, ny)
