"""The specialised FFT shapes of the library against the grids of the 48-cell
batch (host logic, no GPU): every cell's k1 x k2 plane has a register plane
kernel (QX_PLANE_GRIDS in qx_fftplane.h), every z length a register column
kernel (QX_ZCOLS_LENGTHS), and every shape in the list has an instantiation
in one of the qx_fftplane_*.cu files, so that no batch cell falls back to the
shared-memory y/x and z passes."""
import glob
import os
import re

import pytest

from qxmd_b200 import cell

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "qxmd_b200", "csrc")


def _macro_body(name):
    text = open(os.path.join(CSRC, "qx_fftplane.h")).read()
    m = re.search(r"#define %s\(X\)((?:.*\\\n)*.*)" % name, text)
    assert m, name
    return m.group(1)


def plane_grids():
    return {(int(a), int(b)) for a, b in re.findall(r"X\((\d+),\s*(\d+)\)", _macro_body("QX_PLANE_GRIDS"))}


def zcols_lengths():
    return {int(a) for a in re.findall(r"X\((\d+)\)", _macro_body("QX_ZCOLS_LENGTHS"))}


def instantiated():
    grids, zl = set(), set()
    for f in glob.glob(os.path.join(CSRC, "qx_fftplane_*.cu")):
        text = open(f).read()
        grids |= {(int(a), int(b)) for a, b in re.findall(r"^QX_PLANE_GRID\((\d+),\s*(\d+)\)", text, re.M)}
        zl |= {int(a) for a in re.findall(r"^QX_ZCOLS_LENGTH\((\d+)\)", text, re.M)}
    return grids, zl


@pytest.fixture(scope="module")
def batch_grids():
    return [tuple(cell.batch_cell(i).gs.grid) for i in range(48)]


def test_every_listed_shape_is_instantiated():
    grids, zl = instantiated()
    assert plane_grids() == grids
    assert zcols_lengths() == zl


def test_batch_planes_have_register_kernels(batch_grids):
    missing = sorted({(k1, k2) for k1, k2, _ in batch_grids} - plane_grids())
    assert not missing, missing


def test_batch_z_lengths_have_register_kernels(batch_grids):
    missing = sorted({k3 for _, _, k3 in batch_grids} - zcols_lengths())
    assert not missing, missing


def test_listed_lengths_factor_into_register_radices():
    # the register FFTs are built from radices 2, 3, 4, 5 and 7 and one
    # thread holds a line: lengths of at most 64
    def smooth(n):
        for r in (2, 3, 5, 7):
            while n % r == 0:
                n //= r
        return n == 1
    for k1, k2 in plane_grids():
        assert smooth(k1) and smooth(k2) and max(k1, k2) <= 64, (k1, k2)
    for n in zcols_lengths():
        assert smooth(n) and n <= 64, n
