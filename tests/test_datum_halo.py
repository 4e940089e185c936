"""The rows kernel moves the bed of the staged halo cells that lie in another
64 x 64 datum block into the tile's datum, walking only the halo sides that
cross a block edge (csrc/hb_datum_halo.cuh).  Compiled for the CPU, the list
must hold exactly the staged halo cells outside the tile's block, once each,
for every tile position and both tile heights."""
import ctypes
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "chans-hipims-flamegpu_b200", "csrc")


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("halo") / "libdatumhalo.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC,
                    os.path.join(HERE, "datum_halo_check.cpp"), "-o", out], check=True)
    L = ctypes.CDLL(out)
    L.datum_halo_mismatches.argtypes = [ctypes.c_int] * 6 + [ctypes.POINTER(ctypes.c_int)]
    return L


@pytest.mark.parametrize("ty,listed", [(32, 216), (64, 416)])
def test_datum_halo_lists_exactly_the_cells_in_other_blocks(lib, ty, listed):
    n = ctypes.c_int(0)
    # 32-column tiles staged with 40 columns (-4 .. 35), 64 x 64 blocks, 4 x 4 blocks
    assert lib.datum_halo_mismatches(ty, 32, 40, 64, 4, 4, ctypes.byref(n)) == 0
    # 2 rows x 40 + 4 columns x (ty + 2) for every tile: half the 4 x 40 + 8 x ty
    # halo cells of 32-row tiles
    assert n.value == listed
