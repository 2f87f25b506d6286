"""The device layout's set-up on the host (ablate_b200/csrc/fv_setup.hpp), without a GPU: the
canonical cone order, and the record tables (repeated cone-weight sequences and face-geometry
records stored once). tests/setup_records_check.cpp, compiled here with g++, builds the host mesh,
tiles and records from a mesh written by this test and checks that each cell's neighbour offsets
ascend and that the tables expand back to the one-record-per-item arrays bit for bit; this test checks
the class counts on structured and unstructured meshes.
"""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from ablate_b200.mesh import box_mesh, delaunay_mesh

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("setup") / "setup_records_check"
    subprocess.run([gxx, "-std=c++17", "-O2", "-I", str(ROOT / "ablate_b200" / "csrc"), "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "setup_records_check.cpp"), "-o", str(exe)], check=True)
    return exe


def _run(checker, tmp_path, mesh, lsq=True, dif=True):
    p = tmp_path / "mesh.bin"
    shift = mesh.face_shift
    with open(p, "wb") as f:
        np.array([mesh.dim, mesh.n_cells, mesh.n_faces, shift is not None, lsq, dif], dtype=np.int32).tofile(f)
        np.ascontiguousarray(mesh.face_cells, dtype=np.int32).tofile(f)
        for a in (mesh.face_normal, mesh.face_centroid, mesh.cell_centroid, mesh.cell_volume):
            np.ascontiguousarray(a, dtype=np.float64).tofile(f)
        np.ascontiguousarray(mesh.cell_kind, dtype=np.uint8).tofile(f)
        if shift is not None:
            np.ascontiguousarray(shift, dtype=np.float64).tofile(f)
    r = subprocess.run([str(checker), str(p)], capture_output=True, text=True)
    words = r.stdout.split()
    assert r.returncode == 0 and words[-1] == "1", r.stdout + r.stderr
    fields = dict(zip(words[0::2], words[1::2]))
    _run.last = {k: int(v) for k, v in fields.items()}
    return int(words[1]), int(words[3])


def test_periodic_box_has_one_weight_class_and_three_geometry_classes(checker, tmp_path):
    # every cell of a periodic box sees the same neighbours in the same order: one weight sequence;
    # the tile faces have three orientations
    assert _run(checker, tmp_path, box_mesh((16, 16, 16), periodic=(True, True, True), order="morton")) == (1, 3)
    # every 8x8x4 tile of the periodic box has the same local topology: one fused table; it stages its
    # 256 cells, 256 ring-1 and 336 ring-2 cells
    assert _run.last["fused_classes"] == 1 and _run.last["max_ext"] == 848


def test_walled_box_has_a_few_classes(checker, tmp_path):
    # walls in x and y: interior, wall, edge and ghost cells, each kind a few classes
    wc, gc = _run(checker, tmp_path, box_mesh((16, 16, 16), periodic=(False, False, True), order="morton"))
    assert 1 < wc <= 64 and 3 <= gc <= 16


def test_first_order_box_without_weights(checker, tmp_path):
    # no gradients: the weights are zero and only the offsets tell cells apart
    wc, gc = _run(checker, tmp_path, box_mesh((32, 32), order="morton"), lsq=False, dif=False)
    assert 1 <= wc <= 16 and 2 <= gc <= 8


def test_inexact_spacing_keeps_one_weight_record_per_entry(checker, tmp_path):
    # spacing 1/12 is not exact in binary: the offsets, and so the weights, differ in their last bits
    wc, _ = _run(checker, tmp_path, box_mesh((12, 12, 12), periodic=(False, False, True), order="morton"))
    assert wc == 0


def test_unstructured_mesh_keeps_one_record_per_item(checker, tmp_path):
    assert _run(checker, tmp_path, delaunay_mesh(1500, seed=7)) == (0, 0)
