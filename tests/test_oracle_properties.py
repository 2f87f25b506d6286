"""Size-independent properties of the oracle's RHS and of the synthetic meshes (CPU)."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import fv, workloads
from ablate_b200.mesh import box_mesh, delaunay_mesh
from oracle import oracle as orc
from tests import rhs_cases as R


@pytest.mark.parametrize("mesh", ["box", "box_periodic", "box_periodic_xz", "box_morton", "tets"])
def test_lsq_weights_exact_for_linear_fields(mesh):
    # faceInterpolantTests.cpp:224-265 checks exact gradients of linear fields on boxes; here the cell
    # LSQ weights must reproduce a linear field's gradient on every interior cell away from the boundary
    if mesh == "tets":
        m = delaunay_mesh(2000)
    else:
        periodic = {"box": (False,) * 3, "box_periodic": (True,) * 3, "box_periodic_xz": (True, False, True), "box_morton": (True,) * 3}[mesh]
        m = box_mesh((6, 5, 4), upper=(1.2, 1.0, 0.8), periodic=periodic, order="morton" if mesh == "box_morton" else "natural")
    w = orc.lsq_face_weights(m)
    g_true = np.array([1.5, -2.0, 0.75])
    owned = m.cell_kind == L.CELL_OWNED
    fc = m.face_cells
    shift = m.face_shift if m.face_shift is not None else np.zeros((m.n_faces, 3))
    grad = np.zeros((m.n_cells, 3))
    boundary = (m.cell_kind[fc[:, 0]] == L.CELL_BOUNDARY) | (m.cell_kind[fc[:, 1]] == L.CELL_BOUNDARY)
    for f in range(m.n_faces):
        if boundary[f]:
            continue
        a, b = fc[f]
        d = (m.cell_centroid[b] + shift[f] - m.cell_centroid[a]) @ g_true  # u_b - u_a for u = g.x (periodic image)
        grad[a] += w[f, 0] * d
        grad[b] -= w[f, 1] * d
    full = np.array([all(not boundary[f] for f in np.nonzero((fc[:, 0] == c) | (fc[:, 1] == c))[0]) for c in range(m.n_cells)])
    sel = owned & full
    assert sel.sum() > 0
    np.testing.assert_allclose(grad[sel], np.tile(g_true, (sel.sum(), 1)), rtol=0, atol=1e-10)


@pytest.mark.parametrize("name", ["tgv3d_ausmpup_lsq_minmod_visc", "species3d_ns5", "box2d_ausmpup_vanleer_suth", "tets3d_pg_minmod", "tets3d_ns9"])
def test_free_stream_preserved(name):
    w = R.case(name)
    phys, keep = w.physics()
    U = np.tile(w.U[0], (w.mesh.n_cells, 1))
    F, _ = orc.rhs(w.mesh, phys, U, workloads.initial_aux(w))
    assert np.abs(F).max() < 1e-8 * np.abs(U).max()


def test_periodic_conservation():
    # on a fully periodic mesh every face flux enters one cell and leaves another: sum V F = 0
    w = R.case("tgv3d_ausmpup_lsq_minmod_visc")
    phys, keep = w.physics()
    F, _ = orc.rhs(w.mesh, phys, w.U, workloads.initial_aux(w))
    total = (F * w.mesh.cell_volume[:, None]).sum(0)
    scale = np.abs(F * w.mesh.cell_volume[:, None]).sum(0)
    assert np.all(np.abs(total) <= 1e-12 * scale)


@pytest.mark.parametrize("name", R.CASES)
def test_threaded_matches_serial(name):
    # the OpenMP owner-computes variant only reorders the per-cell sums; the walled channel's residual
    # is a small difference of large face fluxes, so reordering moves it by up to ~1e-14 of itself
    w = R.case(name)
    phys, keep = w.physics()
    F1, _ = orc.rhs(w.mesh, phys, w.U, workloads.initial_aux(w), threads=1)
    F4, _ = orc.rhs(w.mesh, phys, w.U, workloads.initial_aux(w), threads=4)
    owned = w.mesh.cell_kind == L.CELL_OWNED
    for block, e in R.block_errors(F4, F1, owned, 2 + w.mesh.dim).items():
        assert e <= 1e-13, (block, e)


def test_mesh_orderings_give_the_same_rhs():
    # Morton renumbering is a permutation: the RHS per physical cell must not change
    a = workloads.tgv3d(8, order="natural")
    b = workloads.tgv3d(8, order="morton")
    pa, ka = a.physics()
    pb, kb = b.physics()
    ia = np.lexsort(a.mesh.cell_centroid.T[::-1])
    ib = np.lexsort(b.mesh.cell_centroid.T[::-1])
    Ub = np.empty_like(b.U)
    Ub[ib] = a.U[ia]  # the same physical state (the seeded noise is drawn in cell order)
    Fa, _ = orc.rhs(a.mesh, pa, a.U, workloads.initial_aux(a))
    Fb, _ = orc.rhs(b.mesh, pb, Ub, workloads.initial_aux(b))
    np.testing.assert_allclose(Fb[ib], Fa[ia], rtol=1e-12, atol=1e-12 * np.abs(Fa).max())


def test_closed_cells():
    # every interior cell of the synthetic meshes is closed: sum over its faces of +-normal = 0
    for m in (box_mesh((5, 4, 3)), box_mesh((4, 4, 4), periodic=(True, True, True), order="morton"), box_mesh((7, 3)), delaunay_mesh(3000)):
        s = np.zeros((m.n_cells, 3))
        np.add.at(s, m.face_cells[:, 0], m.face_normal)
        np.add.at(s, m.face_cells[:, 1], -m.face_normal)
        owned = m.cell_kind == L.CELL_OWNED
        assert np.abs(s[owned]).max() < 1e-15 * max(1.0, np.abs(m.face_normal).max() * 1e3)
