"""The host-buffer RHS (abl_fv_rhs_host: the state and the residual copied in, the residual added to
and copied out, with the residual's copies overlapped with the kernels) against the device-pointer RHS,
bit for bit: on a mesh whose residual is large enough to travel in tile chunks, on small ones, with
ghost rows, and on one whose tiles are not cell ranges."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import workloads
from ablate_b200.mesh import box_mesh
from tests import rhs_cases as R

pytestmark = pytest.mark.gpu


def _cases(name):
    if name == "tgv76":
        return workloads.tgv3d(76)                 # 17.6 MB residual, Morton-numbered cells: chunked copies
    w1 = workloads.tgv3d(16)                       # small residual: one copy each way
    w2 = workloads.wall3d(12)                      # ghosts after the owned rows
    w3 = workloads.tgv3d(12)
    w3.mesh = box_mesh((12, 12, 12), periodic=(True, True, True), order="natural")
    w3.U = workloads.tgv_state(w3.mesh)            # natural numbering: tiles are not ranges
    return {"tgv16": w1, "wall12": w2, "tgv12_natural": w3, "species": R.case("species3d_ns5")}[name]


@pytest.mark.parametrize("name", ["tgv76", "tgv16", "wall12", "tgv12_natural", "species"])
@pytest.mark.parametrize("precision", [L.PRECISION_FP64, L.PRECISION_MIXED])
def test_host_path_adds_the_device_residual(name, precision):
    torch = pytest.importorskip("torch")
    w = _cases(name)
    s = w.solver()
    rng = np.random.default_rng(4)
    F0 = rng.standard_normal(w.U.shape)
    Fh = F0.copy()
    s.ComputeRHSFunction(0.0, w.U, Fh, precision)
    assert s.Status() == L.OK
    dev = torch.device("cuda", 0)
    U = torch.from_numpy(w.U).to(dev)
    Fd = torch.from_numpy(F0).to(dev)
    s.ComputeRHSDevice(0.0, U.data_ptr(), Fd.data_ptr(), precision, torch.cuda.current_stream().cuda_stream)
    np.testing.assert_array_equal(Fh, Fd.cpu().numpy())
    owned = w.mesh.cell_kind == L.CELL_OWNED
    np.testing.assert_array_equal(Fh[~owned], F0[~owned])
    # a second call on the same handle (the pipeline's streams and events are reused)
    Fh2 = F0.copy()
    s.ComputeRHSFunction(0.0, w.U, Fh2, precision)
    np.testing.assert_array_equal(Fh2, Fh)
