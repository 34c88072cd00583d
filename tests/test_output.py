"""Output: the device-computed output fields (asynchronous dump) and the VTK
legacy file of write_vtk_to (crates/cfd_output/src/lib.rs:36-125)."""
import numpy as np
import pytest

from dev_field_efvm_b200 import cases

pytestmark = pytest.mark.gpu


def test_vtk_file_matches_the_state(tmp_path):
    from dev_field_efvm_b200.device import Context

    grid, params, u, ex = cases.vortex_case(32, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    c = Context(grid, params)
    c.upload(u)
    c.step(3)
    s = c.download()
    path = tmp_path / "out.vtk"
    c.write_vtk(str(path))
    lines = path.read_text().splitlines()
    assert lines[:5] == ["# vtk DataFile Version 3.0", "dev_field_efvm output", "ASCII", "DATASET RECTILINEAR_GRID",
                         "DIMENSIONS 33 33 2"]
    assert lines[5] == "X_COORDINATES 33 double"
    x = np.array([float(v) for v in lines[6:39]])
    assert np.allclose(x, np.linspace(0.0, 10.0, 33), atol=1e-12)
    i = lines.index("CELL_DATA 1024")
    assert lines[i + 1] == "SCALARS density double 1"
    rho = np.array([float(v) for v in lines[i + 3:i + 3 + 1024]])
    assert np.allclose(rho, s[..., 0].reshape(-1), rtol=1e-10)
    j = lines.index("VECTORS velocity double")
    vel = np.array([[float(q) for q in ln.split()] for ln in lines[j + 1:j + 1 + 1024]])
    assert np.allclose(vel[:, 0], (s[..., 1] / s[..., 0]).reshape(-1), rtol=1e-10, atol=1e-14)
    assert np.all(vel[:, 2] == 0.0)
    k = lines.index("SCALARS mach double 1")
    assert len(lines) == k + 2 + 1024
    assert all("e+" in v or "e-" in v for v in lines[k + 2:k + 12])


def test_async_output_fields_match_the_synchronous_ones():
    import torch
    from dev_field_efvm_b200.device import Context

    grid, params, u, ex = cases.vortex_case(64, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    c = Context(grid, params)
    c.upload(u)
    c.step(2)
    sync = c.output_fields()
    pinned = torch.empty((7, 64, 64), dtype=torch.float64, pin_memory=True)
    c.output_fields(pinned.numpy(), wait=False)
    c.synchronize()
    assert np.array_equal(pinned.numpy(), sync)
    s = c.download()
    p = 0.4 * (s[..., 4] - 0.5 * (s[..., 1] ** 2 + s[..., 2] ** 2) / s[..., 0])
    assert np.allclose(sync[1], p, rtol=1e-12)
    assert np.all(sync[6] > 0)
