"""akb_stable_time_step_noalloc: the stable time step for callers that cannot
let the library allocate device memory (their memory comes from their own
pool, or they compute inside a loop where runtime allocation is not allowed).

The entry point is checked through the C ABI against the model's own
akb_model_get_stable_time_step on the same mesh and displacement, on two calls
in a row with different displacements (the shared scratch array must not
carry anything from one call to the next).  This file is collected last so a
run that stops at the first failure has run every other test before it."""
import ctypes

import numpy as np
import pytest

import akantu2_b200 as akb
from akantu2_b200 import _capi

pytestmark = pytest.mark.gpu

AKB_NOALLOC_MAX_ELEMENTS = 1 << 20


def _device(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def _noalloc_dt(etype, nodes_d, u_d, conn_d, nb_elements, celerity):
    import torch
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = _capi.lib().akb_stable_time_step_noalloc(
        etype, nodes_d.data_ptr(), u_d.data_ptr(), conn_d.data_ptr(), nb_elements, celerity,
        out.data_ptr(), None)
    _capi.check(rc)
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("mesh_fn,etype", [(lambda: akb.box_hex8(12), _capi.HEXAHEDRON_8),
                                           (lambda: akb.box_tet4(8), _capi.TETRAHEDRON_4),
                                           (lambda: akb.square_tri6(20), _capi.TRIANGLE_6)])
def test_noalloc_matches_model_entry_point(mesh_fn, etype):
    mesh = mesh_fn()
    mesh.nodes += 0.01 * np.sin(5 * mesh.nodes)  # distorted, still valid
    model = akb.SolidMechanicsModel(mesh)
    model.addMaterial("elastic", rho=1.0, E=1.0, nu=0.3)
    model.initFull()
    celerity = np.sqrt((model.getMaterial(0).get("lambda") + 2 * model.getMaterial(0).get("mu"))
                       / model.getMaterial(0).get("rho"))
    nodes_d = _device(mesh.nodes)
    conn_d = _device(mesh.connectivity)
    rng = np.random.default_rng(0)
    for call in range(2):  # two calls in a row, different displacements
        u = 0.002 * rng.standard_normal(mesh.nodes.shape)  # small: no element inverts
        model.setNodal("displacement", u)
        expected = model.getStableTimeStep()
        got = _noalloc_dt(etype, nodes_d, _device(u), conn_d, mesh.getNbElement(), celerity)
        assert expected > 0
        assert abs(got - expected) <= 1e-15 * expected, (call, got, expected)


def test_noalloc_rejects_sizes_beyond_the_maximum():
    import torch
    small = torch.zeros(64, dtype=torch.float64, device="cuda")
    conn = torch.zeros(64, dtype=torch.int32, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _capi.lib().akb_stable_time_step_noalloc(
        _capi.TETRAHEDRON_4, small.data_ptr(), small.data_ptr(), conn.data_ptr(),
        AKB_NOALLOC_MAX_ELEMENTS + 1, 1.0, out.data_ptr(), None)
    assert rc == 1  # AKB_EINVAL, before any launch
    assert b"AKB_NOALLOC_MAX_ELEMENTS" in _capi.lib().akb_last_error()
    assert out.item() == 0.0
