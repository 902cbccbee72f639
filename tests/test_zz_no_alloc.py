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
        etype, nodes_d.data_ptr(), u_d.data_ptr(), nodes_d.shape[0], conn_d.data_ptr(),
        nb_elements, celerity, out.data_ptr(), None)
    _capi.check(rc)
    torch.cuda.synchronize()
    return float(out.item())


def _elastic_model(mesh):
    model = akb.SolidMechanicsModel(mesh)
    model.addMaterial("elastic", rho=1.0, E=1.0, nu=0.3)
    model.initFull()
    mat = model.getMaterial(0)
    return model, np.sqrt((mat.get("lambda") + 2 * mat.get("mu")) / mat.get("rho"))


@pytest.mark.parametrize("mesh_fn,etype", [(lambda: akb.box_hex8(12), _capi.HEXAHEDRON_8),
                                           (lambda: akb.box_tet4(8), _capi.TETRAHEDRON_4),
                                           (lambda: akb.square_tri6(20), _capi.TRIANGLE_6)])
def test_noalloc_matches_model_entry_point(mesh_fn, etype):
    mesh = mesh_fn()
    mesh.nodes += 0.01 * np.sin(5 * mesh.nodes)  # distorted, still valid
    model, celerity = _elastic_model(mesh)
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
        _capi.TETRAHEDRON_4, small.data_ptr(), small.data_ptr(), 16, conn.data_ptr(),
        AKB_NOALLOC_MAX_ELEMENTS + 1, 1.0, out.data_ptr(), None)
    assert rc == 1  # AKB_EINVAL, before any launch
    assert b"AKB_NOALLOC_MAX_ELEMENTS" in _capi.lib().akb_last_error()
    assert out.item() == 0.0


@pytest.mark.parametrize("celerity", [0.0, -1.0, float("nan"), float("inf")])
def test_noalloc_rejects_celerity_that_is_not_finite_and_positive(celerity):
    import torch
    small = torch.zeros(64, dtype=torch.float64, device="cuda")
    conn = torch.zeros(64, dtype=torch.int32, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _capi.lib().akb_stable_time_step_noalloc(
        _capi.TETRAHEDRON_4, small.data_ptr(), small.data_ptr(), 16, conn.data_ptr(), 4,
        celerity, out.data_ptr(), None)
    assert rc == 1
    assert b"celerity" in _capi.lib().akb_last_error()
    torch.cuda.synchronize()
    assert out.item() == 0.0


def test_noalloc_without_elements_gives_the_largest_double():
    import torch
    nodes = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    conn = torch.zeros((1, 4), dtype=torch.int32, device="cuda")
    assert _noalloc_dt(_capi.TETRAHEDRON_4, nodes, nodes, conn, 0, 1.0) == np.finfo(np.float64).max


def test_noalloc_index_out_of_range_gives_nan_and_does_not_stick():
    """A connectivity index >= nb_nodes (or negative) is caught on the device:
    the element reads no node and the result is NaN.  The next valid call on
    the same shared scratch gives the right value again."""
    mesh = akb.box_tet4(3)
    model, celerity = _elastic_model(mesh)
    expected = model.getStableTimeStep()
    nodes_d, u_d = _device(mesh.nodes), _device(np.zeros_like(mesh.nodes))
    for bad_index in (mesh.getNbNodes(), -1):
        conn = mesh.connectivity.copy()
        conn[5, 2] = bad_index
        got = _noalloc_dt(_capi.TETRAHEDRON_4, nodes_d, u_d, _device(conn),
                          mesh.getNbElement(), celerity)
        assert np.isnan(got)
        got = _noalloc_dt(_capi.TETRAHEDRON_4, nodes_d, u_d, _device(mesh.connectivity),
                          mesh.getNbElement(), celerity)
        assert abs(got - expected) <= 1e-15 * expected


def test_noalloc_orders_on_the_callers_stream():
    """The inputs are written by kernels on a non-default stream and the
    entry point is called on that stream with no device-wide synchronisation
    in between: it must see the written displacement, twice in a row."""
    import torch
    mesh = akb.box_hex8(6)
    model, celerity = _elastic_model(mesh)
    rng = np.random.default_rng(3)
    us = [0.002 * rng.standard_normal(mesh.nodes.shape) for _ in range(2)]
    expected = []
    for u in us:
        model.setNodal("displacement", u)
        expected.append(model.getStableTimeStep())
    nodes_d, conn_d = _device(mesh.nodes), _device(mesh.connectivity)
    host_u = [torch.from_numpy(u).pin_memory() for u in us]
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        u_d = torch.zeros(mesh.nodes.shape, dtype=torch.float64, device="cuda")
        outs = [torch.full((1,), -1.0, dtype=torch.float64, device="cuda") for _ in us]
        for hu, out in zip(host_u, outs):
            u_d.copy_(hu, non_blocking=True)
            u_d.mul_(1.0)  # a kernel on the stream writes the input too
            rc = _capi.lib().akb_stable_time_step_noalloc(
                _capi.HEXAHEDRON_8, nodes_d.data_ptr(), u_d.data_ptr(), mesh.getNbNodes(),
                conn_d.data_ptr(), mesh.getNbElement(), celerity, out.data_ptr(),
                ctypes.c_void_p(stream.cuda_stream))
            _capi.check(rc)
    stream.synchronize()
    for out, exp in zip(outs, expected):
        assert abs(out.item() - exp) <= 1e-15 * exp
