"""Shared inputs of the tests: materials, seeded initial states and the
small versions of the benchmark configurations, built identically for the
GPU model and for the CPU oracle."""
import os

import numpy as np

from oracle import oracle as orc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TYPES = ("_tetrahedron_4", "_hexahedron_8", "_triangle_6")
OR_TYPE = {"_tetrahedron_4": orc.TET4, "_hexahedron_8": orc.HEX8, "_triangle_6": orc.TRI6}

# patch-test materials (test/test_model/patch_tests/data/material_check_stress_*.dat)
STEEL_PLANE_STRAIN = dict(type="elastic", name="steel", rho=7800.0, E=2.1e11, nu=0.3)
STEEL_PLANE_STRESS = dict(STEEL_PLANE_STRAIN, Plane_Stress=True)
# lumped-mass test material (material_lumped.dat)
STEEL_LUMPED = dict(type="elastic", name="steel", rho=7800.0, E=2.1e11, nu=0.0)

UNIT_ELASTIC = dict(type="elastic", name="unit", rho=1.0, E=1.0, nu=0.3)
UNIT_NEOHOOKEAN = dict(type="neohookean", name="rubber", rho=1.0, E=1.0, nu=0.3)
UNIT_PLASTIC = dict(type="plastic_linear_isotropic_hardening", name="metal", rho=1.0, E=1.0,
                    nu=0.3, sigma_y=1e-3, h=0.1)

# alpha of patch_test_linear_fixture.hh:158-161
PATCH_ALPHA = np.array([[0.01, 0.02, 0.03, 0.04],
                        [0.05, 0.06, 0.07, 0.08],
                        [0.09, 0.10, 0.11, 0.12]])


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def linear_field(nodes):
    d = nodes.shape[1]
    return PATCH_ALPHA[:d, 0][None, :] + nodes @ PATCH_ALPHA[:d, 1:1 + d].T


def dat_text(mat):
    lines = [f"material {mat['type']} ["]
    for k, v in mat.items():
        if k == "type":
            continue
        if isinstance(v, bool):
            v = "true" if v else "false"
        lines.append(f"  {k} = {v}")
    lines.append("]")
    return "\n".join(lines) + "\n"


def oracle_model(mesh, materials, mat_of_elem=None, qp_rule=0, threads=8):
    return orc.OracleModel(OR_TYPE[mesh.element_type], mesh.nodes, mesh.connectivity,
                           materials, mat_of_elem=mat_of_elem, qp_rule=qp_rule,
                           threads=threads)


def sinusoidal_velocity(nodes, amplitude=0.01):
    """v_z = A sin(pi x) sin(pi y) z (the tet-cube configuration)."""
    v = np.zeros_like(nodes)
    v[:, 2] = amplitude * np.sin(np.pi * nodes[:, 0]) * np.sin(np.pi * nodes[:, 1]) * nodes[:, 2]
    return v


def random_field_velocity(nodes, seed, corr_length=0.1, std=0.02):
    from akantu2_b200 import gaussian_random_field
    return gaussian_random_field(nodes, seed, corr_length, std)


def blocked_face(nodes, axis=2, value=0.0):
    b = np.zeros(nodes.shape, dtype=np.uint8)
    b[np.isclose(nodes[:, axis], value)] = 1
    return b


# ---- travelling-wave bar (test_solid_mechanics_model_dynamics.cc) -----------------------
# A 10 x 1 (x 1) bar of mesh size about 0.6, E = 1, nu = 0, rho = 1, a plane
# P wave and S waves of wave vector k = (0.5, 0, 0) and amplitude A = 0.1; the
# boundary nodes get the analytic displacement and velocity before every step
# (their x component blocked), and the error after t = 5 is
# sqrt(sum over nodes |u - u_exact|^2) / (number of nodes), at most 2e-3.  The
# velocity expression is the reference test's (cosine of the phase).
WAVE_MAT = dict(type="elastic", name="uniterial", rho=1.0, E=1.0, nu=0.0)
WAVE_A, WAVE_K = 0.1, 0.5


def wave_bar(etype):
    import akantu2_b200 as akb
    if etype == "_tetrahedron_4":
        return akb.box_tet4(17, 2, 2, lengths=(10.0, 1.0, 1.0))
    if etype == "_hexahedron_8":
        return akb.box_hex8(17, 2, 2, lengths=(10.0, 1.0, 1.0))
    return akb.square_tri6(17, 2, lengths=(10.0, 1.0))


def wave_solution(X, t):
    """(displacement, velocity) of the analytic waves at the points X, time t."""
    d = X.shape[1]
    lam, mu = 0.0, 0.5  # E = 1, nu = 0
    cp, cs = np.sqrt(lam + 2 * mu), np.sqrt(mu)
    wp, ws = WAVE_K * cp, WAVE_K * cs
    ph_p = WAVE_K * X[:, 0] - wp * t
    ph_s = WAVE_K * X[:, 0] - ws * t
    kpush = np.zeros(d)
    kpush[0] = WAVE_K
    if d == 2:
        shear = [np.array([0.0, WAVE_K])]
    else:  # k x (0, 0, 1) and k x (0, 1, 0)
        shear = [np.array([0.0, -WAVE_K, 0.0]), np.array([0.0, 0.0, WAVE_K])]
    u = WAVE_A * np.outer(np.cos(ph_p), kpush)
    v = WAVE_A * np.outer(wp * np.cos(ph_p), kpush)
    for ks in shear:
        u += WAVE_A * np.outer(np.cos(ph_s), ks)
        v += WAVE_A * np.outer(ws * np.cos(ph_s), ks)
    return u, v


def run_wave(mesh, set_nodal, get_u, step, dt):
    """Drives the wave test through plain callbacks; returns the maximum error."""
    from akantu2_b200 import boundary_nodes
    X = mesh.nodes
    bnd = boundary_nodes(mesh.element_type, mesh.connectivity)
    blocked = np.zeros(X.shape, dtype=np.uint8)
    blocked[bnd, 0] = 1
    u0, v0 = wave_solution(X, 0.0)
    set_nodal("displacement", u0)
    set_nodal("velocity", v0)
    set_nodal("blocked_dofs", blocked)
    steps = int(5.0 / dt)
    t, err = 0.0, -1.0
    for _ in range(steps):
        ub, vb = wave_solution(X[bnd], t)
        u, v = get_u()
        u[bnd], v[bnd] = ub, vb
        set_nodal("displacement", u)
        set_nodal("velocity", v)
        ue, _ = wave_solution(X, t)
        err = max(err, np.sqrt(np.sum((u - ue) ** 2)) / X.shape[0])
        step()
        t += dt
    return err, steps
