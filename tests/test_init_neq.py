"""The non-equilibrium initialisation (Parameter::setUseInitNeq; InitNavierStokesCompressible_Device.cu:
216-501) of the oracle, on the CPU.

The reference writes the equilibrium plus (1 + drho) times a non-equilibrium part per direction pair,
formed from central-difference velocity gradients. Opposite directions share their part, so the part
carries no momentum; its coefficients sum to zero, so it carries no mass; and its xy moment is the
Chapman-Enskog stress -(1 + drho)(d_y u_x + d_x u_y) / (3 omega). The GPU kernel is pinned to the
reference's own kernel and to this oracle in tests/test_gpu_init_neq.py.
"""
import numpy as np

from virtualfluids_b200 import ListGrid, Parameter
from virtualfluids_b200 import _native as N

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1])


def _smooth(g, seed, amp_rho=1e-2, amp_u=0.03, modes=3):
    rng = np.random.default_rng(seed)
    x, y, z = (g.coords[a].astype(np.float64) for a in range(3))
    out = []
    for amp in (amp_rho, amp_u, amp_u, amp_u):
        f = np.zeros(g.number_of_nodes)
        for _ in range(modes):
            k = rng.integers(0, 2, 3) + np.array([1, 0, 0])
            ph = rng.uniform(0, 2 * np.pi, 3)
            f += np.cos(2 * np.pi * k[0] * x / g.nx + ph[0]) * np.cos(2 * np.pi * k[1] * y / g.ny + ph[1]) \
                * np.cos(2 * np.pi * k[2] * z / g.nz + ph[2])
        out.append(f * amp / modes)
    return out


def test_neighbor_inverse_steps_back_to_the_node():
    for periodic in ((True, True, True), (False, True, False), (False, False, False)):
        g = ListGrid(5, 4, 3, periodic=periodic)
        inv, nb = g.neighbor_inverse, g.neighbor
        for k in g.fluid:
            assert inv[k] != 0
            assert nb[2][nb[1][nb[0][inv[k]]]] == k
        assert inv[0] == 0


def test_inverse_neighbours_from_the_plus_one_lists():
    """Imported grids without neighborInverse get it from the +1 lists: the same as the box's own."""
    from virtualfluids_b200.grid import inverse_neighbors
    for periodic in ((True, True, True), (False, True, False), (False, False, False)):
        g = ListGrid(6, 5, 4, periodic=periodic)
        assert np.array_equal(inverse_neighbors(g.neighbor)[g.fluid], g.neighbor_inverse[g.fluid])


def test_neq_init_keeps_density_and_velocity(oracle):
    for periodic in ((True, True, True), (False, True, False)):
        g = ListGrid(12, 10, 8, periodic=periodic)
        rho, ux, uy, uz = _smooth(g, 3)
        neq = oracle.OracleLevel(g, 1.7)
        neq.init(rho, ux, uy, uz, neq=True)
        eq = oracle.OracleLevel(g, 1.7)
        eq.init(rho, ux, uy, uz)
        m = neq.macroscopic()
        fl = g.fluid
        for key, ref in (("rho", rho), ("vx", ux), ("vy", uy), ("vz", uz)):
            np.testing.assert_allclose(m[key][fl], ref[fl], rtol=0, atol=2e-16, err_msg=key)
        assert np.abs(neq.f - eq.f).max() > 1e-6          # the part is there


def test_neq_init_xy_stress_is_the_chapman_enskog_stress(oracle):
    """Linear shear ux = s y, uy = t x on a box with its shell (central differences are exact):
    sum_d cx cy (f_neq - f_eq) = -(1 + drho)(s + t) / (3 omega) at every fluid node."""
    g = ListGrid(7, 6, 5)
    x, y, _ = (g.coords[a].astype(np.float64) for a in range(3))
    s, t, omega, drho = 3e-3, -1e-3, 1.6, 4e-3
    rho = np.full(g.number_of_nodes, drho)
    ux, uy, uz = s * y, t * x, np.zeros(g.number_of_nodes)
    ux[0] = uy[0] = 0.0
    neq = oracle.OracleLevel(g, omega)
    neq.init(rho, ux, uy, uz, neq=True)
    eq = oracle.OracleLevel(g, omega)
    eq.init(rho, ux, uy, uz)
    want = -(1.0 + drho) * (s + t) / (3.0 * omega)
    for k in g.fluid[:: 7]:
        pxy = np.sum(CX * CY * (neq.pre(k) - eq.pre(k)))
        assert abs(pxy - want) < 1e-15, (k, pxy, want)


def test_neq_init_of_a_uniform_flow_is_the_equilibrium_bitwise(oracle):
    g = ListGrid(6, 5, 4, periodic=(True, True, True))
    n = g.number_of_nodes
    fields = [np.full(n, 2e-3), np.full(n, 0.04), np.full(n, -0.01), np.full(n, 0.02)]
    neq = oracle.OracleLevel(g, 1.8)
    neq.init(*fields, neq=True)
    eq = oracle.OracleLevel(g, 1.8)
    eq.init(*fields)
    keep = np.ones(27 * n, dtype=bool)
    keep[np.nonzero(g.geo != N.GEO_FLUID)[0]] = False     # rest slots the neq init marks with 96
    assert np.array_equal(neq.f[keep], eq.f[keep])


def test_neq_init_marks_solid_and_void_rest_slots(oracle):
    g = ListGrid(4, 4, 4)                      # every axis walled: the shell is void
    lv = oracle.OracleLevel(g, 1.8)
    lv.init(neq=True)
    void = np.nonzero(g.geo == N.GEO_VOID)[0]
    assert void.size > 0
    assert np.all(lv.f[void] == 96.0)          # the rest direction's plane holds node k at k


def test_configuration_key_turns_it_on(tmp_path):
    p = tmp_path / "config.txt"
    p.write_text("Viscosity_LB = 0.01\nUseInitNeq = true\n")
    assert Parameter.from_configuration_file(p).use_init_neq
    p.write_text("Viscosity_LB = 0.01\nUseInitNeq = false\n")
    assert not Parameter.from_configuration_file(p).use_init_neq
    assert not Parameter().use_init_neq
