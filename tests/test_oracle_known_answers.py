"""Known-answer pins of the FP64 CPU oracle.

The reference solver (a closed Windows DLL) cannot run here, so the oracle is
pinned by analytic solutions and exact invariants of the method instead.
"""
import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import cases
from oracle.case import initial_field, resolve as case_params
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from _oracle import Oracle


def _params(casedir, name, text, **opt):
    return case_params(cases.write(text, f"{casedir}/{name}.xml"), **opt)


def test_poiseuille_trt_magic_exact(casedir):
    # TRT with Lambda = 3/16 and half-way bounce-back reproduces the parabola
    # to round-off (walls at y = 1/2 and y = ny - 3/2).
    p = _params(casedir, "pois_kat", cases.poiseuille(nx=3, ny=12, nz=3, loops=1, tau=0.8, magic=3 / 16,
                                                       force=1e-6))
    o = Oracle(p)
    o.advance(30000)
    ux = o.field("ux")[1, :, 1]
    nu = (p.tau - 0.5) / 3.0
    H = p.ny - 2
    y = np.arange(p.ny, dtype=np.float64)
    exact = p.force[0] / (2 * nu) * (y - 0.5) * (H + 0.5 - y)
    fl = slice(1, p.ny - 1)
    err = np.max(np.abs(ux[fl] - exact[fl])) / np.max(exact[fl])
    assert err < 1e-10, err


@pytest.mark.parametrize("coll", ["BGK", "MRT"])
def test_poiseuille_other_collisions_converge(casedir, coll):
    # BGK/MRT carry the known tau-dependent wall slip; the profile is still
    # parabolic to O(1e-2) at tau = 0.8.
    p = _params(casedir, f"pois_{coll}", cases.poiseuille(nx=3, ny=12, nz=3, loops=1, collision=coll, force=1e-6))
    o = Oracle(p)
    o.advance(20000)
    ux = o.field("ux")[1, :, 1]
    nu = (p.tau - 0.5) / 3.0
    H = p.ny - 2
    y = np.arange(p.ny, dtype=np.float64)
    exact = p.force[0] / (2 * nu) * (y - 0.5) * (H + 0.5 - y)
    fl = slice(1, p.ny - 1)
    assert np.max(np.abs(ux[fl] - exact[fl])) / np.max(exact[fl]) < 2e-2


def test_flow_mass_conservation(casedir):
    p = _params(casedir, "pois_mass", cases.poiseuille(nx=8, ny=10, nz=6, loops=1, force=1e-5, lattice="D3Q27"))
    o = Oracle(p)
    fl = initial_field(p, "flag") == 0
    m0 = o.field("rho")[fl].sum()
    o.advance(300)
    m1 = o.field("rho")[fl].sum()
    assert abs(m1 - m0) / m0 < 1e-13


def _mp(casedir, name, **kw):
    return _params(casedir, name, cases.multiphase_bubbles(**kw))


def test_multiphase_phi_conservation(casedir):
    p = _mp(casedir, "mp_cons", n=32, nz=32, bubbles=2, rmin=4, rmax=5, width=3.0, gz=-1e-5, loops=1)
    phi0 = initial_field(p, "phi")
    o = Oracle(p, phi=phi0)
    fl = initial_field(p, "flag") == 0
    s0 = o.field("phi")[fl].sum()
    o.advance(200)
    s1 = o.field("phi")[fl].sum()
    assert abs(s1 - s0) / s0 < 1e-12
    assert np.all(np.isfinite(o.field("ux")))


def test_multiphase_flat_interface_stays_tanh(casedir):
    # Gas slab (phi = 0) between two flat interfaces, periodic everywhere:
    # the equilibrium profile 1/2 (1 + tanh(2 d / W)) is (almost) steady.
    p = _mp(casedir, "mp_flat", n=4, nz=48, bubbles=0, width=4.0, gz=0.0, loops=1)
    p.bc[2] = A.MK_BC_PERIODIC
    z = np.arange(p.nz, dtype=np.float64)
    W = p.width
    prof = 0.5 * (1 + np.tanh(2 * (np.abs(z - 23.5) - 10.0) / W))
    phi0 = np.broadcast_to(prof[:, None, None], (p.nz, p.ny, p.nx)).copy()
    o = Oracle(p, phi=phi0)
    o.advance(400)
    phi = o.field("phi")[:, 1, 1]
    # the discrete equilibrium sits within 1e-2 of the continuous tanh ...
    assert np.max(np.abs(phi - prof)) < 1e-2
    # ... and is steady
    o.advance(400)
    assert np.max(np.abs(o.field("phi")[:, 1, 1] - phi)) < 5e-4
    assert np.max(np.abs(o.field("uz"))) < 1e-5


def test_multiphase_static_drop_obeys_laplace(casedir):
    # A gas drop at rest in liquid (no gravity, periodic box).  The model's
    # momentum balance is rho du/dt = -grad(cs^2 rho p*) + mu grad(phi) + rho g,
    # so the hydrodynamic pressure is p = cs^2 rho p*; its jump across the
    # interface is 2 sigma / R (Laplace), within the diffuse-interface error
    # that shrinks as W / R does (R the radius of the drop's gas volume).
    ratio = {}
    for R in (7.0, 10.0):
        p = _mp(casedir, f"mp_laplace_{int(R)}", n=32, bubbles=1, rmin=R, rmax=R, width=3.0, gz=0.0, loops=1,
                boundary="periodic periodic periodic")
        o = Oracle(p, phi=initial_field(p, "phi"))
        o.advance(1200)
        phi, rho, ps = o.field("phi"), o.field("rho"), o.field("pressure")
        pres = rho * ps / 3.0
        r_eff = (3.0 * (1.0 - phi).sum() / (4.0 * np.pi)) ** (1.0 / 3.0)
        jump = pres[phi < 0.01].mean() - pres[phi > 0.99].mean()
        ratio[R] = jump * r_eff / (2.0 * p.sigma)
    assert all(abs(v - 1.0) < 0.12 for v in ratio.values()), ratio
    assert abs(ratio[10.0] - 1.0) < abs(ratio[7.0] - 1.0), ratio


def test_thermal_diffusion_variance_rate(casedir):
    # No seed: phi = -1 everywhere, so T obeys pure D3Q7 diffusion; the
    # variance of a Gaussian grows by 2 D per step along each axis.
    n = 40
    p = _params(casedir, "diff", cases.thermal_dendrite(n=n, loops=1, D=0.1, delta=0.0))
    p.n_objects = 0
    c = (n - 1) / 2
    zz, yy, xx = np.meshgrid(*(np.arange(n, dtype=np.float64),) * 3, indexing="ij")
    r2 = (xx - c) ** 2 + (yy - c) ** 2 + (zz - c) ** 2
    T0 = 1e-3 * np.exp(-r2 / (2 * 2.0 ** 2))
    phi0 = -np.ones_like(T0)
    o = Oracle(p, phi=phi0, T=T0)

    def var_x(T):
        return float(((xx - c) ** 2 * T).sum() / T.sum())

    o.advance(20)
    v1 = var_x(o.field("T"))
    o.advance(40)
    v2 = var_x(o.field("T"))
    rate = (v2 - v1) / 40
    assert abs(rate - 2 * p.D) / (2 * p.D) < 2e-3, rate


def test_thermal_dendrite_cubic_symmetry(casedir):
    n = 25
    p = _params(casedir, "sym", cases.thermal_dendrite(n=n, loops=1, radius=4.0))
    o = Oracle(p, phi=initial_field(p, "phi"))
    o.advance(120)
    phi = o.field("phi")
    assert np.max(np.abs(phi - phi.transpose(0, 2, 1))) < 1e-12
    assert np.max(np.abs(phi - phi.transpose(2, 1, 0))) < 1e-12
    assert np.max(np.abs(phi - phi[::-1, :, :])) < 1e-12
    # the seed has grown (undercooled melt)
    assert (phi > 0).sum() > (initial_field(p, "phi") > 0).sum()


def test_thermal_dendrite_enthalpy_conserved(casedir):
    # sum(T - phi_prev/2) is invariant in a closed box.
    n = 20
    p = _params(casedir, "enth", cases.thermal_dendrite(n=n, loops=1, radius=4.0))
    o = Oracle(p, phi=initial_field(p, "phi"))

    def H():
        phi = o.field("phi")
        dphi = o.field("dphi")
        return float((o.field("T") - 0.5 * (phi - dphi)).sum())

    o.advance(2)
    h0 = H()
    o.advance(150)
    assert abs(H() - h0) / abs(h0) < 1e-12


def test_solutal_no_seed_is_pure_diffusion(casedir):
    # No seed: phi = -1 (liquid, capacity 1, D = D_l), so U diffuses with
    # variance growth 2 D_l per step and the total is conserved.
    n = 40
    p = _params(casedir, "sol_diff", cases.solutal_dendrite(n=n, loops=1, D=0.1, delta=0.0))
    p.n_objects = 0
    c = (n - 1) / 2
    zz, yy, xx = np.meshgrid(*(np.arange(n, dtype=np.float64),) * 3, indexing="ij")
    U0 = 1e-3 * np.exp(-((xx - c) ** 2 + (yy - c) ** 2 + (zz - c) ** 2) / (2 * 2.0 ** 2))
    o = Oracle(p, phi=-np.ones_like(U0), Cc=U0)

    def var_x(U):
        return float(((xx - c) ** 2 * U).sum() / U.sum())

    o.advance(20)
    v1, s1 = var_x(o.field("C")), o.field("C").sum()
    o.advance(40)
    v2, s2 = var_x(o.field("C")), o.field("C").sum()
    assert abs((v2 - v1) / 40 - 2 * p.D) / (2 * p.D) < 2e-3
    assert abs(s2 - s1) / abs(s1) < 1e-12


def test_solutal_seed_grows_rejects_solute_symmetrically(casedir):
    # seed centred between cells: no cell sits where grad phi vanishes
    n = 24
    p = _params(casedir, "sol_seed", cases.solutal_dendrite(n=n, loops=1, seeds=[((11.5, 11.5, 11.5), (0, 0, 0),
                                                                                    4.0)]))
    o = Oracle(p, phi=initial_field(p, "phi"))
    U0 = o.field("C").copy()
    o.advance(150)
    phi, U = o.field("phi"), o.field("C")
    assert (phi > 0).sum() > (initial_field(p, "phi") > 0).sum()
    # solute is rejected into the liquid ahead of the interface: U rises above the far field there
    liquid = phi < -0.5
    assert U[liquid].max() > U0.max() + 1e-3
    assert np.max(np.abs(phi - phi.transpose(0, 2, 1))) < 1e-12
    assert np.max(np.abs(phi - phi.transpose(2, 1, 0))) < 1e-12
    assert np.max(np.abs(U - U.transpose(2, 1, 0))) < 1e-12


# ---------------------------------------------------------------- anisotropy kinds
from _oracle import anisotropy as orc_aniso  # noqa: E402

KINDS = {"cubic": (A.MK_ANISO_CUBIC, 0.05, 0.0), "cbc": (A.MK_ANISO_CBC, 0.03, -0.02),
         "hcp": (A.MK_ANISO_HCP, 0.02, 0.03), "facet": (A.MK_ANISO_FACET, 0.1, 0.05)}


@pytest.mark.parametrize("name", sorted(KINDS))
def test_anisotropy_gradient_matches_finite_differences(name):
    kind, e4, e2 = KINDS[name]
    rng = np.random.default_rng(3)
    for _ in range(20):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        a, g = orc_aniso(kind, e4, e2, n)
        h = 1e-6
        for q in range(3):
            dp, dm = n.copy(), n.copy()
            dp[q] += h
            dm[q] -= h
            fd = (orc_aniso(kind, e4, e2, dp)[0] - orc_aniso(kind, e4, e2, dm)[0]) / (2 * h)
            assert abs(fd - g[q]) < 1e-8, (name, n, q, fd, g[q])


def test_anisotropy_values_at_special_directions():
    e4, e2 = 0.04, 0.03
    s = 1 / np.sqrt(3)
    # cubic: a(100) = 1 + e4, a(111) = 1 - 5 e4 / 3
    assert orc_aniso(A.MK_ANISO_CUBIC, e4, 0, [1, 0, 0])[0] == pytest.approx(1 + e4, abs=1e-15)
    assert orc_aniso(A.MK_ANISO_CUBIC, e4, 0, [s, s, s])[0] == pytest.approx(1 - 5 * e4 / 3, abs=1e-15)
    # cbc: the harmonics average to zero over the sphere; a(100) = 1 + 0.4 e4 + 4/7 e2
    assert orc_aniso(A.MK_ANISO_CBC, e4, e2, [1, 0, 0])[0] == pytest.approx(1 + 0.4 * e4 + 4 / 7 * e2, abs=1e-15)
    # hcp: six-fold in the basal plane, a(c axis) = 1 + e2
    c, sn = np.cos(np.pi / 6), np.sin(np.pi / 6)
    assert orc_aniso(A.MK_ANISO_HCP, e4, e2, [1, 0, 0])[0] == pytest.approx(1 + e4 - e2, abs=1e-15)
    assert orc_aniso(A.MK_ANISO_HCP, e4, e2, [c, sn, 0])[0] == pytest.approx(1 - e4 - e2, abs=1e-14)
    assert orc_aniso(A.MK_ANISO_HCP, e4, e2, [0, 0, 1])[0] == pytest.approx(1 + e2, abs=1e-15)
    for k in range(6):
        t = k * np.pi / 3 + 0.2
        assert orc_aniso(A.MK_ANISO_HCP, e4, e2, [np.cos(t), np.sin(t), 0])[0] == pytest.approx(
            orc_aniso(A.MK_ANISO_HCP, e4, e2, [np.cos(0.2), np.sin(0.2), 0])[0], abs=1e-14)
    # facet: cusp minimum a = 1 at the cube directions, larger elsewhere
    assert orc_aniso(A.MK_ANISO_FACET, 0.1, 0.05, [0, 1, 0])[0] == pytest.approx(1.0, abs=1e-15)
    assert orc_aniso(A.MK_ANISO_FACET, 0.1, 0.05, [s, s, s])[0] > 1.05


@pytest.mark.parametrize("name", ["cbc", "facet"])
def test_cubic_kinds_keep_cubic_symmetry(casedir, name):
    kind, e4, e2 = KINDS[name]
    n = 21
    p = _params(casedir, f"sym_{name}", cases.thermal_dendrite(n=n, loops=1, radius=4.0, eps4=e4, aniso=name,
                                                               eps2=e2))
    assert p.aniso == kind
    o = Oracle(p, phi=initial_field(p, "phi"))
    o.advance(80)
    phi = o.field("phi")
    assert np.max(np.abs(phi - phi.transpose(0, 2, 1))) < 1e-12
    assert np.max(np.abs(phi - phi.transpose(2, 1, 0))) < 1e-12
    assert (phi > 0).sum() > (initial_field(p, "phi") > 0).sum()


def test_hcp_keeps_its_mirror_symmetries_and_differs_from_cubic(casedir):
    n = 21
    p = _params(casedir, "sym_hcp", cases.thermal_dendrite(n=n, loops=1, radius=4.0, eps4=0.03, aniso="hcp",
                                                           eps2=0.02))
    o = Oracle(p, phi=initial_field(p, "phi"))
    o.advance(80)
    phi = o.field("phi")
    for ax in range(3):
        assert np.max(np.abs(phi - np.flip(phi, axis=ax))) < 1e-12
    # six-fold in the basal (x, y) plane: not symmetric under x <-> y, unlike a cubic crystal
    assert np.max(np.abs(phi - phi.transpose(0, 2, 1))) > 1e-6


# ---------------------------------------------------------------- adjoint
@pytest.mark.parametrize("aniso", ["cubic", "facet"])
def test_oracle_adjoint_matches_central_differences(casedir, aniso):
    # the discrete adjoint is the exact gradient of the discrete loop: central
    # differences with h = 1e-4 agree to their O(h^2) truncation
    n, steps, h = 10, 12, 1e-4
    e2 = 0.03 if aniso != "cubic" else 0.0

    def params(eps4, delta):
        return _params(casedir, f"adj_{aniso}", cases.thermal_dendrite(n=n, loops=1, radius=3.0, eps4=eps4,
                                                                        delta=delta, aniso=aniso, eps2=e2))

    def phi_after(p):
        o = Oracle(p, phi=initial_field(p, "phi"), T=initial_field(p, "T"))
        o.advance(steps)
        return o.field("phi")

    target = phi_after(params(0.04, 0.50))
    p0 = params(0.05, 0.55)
    g = Oracle(p0, phi=initial_field(p0, "phi"), T=initial_field(p0, "T")).backward(target, steps)

    def loss(p):
        p.tau0 = p0.tau0  # tau_T and Delta derivatives hold tau0 fixed
        return float(((phi_after(p) - target) ** 2).sum())

    assert g["loss"] == pytest.approx(loss(params(0.05, 0.55)), rel=1e-13)
    fd_e = (loss(params(0.05 + h, 0.55)) - loss(params(0.05 - h, 0.55))) / (2 * h)
    fd_d = (loss(params(0.05, 0.55 + h)) - loss(params(0.05, 0.55 - h))) / (2 * h)
    pp, pm = params(0.05, 0.55), params(0.05, 0.55)
    pp.D += h / 4  # tau_T = 4 D + 1/2
    pm.D -= h / 4
    fd_t = (loss(pp) - loss(pm)) / (2 * h)
    assert g["d_eps4"] == pytest.approx(fd_e, rel=1e-6)
    assert g["d_delta"] == pytest.approx(fd_d, rel=1e-6)
    assert g["d_tau_t"] == pytest.approx(fd_t, rel=1e-6)


# ---------------------------------------------------------------- plates and convection
def test_couette_linear_profile_exact(casedir):
    # moving upper plate, half-way walls at y = 1/2 and y = ny - 3/2: the
    # steady linear profile is exact for the lattice
    U = 1e-2
    p = _params(casedir, "couette", cases.couette(nx=3, ny=14, nz=3, U=U))
    o = Oracle(p)
    o.advance(30000)
    ux = o.field("ux")[1, :, 1]
    H = p.ny - 2
    y = np.arange(p.ny, dtype=np.float64)
    exact = U * (y - 0.5) / H
    fl = slice(1, p.ny - 1)
    assert np.max(np.abs(ux[fl] - exact[fl])) < 1e-9 * U


def test_conduction_between_plates_is_linear_and_nu_is_one(casedir):
    # no buoyancy: the plates impose a linear profile (exact for the D3Q7
    # anti-bounce-back), no flow, Nu = 1
    p = _params(casedir, "cond", cases.convection(nx=8, ny=3, nz=12, Ra=1e3, beta=0.0))
    o = Oracle(p, T=initial_field(p, "T"))
    o.advance(8000)
    T = o.field("T")[:, 1, 3]
    H = p.nz - 2
    z = np.arange(p.nz, dtype=np.float64)
    exact = 1.0 - (z - 0.5) / H
    fl = slice(1, p.nz - 1)
    assert np.max(np.abs(T[fl] - exact[fl])) < 1e-9
    assert np.max(np.abs(o.field("uz"))) < 1e-12


def _nusselt(o, p):
    T, uz = o.field("T"), o.field("uz")
    fl = initial_field(p, "flag") == 0
    H = p.nz - 2
    return 1.0 + (uz * T)[fl].mean() * H / (p.D * (p.wall_value[0] - p.wall_value[1]))


def test_rbc_below_onset_decays_to_conduction(casedir):
    # Ra = 1000 < 1708 (the rigid-rigid critical value): the seeded roll decays
    # (what stays is the O(Ma^2) hydrostatic compressibility residue)
    p = _params(casedir, "rbc_sub", cases.convection(nx=24, ny=3, nz=14, Ra=1000.0))
    o = Oracle(p, T=initial_field(p, "T"))
    o.advance(8000)
    assert abs(_nusselt(o, p) - 1.0) < 1e-3
    assert np.max(np.abs(o.field("uz"))) < 2e-5


def test_rbc_above_onset_convects(casedir):
    # Ra = 1e4, Pr = 0.71, laterally periodic layer of aspect ratio 2 (one
    # roll pair near the critical wavelength): steady rolls.  The periodic-
    # layer value is Nu ~ 2.66 (Clever & Busse 1974, alpha ~ 3.1); this
    # lattice gives 2.72 at H = 12 and 2.67 at H = 24 (converging).
    p = _params(casedir, "rbc_sup", cases.convection(nx=24, ny=3, nz=14, Ra=1e4))
    o = Oracle(p, T=initial_field(p, "T"))
    o.advance(25000)
    nu = _nusselt(o, p)
    assert 2.6 < nu < 2.8, nu


# ----------------------------------------------------- flow + dendrite (a1/a7/a8)
def test_flow_dendrite_uniform_inflow_is_steady(casedir):
    # All liquid at the far-field temperature: the inflow / outflow faces keep
    # the uniform stream u0 and the uniform temperature to round-off.
    p = _params(casedir, "fd_uniform", cases.flow_dendrite(nx=12, ny=6, nz=5, radius=3.0, u_in=0.03))
    sh = (p.nz, p.ny, p.nx)
    o = Oracle(p, phi=-np.ones(sh), T=np.full(sh, -p.delta))
    o.advance(40)
    assert np.abs(o.field("ux") - 0.03).max() < 1e-14
    assert np.abs(o.field("uy")).max() < 1e-14 and np.abs(o.field("uz")).max() < 1e-14
    assert np.abs(o.field("rho") - 1.0).max() < 1e-14
    assert np.abs(o.field("T") + p.delta).max() < 1e-14
    assert np.abs(o.field("phi") + 1.0).max() == 0.0


def test_flow_dendrite_at_rest_is_the_thermal_dendrite(casedir):
    # Closed faces and no inflow: the flow stays at rest (the porous
    # bounce-back of an equilibrium at u = 0 is the identity) and the phase
    # field and temperature are those of the thermal dendrite model.
    p = _params(casedir, "fd_rest", cases.flow_dendrite(nx=20, ny=18, nz=16, radius=4.0, u_in=0.0, inlet=False))
    q = A.MkParams.from_buffer_copy(p)
    q.model = A.MK_MODEL_THERMAL_DENDRITE
    phi, T = initial_field(p, "phi"), initial_field(p, "T")
    o1, o2 = Oracle(p, phi=phi, T=T), Oracle(q, phi=phi, T=T)
    o1.advance(60)
    o2.advance(60)
    assert (o1.field("phi") > 0).sum() > 500  # the seed grew
    assert np.abs(o1.field("phi") - o2.field("phi")).max() < 1e-12
    assert np.abs(o1.field("T") - o2.field("T")).max() < 1e-12
    assert np.abs(o1.field("ux")).max() < 1e-15 and np.abs(o1.field("rho") - 1.0).max() < 1e-14


def test_flow_dendrite_advects_heat_at_the_flow_speed(casedir):
    # A temperature pulse in the uniform stream: its centroid moves at u0
    # (first moment of w T (1 + 4 e.u) is T u) and the heat is conserved.
    p = _params(casedir, "fd_adv", cases.flow_dendrite(nx=64, ny=4, nz=4, radius=3.0, u_in=0.05, D=0.02))
    sh = (p.nz, p.ny, p.nx)
    x = np.arange(p.nx)
    T = np.broadcast_to(-p.delta + 0.1 * np.exp(-((x - 16.0) / 3.0) ** 2), sh).copy()
    o = Oracle(p, phi=-np.ones(sh), T=T)

    def moments():
        e = o.field("T")[0, 0] + p.delta
        return (e * x).sum() / e.sum(), e.sum()

    c0, h0 = moments()
    o.advance(300)
    c1, h1 = moments()
    assert abs((c1 - c0) - 0.05 * 300) < 1e-6
    assert abs(h1 - h0) / h0 < 1e-10


def test_flow_dendrite_solid_stops_the_flow(casedir):
    # The porous bounce-back brings the velocity inside the crystal
    # (phi > 0.99) to below 1 % of the stream around it.
    p = _params(casedir, "fd_core", cases.flow_dendrite(nx=40, ny=24, nz=24, radius=6.0, u_in=0.02, delta=0.3))
    o = Oracle(p, phi=initial_field(p, "phi"), T=initial_field(p, "T"))
    o.advance(400)
    phi = o.field("phi")
    u = np.sqrt(o.field("ux") ** 2 + o.field("uy") ** 2 + o.field("uz") ** 2)
    core = phi > 0.99
    assert core.sum() > 50
    assert u[core].max() < 0.01 * 0.02
    assert u[phi < -0.99].mean() > 0.5 * 0.02
    flag = o.field("flag")
    assert np.array_equal(flag == A.MK_FLAG_SOLID, phi > 0)


# ------------------------------------------------- flow + solutal dendrite (f-2)
def test_flow_solutal_uniform_inflow_is_steady(casedir):
    # All liquid at the far-field supersaturation: the faces keep the uniform
    # stream and the uniform solute to round-off.
    p = _params(casedir, "fs_uniform", cases.flow_solutal_dendrite(nx=12, ny=6, nz=5, radius=3.0, u_in=0.03))
    sh = (p.nz, p.ny, p.nx)
    o = Oracle(p, phi=-np.ones(sh), Cc=np.full(sh, -p.delta))
    o.advance(40)
    assert np.abs(o.field("ux") - 0.03).max() < 1e-14
    assert np.abs(o.field("C") + p.delta).max() < 1e-14
    assert np.abs(o.field("phi") + 1.0).max() == 0.0


def test_flow_solutal_at_rest_is_the_solutal_dendrite(casedir):
    # Closed faces and no inflow: the flow stays at rest and the phase field
    # and the solute are those of the solutal dendrite model.
    p = _params(casedir, "fs_rest", cases.flow_solutal_dendrite(nx=20, ny=18, nz=16, radius=4.0, u_in=0.0,
                                                                inlet=False))
    q = A.MkParams.from_buffer_copy(p)
    q.model = A.MK_MODEL_SOLUTAL_DENDRITE
    phi, U = initial_field(p, "phi"), initial_field(p, "C")
    o1, o2 = Oracle(p, phi=phi, Cc=U), Oracle(q, phi=phi, Cc=U)
    o1.advance(60)
    o2.advance(60)
    assert (o1.field("phi") > 0).sum() > 200  # the seed grew
    assert np.abs(o1.field("phi") - o2.field("phi")).max() < 1e-12
    assert np.abs(o1.field("C") - o2.field("C")).max() < 1e-12
    assert np.abs(o1.field("ux")).max() < 1e-15


def test_flow_solutal_advects_solute_at_the_flow_speed(casedir):
    # A solute pulse in the uniform stream of liquid (capacity 1, no
    # anti-trapping current): its centroid moves at u0 (first moment U u of
    # the advected equilibrium) and the solute is conserved.
    p = _params(casedir, "fs_adv", cases.flow_solutal_dendrite(nx=64, ny=4, nz=4, radius=3.0, u_in=0.05, D=0.02))
    sh = (p.nz, p.ny, p.nx)
    x = np.arange(p.nx)
    U = np.broadcast_to(-p.delta + 0.1 * np.exp(-((x - 16.0) / 3.0) ** 2), sh).copy()
    o = Oracle(p, phi=-np.ones(sh), Cc=U)

    def moments():
        e = o.field("C")[0, 0] + p.delta
        return (e * x).sum() / e.sum(), e.sum()

    c0, m0 = moments()
    o.advance(300)
    c1, m1 = moments()
    assert abs((c1 - c0) - 0.05 * 300) < 1e-6
    assert abs(m1 - m0) / m0 < 1e-10


# ---------------------------------------------------------- multigrain (f-3)
def test_multigrain_single_grain_conserves_phi_and_heat(casedir):
    # one grain: conservative Allen-Cahn (no penalty on grain 0), closed faces:
    # sum phi_0 and the enthalpy sum (T - phi/2) stay exact
    p = _params(casedir, "mg_one", cases.multigrain(n=20, seeds=[(9.5, 9.5, 9.5, 5.0)], loops=10))
    o = Oracle(p, phi=initial_field(p, "phi"), T=initial_field(p, "T"))
    m0 = o.grain(0).sum()
    h0 = (o.field("T") - 0.5 * o.field("phi")).sum()
    o.advance(150)
    assert abs(o.grain(0).sum() - m0) < 1e-10 * abs(m0)
    assert abs((o.field("T") - 0.5 * o.field("phi")).sum() - h0) < 1e-9
    assert np.array_equal(o.field("phi"), o.grain(0))  # N = 1: phi = phi_0


def test_multigrain_flat_interface_is_steady(casedir):
    # the Chai flux holds phi = tanh(x / (sqrt2 W0)); a seed of radius 1000 far
    # away gives a flat front
    p = _params(casedir, "mg_flat", cases.multigrain(n=32, ny=4, nz=4, seeds=[(-984.0, 1.5, 1.5, 1000.0)], loops=10))
    o = Oracle(p, phi=initial_field(p, "phi"), T=initial_field(p, "T"))
    a0 = o.grain(0)[0, 0].copy()
    o.advance(200)
    a1 = o.grain(0)[0, 0].copy()
    o.advance(200)
    a2 = o.grain(0)[0, 0]
    # the lattice settles within 1e-2 of the tanh (its discrete steady profile),
    # then stays put
    assert np.abs(a1 - a0).max() < 1e-2
    assert np.abs(a2 - a1).max() < 1e-5


def test_multigrain_penalty_separates_grains(casedir):
    # two overlapping grains: grain 0 (no penalty) is conserved exactly, grain 1
    # loses order parameter where it overlaps grain 0, and the overlap shrinks
    p = _params(casedir, "mg_two", cases.multigrain(n=32, loops=10))
    o = Oracle(p, phi=initial_field(p, "phi"), T=initial_field(p, "T"))

    def stats():
        g0, g1 = o.grain(0), o.grain(1)
        return g0.sum(), g1.sum(), (0.5 * (1 + g0) * (0.5 * (1 + g1)) ** 2).sum()

    s0, s1, ov0 = stats()
    o.advance(200)
    t0, t1, ov1 = stats()
    assert abs(t0 - s0) < 1e-10 * abs(s0)
    assert t1 < s1
    assert ov1 < 0.5 * ov0
    assert set(np.unique(o.field("grain"))) == {0.0, 1.0}
