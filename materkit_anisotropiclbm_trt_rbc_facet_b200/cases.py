"""BoltzTechs XML cases of the five benchmark configurations.

Each case is a complete BoltzTechs file (the tag set of
MaterKit/BoltzTechs - thermal.xml and BoltzTechs - multiPhaseFlow.xml) plus a
``<b200>`` element with the lattice-unit values the configuration names.  The
generators take overrides so tests run the same case at reduced size.
"""
from __future__ import annotations

import os

_HEADER = """<?xml version="1.0" encoding="utf-8"?>
<MaterKit>
  <calcMode> <dendrite> {dendrite} </dendrite> <flowField> {flow} </flowField> </calcMode>
  <output> <numLoops> {loops} </numLoops> <numFrames> {frames} </numFrames> </output>
  <geometry> <MeshXYZ> {nx} {ny} {nz} </MeshXYZ> <Gravity> 0.0 0.0 0.0 </Gravity> </geometry>
  <numerics> <mk_dx> 1.0 </mk_dx> <mk_dt> 1.0 </mk_dt> <stepSize> -1.0 </stepSize>
    <omega_f> -1.0 </omega_f> <omega_g> -1.0 </omega_g> <omega_h> -1.0 </omega_h> </numerics>
"""


def poiseuille(nx=64, ny=32, nz=32, loops=2000, precision="fp64", collision="TRT", lattice="D3Q19",
               tau=0.8, magic=0.1875, force=1e-6) -> str:
    """Config 1: 3D Poiseuille channel, D3Q19 TRT, walls at y = 0 and y = ny-1."""
    return _HEADER.format(dendrite="false", flow="true", loops=loops, frames=min(loops, 100), nx=nx, ny=ny, nz=nz) + f"""
  <flow> <acceleration> {force} 0.0 0.0 </acceleration> <velocityInlet> 0 0 0 </velocityInlet> </flow>
  <b200>
    <model> flow </model> <lattice> {lattice} </lattice> <collision> {collision} </collision>
    <precision> {precision} </precision> <boundary> periodic walls periodic </boundary>
    <tau> {tau} </tau> <magic> {magic} </magic> <rho0> 1.0 </rho0> <force> {force} 0.0 0.0 </force>
  </b200>
</MaterKit>
"""


def thermal_dendrite(n=128, loops=5000, precision="fp32", eps4=0.05, W0=1.5, lam=10.0, delta=0.55, D=0.1,
                     radius=8.0, tau0=None, center=None, aniso="cubic", eps2=0.0) -> str:
    """Config 2: D3Q7 thermal lattice + anisotropic phase field, one centred seed.

    `aniso` selects the anisotropy kind (cubic, cbc, hcp, facet) with `eps4`
    and `eps2` its two coefficients."""
    c = center if center is not None else ((n - 1) / 2.0,) * 3
    extra = f"<tau0> {tau0} </tau0>" if tau0 else ""
    extra += f" <anisotropyKind> {aniso} </anisotropyKind> <eps2> {eps2} </eps2>"
    return _HEADER.format(dendrite="true", flow="false", loops=loops, frames=min(loops, 100), nx=n, ny=n, nz=n) + f"""
  <phasechange>
    <d0> 0.138486 </d0> <lambda> {lam} </lambda> <anisotropy> {eps4} </anisotropy> <W0> 1.0 </W0> <t0> 1.0 </t0>
    <seed> <number> 1 </number> <center> {c[0]} {c[1]} {c[2]} </center> <angle> 0 0 0 </angle>
      <radius> {radius} </radius> </seed>
  </phasechange>
  <temperature> <iniValue> {-delta} </iniValue> <undercooling> {delta} </undercooling>
    <alphaFluid> {D} </alphaFluid> <alphaSolid> {D} </alphaSolid> <beta> 0.0 </beta> </temperature>
  <b200>
    <model> thermal_dendrite </model> <precision> {precision} </precision>
    <boundary> closed closed closed </boundary>
    <eps4> {eps4} </eps4> <W0> {W0} </W0> <lambda> {lam} </lambda> <delta> {delta} </delta>
    <diffusivity> {D} </diffusivity> {extra}
  </b200>
</MaterKit>
"""


def solutal_dendrite(n=64, ny=None, nz=None, loops=3000, precision="fp32", eps4=0.04, W0=1.5, lam=10.0,
                     delta=0.55, D=0.1, D_s=1e-4, k=0.15, seeds=None, tau0=None, aniso="cubic", eps2=0.0) -> str:
    """Config 4 element: D3Q7 solutal lattice + anisotropic phase field, closed faces.

    `seeds` is a list of (center xyz, angles xyz in degrees, radius); default one
    centred seed of radius 6.  `aniso` / `eps2` as in thermal_dendrite.
    """
    ny = n if ny is None else ny
    nz = n if nz is None else nz
    if seeds is None:
        seeds = [(((n - 1) / 2.0, (ny - 1) / 2.0, (nz - 1) / 2.0), (0.0, 0.0, 0.0), 6.0)]
    cen = " ".join(f"{c[0]} {c[1]} {c[2]}" for c, _, _ in seeds)
    ang = " ".join(f"{a[0]} {a[1]} {a[2]}" for _, a, _ in seeds)
    rad = " ".join(f"{r}" for _, _, r in seeds)
    t0 = f"<tau0> {tau0} </tau0>" if tau0 else ""
    t0 += f" <anisotropyKind> {aniso} </anisotropyKind> <eps2> {eps2} </eps2>"
    return _HEADER.format(dendrite="true", flow="false", loops=loops, frames=min(loops, 100), nx=n, ny=ny, nz=nz) + f"""
  <phasechange>
    <d0> 0.2762 </d0> <lambda> {lam} </lambda> <anisotropy> {eps4} </anisotropy> <W0> 1.0 </W0> <t0> 1.0 </t0>
  </phasechange>
  <composition> <number> 1 </number> <diffFluid> {D} </diffFluid> <diffSolid> {D_s} </diffSolid>
    <iniValue> {-delta} </iniValue> <partition> {k} </partition> </composition>
  <b200>
    <model> solutal_dendrite </model> <precision> {precision} </precision>
    <boundary> closed closed closed </boundary>
    <eps4> {eps4} </eps4> <W0> {W0} </W0> <lambda> {lam} </lambda> <delta> {delta} </delta>
    <diffusivity> {D} </diffusivity> <diffSolid> {D_s} </diffSolid> <partition> {k} </partition> {t0}
    <objects> <number> {len(seeds)} </number> <center> {cen} </center> <angle> {ang} </angle>
      <radius> {rad} </radius> </objects>
  </b200>
</MaterKit>
"""


def multiphase_bubbles(n=256, nz=None, loops=10000, precision="fp32", bubbles=24, rmin=8.0, rmax=16.0,
                       seed=0xB200, width=4.0, sigma=1e-3, rho_ratio=10.0, nu_ratio=10.0, tau_l=0.8,
                       mobility=0.05, gz=-1e-6, contact_angle=90.0, ny=None,
                       boundary="periodic periodic walls") -> str:
    """Config 3 (headline): 256^3 D3Q19 MRT + D3Q19 conservative Allen-Cahn, 24 bubbles.

    Liquid (phi = 1) density 1, gas density 1/rho_ratio; liquid kinematic
    viscosity nu_l = (tau_l - 1/2)/3, gas nu_l / nu_ratio.  `ny` (default n)
    and `boundary` (per axis x y z) reshape the box for tests.
    """
    nz = n if nz is None else nz
    ny = n if ny is None else ny
    nu_l = (tau_l - 0.5) / 3.0
    tau_g = 3.0 * nu_l / nu_ratio + 0.5
    return _HEADER.format(dendrite="false", flow="true", loops=loops, frames=min(loops, 100), nx=n, ny=ny, nz=nz) + f"""
  <multiphases>
    <fluidDense> <kinematicViscosity> {nu_l} </kinematicViscosity> <density> 1.0 </density> </fluidDense>
    <fluidRare> <kinematicViscosity> {nu_l / nu_ratio} </kinematicViscosity> <density> {1.0 / rho_ratio} </density> </fluidRare>
    <force> 0.0 0.0 0.0 </force> <W0> {width} </W0> <Mobility> {mobility} </Mobility> <sigma> {sigma} </sigma>
    <contactAngle> {contact_angle} </contactAngle>
  </multiphases>
  <b200>
    <model> multiphase </model> <collision> MRT </collision> <precision> {precision} </precision>
    <boundary> {boundary} </boundary>
    <rhoL> 1.0 </rhoL> <rhoG> {1.0 / rho_ratio} </rhoG> <tauL> {tau_l} </tauL> <tauG> {tau_g} </tauG>
    <sigma> {sigma} </sigma> <width> {width} </width> <mobility> {mobility} </mobility>
    <contactAngle> {contact_angle} </contactAngle> <force> 0.0 0.0 {gz} </force>
    <random> <bubbles> {bubbles} </bubbles> <radiusMin> {rmin} </radiusMin> <radiusMax> {rmax} </radiusMax>
      <gap> {2 * width} </gap> <seed> {hex(seed)} </seed> </random>
  </b200>
</MaterKit>
"""


def convection(nx=64, ny=3, nz=34, axis="z", Ra=1e4, Pr=0.71, U=0.05, T_hot=1.0, T_cold=0.0, loops=20000,
               precision="fp64", collision="TRT", lattice="D3Q19", beta=None) -> str:
    """Rayleigh-Benard convection: hot plate below, cold plate above along `axis`
    (walls there, periodic elsewhere), gravity g = 1 along -axis.  The free-fall
    velocity U = sqrt(g beta dT H) sets the Mach number; then
    nu = U H sqrt(Pr/Ra), kappa = nu/Pr, tau = 3 nu + 1/2, H the layer
    thickness between the half-way plates.  `beta` overrides the expansion
    coefficient (0: pure conduction)."""
    a = "xyz".index(axis)
    n3 = [nx, ny, nz]
    H = n3[a] - 2
    dT = T_hot - T_cold
    nu = U * H * (Pr / Ra) ** 0.5
    kappa = nu / Pr
    tau = 3.0 * nu + 0.5
    beta = U * U / (dT * H) if beta is None else beta
    g = [0.0, 0.0, 0.0]
    g[a] = -1.0
    bc = ["periodic"] * 3
    bc[a] = "walls"
    return _HEADER.format(dendrite="false", flow="true", loops=loops, frames=min(loops, 100), nx=nx, ny=ny, nz=nz) + f"""
  <b200>
    <model> convection </model> <lattice> {lattice} </lattice> <collision> {collision} </collision>
    <precision> {precision} </precision> <boundary> {" ".join(bc)} </boundary>
    <tau> {tau} </tau> <magic> 0.1875 </magic> <rho0> 1.0 </rho0> <diffusivity> {kappa} </diffusivity>
    <force> {g[0]} {g[1]} {g[2]} </force> <beta> {beta} </beta> <sRef> {0.5 * (T_hot + T_cold)} </sRef>
    <wallAxis> {axis} </wallAxis> <wallValue> {T_hot} {T_cold} </wallValue>
  </b200>
</MaterKit>
"""


def couette(nx=4, ny=18, nz=4, U=1e-2, loops=20000, precision="fp64", collision="TRT", lattice="D3Q19",
            tau=0.8) -> str:
    """Plane Couette flow: plates normal to y, the upper one moving with U along x."""
    return _HEADER.format(dendrite="false", flow="true", loops=loops, frames=min(loops, 100), nx=nx, ny=ny, nz=nz) + f"""
  <b200>
    <model> flow </model> <lattice> {lattice} </lattice> <collision> {collision} </collision>
    <precision> {precision} </precision> <boundary> periodic walls periodic </boundary>
    <tau> {tau} </tau> <magic> 0.1875 </magic> <rho0> 1.0 </rho0> <force> 0 0 0 </force>
    <wallAxis> y </wallAxis> <wallVelocity> 0 0 0 {U} 0 0 </wallVelocity>
  </b200>
</MaterKit>
"""


def flow_dendrite(nx=96, ny=64, nz=64, loops=3000, precision="fp32", u_in=0.02, eps4=0.05, W0=1.5, lam=10.0,
                  delta=0.55, D=0.1, radius=6.0, center=None, tau=0.8, inlet=True, collision="TRT",
                  lattice="D3Q19") -> str:
    """Thermal dendrite in a melt flowing in at x = 0 with `u_in` and out at
    x = nx - 1 (run_flow_thermal_dendrite); periodic across.  `inlet=False`
    closes the x faces (the flow then stays at rest)."""
    c = center if center is not None else (nx / 3.0, (ny - 1) / 2.0, (nz - 1) / 2.0)
    bc = "closed periodic periodic" if inlet else "closed closed closed"
    return _HEADER.format(dendrite="true", flow="true", loops=loops, frames=min(loops, 100), nx=nx, ny=ny, nz=nz) + f"""
  <flow> <acceleration> 0.0 0.0 0.0 </acceleration> <velocityInlet> {u_in} 0.0 0.0 </velocityInlet> </flow>
  <phasechange>
    <d0> 0.138486 </d0> <lambda> {lam} </lambda> <anisotropy> {eps4} </anisotropy> <W0> 1.0 </W0> <t0> 1.0 </t0>
    <seed> <number> 1 </number> <center> {c[0]} {c[1]} {c[2]} </center> <angle> 0 0 0 </angle>
      <radius> {radius} </radius> </seed>
  </phasechange>
  <temperature> <iniValue> {-delta} </iniValue> <undercooling> {delta} </undercooling>
    <alphaFluid> {D} </alphaFluid> <alphaSolid> {D} </alphaSolid> <beta> 0.0 </beta> </temperature>
  <b200>
    <model> flow_dendrite </model> <precision> {precision} </precision> <boundary> {bc} </boundary>
    <lattice> {lattice} </lattice> <collision> {collision} </collision>
    <tau> {tau} </tau> <magic> 0.1875 </magic> <rho0> 1.0 </rho0> <velocity> {u_in} 0 0 </velocity>
    <inlet> {1 if inlet else 0} </inlet>
    <eps4> {eps4} </eps4> <W0> {W0} </W0> <lambda> {lam} </lambda> <delta> {delta} </delta>
    <diffusivity> {D} </diffusivity>
  </b200>
</MaterKit>
"""


def flow_solutal_dendrite(nx=96, ny=64, nz=64, loops=3000, precision="fp32", u_in=0.02, eps4=0.04, W0=1.5,
                          lam=10.0, delta=0.55, D=0.1, D_s=1e-4, k=0.15, radius=6.0, center=None, tau=0.8,
                          inlet=True, collision="TRT", lattice="D3Q19") -> str:
    """Solutal dendrite in a melt flowing in at x = 0 with `u_in` and out at
    x = nx - 1 (run_flow_solutal_dendrite); periodic across.  `inlet=False`
    closes the x faces (the flow then stays at rest)."""
    c = center if center is not None else (nx / 3.0, (ny - 1) / 2.0, (nz - 1) / 2.0)
    bc = "closed periodic periodic" if inlet else "closed closed closed"
    return _HEADER.format(dendrite="true", flow="true", loops=loops, frames=min(loops, 100), nx=nx, ny=ny, nz=nz) + f"""
  <flow> <acceleration> 0.0 0.0 0.0 </acceleration> <velocityInlet> {u_in} 0.0 0.0 </velocityInlet> </flow>
  <phasechange>
    <d0> 0.2762 </d0> <lambda> {lam} </lambda> <anisotropy> {eps4} </anisotropy> <W0> 1.0 </W0> <t0> 1.0 </t0>
    <seed> <number> 1 </number> <center> {c[0]} {c[1]} {c[2]} </center> <angle> 0 0 0 </angle>
      <radius> {radius} </radius> </seed>
  </phasechange>
  <composition> <number> 1 </number> <diffFluid> {D} </diffFluid> <diffSolid> {D_s} </diffSolid>
    <iniValue> {-delta} </iniValue> <partition> {k} </partition> </composition>
  <b200>
    <model> flow_solutal_dendrite </model> <precision> {precision} </precision> <boundary> {bc} </boundary>
    <lattice> {lattice} </lattice> <collision> {collision} </collision>
    <tau> {tau} </tau> <magic> 0.1875 </magic> <rho0> 1.0 </rho0> <velocity> {u_in} 0 0 </velocity>
    <inlet> {1 if inlet else 0} </inlet>
    <eps4> {eps4} </eps4> <W0> {W0} </W0> <lambda> {lam} </lambda> <delta> {delta} </delta>
    <diffusivity> {D} </diffusivity> <diffSolid> {D_s} </diffSolid> <partition> {k} </partition>
  </b200>
</MaterKit>
"""


def multigrain(n=48, loops=1000, precision="fp32", seeds=None, W0=1.5, mobility=1.0, kappa=1.0, delta=0.3,
               D=0.1, nz=None, ny=None) -> str:
    """Multiphase field of grains (run_multiPhaseField): one order parameter
    per seed; `seeds` is a list of (x, y, z, radius), default two touching
    grains along x.  Closed faces."""
    nx = n
    ny = ny or n
    nz = nz or n
    if seeds is None:
        c = ((ny - 1) / 2.0, (nz - 1) / 2.0)
        seeds = [(nx / 2.0 - 6.0, c[0], c[1], 7.0), (nx / 2.0 + 6.0, c[0], c[1], 7.0)]
    centers = " ".join(f"{x} {y} {z}" for x, y, z, _ in seeds)
    radii = " ".join(str(r) for *_, r in seeds)
    angles = " ".join("0 0 0" for _ in seeds)
    return _HEADER.format(dendrite="true", flow="false", loops=loops, frames=min(loops, 100), nx=nx, ny=ny, nz=nz) + f"""
  <phasechange>
    <d0> 0.138486 </d0> <lambda> 10.0 </lambda> <anisotropy> 0.0 </anisotropy> <W0> 1.0 </W0> <t0> 1.0 </t0>
    <seed> <number> {len(seeds)} </number> <center> {centers} </center> <angle> {angles} </angle>
      <radius> {radii} </radius> </seed>
  </phasechange>
  <temperature> <iniValue> {-delta} </iniValue> <undercooling> {delta} </undercooling>
    <alphaFluid> {D} </alphaFluid> <alphaSolid> {D} </alphaSolid> <beta> 0.0 </beta> </temperature>
  <b200>
    <model> multigrain </model> <precision> {precision} </precision> <boundary> closed closed closed </boundary>
    <W0> {W0} </W0> <mobility> {mobility} </mobility> <grainKappa> {kappa} </grainKappa> <delta> {delta} </delta>
    <diffusivity> {D} </diffusivity>
  </b200>
</MaterKit>
"""


def write(text: str, path: str) -> str:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write(text)
    return path
