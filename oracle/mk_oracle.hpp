// mk_oracle.hpp — TEST INFRASTRUCTURE ONLY.
//
// FP64 OpenMP CPU restatement of MaterKit's coupled lattice-Boltzmann /
// phase-field step.  It is the parity checker for the CUDA library and the
// timed CPU baseline; nothing in the product links, loads or calls it.
//
// Parity status: the reference solver bodies live only in the closed Windows
// DLL MaterKit/AiLBFlow.dll (linked at MaterKit/MaterKit.vcxproj:158), which
// cannot run here and is never opened.  Parity against the reference itself is
// therefore UNPINNED.  This oracle is pinned instead by known answers
// (tests/test_oracle_*.py): the analytic Poiseuille profile (exact for TRT with
// Lambda = 3/16 and half-way bounce-back), Gaussian diffusion on D3Q7, the
// flat Allen-Cahn tanh profile, exact mass conservation, and cubic symmetry of
// a centred seed.
//
// Structure follows the reference's per-loop order "propagate, then
// relaxation" for each field (MaterKit/MaterKit.cpp:277-280 flow,
// :322-324 multiphase, :775-781 thermal dendrite, :665-674 solutal dendrite),
// the pull-stream with bounce-back of MaterKit/src/mkFluidsUser.cpp:68-134,
// and the BGK + source relaxation of MaterKit/src/mkFluidsUser.cpp:136-299.
// Stored state after n loops = post-collision populations ("f_out" of
// MaterKit/inc/mkNode.h:135) plus the order parameter phi (mkNode.h:154).
//
// ---------------------------------------------------------------------------
// Model definitions (the exact formulas are inside the closed DLL; these are
// the method's published forms, fixed here as the definition both the oracle
// and the CUDA kernels implement):
//
// Lattices: D3Q19/D3Q27 (cs^2 = 1/3), D3Q7 (w0 = 1/4, wi = 1/8, cs^2 = 1/4).
// Direction order: rest, +-x, +-y, +-z, then xy, xz, yz edges in (+,+),(-,-),
// (+,-),(-,+) pairs, then the 8 corners; opposite directions are adjacent.
//
// FLOW (mkFluidsLBM::propagate/relaxation, mkFluidsLBM.h:47-49; mkNode
// collision_BGK/TRT/MRT*, mkNode.h:74-87):
//   rho = sum f, u = (sum e f + F/2)/rho, feq = w rho (1 + 3eu + 4.5(eu)^2 - 1.5u^2)
//   Guo force Fi = w [3 e.F + 9 (e.u)(e.F) - 3 u.F]
//   BGK  f* = f - (f - feq)/tau + (1 - 1/(2tau)) Fi
//   TRT  symmetric part with tau+ = tau, antisymmetric with tau- = 1/2 + Lambda/(tau - 1/2)
//   MRT  d'Humieres 2002 D3Q19 moments; s_e=1.19 s_eps=1.4 s_q=1.2 s_pi=1.4
//        s_m=1.98, s_nu=1/tau, conserved rates 1; f* = f - Mi[S(m-meq) - (I-S/2)mF]
//
// MULTIPHASE (mkFluidsMultiphase::propagate/relaxation, mkFluidsMultiphase.h:52-57;
// Liang et al., PRE 89 053320 (2014) two-lattice structure, cited at
// mkLattice.h:52-53; conservative Allen-Cahn h-lattice, pressure-normalised g-lattice):
//   phi = sum h (post-stream), rho = rho_g + phi (rho_l - rho_g)
//   grad phi = 3 sum w e phi_nb, lap phi = 6 sum w (phi_nb - phi)   (D3Q19 weights)
//   phi_nb at a non-fluid neighbour = phi + (4/W) cos(theta) phi (1 - phi)  (wetting)
//   beta = 12 sigma / W, kappa = 1.5 sigma W, mu = 4 beta phi (phi-1)(phi-1/2) - kappa lap phi
//   p* = sum g, F = mu grad phi + rho g_acc - p*/3 grad rho, u = sum e g + F/(2 rho)
//   geq = w (p* + 3eu + 4.5(eu)^2 - 1.5u^2), Fbar = w [3 e.F + 9 (e.u)(e.F) - 3 u.F]/rho
//   MRT on g with s_nu = 1/tau(phi), tau = tau_g + phi (tau_l - tau_g)
//   n = grad phi/(|grad phi| + 1e-12), lam = 4 phi (1-phi)/W
//   heq = phi w (1 + 3eu + 4.5(eu)^2 - 1.5u^2)
//   h* = h - (h - heq)/tau_h + (1 - 1/(2 tau_h)) w lam (e.n),  tau_h = 3M + 1/2
//
// THERMAL DENDRITE (mkPhaseField::propagate/relaxation_anisotropy_thermal,
// mkPhaseField.h:41,46; mkThermalField::propagate/relaxation, mkThermalField.h:33-34;
// Karma-Rappel thin-interface model, Chai et al. IJHMT 122 (2018) 631 source
// form as in mkFluidsUser.cpp:262-288):
//   tau0 a^2 dphi/dt = W0^2 div(a^2 grad phi + N) + phi - phi^3 - lam u (1-phi^2)^2
//   a(n) one of the mk_anisotropy kinds (crystal frame n; cubic:
//   1 - 3 eps4 + 4 eps4 sum n_k^4), with da/dn its gradient,
//   N_k = |grad phi| a (da/dn_k - n_k (n . da/dn))   (cubic: |grad phi| a 16 eps4 (n_k^3 - n_k sum n_j^4))
//   D3Q7 g-lattice: geq = w phi, omega_g = 1/(4 W0^2/tau0 + 1/2),
//   g* = g - omega_g (g - geq) + (1 - omega_g/2) w (e.B)/cs^2 + w S,
//   B = -cs^2 [(a^2 - 1) grad phi + N],
//   S = (phi - phi^3 - lam u (1-phi^2)^2)/tau0 + (1 - a^2) (phi^n - phi^(n-1))
//   du/dt = D lap u + (1/2) dphi/dt: D3Q7 t-lattice, omega_T = 1/(4 D + 1/2),
//   t* = t - omega_T (t - w u) + w (phi^n - phi^(n-1))/2
//   The phase-field relaxation at loop n uses u from the previous thermal relaxation.
//
// SOLUTAL DENDRITE (mkPhaseField::relaxation_anisotropy_solute(loops), mkPhaseField.h:48;
// mkSolutalField::propagate/relaxation/ATcurrent, mkSolutalField.h:35-37,65; dilute
// binary alloy of Karma, PRL 87 115701 (2001), phi = +1 solid, U supersaturation):
//   tau0 a^2 dphi/dt = W0^2 div(a^2 grad phi + N) + phi - phi^3 - lam U (1-phi^2)^2
//   c(phi) dU/dt = div(D(phi) grad U - j_at) + (1/2)(1 + (1-k)U) dphi/dt
//   c(phi) = (1 + k - (1-k) phi)/2, D(phi) = D (1-phi)/2 + D_s (1+phi)/2,
//   j_at = -at W0 (1 + (1-k)U) (dphi/dt) n,  at = 1/(2 sqrt 2) (<antiTrapping>)
//   phase field: the thermal-dendrite g-lattice with u -> U.
//   The capacity is applied locally: c dU/dt = div(...) + R is advanced as
//   dU/dt = div((D/c) grad U - j_at/c) + R/c (the grad(1/c) cross terms, nonzero only
//   inside the interface, are dropped).  U-lattice (D3Q7), TRT: pair sums relax to
//   equilibrium with rate 1, pair differences with omega(phi) = 1/(4 D(phi)/c(phi) + 1/2):
//   t0* = w0 U + w0 S,  t_i,j* = w U +- [a - omega (a - w 4 e_i.j_at/c)] + w S,
//   a = (t_i - t_j)/2,  S = (1/2)(1 + (1-k)U) dphi / c(phi),
//   U = sum t (post-stream), phi, dphi of this loop, n = grad phi/(|grad phi| + 1e-6).
//
// FLOW + DENDRITE (run_flow_thermal_dendrite, MaterKit.cpp:467-527) and FLOW +
// SOLUTAL DENDRITE (run_flow_solutal_dendrite, MaterKit.cpp:399-465): per loop
// the flow lattice with the partially saturated porous bounce-back
// (propagate_PBB, relaxation) and the x faces (bdyVelocity), the phase field,
// the scalar lattice advected by the flow's collision velocity u (thermal:
// t_eq = w T (1 + 4 e.u); solutal: the advective flux U u joins the
// anti-trapping current in the first moment, 4 w e.(j_at/c + U u)), then the
// scalar faces (bdy_flowin / bdy_LBflowin): inflow T_b (U_b) = -Delta,
// phi_b = -1, outflow copies the inner neighbour, by non-equilibrium
// extrapolation of w T (1 + 4 e.u).
// ---------------------------------------------------------------------------
#ifndef MK_ORACLE_HPP
#define MK_ORACLE_HPP

#include <stdint.h>
#include "../include/mkb200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_state orc_state;

// Initial macroscopic fields are dense x-fastest arrays of nx*ny*nz doubles;
// any may be NULL (defaults: phi 0 / T,U = -delta / rho = rho0 / u = u0).
orc_state* orc_create(const mk_params* p, const double* phi0, const double* T0, const double* C0,
                      const double* rho0, const double* ux0, const double* uy0, const double* uz0);
void orc_destroy(orc_state* s);
void orc_advance(orc_state* s, int64_t nsteps);
int64_t orc_step(const orc_state* s);
// Returns 0 on success, nonzero for an unknown field.
int orc_get_field(const orc_state* s, int field, double* out);
// Raw post-collision populations of lattice `which` (0 flow/phase, 1 second lattice).
int orc_get_populations(const orc_state* s, int which, double* out);
// Multigrain: the order parameter of one grain (ncell doubles); 1 if out of range.
int orc_get_grain_phi(const orc_state* s, int grain, double* out);
void orc_set_threads(int n);
// Discrete adjoint of the thermal dendrite loop: L = sum (phi - target)^2 after
// `steps` loops from the current state; out = {L, dL/deps4, dL/dDelta,
// dL/dtau_T}.  Stores every state (small cases).  Returns 0 on success.
int orc_backward(orc_state* s, const double* target, int64_t steps, double* out);
// a(n) and da/dn of an anisotropy kind at the crystal-frame unit normal n (tests).
void orc_anisotropy(int kind, double e4, double e2, const double* n, double* a, double* g);
int orc_get_threads(void);

// Reference-structure variant (the reference's node-object layout and its
// schedule(static, 16) sweeps) of the flow model (D3Q19, no moving plates)
// and the thermal dendrite, created from an oracle state and bit-identical
// to orc_advance; NULL for other models.
// Coupling of a dendrite and a multiphase flow of one grid: the flow's fluid
// cells with dendrite phi > 0 turn solid at its next even loop count; the
// dendrite's scalar lattice takes the flow's velocity.  1 for a mismatch.
int orc_update_geometry(orc_state* flow, const orc_state* dendrite);
int orc_update_velocity(orc_state* dendrite, const orc_state* flow);

typedef struct orc_aos orc_aos;
orc_aos* orc_aos_create(const orc_state* s);
void orc_aos_destroy(orc_aos* a);
void orc_aos_advance(orc_aos* a, int64_t nsteps);
int orc_aos_get_populations(const orc_aos* a, int which, double* out);
int orc_aos_get_field(const orc_aos* a, int field, double* out);
size_t orc_aos_node_bytes(void);

#ifdef __cplusplus
}
#endif

#endif
