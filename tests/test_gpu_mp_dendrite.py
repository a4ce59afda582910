"""A thermal dendrite growing in a two-phase flow (run_flow_multiphase_dendrite,
MaterKit/MaterKit.cpp:377-397) through the coupling entry points
mk_update_velocity / mk_update_geometry, against the oracle's coupling in
FP64 at 1e-10 per field; the solid flags agree cell for cell; graph-replayed
flow loops equal eager ones; mismatched handles are refused."""
import os
import subprocess

import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, case_params, cases
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from _oracle import Oracle, rel_l2

pytestmark = pytest.mark.gpu


def _paths(casedir, n=24, prec="fp64"):
    fp = cases.write(cases.multiphase_bubbles(n=n, bubbles=1, rmin=3.0, rmax=3.5, width=2.0, gz=-1e-5,
                                              precision=prec, loops=10), f"{casedir}/gmpd_flow_{prec}.xml")
    dp = cases.write(cases.thermal_dendrite(n=n, loops=10, precision=prec, radius=4.0,
                                            center=(n / 2.0 - 0.5, n / 2.0 - 0.5, n / 3.0)),
                     f"{casedir}/gmpd_dend_{prec}.xml")
    return fp, dp


def _loop(f, d):
    d.update_velocity(f)
    d.advance(1)
    f.update_geometry(d)
    f.advance(1)


def test_coupled_run_matches_oracle(casedir):
    fp, dp = _paths(casedir)
    f, d = Solver(params=case_params(fp)), Solver(params=case_params(dp))
    of, od = Oracle.from_xml(fp), Oracle.from_xml(dp)
    for n in range(14):
        _loop(f, d)
        _loop(of, od)
        if n in (0, 1, 6, 13):
            flag = of.field("flag")
            assert np.array_equal(f.field("flag"), flag), n
            fl = flag == 0
            for name in ("phi", "ux", "uz", "pressure"):
                # the pressure starts at rest: rounding noise until it has grown
                e = rel_l2(f.field(name), of.field(name), fl, floor=1e-9 if name == "pressure" else 1e-12)
                assert e <= 1e-10, (n, "flow", name, e)
            for name in ("phi", "T"):
                e = rel_l2(d.field(name), od.field(name))
                assert e <= 1e-10, (n, "dendrite", name, e)
    assert (f.field("flag") == 2).sum() > 0  # the dendrite made solid cells


def test_flow_graph_equals_eager_with_solids(casedir):
    fp, dp = _paths(casedir, prec="fp32")
    d = Solver(params=case_params(dp))
    d.advance(20)
    a, b = Solver(params=case_params(fp)), Solver(params=case_params(fp))
    a.advance(3)
    b.advance(3)
    a.update_geometry(d)  # pending at an odd count: applied at the next even one
    b.update_geometry(d)
    a.advance(9, graph=True)
    b.advance(9)
    for name in ("phi", "pressure", "uz", "flag"):
        assert np.array_equal(a.field(name), b.field(name)), name
    assert (a.field("flag") == 2).sum() > 0


def test_coupling_checks(casedir):
    fp, dp = _paths(casedir, n=24, prec="fp32")
    f, d = Solver(params=case_params(fp)), Solver(params=case_params(dp))
    fp2, _ = _paths(casedir, n=32, prec="fp32")
    g = Solver(params=case_params(fp2))
    assert f._lib.mk_update_geometry(g.handle, d.handle) == A.MK_ERR_ARG  # another grid
    assert f._lib.mk_update_geometry(d.handle, f.handle) == A.MK_ERR_ARG  # roles swapped
    assert f._lib.mk_update_velocity(f.handle, d.handle) == A.MK_ERR_ARG
    # the flow loses its fused and row-staged forms once it has solids
    f.update_geometry(d)
    assert not f.fused and not f.row_staged


DRIVER = r"""
#include <cstdio>
#include "mkb200_compat.hpp"
using namespace mkb200;
int main(int argc, char** argv) {
  mkSpace sf(argv[1]), sd(argv[2]);
  mkFluidsMultiphase flow(sf);
  mkFluidsMRT dendrite(sd);
  flow.initialize(argv[1], MK_MODEL_MULTIPHASE);
  dendrite.initialize(argv[2], MK_MODEL_THERMAL_DENDRITE);
  flow.initialize_geometry();
  dendrite.initialize_geometry();
  for (int loops = 0; loops < 9; ++loops) {  // run_flow_multiphase_dendrite, MaterKit.cpp:377-397
    dendrite.phasefield_propagate();
    dendrite.relaxation_anisotropy_thermal(flow);
    dendrite.update_velocity(flow);
    dendrite.thermal_propagate();
    dendrite.thermal_relaxation(flow);
    flow.update_geometry(dendrite);
    flow.propagate();
    flow.relaxation();
  }
  mk_diag a = flow.check_variables(9), b = dendrite.check_variables(9);
  std::printf("flow %lld %.17g dendrite %lld %.17g %.17g\n", (long long)a.step, a.phi_sum, (long long)b.step,
              b.phi_sum, b.heat);
  return a.step == 9 && b.step == 9 ? 0 : 1;
}
"""


def test_compat_driver_runs_the_coupled_loop(casedir, tmp_path):
    # the reference's call order through the header-only shim equals the
    # Python loop on the same device kernels
    A.load()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    libdir = os.path.dirname(A.LIB_PATH)
    env = dict(os.environ)
    env.pop("CXX", None)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(root, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lmkb200", f"-Wl,-rpath,{libdir}"], check=True, env=env)
    fp, dp = _paths(casedir, prec="fp32")
    r = subprocess.run([str(exe), fp, dp], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    parts = r.stdout.split()
    f, d = Solver(params=case_params(fp)), Solver(params=case_params(dp))
    for _ in range(9):
        _loop(f, d)
    a, b = f.diagnostics(), d.diagnostics()
    assert parts[0] == "flow" and int(parts[1]) == 9 and int(parts[4]) == 9
    assert float(parts[2]) == a["phi_sum"]
    assert float(parts[5]) == b["phi_sum"] and float(parts[6]) == b["heat"]
