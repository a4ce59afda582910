"""The drop-in path on the device: the reference's own shipped case files
(tests/golden/shipped_cases, comment-stripped copies of MaterKit/BoltzTechs*.xml)
created with mk_create_from_xml and advanced, against the oracle's own reading
of the same files; and the header-only C++ shim advancing a case.

The shipped cases are 2-D (MeshXYZ ... 1) thermal dendrites in physical units
(mk_dx 0.4, mk_dt 0.008: W0 = 2.5, tau0 = 125 lattice units)."""
import os
import subprocess

import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, cases
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from _oracle import Oracle, rel_l2

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _shipped(name):
    return os.path.join(HERE, "golden", "shipped_cases", name)


@pytest.mark.parametrize("name,loops", [("boltztechs_thermal.xml", 40), ("boltztechs_multiphasefield.xml", 30),
                                        ("boltztechs_solutalmultidendrites.xml", 20),
                                        ("boltztechs_solutal.xml", 20)])
def test_shipped_case_fp64_matches_oracle(name, loops):
    path = _shipped(name)
    s = Solver(path, precision="fp64")  # mk_create_from_xml
    o = Oracle.from_xml(path, precision="fp64")
    assert s.shape == (o.params.nz, o.params.ny, o.params.nx)
    for n in (1, 2, loops - 3):
        s.advance(n)
        o.advance(n)
        for f in ("phi", "T", "dphi"):
            e = rel_l2(s.field(f), o.field(f))
            assert e <= 1e-10, (name, s.step, f, e)
    assert np.array_equal(s.field("grain"), o.field("grain"))
    s.close()


def test_shipped_case_default_precision_runs():
    # as shipped (no override): FP32 storage, through the CUDA graph
    path = _shipped("boltztechs_thermal.xml")
    s = Solver(path)
    assert s.params.precision == A.MK_PREC_FP32
    o = Oracle.from_xml(path, precision="fp64")
    s.advance(200, graph=True)
    o.advance(200)
    d = s.diagnostics()
    assert d["n_bad"] == 0 and d["step"] == 200
    assert rel_l2(s.field("phi"), o.field("phi")) < 1e-5
    s.close()


DRIVER = r"""
#include <cstdio>
#include "mkb200_compat.hpp"
using namespace mkb200;
int main(int argc, char** argv) {
  const std::string xml = argv[1];
  int maxLoops = 0, maxFrame = 0;
  readParameters(maxLoops, maxFrame, xml);
  mkSpace space(xml);
  mkFluidsMRT flow(space);
  flow.initialize(xml, MK_MODEL_THERMAL_DENDRITE);
  flow.initialize_geometry();
  for (int loops = 0; loops < 6; ++loops) {
    flow.phasefield_propagate();
    flow.relaxation_anisotropy_thermal();
    flow.thermal_propagate();
    flow.thermal_relaxation();
  }
  mk_diag d = flow.check_variables(6);
  std::printf("step %lld phi_sum %.17g heat %.17g\n", (long long)d.step, d.phi_sum, d.heat);
  return d.step == 6 ? 0 : 1;
}
"""


def test_compat_driver_advances_on_device(tmp_path):
    # the reference-style driver (MaterKit.cpp:743-788 call order) built against
    # the header-only shim advances the case on the device; its sums equal a
    # direct run of the same case through the C ABI
    A.load()
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    libdir = os.path.dirname(A.LIB_PATH)
    env = dict(os.environ)
    env.pop("CXX", None)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lmkb200", f"-Wl,-rpath,{libdir}"], check=True, env=env)
    xml = cases.write(cases.thermal_dendrite(n=16, loops=20, radius=3.0), str(tmp_path / "case.xml"))
    r = subprocess.run([str(exe), xml], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    parts = r.stdout.split()
    assert parts[0] == "step" and parts[1] == "6"
    s = Solver(xml, model="thermal_dendrite")
    s.advance(6)
    d = s.diagnostics()
    assert float(parts[3]) == pytest.approx(d["phi_sum"], rel=1e-12)
    assert float(parts[5]) == pytest.approx(d["heat"], rel=1e-12)
    s.close()
