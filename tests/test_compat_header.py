"""The header-only C++ shim (include/mkb200_compat.hpp) compiles, links against
libmkb200.so and drives a case with the reference's call sequence; without a
device it fails loudly with MK_ERR_NODEVICE instead of falling back."""
import os
import subprocess

from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <cstdio>
#include "mkb200_compat.hpp"
using namespace mkb200;
int main(int argc, char** argv) {
  const std::string xml = argv[1];
  int maxLoops = 0, maxFrame = 0;
  readParameters(maxLoops, maxFrame, xml);
  mkSpace space(xml);
  std::printf("mesh %d %d %d loops %d frames %d\n", space.Mx(), space.My(), space.Mz(), maxLoops, maxFrame);
  mkFluidsMRT flow(space);
  try {
    flow.initialize(xml, MK_MODEL_THERMAL_DENDRITE);
  } catch (const Error& e) {
    std::printf("status %d\n", (int)e.status);
    return e.status == MK_ERR_NODEVICE ? 0 : 1;
  }
  flow.initialize_geometry();
  for (int loops = 0; loops < 4; ++loops) {
    flow.phasefield_propagate();
    flow.relaxation_anisotropy_thermal();
    flow.thermal_propagate();
    flow.thermal_relaxation();
  }
  mk_diag d = flow.check_variables(4);
  std::printf("step %lld phi_sum %.6f\n", (long long)d.step, d.phi_sum);
  return d.step == 4 ? 0 : 1;
}
"""


def test_compat_driver_builds_and_runs(tmp_path):
    A.load()
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    libdir = os.path.dirname(A.LIB_PATH)
    env = dict(os.environ)
    env.pop("CXX", None)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lmkb200", f"-Wl,-rpath,{libdir}"], check=True, env=env)
    xml = cases.write(cases.thermal_dendrite(n=12, loops=20, radius=3.0), str(tmp_path / "case.xml"))
    r = subprocess.run([str(exe), xml], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mesh 12 12 12 loops 20" in r.stdout
