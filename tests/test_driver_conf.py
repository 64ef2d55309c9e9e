"""The C++ driver's initial configurations against the oracle, on the CPU.

The driver builds each chain's starting sigma on the host, from its seed, as
conf_set + conf_transfer do (src/fields.f90:311-507): five `absolute` modes,
then tiling of the thermalisation lattice (NlxT x NlyT x LtrotT) up to the
run size.  The GPU driver tests only reach mode 1 without tiling, so this
test compiles those two functions out of the driver source (its main renamed)
into a small program and compares sigma and the ranf state that continues the
chain with the oracle for every mode and a tiled case.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import z2_oracle as zo
from z2_gauge_zfy_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "z2_gauge_zfy_b200")

HARNESS = r'''
#define main z2_driver_main
#include "%s"
#undef main
int main(int argc, char **argv) {
  Params p;
  if (argc < 3 || !read_params(argv[1], p)) return 2;
  uint32_t iq = (uint32_t)(int32_t)std::atol(argv[2]);
  std::vector<double> st;
  conf_set(p, st, iq);
  const std::vector<double> s = conf_transfer(p, st);
  std::printf("%%u\n", iq);
  for (double v : s) std::printf("%%d\n", (int)v);
  return 0;
}
'''


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    build.build()                       # the driver source links against the library
    d = tmp_path_factory.mktemp("conf")
    src = d / "harness.cpp"
    src.write_text(HARNESS % os.path.join(PKG, "csrc", "z2_main.cpp"))
    exe = d / "harness"
    subprocess.run(["g++", "-O1", "-std=c++17", str(src), "-L" + PKG, "-lz2dqmc",
                    "-Wl,-rpath," + PKG, "-o", str(exe)], check=True)
    return exe


def _params(lat, therm, absolute):
    return ("0.5 1.0 0.52 0.3 1\n%d %d %d 2.0\n%d %d %d\n5 1 1\n.false. 0\n.false. 0\n"
            ".false. 0\n%d\n" % (*lat, *therm, absolute))


@pytest.mark.parametrize("lat, therm", [((4, 4, 40), (4, 4, 40)),     # no tiling
                                        ((4, 6, 20), (2, 3, 10))])    # tiled in x, y, tau
@pytest.mark.parametrize("absolute", [1, 2, 3, 4, 5])
def test_driver_initial_config_matches_oracle(harness, tmp_path, lat, therm, absolute):
    path = tmp_path / "paramC_sets.txt"
    path.write_text(_params(lat, therm, absolute))
    seed = 12439
    out = subprocess.run([str(harness), str(path), str(seed)], capture_output=True, text=True,
                         check=True, timeout=60).stdout.split()
    p = zo.read_params(str(path))
    sig, _, rng = zo.seeded_config(p, zo.Lattice(p.Nlx, p.Nly), seed)
    got = np.array([int(x) for x in out[1:]]).reshape(p.Ltrot, 2 * p.Lq).T
    assert np.array_equal(got, sig), absolute
    assert int(out[0]) == rng.state, absolute
