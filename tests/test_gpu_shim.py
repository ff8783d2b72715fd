"""The drop-in classes (mdtk_b200/mdtk/GpuPotentials.hpp: GpuREBO, GpuAIREBO,
GpuETors, GpuBrenner) inside the reference's own, unmodified FProxy and
SimLoop.  The oracle harness holds them in its FProxy in place of REBO,
AIREBO, ETors or Brenner (oracle/shim_harness.cpp), so FProxy::operator()
(FProxy.cxx:46-61), FGeneral's NL_* calls and SimLoop::execute
(SimLoop.cxx:225-474) drive the GPU path; the results are compared with the
same harness running the reference's own classes.

Bars: energy <= 1e-12 relative and ||dF||/||F|| <= 1e-10 (or FLOOR_FACTOR x
the oracle's 1-ulp floor); 20 SimLoop steps: per-step energies 1e-9 eV per
atom, positions and velocities 1e-9."""
import numpy as np
import pytest

from mdtk_b200 import builders as B
from oracle import ref
from parity import assert_parity, oracle_floor

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "ethane30": (lambda: B.ethane_liquid(30, seed=71, min_dist=1.6, jitter=0.4), ref.POT_AIREBO, 1),
    "ach250": (lambda: B.amorphous_carbon(250, h_fraction=0.3, seed=72), ref.POT_AIREBO, 1),
    "diamond3_rebo_tors": (lambda: B.diamond(3, temp_k=600.0, disp_sigma=0.08, seed=73),
                           ref.POT_REBO | ref.POT_ETORS, 1),
    "ac300_brenner1": (lambda: B.amorphous_carbon(300, seed=74), ref.POT_BRENNER, 1),
    "ach250_brenner2": (lambda: B.amorphous_carbon(250, h_fraction=0.3, seed=75), ref.POT_BRENNER, 2),
}


def _pair(name):
    make, pot, bset = SYSTEMS[name]
    s = make()
    ref.install_gpu_shim()
    out = []
    for p in (pot | ref.POT_GPU, pot):
        r = ref.RefSystem(p, bset)
        r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
        out.append(r)
    return s, pot, bset, out[0], out[1]


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_fproxy_over_gpu_classes_matches_reference_classes(name):
    s, pot, bset, gpu, cpu = _pair(name)
    assert gpu.npot == cpu.npot
    e, et, g = gpu.compute()
    eo, eto, go = cpu.compute()
    floor = oracle_floor(lambda: ref.RefSystem(pot, bset), s)
    assert_parity(e, g, eo, go, floor, label=f"shim {name}")
    # each GPU class returns its own term's energy, as FProxy sums them
    for t in range(cpu.npot):
        assert abs(et[t] - eto[t]) <= max(1e-12 * abs(eo), 4 * floor[0] * abs(eo)), (t, et, eto)
    # FProxy::operator() itself (one call over all potentials)
    ep = np.zeros(1)
    gp = np.zeros((len(s["z"]), 3))
    ref._check(ref.lib().ref_energy_proxy(gpu.h, ref._dp(ep), ref._dp(gp)))
    assert_parity(float(ep[0]), gp, eo, go, floor, label=f"shim FProxy {name}")
    # each class's NeighbourList holds the device's list, as FGeneral::NL reads it
    for k in range(cpu.npot):
        assert np.array_equal(gpu.nl_pairs(k), cpu.nl_pairs(k)), k


@pytest.mark.parametrize("name", ["ethane30", "diamond3_rebo_tors", "ac300_brenner1"])
def test_simloop_execute_over_gpu_classes(name):
    s, pot, bset, gpu, cpu = _pair(name)
    n = len(s["z"])
    a = gpu.run(20, 0.5)
    b = cpu.run(20, 0.5)
    assert np.abs(a["epot"] - b["epot"]).max() / n < 1e-9
    assert np.abs(a["etot"] - b["etot"]).max() / n < 1e-9
    d = a["pos"] - b["pos"]
    per = np.asarray(s["pbc"]) != 0
    d[:, per] -= s["box"][per] * np.round(d[:, per] / s["box"][per])
    assert np.abs(d).max() < 1e-9
    assert np.abs(a["vel"] - b["vel"]).max() < 1e-9
    assert np.array_equal(a["image"], b["image"])
