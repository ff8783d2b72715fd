"""REBO work split and the autotuner: one task per directed bond, one task
per bond, and one bond per lane pair (each lane one end's bond-order terms,
the torsion of a C-C bond a task of its own) route the same terms into the
same records.  The kernels may contract multiply-adds differently and the
lane-pair split adds an end's own gradient in two sums, so forces and
energies agree to rounding; the autotuner only picks the fastest."""
import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "ethane30": lambda: B.ethane_liquid(30, seed=61, min_dist=1.6, jitter=0.4),
    "diamond4_disp": lambda: B.diamond(4, disp_sigma=0.1, seed=62),
    "ach300": lambda: B.amorphous_carbon(300, h_fraction=0.25, seed=63),
    "impact": lambda: B.impact(64, n_target=900),
}


def _ctx(s, mode, precision=M.PREC_FP64, pot=M.POT_AIREBO):
    c = M.Context(potentials=pot, precision=precision, task_mode=mode)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return c


@pytest.mark.parametrize("mode", [2, 3])
@pytest.mark.parametrize("precision", [M.PREC_FP64, M.PREC_FP32_MIXED])
@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_task_modes_agree(name, precision, mode):
    s = SYSTEMS[name]()
    e1, t1, g1 = _ctx(s, 1, precision).compute()
    e2, t2, g2 = _ctx(s, mode, precision).compute()
    tol = 1e-13 if precision == M.PREC_FP64 else 1e-6
    assert np.abs(g1 - g2).max() <= tol * np.abs(g1).max()
    assert abs(e1 - e2) <= tol * np.abs(t1).sum()
    for t in range(3):
        assert abs(t1[t] - t2[t]) <= tol * np.abs(t1).sum(), (t, t1, t2)


@pytest.mark.parametrize("mode", [2, 3])
def test_task_modes_same_trajectory(mode):
    s = SYSTEMS["diamond4_disp"]()
    a, b = _ctx(s, 1), _ctx(s, mode)
    ea = a.run(20, 0.5)
    eb = b.run(20, 0.5)
    assert np.abs(ea[1] - eb[1]).max() < 1e-9 * len(s["z"])
    assert np.abs(a.get_state()[0] - b.get_state()[0]).max() < 1e-10


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_hot_diamond_runs_in_every_split(mode):
    # atoms pushed 0.25 A off the lattice heat up and some take a fifth
    # bond: the default record capacity holds every split's records
    s = B.diamond(4, disp_sigma=0.25, seed=33)
    c = _ctx(s, mode)
    c.run(20, 0.25, energies=False)
    assert np.isfinite(c.get_state()[0]).all()


def test_autotuner_picks_a_mode():
    s = SYSTEMS["ach300"]()
    c = _ctx(s, 0)
    assert c.task_mode()[0] == 1          # before the first run: directed
    c.run(2, 0.25, energies=False)
    mode, t1, t2, t3 = c.task_mode()
    assert mode in (1, 2, 3) and t1 > 0 and t2 > 0 and t3 > 0
    assert mode == 1 + int(np.argmin([t1, t2, t3]))
    # the tuned context reproduces a run fixed to the chosen mode bitwise
    d = _ctx(s, mode)
    d.run(2, 0.25, energies=False)
    assert np.array_equal(c.get_state()[0], d.get_state()[0])
