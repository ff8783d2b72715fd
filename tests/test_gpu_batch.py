"""Batched contexts: many independent systems (uneven sizes, different
boxes and periodicity) stepped by one set of launches.  Each system of a
batch must give what it gives alone, and what the oracle gives."""
import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref
from parity import assert_parity, oracle_floor

pytestmark = pytest.mark.gpu


def _members():
    return [
        B.ethane_liquid(30, seed=51, min_dist=1.6, jitter=0.4),
        B.impact(52, n_target=900),                          # lateral PBC, z open, fixed bottom
        B.amorphous_carbon(300, h_fraction=0.25, seed=53),
        B.c2h6_example(),                                   # no PBC at all
        B.impact(54, n_target=700, e_min_ev=50, e_max_ev=50),
    ]


def _single(s, pot, precision=M.PREC_FP64):
    c = M.Context(potentials=pot, precision=precision)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return c


def _batch(systems, pot, precision=M.PREC_FP64):
    c = M.Context(potentials=pot, precision=precision)
    c.set_batch(systems)
    return c


def _split(x, first):
    return [x[first[k]:first[k + 1]] for k in range(len(first) - 1)]


@pytest.mark.parametrize("precision", [M.PREC_FP64, M.PREC_FP32_MIXED])
def test_batch_forces_equal_single_runs(precision):
    systems = _members()
    bc = _batch(systems, M.POT_AIREBO, precision)
    _, _, g = bc.compute()
    es = bc.batch_energies()
    for k, (s, gk) in enumerate(zip(systems, _split(g, bc.first))):
        e1, et1, g1 = _single(s, M.POT_AIREBO, precision).compute()
        assert np.abs(gk - g1).max() <= 1e-13 * max(np.abs(g1).max(), 1.0), k
        assert abs(es[k, :3].sum() - e1) <= 1e-12 * max(abs(e1), 1.0), (k, es[k], e1)
        assert np.allclose(es[k, :3], et1[:3], rtol=1e-12, atol=1e-12), (k, es[k], et1)


def test_batch_pair_sets_bit_exact():
    systems = _members()
    bc = _batch(systems, M.POT_AIREBO)
    for lst in (0, 1):
        pairs = bc.nl_pairs(lst)
        want = []
        for k, s in enumerate(systems):
            r = ref.RefSystem(ref.POT_AIREBO)
            r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
            want.append(r.nl_pairs(lst) + bc.first[k])
        want = np.concatenate(want)
        assert np.array_equal(pairs, want), lst


def test_batch_members_match_oracle():
    systems = _members()
    bc = _batch(systems, M.POT_AIREBO)
    _, _, g = bc.compute()
    es = bc.batch_energies()
    for k, (s, gk) in enumerate(zip(systems, _split(g, bc.first))):
        r = ref.RefSystem(ref.POT_AIREBO)
        r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
        eo, eto, go = r.compute()
        floor = oracle_floor(lambda: ref.RefSystem(ref.POT_AIREBO), s, samples=2)
        # forces at the FP64 bars; energies term by term against the scale of
        # the terms (REBO and LJ nearly cancel in some members, so a bound
        # relative to the total is meaningless there): 1e-11 of the terms'
        # magnitude, or the oracle's own floor
        assert_parity(eo, gk, eo, go, floor, label=f"member {k}")
        scale = float(np.abs(eto[:3]).sum())
        bound = max(1e-11 * scale, 4 * floor[0] * abs(eo))
        assert np.all(np.abs(es[k, :3] - eto[:3]) <= bound), (k, es[k], eto)


def test_batch_md_tracks_single_runs():
    systems = _members()[:3]
    bc = _batch(systems, M.POT_REBO)
    ep, et = bc.batch_run(30, 0.2)
    pos, vel, _ = bc.get_state()
    for k, s in enumerate(systems):
        c = _single(s, M.POT_REBO)
        ep1, et1 = c.run(30, 0.2)
        p1, v1, _ = c.get_state()
        pk = pos[bc.first[k]:bc.first[k + 1]]
        d = pk - p1
        per = np.asarray(s["pbc"]) > 0
        d[:, per] -= np.asarray(s["box"])[per] * np.round(d[:, per] / np.asarray(s["box"])[per])
        assert np.abs(d).max() < 1e-9, k
        assert np.abs(ep[:, k] - ep1).max() < 1e-9 * len(s["z"]), k


def test_impact_fixed_bottom_and_open_z():
    s = B.impact(55, n_target=1000, e_min_ev=80, e_max_ev=80)
    bc = _batch([s, B.impact(56, n_target=800)], M.POT_AIREBO, M.PREC_FP32_MIXED)
    p0 = bc.get_state()[0]
    bc.batch_run(50, 0.2)
    p1 = bc.get_state()[0]
    fx = np.concatenate([s["fixed"], B.impact(56, n_target=800)["fixed"]]) > 0
    assert np.array_equal(p0[fx], p1[fx])          # fixed atoms never move
    cl = slice(len(s["z"]) - 13, len(s["z"]))
    assert (p1[cl, 2] < p0[cl, 2]).all()            # the cluster falls towards the slab
