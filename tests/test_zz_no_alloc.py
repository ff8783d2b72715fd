"""The allocation-free REBO entry point (mdg_rebo_compute_noalloc) against the
context path (mdg_compute), through the C ABI.

That entry point is for callers that cannot allocate device memory (a host
whose allocator owns all device memory, or a loop that cannot afford the
synchronisation cudaMalloc implies): its intermediates live in a static
device array, and the caller passes device buffers for inputs and outputs.
Here the test allocates those buffers with torch (the test may allocate; the
entry point does not) and checks two calls in a row, plus a third call on the
first system after the scratch held another system."""
import ctypes

import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from parity import TOL_E, TOL_F, rel_e, rel_f

pytestmark = pytest.mark.gpu

MAX_ATOMS = 4096


def _fn():
    L = M.lib()
    f = L.mdg_rebo_compute_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                  ctypes.POINTER(ctypes.c_int32), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _noalloc(s, with_torsion):
    import torch
    n = len(s["z"])
    pos = torch.tensor(np.ascontiguousarray(s["pos"]), dtype=torch.float64, device="cuda")
    z = torch.tensor(s["z"], dtype=torch.int32, device="cuda")
    energy = torch.zeros(2, dtype=torch.float64, device="cuda")
    grad = torch.full((n, 3), 7.0, dtype=torch.float64, device="cuda")  # overwritten by the call
    box = (ctypes.c_double * 3)(*[float(x) for x in s["box"]])
    pbc = (ctypes.c_int32 * 3)(*[int(x) for x in s["pbc"]])
    stream = torch.cuda.current_stream().cuda_stream
    rc = _fn()(n, pos.data_ptr(), z.data_ptr(), box, pbc, 1 if with_torsion else 0, energy.data_ptr(),
               grad.data_ptr(), stream)
    if rc != 0:
        raise M.MdgError(rc, M.lib().mdg_last_error().decode())
    torch.cuda.synchronize()
    return energy.cpu().numpy(), grad.cpu().numpy()


def _context(s, with_torsion):
    pot = M.POT_REBO | (M.POT_ETORS if with_torsion else 0)
    ctx = M.Context(potentials=pot)
    ctx.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"])
    e, et, g = ctx.compute()
    return et, g


def _check(e_na, g_na, et, g):
    assert rel_e(e_na[0], et[0]) <= TOL_E
    assert abs(e_na[1] - et[2]) <= TOL_E * max(abs(et[0]), 1.0)
    assert rel_f(g_na, g) <= TOL_F


def test_noalloc_matches_context_path_on_consecutive_calls():
    s1 = B.amorphous_carbon(300, h_fraction=0.3, seed=41)
    s2 = B.diamond(3, disp_sigma=0.15, seed=42)
    et1, g1 = _context(s1, True)
    et2, g2 = _context(s2, True)
    e, g = _noalloc(s1, True)
    _check(e, g, et1, g1)
    e, g = _noalloc(s2, True)
    _check(e, g, et2, g2)
    # the scratch now holds s2's intermediates; a call on s1 must not see them
    e, g = _noalloc(s1, True)
    _check(e, g, et1, g1)


def test_noalloc_without_torsion():
    s = B.ethane_liquid(30, seed=43, min_dist=1.6, jitter=0.4)
    et, g = _context(s, False)
    for _ in range(2):
        e, gg = _noalloc(s, False)
        _check(e, gg, et, g)
        assert e[1] == 0.0


def test_noalloc_rejects_systems_above_its_limit():
    s = B.diamond(9)  # 5832 atoms > 4096
    assert len(s["z"]) > MAX_ATOMS
    with pytest.raises(M.MdgError) as err:
        _noalloc(s, False)
    assert err.value.code == -1
    assert "4096" in str(err.value)
