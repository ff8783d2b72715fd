"""Adjoint of the velocity-Verlet trajectory (pure carbon, REBO + LJ +
torsion) through the C ABI.

* the force-field products of one dual pass: J^T u and J u against central
  finite differences of the FP64 gradient (J symmetric without torsion; with
  the reference's torsion derivative J is not, and the transpose is checked
  through v . J^T u = u . J v), the exact energy gradient, dE/dtheta and
  d(u . g)/dtheta against finite differences in the parameters;
* trajectory gradients (parameters, x0, v0) against central finite
  differences of the GPU forward run and of the reference's own SimLoop run
  with the same parameters (the FP64 reference gradient), over a horizon
  where central differences converge (10 steps of the 3,000 K system);
* over long horizons, against the tangent-linear model: the linearised
  trajectory propagated forward with J u products and the parameter forcing
  dg/dtheta from central differences of single force evaluations.  Hot
  amorphous carbon is chaotic and the reference's spline arithmetic has a
  noise floor, so central differences of a 200-step loss do not converge for
  any step size (measured from 1e-5 down to 1e-11); the tangent-linear model
  is the exact linearisation the adjoint must reproduce;
* independence of the checkpoint interval, determinism;
* a torch.autograd.Function around the ABI (test harness only);
* the adjoint workload: 4,096-atom amorphous carbon at 2.0 g/cm^3,
  pre-relaxed 500 steps at 3,000 K, 200 steps of 0.5 fs with a checkpoint
  every 20, loss = mean |x_200 - x_target|^2 + lambda E_total.

Tolerances: 1e-6 relative for the single-evaluation products (central
differences with h ~ 1e-5 leave ~1e-8), 1e-4 for trajectory gradients
against finite differences (the bound the adjoint is specified to), 1e-5
against the tangent-linear model (its parameter forcing carries the ~1e-7
error of a central difference of the force), 1e-8 for initial-condition
directions (no finite difference involved)."""
import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref

pytestmark = pytest.mark.gpu

DT = 0.5
LAM = 1e-5          # weight of the total energy (eV^-1) in the loss
CONV = B.EV_PER_AMU_A2FS2

_SYS = {}


def ac(n, seed, temp_k=0.0):
    key = (n, seed, temp_k)
    if key not in _SYS:
        s = B.amorphous_carbon(n, density_g_cm3=2.0, min_sep=1.2, seed=seed)
        s["vel"] = B.thermal_velocities(s["z"], temp_k, np.random.default_rng(seed + 1000))
        _SYS[key] = s
    return _SYS[key]


def hot216():
    """216 C at 2.0 g/cm^3 (box 12.4 A), relaxed 100 steps at 3,000 K."""
    key = "hot216"
    if key not in _SYS:
        s = B.amorphous_carbon(216, density_g_cm3=2.0, min_sep=1.2, seed=61)
        _SYS[key] = B.relax_hot(s, 100, 3000.0, DT, M.POT_AIREBO, seed=62)
    return _SYS[key]


def ctx_for(s, pot=M.POT_AIREBO, params=None, vel=None):
    # One REBO task mode for every run (no autotuner): the two modes agree to
    # rounding, and over 200 steps of hot carbon rounding-level differences
    # of the force grow by ~e^12, enough to change the trajectory's gradient.
    c = M.Context(potentials=pot, task_mode=1)
    for k, v in (params or {}).items():
        c.set_param(k, v)
    c.set_system(s["z"], s["pos"], s["vel"] if vel is None else vel, s["box"], s["pbc"], s["fixed"])
    return c


def grad_at(c, pos):
    c.set_state(pos)
    return c.compute()


def default_params():
    c = M.Context(potentials=M.POT_AIREBO)
    return np.array([c.get_param(k) for k in range(M.NPARAM)])


# ---------------------------------------------------------------- products
def test_force_product_symmetric_without_torsion():
    s = ac(300, 71)
    c = ctx_for(s, M.POT_REBO | M.POT_AIREBO_LJ)
    rng = np.random.default_rng(1)
    u = rng.normal(size=s["pos"].shape)
    _, _, g0 = c.compute()
    out = c.force_product(u)
    # the values of the dual pass are the FP64 path's gradient
    assert np.linalg.norm(out["grad"] - g0) <= 1e-12 * np.linalg.norm(g0)
    h = 1e-5
    x = s["pos"].copy()
    fd = (grad_at(c, x + h * u)[2] - grad_at(c, x - h * u)[2]) / (2 * h)
    err = np.linalg.norm(out["ju"] - fd) / np.linalg.norm(fd)
    assert err < 1e-6, err
    c.set_state(x)
    assert np.array_equal(c.force_product(u, transpose=False)["ju"], out["ju"])


def test_force_product_transpose_with_torsion():
    s = ac(300, 72)
    c = ctx_for(s, M.POT_AIREBO)
    rng = np.random.default_rng(2)
    x = s["pos"].copy()
    h = 1e-5
    for trial in range(3):
        u = rng.normal(size=x.shape)
        v = rng.normal(size=x.shape)
        c.set_state(x)
        jtu = c.force_product(u)["ju"]
        jv = (grad_at(c, x + h * v)[2] - grad_at(c, x - h * v)[2]) / (2 * h)
        a, b = float(np.sum(v * jtu)), float(np.sum(u * jv))
        assert abs(a - b) <= 1e-6 * np.linalg.norm(v) * np.linalg.norm(jtu), (trial, a, b)
        # the forward product is J v itself
        c.set_state(x)
        jv_d = c.force_product(v, transpose=False)["ju"]
        assert np.linalg.norm(jv_d - jv) <= 1e-6 * np.linalg.norm(jv), trial
    # the exact gradient of the energy (the reference's torsion force is not)
    c.set_state(x)
    ge = c.force_product(np.zeros_like(x))["grad"]
    v = rng.normal(size=x.shape)
    fd = (grad_at(c, x + h * v)[0] - grad_at(c, x - h * v)[0]) / (2 * h)
    assert abs(np.sum(v * ge) - fd) <= 1e-7 * np.linalg.norm(v) * np.linalg.norm(ge), (np.sum(v * ge), fd)


def test_parameter_derivatives():
    s = ac(300, 73)
    rng = np.random.default_rng(3)
    u = rng.normal(size=s["pos"].shape)
    p0 = default_params()
    out = ctx_for(s).force_product(u)
    for k in range(M.NPARAM):
        h = 1e-6 * p0[k]
        e, up = [], []
        for sgn in (1, -1):
            c = ctx_for(s, params={k: p0[k] + sgn * h})
            ee, _, g = c.compute()
            e.append(ee)
            up.append(float(np.sum(u * g)))
        fd_e = (e[0] - e[1]) / (2 * h)
        fd_p = (up[0] - up[1]) / (2 * h)
        assert abs(out["de_dparam"][k] - fd_e) <= 1e-6 * abs(fd_e) + 1e-9, (M.PARAM_NAMES[k], out["de_dparam"][k], fd_e)
        assert abs(out["dprod_dparam"][k] - fd_p) <= 1e-6 * abs(fd_p) + 1e-9, (M.PARAM_NAMES[k], out["dprod_dparam"][k], fd_p)


# ---------------------------------------------------------------- trajectories
def loss_of(xN, vN, epot, z, target):
    m = B.masses(z)
    ekin = 0.5 * np.sum(m[:, None] * vN ** 2) / CONV
    return float(np.mean(np.sum((xN - target) ** 2, axis=1)) + LAM * (epot + ekin))


def seeds_of(xN, vN, z, target):
    n = len(z)
    m = B.masses(z)
    return 2.0 * (xN - target) / n, LAM * m[:, None] * vN / CONV, LAM


def gpu_loss(s, nsteps, target, params=None, pos=None, vel=None, every=20):
    c = M.Context(potentials=M.POT_AIREBO, task_mode=1)
    for k, v in (params or {}).items():
        c.set_param(k, v)
    c.set_system(s["z"], s["pos"] if pos is None else pos, s["vel"] if vel is None else vel, s["box"], s["pbc"],
                 s["fixed"])
    xN, vN, ep = c.adjoint_forward(nsteps, DT, every)
    return loss_of(xN, vN, ep, s["z"], target)


def ref_loss(s, nsteps, target, params=None):
    r = ref.RefSystem(ref.POT_AIREBO)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    for k, v in (params or {}).items():
        r.set_param(k, v)
    out = r.run(nsteps, DT)
    xN = out["pos"] + out["image"] * np.asarray(s["box"])[None, :]
    return loss_of(xN, out["vel"], out["epot"][-1], s["z"], target)


def adjoint(s, nsteps, every, target=None, seed=5):
    c = ctx_for(s)
    xN, vN, ep = c.adjoint_forward(nsteps, DT, every)
    if target is None:
        target = xN + 0.01 * np.random.default_rng(seed).normal(size=xN.shape)
    sx, sv, se = seeds_of(xN, vN, s["z"], target)
    gp, gx, gv = c.adjoint_backward(sx, sv, se)
    return gp, gx, gv, target, c


NSTEPS = 40      # long horizon (tangent-linear checks, checkpoint tests)
NFD = 10         # finite-difference horizon: central differences converge to ~1e-6 here
HFD = 1e-5       # relative finite-difference step


def test_adjoint_matches_gpu_finite_differences():
    s = hot216()
    gp, gx, gv, target, _ = adjoint(s, NFD, 3)
    p0 = default_params()
    for k in range(M.NPARAM):
        h = HFD * p0[k]
        fd = (gpu_loss(s, NFD, target, {k: p0[k] + h}) - gpu_loss(s, NFD, target, {k: p0[k] - h})) / (2 * h)
        assert abs(gp[k] - fd) <= 1e-4 * abs(fd), (M.PARAM_NAMES[k], gp[k], fd)
    rng = np.random.default_rng(9)
    d = rng.normal(size=s["pos"].shape)
    h = 1e-6
    fd = (gpu_loss(s, NFD, target, pos=s["pos"] + h * d) - gpu_loss(s, NFD, target, pos=s["pos"] - h * d)) / (2 * h)
    assert abs(np.sum(gx * d) - fd) <= 1e-4 * abs(fd), (np.sum(gx * d), fd)
    d = rng.normal(size=s["pos"].shape) * 0.01
    fd = (gpu_loss(s, NFD, target, vel=s["vel"] + h * d) - gpu_loss(s, NFD, target, vel=s["vel"] - h * d)) / (2 * h)
    assert abs(np.sum(gv * d) - fd) <= 1e-4 * abs(fd), (np.sum(gv * d), fd)


def test_adjoint_matches_reference_finite_differences():
    """The gradient from the FP64 reference: central differences of the
    unmodified SimLoop run of the oracle with each parameter moved."""
    s = hot216()
    gp, _, _, target, _ = adjoint(s, NFD, 3)
    p0 = default_params()
    for k in range(M.NPARAM):
        h = HFD * p0[k]
        fd = (ref_loss(s, NFD, target, {k: p0[k] + h}) - ref_loss(s, NFD, target, {k: p0[k] - h})) / (2 * h)
        assert abs(gp[k] - fd) <= 1e-4 * abs(fd), (M.PARAM_NAMES[k], gp[k], fd)


def tangent_linear(s, nsteps, target, directions=None, hrel=1e-7):
    """dL along each parameter (directions None) or along initial-position
    directions [m, n, 3], by the tangent-linear model of the same trajectory:
    dx' = dx + dv dt + da dt^2/2, da' = -c/m (J(x') dx' + dg/dtheta(x')),
    dv' = dv + (da + da') dt/2, with J u from the dual pass (transpose=False)
    and dg/dtheta from central differences of single force evaluations.

    The difference step is 1e-7 relative: the LJ switch S(t_r) has jumps of
    its second derivative at r = sigma and r = 2^(1/6) sigma, so a step of
    h sigma in sigma straddles them for every pair within h sigma of either
    distance (about 3e4 pairs per Angstrom at 4,096 atoms of 2.0 g/cm^3:
    one pair per step at h = 1e-5, whose difference then is no derivative;
    measured on the 200-step workload: 8e-3 relative at h = 1e-5, 8e-10 at
    1e-7)."""
    c = ctx_for(s)
    traj = [c.get_state()[0]]
    for _ in range(nsteps):
        c.run(1, DT, energies=False)
        traj.append(c.get_state()[0])
    xN, vN, img = c.get_state()
    xN = xN + img * np.asarray(s["box"])[None, :]
    m = B.masses(s["z"])[:, None]
    n = len(s["z"])
    p0 = default_params()
    if directions is None:
        nd = M.NPARAM
        pert = []
        for k in range(M.NPARAM):
            pert.append([ctx_for(s, params={k: p0[k] * (1 + sg * hrel)}) for sg in (1, -1)])

        def forcing(x):
            out = np.zeros((nd, n, 3))
            for k in range(nd):
                gp_ = grad_at(pert[k][0], x)[2]
                gm_ = grad_at(pert[k][1], x)[2]
                out[k] = (gp_ - gm_) / (2 * hrel * p0[k])
            return out
        dx = np.zeros((nd, n, 3))
    else:
        nd = len(directions)

        def forcing(x):
            return np.zeros((nd, n, 3))
        dx = np.array(directions, dtype=float)
    dv = np.zeros_like(dx)

    def jprod(x, d):
        c.set_state(x)
        return np.array([c.force_product(d[k], transpose=False)["ju"] for k in range(nd)])
    da = -CONV / m * (jprod(traj[0], dx) + forcing(traj[0]))
    for step in range(nsteps):
        dx = dx + dv * DT + da * DT * DT / 2.0
        da_new = -CONV / m * (jprod(traj[step + 1], dx) + forcing(traj[step + 1]))
        dv = dv + (da + da_new) * DT / 2.0
        da = da_new
    c.set_state(traj[nsteps])
    fin = c.force_product(np.zeros((n, 3)))
    sx, sv, se = seeds_of(xN, vN, s["z"], target)
    dl = np.array([np.sum(sx * dx[k]) + np.sum(sv * dv[k]) + se * np.sum(fin["grad"] * dx[k]) for k in range(nd)])
    if directions is None:
        dl += se * fin["de_dparam"]
    return dl


def test_adjoint_matches_tangent_linear_model():
    s = hot216()
    gp, gx, _, target, _ = adjoint(s, NSTEPS, 7)
    tl = tangent_linear(s, NSTEPS, target)
    for k in range(M.NPARAM):
        assert abs(gp[k] - tl[k]) <= 1e-5 * abs(tl[k]), (M.PARAM_NAMES[k], gp[k], tl[k])
    d = np.random.default_rng(12).normal(size=(2,) + s["pos"].shape)
    tl = tangent_linear(s, NSTEPS, target, directions=d)
    for q in range(2):
        a = float(np.sum(gx * d[q]))
        assert abs(a - tl[q]) <= 1e-8 * abs(tl[q]), (q, a, tl[q])


def test_checkpoint_interval_and_determinism():
    s = hot216()
    a = adjoint(s, NSTEPS, 7)
    b = adjoint(s, NSTEPS, NSTEPS, target=a[3])
    c = adjoint(s, NSTEPS, 7, target=a[3])
    for x, y in zip(a[:3], c[:3]):
        assert np.array_equal(x, y)  # bitwise repeatable
    for x, y in zip(a[:3], b[:3]):
        assert np.linalg.norm(x - y) <= 1e-10 * np.linalg.norm(y)


def test_backward_leaves_final_state():
    s = hot216()
    c = ctx_for(s)
    xN, vN, _ = c.adjoint_forward(10, DT, 3)
    c.adjoint_backward(np.ones_like(xN), None, 0.0)
    p, v, img = c.get_state()
    assert np.allclose(p + img * np.asarray(s["box"])[None, :], xN, rtol=0, atol=1e-12)
    assert np.array_equal(v, vN)


# ---------------------------------------------------------------- torch wrapper
def test_torch_autograd_function():
    torch = pytest.importorskip("torch")

    class Trajectory(torch.autograd.Function):
        """(params, x0, v0) -> (x_N unwrapped, v_N, E_pot(x_N)) through the
        mdg adjoint ABI."""

        @staticmethod
        def forward(fctx, params, x0, v0, s, nsteps, every):
            c = M.Context(potentials=M.POT_AIREBO)
            for k in range(M.NPARAM):
                c.set_param(k, float(params[k]))
            c.set_system(s["z"], x0.detach().numpy(), v0.detach().numpy(), s["box"], s["pbc"], s["fixed"])
            xN, vN, ep = c.adjoint_forward(nsteps, DT, every)
            fctx.c = c
            return torch.from_numpy(xN), torch.from_numpy(vN), torch.tensor(ep, dtype=torch.float64)

        @staticmethod
        def backward(fctx, gx, gv, ge):
            gp, gx0, gv0 = fctx.c.adjoint_backward(gx.numpy(), gv.numpy(), float(ge))
            return torch.from_numpy(gp), torch.from_numpy(gx0), torch.from_numpy(gv0), None, None, None

    s = hot216()
    params = torch.tensor(default_params(), dtype=torch.float64, requires_grad=True)
    x0 = torch.tensor(s["pos"], requires_grad=True)
    v0 = torch.tensor(s["vel"], requires_grad=True)
    xN, vN, ep = Trajectory.apply(params, x0, v0, s, 20, 6)
    target = xN.detach() + 0.01 * torch.from_numpy(np.random.default_rng(11).normal(size=xN.shape))
    m = torch.from_numpy(B.masses(s["z"]))
    loss = ((xN - target) ** 2).sum(1).mean() + LAM * (ep + 0.5 * (m[:, None] * vN ** 2).sum() / CONV)
    loss.backward()
    gp, gx, gv, _, _ = adjoint(s, 20, 6, target=target.numpy())
    # the seeds torch forms equal ours to rounding
    for a, b in ((params.grad.numpy(), gp), (x0.grad.numpy(), gx), (v0.grad.numpy(), gv)):
        assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b)


# ---------------------------------------------------------------- the adjoint workload
def test_adjoint_workload_4096_amorphous_carbon():
    """4,096 C at 2.0 g/cm^3 (box 34.43 A), pre-relaxed 500 steps at 3,000 K;
    200 steps of 0.5 fs, checkpoint every 20.  The six parameter gradients
    of the 200-step loss against the tangent-linear model, and of a 10-step
    loss against central finite differences."""
    s0 = B.amorphous_carbon(4096, density_g_cm3=2.0, min_sep=1.2, seed=81)
    assert abs(s0["box"][0] - 34.43) < 0.01
    s = B.relax_hot(s0, 500, 3000.0, DT, M.POT_AIREBO, seed=82)
    gp, gx, _, target, _ = adjoint(s, 200, 20, seed=83)
    assert np.all(np.isfinite(gp)) and np.all(np.isfinite(gx))
    tl = tangent_linear(s, 200, target)
    for k in range(M.NPARAM):
        assert abs(gp[k] - tl[k]) <= 1e-5 * abs(tl[k]), (M.PARAM_NAMES[k], gp[k], tl[k])
    # central differences over a short horizon: the step must be small enough
    # for the linear regime of this hot system and large enough for the
    # reference arithmetic's noise floor; the adjoint must agree with the
    # difference at one of three steps
    gp10, _, _, t10, _ = adjoint(s, NFD, NFD, seed=84)
    p0 = default_params()
    for k in range(M.NPARAM):
        errs = []
        for hr in (1e-5, 1e-6, 1e-7):
            h = hr * p0[k]
            fd = (gpu_loss(s, NFD, t10, {k: p0[k] + h}) - gpu_loss(s, NFD, t10, {k: p0[k] - h})) / (2 * h)
            errs.append(abs(gp10[k] - fd) / abs(fd))
        assert min(errs) <= 1e-4, (M.PARAM_NAMES[k], gp10[k], errs)
