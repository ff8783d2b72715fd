"""Seeded synthetic hydrocarbon systems (the reference ships no builders).

Every builder returns a dict with
    z      int32 [n]      atomic numbers (6 = C, 1 = H)
    pos    float64 [n,3]  positions, Angstrom
    vel    float64 [n,3]  velocities, Angstrom/fs
    box    float64 [3]    periods (Angstrom); ignored on non-periodic axes
    pbc    int32 [3]      1 = periodic axis
    fixed  uint8 [n]      1 = atom held fixed (Atom::fix, mdtk/Atom.hpp:58)

Masses and constants are the reference's (mdtk/Atom.hpp:104-105,
mdtk/consts.cxx:28-36): C 12 amu, H 1 amu, kb = 8.617343e-5 eV/K.
Velocities follow the recipe: Gaussian per component with sigma =
sqrt(kb T / M), zero net momentum (AtomsArray::removeMomentum,
mdtk/AtomsContainer.cxx:269-278), then rescaled so that the reference's
temperatureWithoutFixed() (mdtk/SimLoop.cxx:548-568: Ekin / (1.5 kb N), no
degree-of-freedom correction) equals T.
"""
from __future__ import annotations

import math
from typing import Dict

import numpy as np

KB_EV = 8.617343e-5
EV_ERG = 1.6021e-12
AMU_G = 1.6605655e-24
# 1 eV/amu expressed in (Angstrom/fs)^2, with the reference's constants
EV_PER_AMU_A2FS2 = EV_ERG / AMU_G * 1e16 / 1e30
MASS = {6: 12.0, 1: 1.0}


# Atom::setAttributesByElementID (mdtk/Atom.hpp:100-115): amu by atomic number
MASS_AMU = {1: 1.0, 6: 12.0, 29: 63.546, 47: 107.868, 79: 196.967, 18: 39.948, 54: 131.293}


def masses(z: np.ndarray) -> np.ndarray:
    z = np.asarray(z)
    out = np.empty(z.shape, float)
    for k, m in MASS_AMU.items():
        out[z == k] = m
    return out


def temperature(z, vel, fixed=None) -> float:
    """temperatureWithoutFixed (mdtk/SimLoop.cxx:548-568) in K."""
    m = masses(z)
    free = np.ones(len(z), bool) if fixed is None else (np.asarray(fixed) == 0)
    if not free.any():
        return 0.0
    ek = 0.5 * np.sum(m[free, None] * vel[free] ** 2) / EV_PER_AMU_A2FS2
    return ek / (1.5 * KB_EV * free.sum())


def thermal_velocities(z, temp_k: float, rng: np.random.Generator, fixed=None) -> np.ndarray:
    n = len(z)
    m = masses(z)
    free = np.ones(n, bool) if fixed is None else (np.asarray(fixed) == 0)
    vel = np.zeros((n, 3))
    if temp_k <= 0 or not free.any():
        return vel
    sig = np.sqrt(KB_EV * temp_k / m * EV_PER_AMU_A2FS2)
    vel[free] = rng.normal(size=(free.sum(), 3)) * sig[free, None]
    p = np.sum(m[free, None] * vel[free], axis=0)
    vel[free] -= p / m[free].sum()
    t_now = temperature(z, vel, fixed)
    if t_now > 0:
        vel *= math.sqrt(temp_k / t_now)
    return vel


def _system(z, pos, vel, box, pbc, fixed=None) -> Dict[str, np.ndarray]:
    n = len(z)
    return {
        "z": np.ascontiguousarray(z, dtype=np.int32),
        "pos": np.ascontiguousarray(pos, dtype=np.float64).reshape(n, 3),
        "vel": np.ascontiguousarray(vel, dtype=np.float64).reshape(n, 3),
        "box": np.ascontiguousarray(box, dtype=np.float64),
        "pbc": np.ascontiguousarray(pbc, dtype=np.int32),
        "fixed": np.zeros(n, np.uint8) if fixed is None else np.ascontiguousarray(fixed, dtype=np.uint8),
    }


def diamond(nx: int, ny: int = None, nz: int = None, a: float = 3.567, temp_k: float = 0.0,
            disp_sigma: float = 0.0, seed: int = 0) -> Dict[str, np.ndarray]:
    """Diamond-cubic carbon, nx*ny*nz cubic cells of 8 atoms, periodic box."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    basis = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]], float)
    basis = np.vstack([basis, basis + 0.25])
    cells = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    pos = ((cells[:, None, :] + basis[None, :, :]).reshape(-1, 3)) * a
    rng = np.random.default_rng(seed)
    if disp_sigma > 0:
        pos = pos + rng.normal(scale=disp_sigma, size=pos.shape)
    box = np.array([nx, ny, nz], float) * a
    pos = np.mod(pos, box)
    z = np.full(len(pos), 6, np.int32)
    vel = thermal_velocities(z, temp_k, rng)
    return _system(z, pos, vel, box, [1, 1, 1])


def _ethane_template(r_cc: float = 1.54, r_ch: float = 1.09) -> np.ndarray:
    """Staggered ethane, C-C along x, tetrahedral H-C-C; returns [8,3] with C0, C1, H*6."""
    th = math.acos(-1.0 / 3.0)  # tetrahedral angle
    c0 = np.array([-r_cc / 2, 0, 0])
    c1 = np.array([r_cc / 2, 0, 0])
    out = [c0, c1]
    for ci, sgn, phase in ((c0, -1.0, 0.0), (c1, 1.0, math.pi / 3)):
        for k in range(3):
            ang = phase + 2 * math.pi * k / 3
            d = np.array([sgn * -math.cos(th), math.sin(th) * math.cos(ang), math.sin(th) * math.sin(ang)])
            out.append(ci + r_ch * d)
    return np.array(out)


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def ethane_liquid(n_mol: int, density_g_cm3: float = 0.55, temp_k: float = 300.0, seed: int = 0,
                  min_dist: float = 2.0, jitter: float = 0.25) -> Dict[str, np.ndarray]:
    """n_mol ethane molecules (staggered, C-C 1.54 A, C-H 1.09 A, tetrahedral
    H-C-C) in a periodic cubic box whose size gives the requested density
    (reference masses: 30 amu per molecule).

    Random sequential insertion jams well below liquid density, so each
    molecule takes a randomly chosen site of a lattice filling the box,
    a seeded random displacement of up to `jitter` A per axis and a uniformly
    random orientation; orientations are redrawn until every intermolecular
    atom pair is at least min_dist apart.  The lattice is FCC or simple cubic,
    whichever spaces the sites further apart for this molecule count."""
    mass_g = n_mol * 30.0 * AMU_G
    L = (mass_g / density_g_cm3) ** (1.0 / 3.0) * 1e8
    rng = np.random.default_rng(seed)
    # the lattice (FCC or simple cubic) whose nearest-neighbour spacing is larger
    m = 1
    while 4 * m ** 3 < n_mol:
        m += 1
    k = 1
    while k ** 3 < n_mol:
        k += 1
    if L / (m * math.sqrt(2.0)) >= L / k:
        basis = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])
        ncell = m
    else:
        basis = np.zeros((1, 3))
        ncell = k
    a = L / ncell
    cells = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell), indexing="ij"), -1).reshape(-1, 3)
    sites = ((cells[:, None, :] + basis[None]).reshape(-1, 3) + 0.25) * a
    order = sites[rng.permutation(len(sites))]
    # the first n_mol sites of the permutation are used in turn; a site where no
    # orientation fits (its neighbours jammed it) is given up for the next
    # unused site, so every seed builds while the lattice has spare sites
    spare = list(order[n_mol:][::-1])
    tmpl = _ethane_template()
    ng = max(1, int(L // min_dist))
    csz = L / ng
    grid: Dict[tuple, list] = {}
    placed = []
    for center0 in order[:n_mol]:
        at, keys = _place_ethane(rng, tmpl, center0, L, jitter, min_dist, grid, csz, ng)
        while at is None:
            if not spare:
                raise RuntimeError("ethane_liquid: no clash-free orientation; lower the density or min_dist")
            at, keys = _place_ethane(rng, tmpl, spare.pop(), L, jitter, min_dist, grid, csz, ng)
        for p, k in zip(at, keys):
            grid.setdefault(k, []).append(p)
        placed.append(at)
    pos = np.concatenate(placed, 0)
    z = np.tile(np.array([6, 6, 1, 1, 1, 1, 1, 1], np.int32), n_mol)
    vel = thermal_velocities(z, temp_k, rng)
    return _system(z, pos, vel, [L, L, L], [1, 1, 1])


def _place_ethane(rng, tmpl, center0, L, jitter, min_dist, grid, csz, ng, attempts: int = 5000):
    """A random orientation and jitter of one ethane molecule about a lattice
    site with every atom at least min_dist from the atoms already placed:
    (atoms, their grid cells), or (None, None) when `attempts` draws all clash."""
    for _ in range(attempts):
        R = _random_rotations(rng, 1)[0]
        center = center0 + rng.uniform(-jitter, jitter, size=3)
        at = np.mod((tmpl @ R.T) + center, L)
        keys = [tuple((p // csz).astype(int) % ng) for p in at]
        ok = True
        for p, ci in zip(at, keys):
            near = []
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        lst = grid.get(((ci[0] + dx) % ng, (ci[1] + dy) % ng, (ci[2] + dz) % ng))
                        if lst:
                            near.extend(lst)
            if near:
                d = p - np.array(near)
                d -= L * np.round(d / L)
                if np.min(np.einsum("ij,ij->i", d, d)) < min_dist * min_dist:
                    ok = False
                    break
        if ok:
            return at, keys
    return None, None


def amorphous_carbon(n: int, density_g_cm3: float = 2.0, min_sep: float = 1.2, temp_k: float = 0.0,
                     h_fraction: float = 0.0, seed: int = 0) -> Dict[str, np.ndarray]:
    """Random carbon (optionally with a fraction of H) at the given density,
    random sequential placement with a minimum separation, periodic cubic box."""
    rng = np.random.default_rng(seed)
    z = np.full(n, 6, np.int32)
    if h_fraction > 0:
        z[rng.random(n) < h_fraction] = 1
    mass_g = masses(z).sum() * AMU_G
    L = (mass_g / density_g_cm3) ** (1.0 / 3.0) * 1e8
    ncell = max(1, int(L // min_sep))
    csz = L / ncell
    grid: Dict[tuple, list] = {}
    pos = np.zeros((n, 3))
    i = 0
    tries = 0
    while i < n:
        tries += 1
        if tries > 2000 * n:
            raise RuntimeError("amorphous_carbon: could not place atoms")
        p = rng.uniform(0, L, size=3)
        ci = tuple((p // csz).astype(int) % ncell)
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    lst = grid.get(((ci[0] + dx) % ncell, (ci[1] + dy) % ncell, (ci[2] + dz) % ncell))
                    if not lst:
                        continue
                    d = p - np.array(lst)
                    d -= L * np.round(d / L)
                    if np.min(np.einsum("ij,ij->i", d, d)) < min_sep * min_sep:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        grid.setdefault(ci, []).append(p)
        pos[i] = p
        i += 1
    vel = thermal_velocities(z, temp_k, rng)
    return _system(z, pos, vel, [L, L, L], [1, 1, 1])


def c2h6_example() -> Dict[str, np.ndarray]:
    """The reference's 8-atom ethane example (examples/C2H6/main.cpp:38-45),
    non-periodic, at rest."""
    pos = np.array([
        [0.0, 0.0, 0.0], [1.5, 0.0, 0.0],
        [1.9, 0.0, 1.0], [1.9, -0.9, -0.5], [1.9, 0.9, -0.5],
        [-0.4, 0.0, 1.0], [-0.4, -0.9, -0.2], [-0.4, 0.8, -0.2],
    ])
    z = np.array([6, 6, 1, 1, 1, 1, 1, 1], np.int32)
    return _system(z, pos, np.zeros((8, 3)), [0.0, 0.0, 0.0], [0, 0, 0])


def graphite_slab(n_layers: int, nx: int, ny: int, cc: float = 1.42, interlayer: float = 3.35,
                  temp_k: float = 0.0, seed: int = 0, fix_bottom: bool = True) -> Dict[str, np.ndarray]:
    """AB-stacked graphite slab, lateral PBC (orthorhombic 4-atom cell per layer
    repeated nx * ny), z non-periodic, bottom layer fixed."""
    a = cc * math.sqrt(3.0)
    cell = np.array([a, 3.0 * cc])
    base = np.array([[0.0, 0.0], [a / 2, cc / 2], [a / 2, 1.5 * cc], [0.0, 2.0 * cc]])
    layers = []
    for l in range(n_layers):
        shift = np.array([0.0, cc]) if l % 2 else np.array([0.0, 0.0])
        for ix in range(nx):
            for iy in range(ny):
                xy = base + shift + np.array([ix, iy]) * cell
                layers.append(np.column_stack([xy, np.full(4, l * interlayer)]))
    pos = np.concatenate(layers, 0)
    box = np.array([nx * cell[0], ny * cell[1], 0.0])
    pos[:, 0] = np.mod(pos[:, 0], box[0])
    pos[:, 1] = np.mod(pos[:, 1], box[1])
    z = np.full(len(pos), 6, np.int32)
    fixed = np.zeros(len(pos), np.uint8)
    if fix_bottom:
        fixed[np.abs(pos[:, 2]) < 1e-9] = 1
    rng = np.random.default_rng(seed)
    vel = thermal_velocities(z, temp_k, rng, fixed)
    return _system(z, pos, vel, box, [1, 1, 0], fixed)


def impact(seed: int, n_target: int = None, e_min_ev: float = 10.0, e_max_ev: float = 100.0,
           temp_k: float = 0.0, cluster_atoms: int = 13) -> Dict[str, np.ndarray]:
    """One cluster-impact system: an AB graphite slab of about n_target atoms
    (uniform in [800, 6000] when not given; whole layers x lateral repeats,
    lateral periods >= 11 A so that checkMIC(2 x 5.5 A) holds), z open,
    bottom layer fixed, and a random C cluster (min separation 1.3 A) 8 A
    above the top layer moving straight down with kinetic energy uniform in
    [e_min_ev, e_max_ev] (AtomsArray::setTranslationalEnergy,
    mdtk/AtomsContainer.cxx:313-323: every cluster atom gets the same
    velocity)."""
    rng = np.random.default_rng(seed)
    if n_target is None:
        n_target = int(rng.integers(800, 6001))
    n_layers = int(rng.integers(2, 7))
    cells = max(1.0, n_target / (4.0 * n_layers))
    ny = max(3, int(round(math.sqrt(cells * 2.46 / 4.26))))
    nx = max(5, int(round(cells / ny)))
    slab = graphite_slab(n_layers, nx, ny, temp_k=temp_k, seed=seed)
    box = slab["box"]
    top = slab["pos"][:, 2].max()
    # cluster: rejection sampling in a ball
    cl = []
    radius = 2.6
    while len(cl) < cluster_atoms:
        p = rng.uniform(-radius, radius, 3)
        if np.linalg.norm(p) > radius:
            continue
        if all(np.linalg.norm(p - q) >= 1.3 for q in cl):
            cl.append(p)
    cl = np.array(cl)
    centre = np.array([rng.uniform(0, box[0]), rng.uniform(0, box[1]), top + 8.0])
    cl = cl - cl.mean(axis=0) + centre
    cl[:, 2] = np.maximum(cl[:, 2], top + 8.0 - radius)
    cl[:, 0] = np.mod(cl[:, 0], box[0])
    cl[:, 1] = np.mod(cl[:, 1], box[1])
    e_kin = rng.uniform(e_min_ev, e_max_ev)
    m_tot = 12.0 * cluster_atoms
    v = math.sqrt(2.0 * e_kin / m_tot * EV_PER_AMU_A2FS2)
    z = np.concatenate([slab["z"], np.full(cluster_atoms, 6, np.int32)])
    pos = np.concatenate([slab["pos"], cl])
    vel = np.concatenate([slab["vel"], np.tile([0.0, 0.0, -v], (cluster_atoms, 1))])
    fixed = np.concatenate([slab["fixed"], np.zeros(cluster_atoms, np.uint8)])
    return _system(z, pos, vel, box, [1, 1, 0], fixed)


def impact_batch(n_systems: int, seed: int = 0, **kw):
    """n_systems independent impact systems of uneven size (seeds seed, seed+1, ...)."""
    return [impact(seed + k, **kw) for k in range(n_systems)]


def relax_hot(s: Dict[str, np.ndarray], steps: int, temp_k: float, dt: float, potentials: int,
              seed: int = 0, device: int = 0) -> Dict[str, np.ndarray]:
    """Pre-relaxation of a random packing: `steps` velocity-Verlet steps on
    the GPU (mdg) with the velocities rescaled to temp_k after every step (a
    seeded Maxwell-Boltzmann start).  Returns a copy of s with the relaxed,
    wrapped positions and the final velocities; the same on every run."""
    from mdtk_b200 import Context

    rng = np.random.default_rng(seed)
    out = dict(s)
    vel = thermal_velocities(s["z"], temp_k, rng, s.get("fixed"))
    # one fixed REBO work split: the two splits agree to rounding only, and
    # 500 hot steps would turn a timing-dependent choice into a different state
    ctx = Context(potentials=potentials, device=device, task_mode=1)
    ctx.set_system(s["z"], s["pos"], vel, s["box"], s["pbc"], s.get("fixed"))
    for _ in range(steps):
        ctx.run(1, dt, energies=False)
        pos, v, _ = ctx.get_state()
        t_now = temperature(s["z"], v, s.get("fixed"))
        if t_now > 0:
            v = v * math.sqrt(temp_k / t_now)
        ctx.set_state(pos, v)
    pos, v, _ = ctx.get_state()
    ctx.close()
    out["pos"] = pos
    out["vel"] = v
    return out


# fcc lattice constants of the Ackland potential's metals (Ackland.cxx:330, 352, 374)
FCC_A = {29: 3.615, 47: 4.086, 79: 4.078}


def fcc(z: int, nx: int, ny: int = None, nz: int = None, a: float = None, temp_k: float = 0.0,
        disp_sigma: float = 0.0, pbc=(1, 1, 1), seed: int = 0) -> Dict[str, np.ndarray]:
    """An fcc metal crystal (Cu 29, Ag 47, Au 79), nx*ny*nz cubic cells of 4 atoms."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    a = FCC_A[z] if a is None else a
    basis = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]], float) + 0.25
    cells = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    pos = ((cells[:, None, :] + basis[None, :, :]).reshape(-1, 3)) * a
    rng = np.random.default_rng(seed)
    if disp_sigma > 0:
        pos = pos + rng.normal(scale=disp_sigma, size=pos.shape)
    box = np.array([nx, ny, nz], float) * a
    pos = np.where(np.asarray(pbc)[None, :] != 0, np.mod(pos, box), pos)
    zz = np.full(len(pos), z, np.int32)
    vel = thermal_velocities(zz, temp_k, rng)
    return _system(zz, pos, vel, box, list(pbc))


def add_atoms(s: Dict[str, np.ndarray], z, pos, vel=None, fixed=None) -> Dict[str, np.ndarray]:
    """s with more atoms appended (a projectile, an adsorbate)."""
    z = np.atleast_1d(np.asarray(z, np.int32))
    pos = np.asarray(pos, float).reshape(-1, 3)
    vel = np.zeros_like(pos) if vel is None else np.asarray(vel, float).reshape(-1, 3)
    fx = np.zeros(len(z), np.uint8) if fixed is None else np.asarray(fixed, np.uint8)
    return _system(np.concatenate([s["z"], z]), np.concatenate([s["pos"], pos]), np.concatenate([s["vel"], vel]),
                   s["box"], s["pbc"], np.concatenate([s["fixed"], fx]))
