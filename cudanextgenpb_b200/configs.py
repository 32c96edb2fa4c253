"""Workloads: the charged Born sphere and seeded synthetic molecules.

The synthetic molecules stand in for real proteins (no dataset is used): atom
centres are a seeded random subset of face-centred-cubic lattice sites with
nearest-neighbour distance 2.5 A inside a sphere, radii drawn from
{1.2 (H): 0.5, 1.7 (C): 0.3, 1.55 (N): 0.1, 1.52 (O): 0.1} A, partial charges
N(0, 0.35) e shifted so the molecule carries a chosen integer net charge.  A
lattice subset is used because random sequential addition cannot reach the
packing density that 2,000 centres at >= 2.5 A inside an 18 A sphere need.
"""
from __future__ import annotations

import math

import numpy as np

# include/pb_class.h:47-54
E_0, KB, E_CH, N_AV, ANGS, PI = 8.85418781762e-12, 1.380649e-23, 1.602176634e-19, 6.022e23, 1e-10, math.pi


def scaled_constants(e_in=2.0, e_out=80.0, ionic=0.145, T=298.15):
    """eps_in, eps_out (kT/e units) and kappa as computed at src/pb_class.cpp:1800-1806."""
    eps_in = 4.0 * PI * E_0 * e_in * KB * T * ANGS / (E_CH * E_CH)
    eps_out = 4.0 * PI * E_0 * e_out * KB * T * ANGS / (E_CH * E_CH)
    c0 = 1.0e3 * N_AV * ionic
    k2 = 2.0 * c0 * ANGS * ANGS * E_CH * E_CH / (E_0 * e_out * KB * T)
    return eps_in, eps_out, math.sqrt(k2)


def born_energy(a=2.0, q=1.0, e_in=2.0, e_out=80.0, ionic=0.145, T=298.15):
    """Analytic solvation energy [kT] of a charge q at the centre of a sphere of radius a
    in an ionic solvent (Born / Debye-Hueckel): q^2/2a (1/(eps_out(1+kappa a)) - 1/eps_in)."""
    eps_in, eps_out, k = scaled_constants(e_in, e_out, ionic, T)
    return 0.5 * q * q * (1.0 / (eps_out * (1.0 + k * a)) - 1.0 / eps_in) / a


_BORN_TEMPLATE = r"""
[mesh]
mesh_shape = 2
x1 = {lo}
x2 = {hi}
y1 = {lo}
y2 = {hi}
z1 = {lo}
z2 = {hi}
unilevel = {unilevel}
loc_refinement = 1
minlevel = {unilevel}
maxlevel = {maxlevel}
[../]
[model]
bc_type = {bc_type}
molecular_dielectric_constant = 2
solvent_dielectric_constant = 80
ionic_strength = 0.145
T = 298.15
calc_energy = 2
calc_coulombic = 1
[../]
[algorithm]
linear_solver = lis
solver_options = -i\ bicgstab\ -p\ jacobi\ -tol\ 1.e-8
[../]
"""


def born_options(unilevel=5, maxlevel=6, half=8.0, bc_type=3):
    """Born sphere: box [-half, half]^3 (4x the 4 A sphere extent for half = 8), uniform
    level `unilevel` (2 nodes/A at 5), surface refined to `maxlevel`, analytic Dirichlet data,
    BiCGStab + Jacobi to 1e-8."""
    return _BORN_TEMPLATE.format(lo=-half, hi=half, unilevel=unilevel, maxlevel=maxlevel, bc_type=bc_type)


BORN_OPTIONS = born_options()


BORN_ATOM = (np.zeros((1, 3)), np.array([1.0]), np.array([2.0]))


def synthetic_molecule(n_atoms: int, radius: float, net_charge: float, seed: int):
    """Seeded synthetic molecule (positions n x 3, charges, radii)."""
    rng = np.random.default_rng(seed)
    a = 2.5 * math.sqrt(2.0)  # FCC cube edge for nearest-neighbour 2.5 A
    m = int(math.ceil(radius / a)) + 1
    g = np.arange(-m, m + 1)
    base = np.array(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1).T.astype(np.float64)
    offs = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    sites = (base[:, None, :] + offs[None, :, :]).reshape(-1, 3) * a
    sites = sites[np.linalg.norm(sites, axis=1) <= radius]
    if len(sites) < n_atoms:
        raise ValueError("sphere of radius %g holds only %d lattice sites" % (radius, len(sites)))
    pos = sites[rng.choice(len(sites), size=n_atoms, replace=False)]
    pos = pos + rng.uniform(-0.05, 0.05, size=pos.shape)  # break exact lattice alignment with the mesh
    radii = rng.choice(np.array([1.2, 1.7, 1.55, 1.52]), size=n_atoms, p=[0.5, 0.3, 0.1, 0.1])
    q = rng.normal(0.0, 0.35, size=n_atoms)
    q += (net_charge - q.sum()) / n_atoms
    return pos, q, radii


def globular_options(scale=2.0, perfil1=0.9, perfil2=0.2, levels=3, bc_type=1, solver="-i\\ cg\\ -p\\ jacobi\\ -tol\\ 1.e-8"):
    """mesh_shape 0 (derefined cubic box scaled by `scale`), `levels` surface refinement levels."""
    return r"""
[mesh]
mesh_shape = 0
perfil1 = %g
perfil2 = %g
scale = %g
loc_refinement = 1
unilevel = 5
minlevel = 3
maxlevel = @MAXLEVEL@
[../]
[model]
bc_type = %d
molecular_dielectric_constant = 2
solvent_dielectric_constant = 80
ionic_strength = 0.145
T = 298.15
calc_energy = 2
calc_coulombic = 1
[../]
[algorithm]
linear_solver = lis
solver_options = %s
[../]
""" % (perfil1, perfil2, scale, bc_type, solver), levels


def scale_level_for(pos, radii, scale=2.0, perfil2=0.2, prb_radius=1.4):
    """scale_level that create_mesh (mesh_shape 0) derives, src/pb_class.cpp:152-167."""
    maxr = float(np.max(radii))
    l = (pos.max(axis=0) + maxr + 2 * prb_radius) - (pos.min(axis=0) - maxr - 2 * prb_radius)
    lmax = float(l.max())
    size, lvl = 1.0 / scale, 0
    for _ in range(29):
        size *= 2
        lvl += 1
        if lmax / size < perfil2:
            break
    return lvl


def make_globular_problem(n_atoms, radius, net_charge, seed, scale=2.0, levels=3, perfil1=0.9, perfil2=0.2,
                          solver="-i\\ cg\\ -p\\ jacobi\\ -tol\\ 1.e-8", bc_type=1):
    """Host problem for a synthetic molecule with `levels` surface refinement levels."""
    from .pb import Problem
    pos, q, r = synthetic_molecule(n_atoms, radius, net_charge, seed)
    text, lv = globular_options(scale, perfil1, perfil2, levels, bc_type, solver)
    sl = scale_level_for(pos, r, scale, perfil2)
    prob = Problem(text.replace("@MAXLEVEL@", str(sl + lv)))
    prob.set_atoms(pos, q, r)
    return prob


def make_born_problem(unilevel=5, maxlevel=6, half=8.0, bc_type=3):
    from .pb import Problem
    prob = Problem(born_options(unilevel, maxlevel, half, bc_type))
    prob.set_atoms(*BORN_ATOM)
    return prob


def radius_for(n_atoms: int) -> float:
    """Smallest radius (0.5 A steps) whose sphere holds the n atoms at <= 90%
    of the FCC lattice sites (the 2,000-atom configuration uses 18 A)."""
    a = 2.5 * math.sqrt(2.0)
    r = max(4.0, round((n_atoms / 0.9 / (4.0 / a ** 3) / (4.0 / 3.0 * math.pi)) ** (1.0 / 3.0) * 2) / 2)
    while True:
        m = int(math.ceil(r / a)) + 1
        g = np.arange(-m, m + 1)
        base = np.array(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1).T.astype(np.float64)
        offs = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
        sites = (base[:, None, :] + offs[None, :, :]).reshape(-1, 3) * a
        if (np.linalg.norm(sites, axis=1) <= r).sum() * 0.9 >= n_atoms:
            return r
        r += 0.5


def molecule_specs(count: int, lo: int, hi: int, seed: int):
    """Seeded molecule specs for batches and request streams: atom counts
    log-uniform in [lo, hi], integer net charges in [-5, 5]; each spec is
    (n_atoms, radius, net_charge, seed)."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count)).astype(int)
    net = rng.integers(-5, 6, size=count)
    return [(int(k), radius_for(int(k)), float(c), int(seed * 1000 + j)) for j, (k, c) in enumerate(zip(n, net))]
