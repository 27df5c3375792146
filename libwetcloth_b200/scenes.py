"""Seeded synthetic liquid scenes.

The reference seeds liquid from signed-distance "source" fields with jittered
resampling that draws ``rand()`` inside TBB loops
(libWetCloth/Core/DistanceFields.cpp:157-240), so its particle sets are not
reproducible.  These generators replace it with numpy ``default_rng`` streams;
per-particle attributes follow ``TwoDScene::sampleLiquidDistanceFields``
(libWetCloth/Core/TwoDScene.cpp:5564-5605): radius r, volume 4/3*pi*r^3,
mass rho*volume, zero affine matrix.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class SceneParams:
    """Scene-wide parameters of the fluid step (the liquid subset of
    ``LiquidInfo``, libWetCloth/Core/TwoDScene.h:35-91, plus bucket info and the
    solid box walls)."""

    dx: float = 1.0 / 64.0
    gravity: tuple = (0.0, -9.81, 0.0)
    liquid_density: float = 1000.0
    flip_coeff: float = 0.99
    liquid_boundary_friction: float = 0.0
    box_center: tuple = (0.5, 0.5, 0.5)
    box_half: tuple = (0.5, 0.5, 0.5)
    box_radius: float = 0.0
    criterion: float = 1e-6
    maxiters: int = 1000
    viscosity: float = 0.0        # LiquidInfo::viscosity; 0 = compute_viscosity off
    viscosity_substeps: int = 1   # LinearizedImplicitEuler viscosity sub-steps
    elasto_flip_coeff: float = 0.95       # LiquidInfo elasto_flip_coeff
    elasto_flip_asym_coeff: float = 1.0   # LiquidInfo elasto_flip_asym_coeff
    elasto_advect_coeff: float = 1.0      # LiquidInfo elasto_advect_coeff
    drag_viscosity: float = 8.9e-3        # LiquidInfo viscosity as the drag reads it
    # LiquidInfo::implicit_viscosity (stepImplicitViscosityDiagonalPCG) and the
    # stepper's viscous criterion
    viscosity_implicit: bool = False
    viscosity_criterion: float = 1e-6
    # correctLiquidParticles (TwoDScene.cpp:1967): LiquidInfo correction_strength
    # (0 turns it off), correction_step, correction_multiplier, and the seed of
    # the stream that picks each sub-step's particle subset
    correction_strength: float = 0.0
    correction_step: int = 8
    correction_multiplier: float = 2.0
    correction_seed: int = 0
    # relabel + mergeLiquidParticles before each sub-step, the seed of its
    # draws, and LiquidInfo::particle_cell_multiplier (V_fine)
    particle_merge: bool = False
    merge_seed: int = 0
    particle_split: bool = False   # relabel + splitLiquidParticles before each sub-step
    split_seed: int = 0
    particle_cell_multiplier: float = 0.3535533906
    # terminateParticles (TwoDScene.cpp:1756): one terminator box (a distance
    # field with usage "terminator"); inside=True removes the liquid particles
    # that leave it, inside=False the ones that enter it
    terminator: bool = False
    terminator_center: tuple = (0.5, 0.5, 0.5)
    terminator_half: tuple = (0.5, 0.5, 0.5)
    terminator_radius: float = 0.0
    terminator_inside: bool = True


def particle_radius(dx: float, ppc: int) -> float:
    """Radius whose sphere volume is dx^3/ppc (one particle per 1/ppc of a
    cell), i.e. particle_cell_multiplier * dx / sqrt(3) with the multiplier
    chosen so that every particle is classified 'optimal' by the reference."""
    return dx * (3.0 / (4.0 * math.pi * ppc)) ** (1.0 / 3.0)


def attributes(n: int, dx: float, ppc: int, rho: float):
    r = particle_radius(dx, ppc)
    vol = 4.0 / 3.0 * math.pi * r * r * r
    return (np.full(n, rho * vol), np.full(n, vol), np.full(n, r))


def liquid_block(dx: float, lo, hi, ppc: int, seed: int) -> np.ndarray:
    """Jittered particles filling the box [lo, hi].

    ppc == 8: one particle per (dx/2)^3 sub-cell whose centre lies in the box,
    uniformly jittered inside its sub-cell.  Other ppc: ppc particles per cell
    whose centre lies in the box, uniform inside the cell.
    """
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    if ppc == 8:
        h = dx * 0.5
        per = 1
    else:
        h = dx
        per = ppc
    i0 = np.floor(lo / h).astype(np.int64)
    i1 = np.ceil(hi / h).astype(np.int64)
    axes = [np.arange(i0[d], i1[d]) for d in range(3)]
    cz, cy, cx = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    cells = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1)
    centre = (cells + 0.5) * h
    keep = np.all((centre >= lo) & (centre <= hi), axis=1)
    cells = cells[keep]
    cells = np.repeat(cells, per, axis=0)
    jitter = rng.random((cells.shape[0], 3))
    return (cells + jitter) * h


def curl_noise_velocity(x: np.ndarray, n: int, sigma_cells: float,
                        amplitude: float, seed: int) -> np.ndarray:
    """Divergence-free velocity: curl of Gaussian-smoothed white noise on an
    n^3 grid over the unit box (sigma in cells), scaled so that max |v| equals
    ``amplitude`` on the grid, trilinearly interpolated to ``x``."""
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n) * 2.0 * math.pi
    kx, ky, kz = np.meshgrid(k, k, k, indexing="ij")
    g = np.exp(-0.5 * (sigma_cells ** 2) * (kx * kx + ky * ky + kz * kz))
    psi = []
    for _ in range(3):
        w = rng.standard_normal((n, n, n))
        psi.append(np.real(np.fft.ifftn(np.fft.fftn(w) * g)))
    h = 1.0 / n

    def d(f, axis):
        return (np.roll(f, -1, axis) - np.roll(f, 1, axis)) / (2.0 * h)

    vx = d(psi[2], 1) - d(psi[1], 2)
    vy = d(psi[0], 2) - d(psi[2], 0)
    vz = d(psi[1], 0) - d(psi[0], 1)
    vmax = float(np.sqrt(vx * vx + vy * vy + vz * vz).max())
    s = amplitude / vmax
    vel = np.stack([vx * s, vy * s, vz * s], axis=-1)
    # trilinear interpolation at sample points (grid values at cell centres)
    p = x / h - 0.5
    i = np.floor(p).astype(np.int64)
    f = p - i
    out = np.zeros_like(x)
    for dz in (0, 1):
        for dy in (0, 1):
            for dxx in (0, 1):
                w = ((f[:, 0] if dxx else 1 - f[:, 0]) *
                     (f[:, 1] if dy else 1 - f[:, 1]) *
                     (f[:, 2] if dz else 1 - f[:, 2]))
                ii = np.clip(i[:, 0] + dxx, 0, n - 1)
                jj = np.clip(i[:, 1] + dy, 0, n - 1)
                kk = np.clip(i[:, 2] + dz, 0, n - 1)
                out += w[:, None] * vel[ii, jj, kk]
    return out


@dataclasses.dataclass
class ElastoSet:
    """Elasto (cloth / yarn) particles, which the reference stores ahead of
    the liquid ones (TwoDScene::isFluid, libWetCloth/Core/TwoDScene.cpp:6921).
    Arrays follow the reference's per-particle members: x4 / v4 = m_x / m_v
    (position or velocity plus the twist component), B = m_B (row-major 3x3),
    m4 / fm4 = m_m / m_fluid_m, rest_vol = m_rest_vol, rest_vf =
    m_rest_volume_fraction, fluid_vol = m_fluid_vol (liquid held in the
    cloth), shape_factor, orientation = m_orientation, surfel != 0 where
    m_particle_to_surfel >= 0, radius."""

    x4: np.ndarray
    v4: np.ndarray
    B: np.ndarray
    m4: np.ndarray
    fm4: np.ndarray
    rest_vol: np.ndarray
    rest_vf: np.ndarray
    fluid_vol: np.ndarray
    shape_factor: np.ndarray
    orientation: np.ndarray
    surfel: np.ndarray
    radius: np.ndarray

    @property
    def n(self) -> int:
        return self.x4.shape[0]


@dataclasses.dataclass
class Scene:
    params: SceneParams
    x: np.ndarray
    v: np.ndarray
    mass: np.ndarray
    vol: np.ndarray
    radius: np.ndarray
    C: np.ndarray | None = None
    name: str = ""
    elasto: ElastoSet | None = None


def cloth_sheet(lo, hi, y: float, spacing: float, seed: int, thickness: float = 0.004,
                density: float = 1320.0, rest_vf: float = 0.5, wetness: float = 0.3,
                liquid_density: float = 1000.0, speed: float = 0.5,
                surfel_every: int = 0) -> ElastoSet:
    """A seeded cloth sheet of vertices on a regular grid in the plane y,
    spanning [lo, hi] in x and z, with the per-vertex attributes of
    TwoDSceneXMLParser::loadClothes (App/TwoDSceneXMLParser.cpp:1455-1470):
    volume = rest area x thickness, mass = density x volume x rest volume
    fraction.  Each vertex holds liquid of volume wetness x (1 - rest_vf) x
    volume; velocities, affine matrices, twists, shape factors and normal tilts
    are seeded random.  surfel_every = k > 0 marks every k-th vertex a
    surfel."""
    rng = np.random.default_rng(seed)
    xs = np.arange(lo[0], hi[0] + 0.5 * spacing, spacing)
    zs = np.arange(lo[1], hi[1] + 0.5 * spacing, spacing)
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    n = X.size
    x4 = np.zeros((n, 4))
    x4[:, 0] = X.reshape(-1) + rng.uniform(-0.1, 0.1, n) * spacing
    x4[:, 1] = y + rng.uniform(-0.1, 0.1, n) * spacing
    x4[:, 2] = Z.reshape(-1) + rng.uniform(-0.1, 0.1, n) * spacing
    x4[:, 3] = rng.uniform(-0.5, 0.5, n)
    v4 = np.zeros((n, 4))
    v4[:, :3] = rng.normal(0.0, 0.1 * speed, (n, 3))
    v4[:, 1] -= speed
    v4[:, 3] = rng.normal(0.0, 1.0, n)
    B = rng.normal(0.0, 1.0, (n, 9))
    vol = spacing * spacing * thickness
    mass = density * vol * rest_vf
    m4 = np.zeros((n, 4))
    m4[:, :3] = mass
    m4[:, 3] = mass * thickness * thickness * 0.25
    fvol = wetness * (1.0 - rest_vf) * vol
    fm4 = np.zeros((n, 4))
    fm4[:, :3] = liquid_density * fvol
    tilt = rng.normal(0.0, 0.2, (n, 3))
    tilt[:, 1] = 1.0
    orientation = tilt / np.linalg.norm(tilt, axis=1, keepdims=True)
    surfel = np.zeros(n, dtype=np.int32)
    if surfel_every > 0:
        surfel[::surfel_every] = 1
        v4[surfel != 0] = 0.0
    return ElastoSet(x4=x4, v4=v4, B=B, m4=m4, fm4=fm4, rest_vol=np.full(n, vol),
                     rest_vf=np.full(n, rest_vf), fluid_vol=np.full(n, fvol),
                     shape_factor=rng.uniform(0.2, 0.8, n), orientation=orientation,
                     surfel=surfel, radius=np.full(n, 0.5 * thickness))


def liquid_on_sheet(n_cells: int = 32, ppc: int = 8, seed: int = 3, sheet_spacing=None,
                    surfel_every: int = 0, center=(0.5, 0.75, 0.5)) -> Scene:
    """A falling liquid sphere (r 0.15 at `center`, v = (0, -1, 0) plus a
    spin of 3 rad/s about y) and a cloth sheet at y = 0.4 spanning [0.1, 0.9]
    in x and z; with the centre at y = 0.45 the sphere straddles the sheet."""
    dx = 1.0 / n_cells
    prm = SceneParams(dx=dx)
    c = np.array(center, dtype=np.float64)
    x = liquid_block(dx, tuple(c - 0.15), tuple(c + 0.15), ppc, seed)
    x = x[np.linalg.norm(x - c, axis=1) <= 0.15]
    v = np.cross(np.array([0.0, 3.0, 0.0]), x - c)
    v[:, 1] = -1.0
    m, vol, r = attributes(x.shape[0], dx, ppc, prm.liquid_density)
    h = sheet_spacing if sheet_spacing is not None else 0.5 * dx
    sheet = cloth_sheet((0.1, 0.1), (0.9, 0.9), 0.4, h, seed + 1, surfel_every=surfel_every)
    return Scene(prm, x, v, m, vol, r, elasto=sheet,
                 name=f"liquid_on_sheet_{n_cells}^3_{ppc}ppc_{sheet.n}v")


def dam_break(n_cells: int = 64, ppc: int = 8, seed: int = 0,
              block_hi=(0.4, 0.8, 0.4)) -> Scene:
    """Liquid dam break in the unit box: block [0, block_hi] at ppc particles
    per cell, zero initial velocity, rho 1000, g -9.81 y, free-slip walls."""
    dx = 1.0 / n_cells
    prm = SceneParams(dx=dx)
    x = liquid_block(dx, (0.0, 0.0, 0.0), block_hi, ppc, seed)
    m, vol, r = attributes(x.shape[0], dx, ppc, prm.liquid_density)
    return Scene(prm, x, np.zeros_like(x), m, vol, r,
                 name=f"dam_break_{n_cells}^3_{ppc}ppc")


def differentiation_block(n_cells: int = 64, ppc: int = 8, seed: int = 2,
                          sigma: float = 0.2, viscosity: float = 1e-3) -> Scene:
    """The dam-break block [0,0.4]x[0,0.8]x[0,0.4] (particle seed 0) with a
    seeded Gaussian initial velocity (each component N(0, sigma^2), seed
    `seed`) and the explicit viscosity on: the scene of the 200-step
    gradient run."""
    sc = dam_break(n_cells, ppc, 0)
    sc.v = np.random.default_rng(seed).normal(0.0, sigma, sc.x.shape)
    sc.params.viscosity = viscosity
    sc.name = f"differentiation_{n_cells}^3_{ppc}ppc"
    return sc


def fine_volume(dx: float, cell_multiplier: float = 0.3535533906) -> float:
    """V_fine of relabelLiquidParticles (TwoDScene.cpp:2484-2489): the
    volume of a sphere of radius dx * cell_multiplier / sqrt(3)."""
    r = 1.0 / np.sqrt(3.0) * dx * cell_multiplier
    return 4.0 / 3.0 * np.pi * r * r * r


def mixed_volumes(sc: Scene, seed: int = 0, mrel=(0.3, 0.7, 1.0, 1.5, 2.5)) -> Scene:
    """The scene with every liquid particle's volume set to V_fine times a
    seeded choice from mrel (radius and mass to match), so that the merge and
    split classes S, s, o, l and L all occur."""
    rng = np.random.default_rng(seed)
    vf = fine_volume(sc.params.dx)
    vol = vf * rng.choice(np.asarray(mrel, dtype=np.float64), size=sc.x.shape[0])
    sc.vol = vol
    sc.mass = vol * sc.params.liquid_density
    sc.radius = np.cbrt(vol * 0.75 / np.pi)
    return sc


def half_box(n_cells: int = 256, ppc: int = 2, seed: int = 1,
             amplitude: float = 0.5, sigma_cells: float = 4.0) -> Scene:
    """Half-filled unit box (y < 0.5) at ppc particles per cell with a random
    divergence-free initial velocity (curl of Gaussian noise)."""
    dx = 1.0 / n_cells
    prm = SceneParams(dx=dx)
    x = liquid_block(dx, (0.0, 0.0, 0.0), (1.0, 0.5, 1.0), ppc, seed)
    v = curl_noise_velocity(x, n_cells, sigma_cells, amplitude, seed)
    m, vol, r = attributes(x.shape[0], dx, ppc, prm.liquid_density)
    return Scene(prm, x, v, m, vol, r,
                 name=f"half_box_{n_cells}^3_{ppc}ppc")


def batch_scenes(count: int = 256, seed: int = 4, n_range=(32, 96), np_range=(10_000, 1_000_000),
                 ppc: int = 8):
    """Seeded independent scenes of uneven size: grid n ~ U{n_range}^3, a
    liquid block of about N_p ~ U[np_range] particles (capped by the box) at a
    seeded position, viscosity log-uniform in [1e-3, 1], density U[800, 1300]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        dx = 1.0 / n
        target = float(rng.uniform(np_range[0], np_range[1]))
        cells = min(target / ppc, 0.6 * n ** 3)
        # block with aspect (1, 2, 1) scaled to the cell count, inside the box
        side = (cells / 2.0) ** (1.0 / 3.0) * dx
        size = np.minimum(np.array([side, 2.0 * side, side]), 0.9)
        lo = rng.uniform(0.0, 1.0 - size)
        lo[1] = 0.0
        prm = SceneParams(dx=dx, liquid_density=float(rng.uniform(800.0, 1300.0)),
                          viscosity=float(10.0 ** rng.uniform(-3.0, 0.0)))
        x = liquid_block(dx, lo, lo + size, ppc, seed * 1000 + k)
        m, vol, r = attributes(x.shape[0], dx, ppc, prm.liquid_density)
        out.append(Scene(prm, x, np.zeros_like(x), m, vol, r, name=f"batch{k}_{n}^3_{x.shape[0]}p"))
    return out
