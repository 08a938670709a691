"""Seeded synthetic phantoms and spot plans for the benchmark workloads.

No clinical data is involved: every CT is generated from a seed with
``numpy.random.default_rng``.  Workloads (volumes are numpy (nz, ny, nx)):

  water_cube()            120^3 at 2.5 mm, HU 0 in a centred 200 mm cube,
                          air outside; one beam at gantry 0; spots on a 5 mm
                          lattice over a centred 50 mm target; 10 energy
                          layers whose R80 spans the target depth; mu = 1.
  heterogeneous(seed, angles, n_spots)
                          256x256x160 at 2 mm, water with a 10 mm air margin,
                          seeded axis-aligned slabs and spheres (radius
                          10-30 mm) of bone (HU 1000) and lung (HU -700), a
                          seeded ellipsoidal target (semi-axes 30-45 mm); per
                          beam a 5 mm lattice over the target's beam's-eye
                          projection and layers spanning its WET range; mu in
                          [0.5, 1.5].  Prescription 60 in the target, 0
                          outside; voxel weights 1 / 0.1.

The isocentre is the target centre, placed off the voxel lattice, so that no
sample of the WET smoothing lands exactly on a half-voxel boundary.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from .plan_impt import IMPTBeam, IMPTDoseGrid, IMPTPlan

_PLAN_CACHE = {}


def _new_plan(machine="HitachiProbeatJHU") -> IMPTPlan:
    """IMPTPlan with the machine's models (parsed once, then shallow-copied)."""
    base = _PLAN_CACHE.get(machine)
    if base is None:
        base = IMPTPlan(machine)
        _PLAN_CACHE[machine] = base
    p = IMPTPlan.__new__(IMPTPlan)
    p.__dict__.update(base.__dict__)
    p.beam_list = []
    p.n_beams = 0
    p.Prescriptions = []
    return p


@dataclass
class SynthCase:
    name: str
    grid: IMPTDoseGrid
    plan: IMPTPlan
    target: np.ndarray                      # bool (nz, ny, nx)
    presc: Optional[np.ndarray] = None      # float32 (nz, ny, nx)
    weights: Optional[np.ndarray] = None    # float32 (nz, ny, nx)
    info: dict = field(default_factory=dict)

    @property
    def n_spots(self) -> int:
        return int(sum(np.asarray(b.spot_list).reshape(-1, 4).shape[0] for b in self.plan.beam_list))

    def objective_fields(self):
        presc = np.where(self.target, 60.0, 0.0).astype(np.float32)
        w = np.where(self.target, 1.0, 0.1).astype(np.float32)
        return presc, w


# ---------------------------------------------------------------- geometry

def beam_frame(gantry_deg: float, couch_deg: float, sad: float):
    """Source position (image frame, relative to iso) and image->head
    rotation for a beam, in float64 (used only to lay out spots)."""
    ga = np.deg2rad(np.fmod(gantry_deg + 180.0, 360.0))
    ta = np.deg2rad(couch_deg)
    sg, cg, st, ct = np.sin(ga), np.cos(ga), np.sin(ta), np.cos(ta)
    xg, yg = -sad * sg, sad * cg
    src = np.array([xg * ct, yg, -xg * st])

    def to_head(p):
        p = np.asarray(p, dtype=np.float64)
        x, y, z = p[..., 0], p[..., 1], p[..., 2]
        xt = x * ct - z * st
        zt = x * st + z * ct
        xg_ = xt * cg + y * sg
        yg_ = -xt * sg + y * cg
        return np.stack([-xg_, zt, yg_], axis=-1)

    return src, to_head


def hu_to_rlsp_np(hu, machine="HitachiProbeatJHU"):
    from .plan_impt import _hu_curve
    xh, yh = _hu_curve(machine)
    return np.array(np.interp(hu, xh, yh), dtype=np.single)


def _wet_samples(rlsp, origin, spacing, iso, src, pts_rel):
    """WET (mm) from points (image frame, relative to iso) to the grid edge
    toward the source: trilinear march in 1 mm steps (layer selection only)."""
    from scipy.ndimage import map_coordinates
    nz, ny, nx = rlsp.shape
    u = src[None, :] - pts_rel
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    diag = spacing * np.sqrt(nx * nx + ny * ny + nz * nz)
    t = np.arange(0.0, diag + 1.0, 1.0)
    wet = np.zeros(len(pts_rel))
    for q in range(len(pts_rel)):
        p = pts_rel[q][None, :] + t[:, None] * u[q][None, :] + iso - origin
        idx = p / spacing
        vals = map_coordinates(rlsp, [idx[:, 2], idx[:, 1], idx[:, 0]], order=1, mode="constant",
                               cval=0.0)
        wet[q] = np.clip(vals, 0.0, None).sum()
    return wet


def _pick_energies(model, r80_lo: float, r80_hi: float, n_layers: int):
    r80 = model.divergence_params[:, 1].astype(np.float64)
    want = np.linspace(r80_lo, r80_hi, max(n_layers, 1))
    ids = sorted({int(np.argmin(np.abs(r80 - w))) for w in want})
    return ids


def _lattice_over(target_head_iso_xy, pitch=5.0, margin=5.0):
    """Lattice points (pitch) within `margin` of any projected target point."""
    from scipy.spatial import cKDTree
    lo = np.floor((target_head_iso_xy.min(axis=0) - margin) / pitch) * pitch
    hi = np.ceil((target_head_iso_xy.max(axis=0) + margin) / pitch) * pitch
    gx = np.arange(lo[0], hi[0] + 0.5 * pitch, pitch)
    gy = np.arange(lo[1], hi[1] + 0.5 * pitch, pitch)
    X, Y = np.meshgrid(gx, gy, indexing="ij")
    cand = np.stack([X.ravel(), Y.ravel()], axis=1)
    d, _ = cKDTree(target_head_iso_xy).query(cand)
    return cand[d <= margin]


# --------------------------------------------------------------- workloads

def water_cube(machine="HitachiProbeatJHU") -> SynthCase:
    n, s = 120, 2.5
    g = IMPTDoseGrid()
    g.origin = np.array([-n * s / 2.0] * 3)
    g.spacing = np.array([s, s, s])
    g.size = np.array([n, n, n])
    hu = np.full((n, n, n), -1000.0, dtype=np.single)
    lo, hi = 20, 100  # 200 mm cube = 80 voxels, centred
    hu[lo:hi, lo:hi, lo:hi] = 0.0
    g.HU = hu
    plan = _new_plan(machine)
    beam = IMPTBeam()
    beam.dicom_rangeshifter_label = '0'
    beam.gantry_angle = 0.0
    beam.couch_angle = 0.0
    beam.iso = np.array([0.0, 0.0, 0.0], dtype=np.single)
    model = plan.beam_models[0]
    # beam enters at y = -100 mm; the 50 mm target spans depths 75..125 mm
    rl = 1.00653  # RLSP of water (HU 0) on this machine's curve
    ids = _pick_energies(model, 78.0 * rl, 128.0 * rl, 10)
    xs = np.arange(-25.0, 25.0 + 1e-3, 5.0)
    rows = [[x, y, 1.0, e] for e in ids for x in xs for y in xs]
    beam.spot_list = np.array(rows, dtype=np.single)
    beam.n_spots = len(rows)
    plan.addBeam(beam)
    c = (np.arange(n) + 0.5) * s - n * s / 2.0 - s / 2.0
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    target = (np.abs(xx) <= 25.0) & (np.abs(yy) <= 25.0) & (np.abs(zz) <= 25.0)
    return SynthCase("water_cube_120_2.5mm", g, plan, target,
                     info={"energy_ids": ids, "beams": 1})


def heterogeneous(seed: int = 2, angles: Sequence[float] = (0.0, 120.0, 240.0),
                  n_spots: int = 8000, shape=(160, 256, 256), spacing: float = 2.0,
                  machine="HitachiProbeatJHU", n_slabs: int = 3, n_spheres: int = 6,
                  semi_range=(30.0, 45.0), centre_jitter: float = 20.0,
                  body_inset: float = 30.0, pitch: float = 5.0) -> SynthCase:
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    s = float(spacing)
    g = IMPTDoseGrid()
    ext = np.array([nx, ny, nz], dtype=np.float64) * s
    g.origin = -ext / 2.0
    g.spacing = np.array([s, s, s])
    g.size = np.array(shape)
    # voxel centre coordinates (patient frame), per axis
    cx = g.origin[0] + np.arange(nx) * s
    cy = g.origin[1] + np.arange(ny) * s
    cz = g.origin[2] + np.arange(nz) * s
    hu = np.zeros(shape, dtype=np.single)
    margin = int(round(10.0 / s))
    hu[:margin] = hu[-margin:] = -1000.0
    hu[:, :margin] = hu[:, -margin:] = -1000.0
    hu[:, :, :margin] = hu[:, :, -margin:] = -1000.0
    body_lo = g.origin + margin * s + body_inset
    body_hi = g.origin + ext - margin * s - body_inset
    for _ in range(n_slabs):
        axis = int(rng.integers(0, 3))
        thick = rng.uniform(10.0, 30.0)
        c0 = rng.uniform(body_lo, body_hi)
        half = rng.uniform(40.0, 110.0, size=3)
        half[axis] = thick / 2.0
        val = 1000.0 if rng.random() < 0.5 else -700.0
        sl = [slice(np.searchsorted(ax, c - h), np.searchsorted(ax, c + h))
              for ax, c, h in zip((cx, cy, cz), c0, half)]
        hu[sl[2], sl[1], sl[0]] = val
    for _ in range(n_spheres):
        r = rng.uniform(10.0, 30.0)
        c0 = rng.uniform(body_lo, body_hi)
        val = 1000.0 if rng.random() < 0.5 else -700.0
        zs = slice(np.searchsorted(cz, c0[2] - r), np.searchsorted(cz, c0[2] + r))
        ys = slice(np.searchsorted(cy, c0[1] - r), np.searchsorted(cy, c0[1] + r))
        xs = slice(np.searchsorted(cx, c0[0] - r), np.searchsorted(cx, c0[0] + r))
        Z, Y, X = np.meshgrid(cz[zs], cy[ys], cx[xs], indexing="ij")
        m = (X - c0[0]) ** 2 + (Y - c0[1]) ** 2 + (Z - c0[2]) ** 2 <= r * r
        blk = hu[zs, ys, xs]
        blk[m] = val
    # target ellipsoid, centre off the voxel lattice
    semi = rng.uniform(semi_range[0], semi_range[1], size=3)
    tc = rng.uniform(-centre_jitter, centre_jitter, size=3) + rng.uniform(0.1, 0.9, size=3) * s
    target = ((((cx - tc[0]) / semi[0]) ** 2)[None, None, :] +
              (((cy - tc[1]) / semi[1]) ** 2)[None, :, None] +
              (((cz - tc[2]) / semi[2]) ** 2)[:, None, None]) <= 1.0
    g.HU = hu
    rlsp = hu_to_rlsp_np(hu, machine)

    plan = _new_plan(machine)
    model = plan.beam_models[0]
    sad = (model.VSADX + model.VSADY) / 2.0
    iso = tc.astype(np.single)
    tidx = np.argwhere(target)
    tpts = np.stack([cx[tidx[:, 2]], cy[tidx[:, 1]], cz[tidx[:, 0]]], axis=1) - tc
    per_beam = n_spots / max(len(angles), 1)
    sub = tpts[rng.choice(len(tpts), size=min(300, len(tpts)), replace=False)]
    for ang in angles:
        src, to_head = beam_frame(ang, 0.0, sad)
        h = to_head(tpts)
        proj = np.stack([h[:, 0] / (1.0 - h[:, 2] / model.VSADX),
                         h[:, 1] / (1.0 - h[:, 2] / model.VSADY)], axis=1)
        lat = _lattice_over(proj[:: max(1, len(proj) // 20000)], pitch=pitch)
        wet = _wet_samples(rlsp, g.origin, s, tc, src, sub)
        n_layers = max(1, int(round(per_beam / max(len(lat), 1))))
        ids = _pick_energies(model, wet.min() - 2.0, wet.max() + 3.0, n_layers)
        rows = []
        for e in ids:
            mu = rng.uniform(0.5, 1.5, size=len(lat))
            rows.append(np.column_stack([lat, mu, np.full(len(lat), e)]))
        beam = IMPTBeam()
        beam.dicom_rangeshifter_label = '0'
        beam.gantry_angle = float(ang)
        beam.couch_angle = 0.0
        beam.iso = iso.copy()
        beam.spot_list = np.concatenate(rows).astype(np.single)
        beam.n_spots = beam.spot_list.shape[0]
        plan.addBeam(beam)
    case = SynthCase(f"heterogeneous_{nx}x{ny}x{nz}_{s:g}mm_{len(angles)}beams", g, plan, target,
                     info={"seed": seed, "angles": list(angles), "semi_axes": semi.tolist(),
                           "target_centre": tc.tolist()})
    case.presc, case.weights = case.objective_fields()
    return case


def config_forward_heterogeneous(seed: int = 2) -> SynthCase:
    """3 beams at 0/120/240 degrees, ~8,000 spots."""
    return heterogeneous(seed, (0.0, 120.0, 240.0), 8000)


def config_gradient(seed: int = 3) -> SynthCase:
    """4 beams, ~20,000 spots (5 mm lattice over a target of 7-10 cm axes),
    with the quadratic objective's fields."""
    return heterogeneous(seed, (0.0, 90.0, 180.0, 270.0), 20000, semi_range=(35.0, 50.0))


def small_heterogeneous(seed: int = 7, angles=(0.0, 135.0), n_spots=300,
                        shape=(40, 48, 56), spacing=3.0) -> SynthCase:
    """Small heterogeneous case that the FP64 oracle finishes in seconds."""
    return heterogeneous(seed, angles, n_spots, shape=shape, spacing=spacing, n_slabs=1,
                         n_spheres=2, semi_range=(10.0, 16.0), centre_jitter=5.0,
                         body_inset=15.0)


def batch_cases(seed: int = 4, n_plans: int = 32, min_shape=(64, 64, 64),
                max_shape=(160, 200, 200), spacings=(2.0, 2.5, 3.0), beams=(1, 4),
                spots=(500, 20000)):
    """Independent plans of uneven size for the batched mode: grid (nz, ny, nx)
    drawn per plan between min_shape and max_shape, spacing from `spacings`,
    1-4 beams at seeded gantry angles, 500-20,000 spots, heterogeneity as in
    `heterogeneous`, target size scaled to the grid."""
    rng = np.random.default_rng(seed)
    out = []
    for p in range(n_plans):
        shape = tuple(int(rng.integers(lo, hi + 1)) for lo, hi in zip(min_shape, max_shape))
        s = float(rng.choice(spacings))
        nb = int(rng.integers(beams[0], beams[1] + 1))
        angles = tuple(float(a) for a in np.sort(rng.uniform(0.0, 360.0, nb)))
        ext = min(shape) * s
        semi = (0.10 * ext, 0.16 * ext)
        case = heterogeneous(seed=int(rng.integers(1 << 30)), angles=angles,
                             n_spots=int(rng.integers(spots[0], spots[1] + 1)), shape=shape,
                             spacing=s, n_slabs=2, n_spheres=3, semi_range=semi,
                             centre_jitter=0.05 * ext, body_inset=0.1 * ext)
        case.name = f"batch{p}_{shape[2]}x{shape[1]}x{shape[0]}_{s:g}mm_{nb}beams"
        out.append(case)
    return out


def config_optimisation(seed: int = 3) -> SynthCase:
    """512x512x200 at 1 mm, 4 beams, ~60,000 spots (3 mm lattice; 59,579 at
    seed 3), with the objective's fields: the large optimisation loop."""
    return heterogeneous(seed, (0.0, 90.0, 180.0, 270.0), 64000, shape=(200, 512, 512),
                         spacing=1.0, semi_range=(40.0, 60.0), centre_jitter=15.0,
                         body_inset=40.0, pitch=3.0)
