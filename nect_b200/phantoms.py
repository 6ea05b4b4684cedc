"""Seeded synthetic phantoms and exact line-integral projections.

Stand-ins for the reference's data (its demo data sets are downloaded from
Zenodo and its porous phantoms need porespy, neither available here), built to
the shapes, sizes and value ranges of the benchmark workloads:

* ``ellipsoid_phantom``: additive sum of seeded random ellipsoids in the unit
  cube (static parallel-beam workload, 128^3, 20 ellipsoids).
* ``porous_phantom``: a cylinder (attenuation 0.2) filled to 60 % with
  non-overlapping spheres (attenuation 0.8, radii U[3, 12] voxels) by
  collective rearrangement: the radii are drawn until their volume is the
  target fraction, the spheres start at seeded random places and overlapping
  pairs are pushed apart (and spheres back into the cylinder) until no two
  overlap (static cone-beam workload, 256^3).  Random sequential insertion
  jams near 40 %; the rearrangement reaches the target, and the achieved
  fraction is reported.
* ``dynamic_porous``: the porous medium plus a brine front (attenuation 0.5)
  rising in z as a sigmoid in t with a value-noise-perturbed interface, and 30
  grains that shrink linearly in time (4D workload).

Projections are exact line integrals (sums of analytic chord lengths), the
limit the ray-marched integrals of the workload description converge to;
rays follow the sampler's conventions (nect/sampling/ct_sampling.cu:226-389:
source at -DSO on x, detector column -> -y, row -> z, rotation about z after
the centre-of-rotation shift).  The time-dependent brine front has no closed
form and is ray-marched at 4 samples per voxel.  Everything runs in torch on
the given device and is used only to make inputs (it is not part of the
training path).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch


# ---------------------------------------------------------------- rays ----
def detector_rays(geometry, angle: float, device, dtype=torch.float64):
    """World-space ray origins/directions [P,3] (x,y,z) for every detector pixel.

    Uses the nect_b200.sampling.Geometry conventions (detector binning 1)."""
    nr, nc = geometry.nDetector
    rows = torch.arange(nr, device=device, dtype=dtype)
    cols = torch.arange(nc, device=device, dtype=dtype)
    u = (cols - (nc - 1) / 2) * geometry.dDetector[1] + geometry.offDetector[1]
    v = (rows - (nr - 1) / 2) * geometry.dDetector[0] + geometry.offDetector[0]
    V, U = torch.meshgrid(v, u, indexing="ij")
    y = -U.reshape(-1)
    z = V.reshape(-1)
    P = y.numel()
    if geometry.mode == "cone":
        src = torch.tensor([-geometry.DSO, 0.0, 0.0], device=device, dtype=dtype).expand(P, 3)
        det = torch.stack([torch.full_like(y, geometry.DSD - geometry.DSO), y, z], 1)
    else:
        L = 2.0 * max(geometry.sVoxel)
        src = torch.stack([torch.full_like(y, -L), y, z], 1)
        det = torch.stack([torch.full_like(y, L), y, z], 1)
    c, s = math.cos(angle), math.sin(angle)

    def rot(p):
        x, yy, zz = p[:, 0], p[:, 1] - geometry.COR, p[:, 2]
        return torch.stack([c * x - s * yy, s * x + c * yy, zz], 1)

    a, b = rot(src), rot(det)
    d = b - a
    return a, d / d.norm(dim=1, keepdim=True)


def _sphere_chords(o, d, centers, radii, chunk=2048):
    """Sum over spheres handled by the caller: returns [P, S] chord lengths."""
    out = []
    for i in range(0, centers.shape[0], chunk):
        c = centers[i:i + chunk]
        r = radii[i:i + chunk]
        oc = o[:, None, :] - c[None]
        b = (oc * d[:, None, :]).sum(-1)
        q = (oc * oc).sum(-1) - b * b
        h = r[None] ** 2 - q
        out.append(2 * torch.sqrt(torch.clamp(h, min=0)))
    return torch.cat(out, 1)


def _cylinder_chord(o, d, radius, half_height):
    """Chord of each line with {x^2 + y^2 <= r^2, |z| <= h}."""
    a = d[:, 0] ** 2 + d[:, 1] ** 2
    b = 2 * (o[:, 0] * d[:, 0] + o[:, 1] * d[:, 1])
    c = o[:, 0] ** 2 + o[:, 1] ** 2 - radius ** 2
    disc = b * b - 4 * a * c
    ok = (disc > 0) & (a > 1e-12)
    sq = torch.sqrt(torch.clamp(disc, min=0))
    t0 = torch.where(ok, (-b - sq) / (2 * a).clamp(min=1e-12), torch.zeros_like(a))
    t1 = torch.where(ok, (-b + sq) / (2 * a).clamp(min=1e-12), torch.zeros_like(a))
    # clip by the slab |z| <= h
    dz = d[:, 2]
    safe = torch.where(dz.abs() > 1e-12, dz, torch.full_like(dz, 1e-12))
    z0 = (-half_height - o[:, 2]) / safe
    z1 = (half_height - o[:, 2]) / safe
    zl, zh = torch.minimum(z0, z1), torch.maximum(z0, z1)
    flat = dz.abs() <= 1e-12
    inside_slab = o[:, 2].abs() <= half_height
    zl = torch.where(flat, torch.where(inside_slab, torch.full_like(zl, -1e30), torch.full_like(zl, 1e30)), zl)
    zh = torch.where(flat, torch.where(inside_slab, torch.full_like(zh, 1e30), torch.full_like(zh, -1e30)), zh)
    lo, hi = torch.maximum(t0, zl), torch.minimum(t1, zh)
    return torch.where(ok, torch.clamp(hi - lo, min=0), torch.zeros_like(a))


# ------------------------------------------------------- ellipsoids (C1) ----
@dataclass
class EllipsoidPhantom:
    centers: np.ndarray   # [E,3] world (x,y,z), unit cube centred at 0
    axes: np.ndarray      # [E,3] semi-axes
    rot: np.ndarray       # [E,3,3] rotation (columns = ellipsoid axes)
    mu: np.ndarray        # [E]


def ellipsoid_phantom(n: int = 20, seed: int = 0, size: float = 1.0) -> EllipsoidPhantom:
    """Centres U[-0.6,0.6]^3 in the cube [-1,1]^3 scaled to a cube of side
    ``size`` (unit cube: U[-0.3,0.3] in world units), semi-axes U[0.05,0.35]
    of the [-1,1] cube (unit cube: U[0.025,0.175]), uniform random rotations,
    attenuation U[0.1,1.0] per unit of the cube."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-0.6, 0.6, (n, 3)) * 0.5 * size
    axes = rng.uniform(0.05, 0.35, (n, 3)) * 0.5 * size
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    rot = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)
    mu = rng.uniform(0.1, 1.0, n)
    return EllipsoidPhantom(centers, axes, rot, mu)


def ellipsoid_projection(ph: EllipsoidPhantom, geometry, angle: float, device) -> torch.Tensor:
    o, d = detector_rays(geometry, angle, device)
    C = torch.as_tensor(ph.centers, device=device)
    A = torch.as_tensor(ph.axes, device=device)
    Rm = torch.as_tensor(ph.rot, device=device)
    mu = torch.as_tensor(ph.mu, device=device)
    oc = o[:, None, :] - C[None]                       # [P,E,3]
    ol = torch.einsum("pei,eij->pej", oc, Rm) / A[None]
    dl = torch.einsum("pi,eij->pej", d, Rm) / A[None]
    a = (dl * dl).sum(-1)
    b = 2 * (ol * dl).sum(-1)
    c = (ol * ol).sum(-1) - 1
    disc = torch.clamp(b * b - 4 * a * c, min=0)
    chord = torch.sqrt(disc) / a                       # t2 - t1 with |d| = 1
    return (chord * mu[None]).sum(1).to(torch.float32).reshape(geometry.nDetector[0], geometry.nDetector[1])


def ellipsoid_volume(ph: EllipsoidPhantom, n: int, device) -> torch.Tensor:
    """Voxel-centre samples [z,y,x] of the attenuation on an n^3 grid."""
    c = (torch.arange(n, device=device, dtype=torch.float64) + 0.5) / n - 0.5
    Z, Y, X = torch.meshgrid(c, c, c, indexing="ij")
    p = torch.stack([X, Y, Z], -1).reshape(-1, 3)
    vol = torch.zeros(p.shape[0], device=device, dtype=torch.float64)
    for e in range(len(ph.mu)):
        lp = (p - torch.as_tensor(ph.centers[e], device=device)) @ torch.as_tensor(ph.rot[e], device=device)
        inside = ((lp / torch.as_tensor(ph.axes[e], device=device)) ** 2).sum(1) <= 1
        vol += inside.double() * ph.mu[e]
    return vol.reshape(n, n, n).float()


# ------------------------------------------------------ porous medium (C2) ----
@dataclass
class PorousPhantom:
    radius: float          # cylinder radius (world units = voxels)
    half_height: float
    mu_cyl: float
    mu_grain: float
    centers: np.ndarray    # [G,3] (x,y,z)
    radii: np.ndarray      # [G]
    packing: float         # achieved grain volume fraction of the cylinder


def _overlaps(c: np.ndarray, r: np.ndarray):
    """(i, j, unit vector i->j, overlap) of the overlapping sphere pairs."""
    from scipy.spatial import cKDTree

    pairs = cKDTree(c).query_pairs(2 * float(r.max()), output_type="ndarray")
    if pairs.size == 0:
        return (np.zeros(0, int),) * 2 + (np.zeros((0, 3)), np.zeros(0))
    i, j = pairs[:, 0], pairs[:, 1]
    d = c[j] - c[i]
    dist = np.sqrt((d * d).sum(1))
    ov = r[i] + r[j] - dist
    hit = ov > 0
    return i[hit], j[hit], d[hit] / np.maximum(dist[hit], 1e-9)[:, None], ov[hit]


def _push_apart(c: np.ndarray, r: np.ndarray, R: float, H: float, sweeps: int, tol: float) -> float:
    """Collective rearrangement: every sweep moves the two spheres of each
    overlapping pair apart along their axis by 1.5 x the overlap (shared in
    proportion to the other sphere's volume; over-relaxed, as the pushes of
    neighbouring pairs partly cancel) and returns spheres that left the
    cylinder to its wall.  Stops when the largest overlap is below tol
    (voxels); returns the largest remaining overlap."""
    worst = 0.0
    for _ in range(sweeps):
        i, j, u, ov = _overlaps(c, r)
        worst = float(ov.max()) if ov.size else 0.0
        if worst < tol:
            break
        wi = r[j] ** 3 / (r[i] ** 3 + r[j] ** 3)
        step = (1.5 * ov + 2e-3)[:, None] * u
        move = np.zeros_like(c)
        np.add.at(move, i, -wi[:, None] * step)
        np.add.at(move, j, (1 - wi)[:, None] * step)
        c += move
        rho = np.sqrt(c[:, 0] ** 2 + c[:, 1] ** 2)
        lim = np.maximum(R - r, 0.0)
        out = rho > lim
        c[out, :2] *= (lim[out] / rho[out])[:, None]
        c[:, 2] = np.clip(c[:, 2], -H + r, H - r)
    return worst


def porous_phantom(n: int = 256, seed: int = 0, r_min: float = 3.0, r_max: float = 12.0, target: float = 0.6,
                   attempts: int = 8000) -> PorousPhantom:
    """Cylinder of radius and half height n/2 - 0.5 voxels filled to ``target``
    with non-overlapping spheres of radius U[r_min, r_max] (collective
    rearrangement, at most ``attempts`` sweeps; see the module doc).  The
    pairs still overlapping by less than 0.01 voxel when it stops are
    separated by shrinking both radii by their overlap."""
    rng = np.random.default_rng(seed)
    R, H = n / 2 - 0.5, n / 2 - 0.5
    vol_cyl = math.pi * R * R * 2 * H
    radii, filled = [], 0.0
    while filled < target * vol_cyl:
        r = float(rng.uniform(r_min, r_max))
        radii.append(r)
        filled += 4 / 3 * math.pi * r ** 3
    r = np.array(radii)
    rho = (R - r) * np.sqrt(rng.uniform(size=r.size))
    th = rng.uniform(0, 2 * math.pi, r.size)
    c = np.stack([rho * np.cos(th), rho * np.sin(th), rng.uniform(-H + r, H - r)], 1)
    _push_apart(c, r, R, H, attempts, tol=1e-2)
    for _ in range(8):   # remaining small overlaps: shrink both spheres of each pair
        i, j, _, ov = _overlaps(c, r)
        if ov.size == 0:
            break
        shrink = np.zeros_like(r)
        np.maximum.at(shrink, i, ov / 2 + 1e-4)
        np.maximum.at(shrink, j, ov / 2 + 1e-4)
        r = r - shrink
    i, j, _, ov = _overlaps(c, r)
    if ov.size:   # never expected: drop what still overlaps
        keep = np.ones(r.size, bool)
        keep[j] = False
        c, r = c[keep], r[keep]
    packing = float((4 / 3 * math.pi * r ** 3).sum() / vol_cyl)
    return PorousPhantom(R, H, 0.2, 0.8, c, r, packing)


def porous_projection(ph: PorousPhantom, geometry, angle: float, device, chunk: int | None = None,
                      grain_scale: np.ndarray | None = None) -> torch.Tensor:
    o, d = detector_rays(geometry, angle, device)
    if chunk is None:  # bound the [rays, grains, 3] temporaries to ~400 MB
        chunk = max(256, int(4e8 / (max(len(ph.radii), 1) * 3 * 8)))
    C = torch.as_tensor(ph.centers, device=device)
    r = torch.as_tensor(ph.radii if grain_scale is None else ph.radii * grain_scale, device=device)
    out = torch.empty(o.shape[0], device=device, dtype=torch.float64)
    for i in range(0, o.shape[0], chunk):
        oo, dd = o[i:i + chunk], d[i:i + chunk]
        cyl = _cylinder_chord(oo, dd, ph.radius, ph.half_height)
        sph = _sphere_chords(oo, dd, C, r).sum(1)
        out[i:i + chunk] = ph.mu_cyl * cyl + (ph.mu_grain - ph.mu_cyl) * sph
    return out.to(torch.float32).reshape(geometry.nDetector[0], geometry.nDetector[1])


def porous_volume(ph: PorousPhantom, n: int, device) -> torch.Tensor:
    c = torch.arange(n, device=device, dtype=torch.float32) - (n - 1) / 2
    Z, Y, X = torch.meshgrid(c, c, c, indexing="ij")
    vol = ((X ** 2 + Y ** 2 <= ph.radius ** 2) & (Z.abs() <= ph.half_height)).float() * ph.mu_cyl
    C = torch.as_tensor(ph.centers, device=device, dtype=torch.float32)
    Rr = torch.as_tensor(ph.radii, device=device, dtype=torch.float32)
    for j in range(C.shape[0]):
        cx, cy, cz = C[j]
        r = float(Rr[j])
        lo = [max(0, int(math.floor(float(v) + (n - 1) / 2 - r))) for v in (cz, cy, cx)]
        hi = [min(n, int(math.ceil(float(v) + (n - 1) / 2 + r)) + 1) for v in (cz, cy, cx)]
        sub = (Z[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] - cz) ** 2 + (Y[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] - cy) ** 2 \
            + (X[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] - cx) ** 2
        v = vol[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        v[sub <= r * r] = ph.mu_grain
    return vol


# ------------------------------------------------ dynamic porous medium (C3) ----
@dataclass
class DynamicPorousPhantom:
    base: PorousPhantom
    shrink: np.ndarray        # [G] radius loss per unit t (0 for grains that do not shrink)
    noise: np.ndarray         # [K,K,K] value-noise lattice in [-1, 1]
    mu_brine: float = 0.5
    front_width: float = 4.0  # voxels
    noise_amp: float = 12.0   # voxels of interface displacement

    def radii(self, t: float) -> np.ndarray:
        return np.maximum(self.base.radii - self.shrink * t, 0.0)

    def front_z(self, t: float) -> float:
        """Height of the unperturbed front: rises through the cylinder as t goes 0 -> 1."""
        h = self.base.half_height
        return -h - 2 * self.front_width + (2 * h + 4 * self.front_width) * t


def dynamic_porous(n: int = 256, seed: int = 0, n_shrinking: int = 30, lattice: int = 9,
                   attempts: int = 8000) -> DynamicPorousPhantom:
    """The porous medium plus a brine front (attenuation 0.5) rising in z as
    sigmoid((z0(t) + noise(x) - z) / w), its interface displaced by seeded
    trilinear value noise, and ``n_shrinking`` grains whose radii shrink
    linearly at U[0.2, 1.0] voxels per unit t.  The brine adds
    (0.5 - 0.2) * front over the whole cylinder (grains included), so every
    part of the object has a closed form except the front, which is
    ray-marched."""
    base = porous_phantom(n, seed=seed, attempts=attempts)
    rng = np.random.default_rng(seed + 1)
    shrink = np.zeros(len(base.radii))
    pick = rng.choice(len(base.radii), size=min(n_shrinking, len(base.radii)), replace=False)
    shrink[pick] = rng.uniform(0.2, 1.0, pick.size)
    noise = rng.uniform(-1.0, 1.0, (lattice, lattice, lattice))
    return DynamicPorousPhantom(base, shrink, noise)


def _front(ph: DynamicPorousPhantom, x: torch.Tensor, t: float) -> torch.Tensor:
    """Brine fraction in [0,1] at world points x [..., 3] (x, y, z), voxel units."""
    b = ph.base
    K = ph.noise.shape[0]
    lat = torch.as_tensor(ph.noise, device=x.device, dtype=x.dtype)
    # lattice spans the cylinder's bounding box
    g = torch.stack([(x[..., 0] + b.radius) / (2 * b.radius), (x[..., 1] + b.radius) / (2 * b.radius),
                     (x[..., 2] + b.half_height) / (2 * b.half_height)], -1).clamp(0, 1) * (K - 1)
    i0 = g.floor().long().clamp(max=K - 2)
    f = g - i0
    val = torch.zeros(x.shape[:-1], device=x.device, dtype=x.dtype)
    for cx in (0, 1):
        for cy in (0, 1):
            for cz in (0, 1):
                w = ((f[..., 0] if cx else 1 - f[..., 0]) * (f[..., 1] if cy else 1 - f[..., 1])
                     * (f[..., 2] if cz else 1 - f[..., 2]))
                val = val + w * lat[i0[..., 0] + cx, i0[..., 1] + cy, i0[..., 2] + cz]
    return torch.sigmoid((ph.front_z(t) + ph.noise_amp * val - x[..., 2]) / ph.front_width)


def dynamic_porous_projection(ph: DynamicPorousPhantom, geometry, angle: float, t: float, device,
                              samples_per_voxel: int = 4, chunk: int = 8192) -> torch.Tensor:
    """Line integrals at (angle, t): exact chords of the cylinder and of the
    grains at their radii at t, plus the brine front ray-marched at
    ``samples_per_voxel`` midpoint samples per voxel of path inside the
    cylinder."""
    b = ph.base
    static = porous_projection(b, geometry, angle, device,
                               grain_scale=np.divide(ph.radii(t), b.radii, out=np.zeros_like(b.radii),
                                                     where=b.radii > 0)).double().reshape(-1)
    o, d = detector_rays(geometry, angle, device)
    # entry/exit of the cylinder's bounding box along each ray
    lo = torch.tensor([-b.radius, -b.radius, -b.half_height], device=device, dtype=torch.float64)
    hi = -lo
    safe = torch.where(d.abs() > 1e-12, d, torch.full_like(d, 1e-12))
    t0 = torch.minimum((lo - o) / safe, (hi - o) / safe).max(1).values
    t1 = torch.maximum((lo - o) / safe, (hi - o) / safe).min(1).values
    L = torch.clamp(t1 - t0, min=0)
    n_s = int(math.ceil(float(L.max()) * samples_per_voxel)) if L.numel() else 0
    brine = torch.zeros_like(L)
    if n_s > 0:
        u = (torch.arange(n_s, device=device, dtype=torch.float64) + 0.5) / n_s
        for i in range(0, o.shape[0], chunk):
            tt = t0[i:i + chunk, None] + u[None] * L[i:i + chunk, None]                   # [c, n_s]
            pts = o[i:i + chunk, None, :] + tt[..., None] * d[i:i + chunk, None, :]       # [c, n_s, 3]
            inside = (pts[..., 0] ** 2 + pts[..., 1] ** 2 <= b.radius ** 2) & (pts[..., 2].abs() <= b.half_height)
            fr = _front(ph, pts, t) * inside
            brine[i:i + chunk] = fr.sum(1) * (L[i:i + chunk] / n_s)
    out = static + (ph.mu_brine - b.mu_cyl) * brine
    return out.to(torch.float32).reshape(geometry.nDetector[0], geometry.nDetector[1])


def dynamic_porous_volume(ph: DynamicPorousPhantom, n: int, t: float, device) -> torch.Tensor:
    """Voxel-centre attenuation [z, y, x] at time t."""
    b = ph.base
    shrunk = PorousPhantom(b.radius, b.half_height, b.mu_cyl, b.mu_grain, b.centers, ph.radii(t), b.packing)
    vol = porous_volume(shrunk, n, device).double()
    c = torch.arange(n, device=device, dtype=torch.float64) - (n - 1) / 2
    Z, Y, X = torch.meshgrid(c, c, c, indexing="ij")
    pts = torch.stack([X, Y, Z], -1)
    inside = (X ** 2 + Y ** 2 <= b.radius ** 2) & (Z.abs() <= b.half_height)
    vol = vol + (ph.mu_brine - b.mu_cyl) * _front(ph, pts, t) * inside
    return vol.float()


def poisson_projections(projs: torch.Tensor, width: float, photons: float = 1e4, seed: int = 0) -> torch.Tensor:
    """Poisson noise on line integrals ``projs`` (voxel units): counts
    I = Poisson(photons * exp(-p / width)) on the attenuation per object
    width, so that exp(-p) stays in the detector's range, and
    p' = -ln(I / photons) * width with I clamped to [1, photons].  The upper
    clamp (a flat-field-corrected reading does not exceed the open beam)
    keeps p' >= 0, so the data set's minimum is 0 as the reference's export
    (sigma * (max - min) / max_distance_traveled + min) assumes."""
    gen = torch.Generator(device=projs.device).manual_seed(seed)
    counts = torch.poisson(photons * torch.exp(-projs.double() / width), generator=gen)
    return (-torch.log(torch.clamp(counts, min=1.0, max=photons) / photons) * width).float()


def minmax_scale(projs: torch.Tensor):
    """Dataset-wide min-max scaling to [0,1] (nect/data.py:177-183)."""
    mn = projs.min()
    projs = projs - mn
    mx = projs.max()
    return projs / mx, float(mn), float(mx)
