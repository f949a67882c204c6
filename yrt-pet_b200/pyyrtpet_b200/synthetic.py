"""Seeded synthetic scanners, phantoms and list-mode events.

The reference measures on clinical and simulated datasets that are not
available here; these generators produce inputs with the shapes, sizes and
value distributions of the five benchmark configurations instead:

  C1  16 rings x 256 crystals, R = 300 mm; image 128x128x64 @ 2 mm; 1M events
  C2  80 rings x 672 crystals, R = 410 mm; image 256x256x160 @ 2 mm; 50M TOF
      events (214 ps FWHM), water mu-map, lognormal crystal efficiencies,
      20 % uniform randoms
  C3  C1 scanner histogram (DD + PSF), image 200x200x100 @ 2.5 mm
  C4  C1 scanner, 8 phantoms x 5M TOF events
  C5  C2 scanner, 24 frames with rigid motion

Emission points are drawn from the phantom activity (water cylinder r=100 mm
of activity 1 with three spheres r = 5, 10, 15 mm of activity 4 on a ring at
r = 50 mm, z = 0), directions are isotropic, and each line is intersected with
the cylinder of crystal centres (R + depth/2).  Hits map to the nearest
crystal by angle and to a ring by z; lines outside the axial FOV or beyond the
ring-difference / angle limits of the histogram are discarded.  TOF follows
the reference convention tof = (2 |x_e - p1| - |p1 - p2|) / c + noise.
Generation runs in torch on any device with an explicit generator per seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from .core import ImageParams, Scanner

C_MM_PS = 0.299792458


def scanner_c1(max_ring_diff: int = 15) -> Scanner:
    return Scanner("c1", 64, 4, 4, 10, 300, 256, 16, 1, max_ring_diff, 2, 1)


def scanner_c2() -> Scanner:
    return Scanner("c2", 256, 3.2, 3.2, 20, 410, 672, 80, 1, 79, 2, 1)


def image_c1() -> ImageParams:
    return ImageParams(128, 128, 64, 256, 256, 128)


def image_c2() -> ImageParams:
    return ImageParams(256, 256, 160, 512, 512, 320)


def image_c3() -> ImageParams:
    return ImageParams(200, 200, 100, 500, 500, 250)


@dataclass
class Phantom:
    cyl_radius: float = 100.0
    cyl_half_length: float = 32.0
    background: float = 1.0
    sphere_activity: float = 4.0
    spheres: tuple = ((50.0, 0.0, 0.0, 5.0), (-25.0, 43.30127, 0.0, 10.0),
                      (-25.0, -43.30127, 0.0, 15.0))

    def activity(self, x, y, z):
        inside = (x * x + y * y <= self.cyl_radius ** 2) & \
                 (z.abs() <= self.cyl_half_length)
        a = torch.where(inside, torch.full_like(x, self.background),
                        torch.zeros_like(x))
        for (cx, cy, cz, r) in self.spheres:
            s = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2 <= r * r
            a = torch.where(s, torch.full_like(x, self.sphere_activity), a)
        return a

    def image(self, ip: ImageParams, device="cpu") -> torch.Tensor:
        """Voxelised activity (voxel centres), shape (1, nz, ny, nx)."""
        xs = (torch.arange(ip.nx, device=device) + 0.5) * ip.vx - ip.length_x / 2
        ys = (torch.arange(ip.ny, device=device) + 0.5) * ip.vy - ip.length_y / 2
        zs = (torch.arange(ip.nz, device=device) + 0.5) * ip.vz - ip.length_z / 2
        z, y, x = torch.meshgrid(zs, ys, xs, indexing="ij")
        return self.activity(x, y, z)[None].float().contiguous()

    def mu_image(self, ip: ImageParams, mu_stored: float = 0.096,
                 device="cpu") -> torch.Tensor:
        """Water cylinder attenuation map.  The reference's ACF is
        exp(-0.1 * integral), i.e. mu in cm^-1 over mm paths: water
        0.0096 /mm is stored as 0.096."""
        xs = (torch.arange(ip.nx, device=device) + 0.5) * ip.vx - ip.length_x / 2
        ys = (torch.arange(ip.ny, device=device) + 0.5) * ip.vy - ip.length_y / 2
        zs = (torch.arange(ip.nz, device=device) + 0.5) * ip.vz - ip.length_z / 2
        z, y, x = torch.meshgrid(zs, ys, xs, indexing="ij")
        inside = (x * x + y * y <= self.cyl_radius ** 2) & \
                 (z.abs() <= self.cyl_half_length)
        return (inside.float() * mu_stored)[None].contiguous()


def random_phantom(seed: int, half_length: float) -> Phantom:
    """C1-family phantom with random sphere positions and contrasts."""
    g = np.random.default_rng(seed)
    spheres = []
    for r in (5.0, 10.0, 15.0):
        rad = g.uniform(0, 100 - r - 5)
        ang = g.uniform(0, 2 * np.pi)
        spheres.append((rad * np.cos(ang), rad * np.sin(ang),
                        g.uniform(-max(half_length - r, 0), max(half_length - r, 0)), r))
    return Phantom(cyl_half_length=half_length,
                   sphere_activity=float(g.uniform(2.0, 6.0)),
                   spheres=tuple(spheres))


def valid_ring_pairs(scanner: Scanner) -> np.ndarray:
    """dpr x dpr boolean table of in-ring crystal pairs that have a
    Histogram3D bin (Histogram3D::getDetPairInSameRing over all r, phi)."""
    n = scanner.detsPerRing
    r_cut = scanner.minAngDiff // 2
    if scanner.minAngDiff % 2 != 0 and n % 4 == 0:
        r_cut += 1
    num_r = n // 2 + 1 - scanner.minAngDiff
    r = np.arange(num_r)[:, None]
    phi = np.arange(n)[None, :]
    d02 = np.where(phi % 2 != 0, n // 2 + 1, n // 2)
    dr1 = r - n // 4 + r_cut
    dr2 = d02 - (r - n // 4 + r_cut)
    dr1 = np.where(dr1 < 0, dr1 + n, dr1)
    dr2 = np.where(dr2 < 0, dr2 + n, dr2)
    a = (dr1 + phi // 2) % n
    b = (dr2 + phi // 2) % n
    ok = np.zeros((n, n), bool)
    ok[a.ravel(), b.ravel()] = True
    ok[b.ravel(), a.ravel()] = True
    np.fill_diagonal(ok, False)
    return ok


@dataclass
class Events:
    d1: torch.Tensor
    d2: torch.Tensor
    tof: Optional[torch.Tensor] = None
    is_random: Optional[torch.Tensor] = None

    def numpy(self):
        out = {"d1": self.d1.cpu().numpy().astype(np.uint32),
               "d2": self.d2.cpu().numpy().astype(np.uint32)}
        if self.tof is not None:
            out["tof"] = self.tof.cpu().numpy().astype(np.float32)
        return out


def _chord_in_cylinder(x, d, radius, half_len):
    """Length of the line x + t d (|d| = 1) inside a finite z-cylinder."""
    a = d[:, 0] ** 2 + d[:, 1] ** 2
    b = 2 * (x[:, 0] * d[:, 0] + x[:, 1] * d[:, 1])
    c = x[:, 0] ** 2 + x[:, 1] ** 2 - radius ** 2
    disc = (b * b - 4 * a * c).clamp_min(0)
    sq = disc.sqrt()
    a_safe = torch.where(a > 1e-12, a, torch.ones_like(a))
    t0 = (-b - sq) / (2 * a_safe)
    t1 = (-b + sq) / (2 * a_safe)
    dz = torch.where(d[:, 2].abs() > 1e-12, d[:, 2], torch.full_like(d[:, 2], 1e-12))
    tz0 = (-half_len - x[:, 2]) / dz
    tz1 = (half_len - x[:, 2]) / dz
    lo = torch.maximum(t0, torch.minimum(tz0, tz1))
    hi = torch.minimum(t1, torch.maximum(tz0, tz1))
    return (hi - lo).clamp_min(0)


def generate_events(scanner: Scanner, n: int, seed: int, *,
                    phantom: Optional[Phantom] = None,
                    tof_fwhm_ps: Optional[float] = None,
                    mu_per_mm: float = 0.0,
                    crystal_eff: Optional[torch.Tensor] = None,
                    randoms_fraction: float = 0.0,
                    device="cpu", chunk: int = 1 << 22) -> Events:
    """n list-mode events (detector pairs, optional TOF in ps)."""
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    ph = phantom or Phantom(cyl_half_length=scanner.axialFOV / 2)
    ok_pairs = torch.from_numpy(valid_ring_pairs(scanner)).to(device)
    dpr, rings = scanner.detsPerRing, scanner.numRings
    Rc = scanner.scannerRadius + scanner.crystalDepth / 2
    zgap = scanner.axialFOV / rings
    amax = max(ph.background, ph.sphere_activity)
    n_rand = int(round(n * randoms_fraction))
    n_true = n - n_rand
    eff_max = float(crystal_eff.max()) if crystal_eff is not None else 1.0
    out_d1, out_d2, out_tof = [], [], []
    got = 0
    hl = ph.cyl_half_length
    while got < n_true:
        m = chunk
        x = torch.empty((m, 3), device=device)
        x[:, 0] = torch.rand(m, generator=g, device=device) * 2 * ph.cyl_radius - ph.cyl_radius
        x[:, 1] = torch.rand(m, generator=g, device=device) * 2 * ph.cyl_radius - ph.cyl_radius
        x[:, 2] = torch.rand(m, generator=g, device=device) * 2 * hl - hl
        act = ph.activity(x[:, 0], x[:, 1], x[:, 2])
        keep = torch.rand(m, generator=g, device=device) * amax < act
        x = x[keep]
        m = x.shape[0]
        u = torch.rand(m, generator=g, device=device) * 2 - 1
        phi = torch.rand(m, generator=g, device=device) * 2 * math.pi
        s = (1 - u * u).clamp_min(0).sqrt()
        d = torch.stack([s * torch.cos(phi), s * torch.sin(phi), u], 1)
        a = d[:, 0] ** 2 + d[:, 1] ** 2
        b = 2 * (x[:, 0] * d[:, 0] + x[:, 1] * d[:, 1])
        c = x[:, 0] ** 2 + x[:, 1] ** 2 - Rc * Rc
        good = a > 1e-9
        sq = (b * b - 4 * a * c).clamp_min(0).sqrt()
        a_s = torch.where(good, a, torch.ones_like(a))
        t1 = (-b - sq) / (2 * a_s)
        t2 = (-b + sq) / (2 * a_s)
        h1 = x + t1[:, None] * d
        h2 = x + t2[:, None] * d
        ang = 2 * math.pi / dpr
        c1 = torch.round(torch.atan2(h1[:, 1], h1[:, 0]) / ang).long() % dpr
        c2 = torch.round(torch.atan2(h2[:, 1], h2[:, 0]) / ang).long() % dpr
        r1 = torch.floor((h1[:, 2] + scanner.axialFOV / 2) / zgap).long()
        r2 = torch.floor((h2[:, 2] + scanner.axialFOV / 2) / zgap).long()
        good &= (r1 >= 0) & (r1 < rings) & (r2 >= 0) & (r2 < rings)
        good &= (r1 - r2).abs() <= scanner.maxRingDiff
        good &= ok_pairs[c1.clamp(0, dpr - 1), c2.clamp(0, dpr - 1)]
        d1 = c1 + r1.clamp(0, rings - 1) * dpr
        d2 = c2 + r2.clamp(0, rings - 1) * dpr
        if mu_per_mm > 0:
            chord = _chord_in_cylinder(x, d, ph.cyl_radius, hl)
            good &= torch.rand(x.shape[0], generator=g, device=device) < torch.exp(-mu_per_mm * chord)
        if crystal_eff is not None:
            e = crystal_eff[d1.clamp(0, len(crystal_eff) - 1)] * \
                crystal_eff[d2.clamp(0, len(crystal_eff) - 1)] / (eff_max * eff_max)
            good &= torch.rand(x.shape[0], generator=g, device=device) < e
        x, d1, d2, t1 = x[good], d1[good], d2[good], t1[good]
        h1 = h1[good]
        # Randomly swap the endpoint order so both orders occur.
        sw = torch.rand(d1.shape[0], generator=g, device=device) < 0.5
        d1, d2 = torch.where(sw, d2, d1), torch.where(sw, d1, d2)
        out_d1.append(d1)
        out_d2.append(d2)
        if tof_fwhm_ps:
            lut = torch.from_numpy(scanner.createLUT()[:, :3]).to(device)
            p1 = lut[d1]
            p2 = lut[d2]
            L = (p1 - p2).norm(dim=1)
            dist = (x - p1).norm(dim=1)
            sig = tof_fwhm_ps / 2.3548
            tof = (2 * dist - L) / C_MM_PS + torch.randn(
                d1.shape[0], generator=g, device=device) * sig
            out_tof.append(tof.float())
        got += d1.shape[0]
    d1 = torch.cat(out_d1)[:n_true]
    d2 = torch.cat(out_d2)[:n_true]
    tof = torch.cat(out_tof)[:n_true] if tof_fwhm_ps else None
    is_random = None
    if n_rand > 0:
        rd1, rd2, rtof = _uniform_lors(scanner, n_rand, g, ok_pairs, device,
                                       tof_fwhm_ps)
        perm = torch.randperm(n, generator=g, device=device)
        d1 = torch.cat([d1, rd1])[perm]
        d2 = torch.cat([d2, rd2])[perm]
        is_random = torch.cat([torch.zeros(n_true, dtype=torch.bool, device=device),
                               torch.ones(n_rand, dtype=torch.bool, device=device)])[perm]
        if tof is not None:
            tof = torch.cat([tof, rtof])[perm]
    return Events(d1.to(torch.int64), d2.to(torch.int64), tof, is_random)


def _uniform_lors(scanner, n, g, ok_pairs, device, tof_fwhm_ps):
    dpr, rings = scanner.detsPerRing, scanner.numRings
    outs1, outs2 = [], []
    got = 0
    while got < n:
        m = max(2 * (n - got), 1024)
        c1 = torch.randint(0, dpr, (m,), generator=g, device=device)
        c2 = torch.randint(0, dpr, (m,), generator=g, device=device)
        r1 = torch.randint(0, rings, (m,), generator=g, device=device)
        r2 = torch.randint(0, rings, (m,), generator=g, device=device)
        good = ok_pairs[c1, c2] & ((r1 - r2).abs() <= scanner.maxRingDiff)
        outs1.append((c1 + r1 * dpr)[good])
        outs2.append((c2 + r2 * dpr)[good])
        got += int(good.sum())
    d1 = torch.cat(outs1)[:n]
    d2 = torch.cat(outs2)[:n]
    tof = None
    if tof_fwhm_ps:
        lut = torch.from_numpy(scanner.createLUT()[:, :3]).to(device)
        L = (lut[d1] - lut[d2]).norm(dim=1)
        tof = ((torch.rand(n, generator=g, device=device) * 2 - 1) * L / C_MM_PS).float()
    return d1, d2, tof


def crystal_efficiencies(scanner: Scanner, seed: int, sigma: float = 0.1,
                         device="cpu") -> torch.Tensor:
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return torch.exp(torch.randn(scanner.getNumDets(), generator=g,
                                 device=device) * sigma).float()


def frame_counts_loguniform(num_frames: int, lo: float, hi: float,
                            seed: int) -> np.ndarray:
    g = np.random.default_rng(seed)
    return np.round(np.exp(g.uniform(np.log(lo), np.log(hi), num_frames))).astype(np.int64)


def rigid_transforms(num_frames: int, seed: int, max_deg: float = 3.0,
                     max_mm: float = 5.0) -> np.ndarray:
    """(num_frames, 12) in transform_t order (r00 r01 r02 tx r10 r11 r12 ty
    r20 r21 r22 tz): rotation <= max_deg about a random axis, translation
    <= max_mm per axis."""
    g = np.random.default_rng(seed)
    out = np.zeros((num_frames, 12), np.float32)
    for f in range(num_frames):
        axis = g.normal(size=3)
        axis /= np.linalg.norm(axis)
        th = np.deg2rad(g.uniform(0, max_deg))
        K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]],
                      [-axis[1], axis[0], 0]])
        R = np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K
        t = g.uniform(-max_mm, max_mm, 3)
        out[f] = np.concatenate([R, t[:, None]], axis=1).ravel()
    return out
