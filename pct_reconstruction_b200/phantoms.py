"""Synthetic phantoms and proton scans (seeded, deterministic).

The reference reconstructs measured or Monte-Carlo tracker data read from files; no data set is
shipped with it.  These generators stand in for that data with the shapes, sizes and value
distributions of the benchmark configurations:

* ``water_cylinder_phantom`` -- a water cylinder with four cylindrical inserts (RSP 0.3, 0.95,
  1.05, 1.6), discrete gantry angles;
* ``head_phantom`` -- an ellipsoidal head (semi-axes 8.5/7.0/3.5 cm) whose regions take RSP
  values from {0.0, 0.95, 1.04, 1.7};
* ``random_ellipsoid_phantom`` -- unions of random ellipsoids with RSP in [0.2, 1.8].

``simulate_tracks`` propagates protons through a phantom along the beam axis u in steps of
``step`` cm with Gaussian multiple Coulomb scattering: per step the lateral angle gets an increment
with the Highland width computed from the water-equivalent step length and the 200 MeV
1/(beta^2 p^2) polynomial of B.h:749-754; WEPL is the RSP line integral along the simulated path
plus Gaussian noise.  ``reconstruction_histories`` turns the tracks into the arrays the DROP stage
consumes (hull entry/exit points and angles, WEPL, first MLP voxel), which is what the reference
holds after reconstruction_cuts (B.cu:8296).  Everything runs in torch on the given device.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import torch

# 1/(beta^2 p^2) fit at 200 MeV, MeV^-2, in powers of depth (cm) (B.h:749-754)
A_COEFFS = (7.457e-6, 4.548e-7, -5.777e-8, 1.301e-8, -9.228e-10, 2.687e-11)
E_0, X_0 = 13.6, 36.08


@dataclass
class Ellipsoid:
    cx: float
    cy: float
    cz: float
    ax: float
    ay: float
    az: float
    rsp: float
    mode: str = "set"  # "set": value replaces what is below it


@dataclass
class Phantom:
    objects: list = field(default_factory=list)
    background: float = 0.0
    name: str = "phantom"
    # outer boundary used as the object hull (an ellipsoid); None -> first object
    hull: Ellipsoid | None = None

    def rsp(self, x: torch.Tensor, y: torch.Tensor, z: torch.Tensor) -> torch.Tensor:
        out = torch.full_like(x, self.background)
        for o in self.objects:
            inside = ((x - o.cx) / o.ax) ** 2 + ((y - o.cy) / o.ay) ** 2 + ((z - o.cz) / o.az) ** 2 <= 1.0
            out = torch.where(inside, torch.full_like(x, o.rsp), out)
        return out

    def hull_ellipsoid(self) -> Ellipsoid:
        return self.hull if self.hull is not None else self.objects[0]


def water_cylinder_phantom(radius=8.0, height=1e3) -> Phantom:
    """Water cylinder (RSP 1.0) with 4 cylindrical inserts of radius 1 cm (cylinders are
    ellipsoids with a very long z axis)."""
    objs = [Ellipsoid(0, 0, 0, radius, radius, height, 1.0)]
    for k, rsp in enumerate((0.3, 0.95, 1.05, 1.6)):
        a = math.pi / 4 + k * math.pi / 2
        objs.append(Ellipsoid(3.5 * math.cos(a), 3.5 * math.sin(a), 0, 1.0, 1.0, height, rsp))
    return Phantom(objs, 0.0, "water_cylinder")


def head_phantom() -> Phantom:
    """Ellipsoidal head: skull shell RSP 1.7, brain 1.04, ventricles 0.95, sinus/air 0.0."""
    objs = [
        Ellipsoid(0, 0, 0, 8.5, 7.0, 3.5, 1.7),
        Ellipsoid(0, 0, 0, 8.0, 6.5, 3.1, 1.04),
        Ellipsoid(-1.2, 0.6, 0.0, 1.0, 2.0, 1.2, 0.95),
        Ellipsoid(1.2, 0.6, 0.0, 1.0, 2.0, 1.2, 0.95),
        Ellipsoid(0.0, -5.0, -0.5, 1.5, 0.8, 0.8, 0.0),
        Ellipsoid(2.5, -2.0, 1.0, 0.7, 0.7, 0.7, 1.7),
    ]
    return Phantom(objs, 0.0, "head")


def random_ellipsoid_phantom(seed: int, extent=(8.0, 8.0, 3.0), count=6) -> Phantom:
    g = torch.Generator().manual_seed(seed)
    r = lambda lo, hi: lo + (hi - lo) * torch.rand((), generator=g).item()
    outer = Ellipsoid(0, 0, 0, extent[0] * r(0.8, 1.0), extent[1] * r(0.8, 1.0), extent[2] * r(0.8, 1.0), r(0.8, 1.2))
    objs = [outer]
    for _ in range(count):
        objs.append(Ellipsoid(r(-0.5, 0.5) * outer.ax, r(-0.5, 0.5) * outer.ay, r(-0.4, 0.4) * outer.az,
                              r(0.1, 0.35) * outer.ax, r(0.1, 0.35) * outer.ay, r(0.2, 0.5) * outer.az, r(0.2, 1.8)))
    return Phantom(objs, 0.0, f"random_{seed}", hull=outer)


def inv_beta2p2(depth: torch.Tensor) -> torch.Tensor:
    out = torch.zeros_like(depth)
    for k, a in enumerate(A_COEFFS):
        out = out + a * depth ** k
    return out


@dataclass
class Tracks:
    """Simulated proton tracks in the object frame (cm, rad)."""
    angle: torch.Tensor       # gantry/beam angle (rad) of each history
    t0: torch.Tensor          # lateral start offset in the gantry frame
    v0: torch.Tensor          # vertical start offset
    x_entry: torch.Tensor
    y_entry: torch.Tensor
    z_entry: torch.Tensor
    x_exit: torch.Tensor
    y_exit: torch.Tensor
    z_exit: torch.Tensor
    xy_entry_angle: torch.Tensor
    xz_entry_angle: torch.Tensor
    xy_exit_angle: torch.Tensor
    xz_exit_angle: torch.Tensor
    wepl: torch.Tensor
    hit: torch.Tensor         # True when the track crossed the hull
    # gantry frame (u along the beam): straight-line segments before and after the object
    u_in: torch.Tensor
    u_out: torch.Tensor
    t_in: torch.Tensor
    v_in: torch.Tensor
    slope_t_in: torch.Tensor
    slope_v_in: torch.Tensor
    t_out: torch.Tensor
    v_out: torch.Tensor
    slope_t_out: torch.Tensor
    slope_v_out: torch.Tensor


def _hull_crossings(h: Ellipsoid, angle, t0, v0, span):
    """Straight-line entry/exit parameters u of the ray (u*cos - t0*sin, u*sin + t0*cos) through
    the hull ellipse (2-D, in the xy plane)."""
    c, s = torch.cos(angle), torch.sin(angle)
    # point(u) = (u c - t0 s, u s + t0 c) ; ((x-cx)/ax)^2 + ((y-cy)/ay)^2 = 1
    px0, py0 = -t0 * s - h.cx, t0 * c - h.cy
    A = (c / h.ax) ** 2 + (s / h.ay) ** 2
    B = 2 * (px0 * c / h.ax ** 2 + py0 * s / h.ay ** 2)
    Cc = (px0 / h.ax) ** 2 + (py0 / h.ay) ** 2 - 1
    disc = B * B - 4 * A * Cc
    ok = disc > 0
    sq = torch.sqrt(torch.clamp(disc, min=0))
    u_in = (-B - sq) / (2 * A)
    u_out = (-B + sq) / (2 * A)
    return ok, torch.clamp(u_in, -span, span), torch.clamp(u_out, -span, span)


def simulate_tracks(phantom: Phantom, n: int, *, seed: int, device="cpu", continuous_angles=False,
                    angle_interval_deg=4.0, t_extent=18.0, v_extent=4.0, step=0.1, wepl_sigma=0.15,
                    span=10.0, chunk=4_000_000) -> Tracks:
    """Simulate n proton histories crossing `phantom` (see module docstring)."""
    dev = torch.device(device)
    g = torch.Generator(device=dev).manual_seed(seed)
    parts = []
    for start in range(0, n, chunk):
        m = min(chunk, n - start)
        parts.append(_simulate_chunk(phantom, m, g, dev, continuous_angles, angle_interval_deg, t_extent, v_extent,
                                     step, wepl_sigma, span))
    return Tracks(*[torch.cat([getattr(p, f) for p in parts]) for f in Tracks.__dataclass_fields__])


def _simulate_chunk(phantom, n, g, dev, continuous, interval, t_extent, v_extent, step, wepl_sigma, span) -> Tracks:
    f64 = torch.float64
    rnd = lambda: torch.rand(n, generator=g, device=dev, dtype=f64)
    nrm = lambda: torch.randn(n, generator=g, device=dev, dtype=f64)
    if continuous:
        angle = rnd() * (2 * math.pi)
    else:
        k = torch.floor(rnd() * (360.0 / interval))
        angle = k * (interval * math.pi / 180.0)
    t0 = (rnd() - 0.5) * t_extent
    v0 = (rnd() - 0.5) * v_extent
    # small beam divergence
    th_t = nrm() * 0.002
    th_v = nrm() * 0.002
    h = phantom.hull_ellipsoid()
    ok, u_in, u_out = _hull_crossings(h, angle, t0, v0, span)
    c, s = torch.cos(angle), torch.sin(angle)
    t, v = t0.clone(), v0.clone()
    ang_t, ang_v = th_t.clone(), th_v.clone()
    wepl = torch.zeros(n, device=dev, dtype=f64)
    depth = torch.zeros(n, device=dev, dtype=f64)
    t_entry = v_entry = None
    # propagate straight to the hull entry, then step through the object
    t = t + ang_t * (u_in + span)
    v = v + ang_v * (u_in + span)
    t_entry, v_entry = t.clone(), v.clone()
    ent_t, ent_v = ang_t.clone(), ang_v.clone()
    length = torch.clamp(u_out - u_in, min=0)
    nsteps = int(math.ceil(float(length.max().item()) / step)) if n else 0
    for i in range(nsteps):
        du = torch.clamp(length - i * step, min=0, max=step)
        active = du > 0
        u = u_in + i * step + 0.5 * du
        x = u * c - t * s
        y = u * s + t * c
        rsp = phantom.rsp(x, y, v)
        wl = rsp * du  # water-equivalent step
        depth = depth + wl
        wepl = wepl + wl
        lw = torch.clamp(wl, min=1e-9)
        sig2 = (E_0 * (1 + 0.038 * torch.log(lw / X_0))) ** 2 * inv_beta2p2(depth) * lw / X_0
        sig = torch.sqrt(torch.clamp(sig2, min=0)) * (wl > 1e-6)
        dth_t = nrm() * sig
        dth_v = nrm() * sig
        t = t + (ang_t + 0.5 * dth_t) * du
        v = v + (ang_v + 0.5 * dth_v) * du
        ang_t = torch.where(active, ang_t + dth_t, ang_t)
        ang_v = torch.where(active, ang_v + dth_v, ang_v)
    wepl = wepl + nrm() * wepl_sigma
    xe, ye = u_in * c - t_entry * s, u_in * s + t_entry * c
    xo, yo = u_out * c - t * s, u_out * s + t * c
    return Tracks(angle, t0, v0, xe, ye, v_entry, xo, yo, v,
                  angle + torch.atan(ent_t), torch.atan(ent_v), angle + torch.atan(ang_t), torch.atan(ang_v), wepl,
                  ok & (length > 4 * step), u_in, u_out, t_entry, v_entry, ent_t, ent_v, t, v, ang_t, ang_v)


def tracker_data(tracks: Tracks, planes=(-15.0, -10.0, 10.0, 15.0)) -> dict:
    """Tracker hits of each history on two entry and two exit planes (gantry frame, cm), in the
    arrays the reference reads (t/u/v_in_1, _in_2, _out_1, _out_2; B.cu:4361-4766 after its
    mm->cm conversion), plus WEPL and the gantry angle in degrees (float; integral for
    discrete-angle scans)."""
    u_in1, u_in2, u_out1, u_out2 = planes
    out = {}
    for name, u, side in (("in_1", u_in1, "in"), ("in_2", u_in2, "in"), ("out_1", u_out1, "out"),
                          ("out_2", u_out2, "out")):
        if side == "in":
            t = tracks.t_in + tracks.slope_t_in * (u - tracks.u_in)
            v = tracks.v_in + tracks.slope_v_in * (u - tracks.u_in)
        else:
            t = tracks.t_out + tracks.slope_t_out * (u - tracks.u_out)
            v = tracks.v_out + tracks.slope_v_out * (u - tracks.u_out)
        out["t_" + name] = t.to(torch.float32)
        out["u_" + name] = torch.full_like(t, u).to(torch.float32)
        out["v_" + name] = v.to(torch.float32)
    out["WEPL"] = tracks.wepl.to(torch.float32)
    out["gantry_angle"] = torch.remainder(tracks.angle * (180.0 / math.pi), 360.0).to(torch.float32)
    return out


def voxel_of(cfg, x, y, z):
    """Voxel index of points, as calculate_voxel_GPU computes it (B.cu:11091)."""
    vx = torch.floor(torch.abs(x - (-cfg.RECON_CYL_RADIUS)) / cfg.VOXEL_WIDTH).to(torch.int64)
    vy = torch.floor(torch.abs(y - cfg.RECON_CYL_RADIUS) / cfg.VOXEL_HEIGHT).to(torch.int64)
    vz = torch.floor(torch.abs(z - cfg.RECON_CYL_HEIGHT / 2) / cfg.VOXEL_THICKNESS).to(torch.int64)
    return vx + vy * cfg.COLUMNS + vz * cfg.COLUMNS * cfg.ROWS


def reconstruction_histories(cfg, tracks: Tracks) -> dict:
    """DROP-stage arrays (float32 SoA + uint32 first voxel) for the tracks that crossed the hull
    inside the reconstruction cylinder, in simulation order."""
    keep = tracks.hit & (tracks.z_entry.abs() < cfg.RECON_CYL_HEIGHT / 2) & (tracks.z_exit.abs() < cfg.RECON_CYL_HEIGHT / 2)
    r2 = cfg.RECON_CYL_RADIUS ** 2
    keep &= (tracks.x_entry ** 2 + tracks.y_entry ** 2 < r2) & (tracks.x_exit ** 2 + tracks.y_exit ** 2 < r2)
    idx = torch.nonzero(keep).squeeze(1)
    out = {}
    for name in ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit",
                 "xy_entry_angle", "xz_entry_angle", "xy_exit_angle", "xz_exit_angle"):
        out[name] = getattr(tracks, name)[idx].to(torch.float32).contiguous()
    out["WEPL"] = tracks.wepl[idx].to(torch.float32).contiguous()
    fv = voxel_of(cfg, out["x_entry"].double(), out["y_entry"].double(), out["z_entry"].double())
    out["first_MLP_voxel"] = fv.to(torch.int64).to(torch.int32).contiguous()  # reinterpreted as uint32
    return out


def truth_image(cfg, phantom: Phantom, device="cpu") -> torch.Tensor:
    """Phantom RSP sampled at voxel centres, reference voxel order (row 0 at +y, slice 0 at +z)."""
    dev = torch.device(device)
    col = torch.arange(cfg.COLUMNS, device=dev, dtype=torch.float64)
    row = torch.arange(cfg.ROWS, device=dev, dtype=torch.float64)
    sl = torch.arange(cfg.SLICES, device=dev, dtype=torch.float64)
    x = -cfg.RECON_CYL_RADIUS + (col + 0.5) * cfg.VOXEL_WIDTH
    y = cfg.RECON_CYL_RADIUS - (row + 0.5) * cfg.VOXEL_HEIGHT
    z = cfg.RECON_CYL_HEIGHT / 2 - (sl + 0.5) * cfg.VOXEL_THICKNESS
    Z, Y, X = torch.meshgrid(z, y, x, indexing="ij")
    return phantom.rsp(X, Y, Z).to(torch.float32).reshape(-1)


def hull_image(cfg, phantom: Phantom, device="cpu") -> torch.Tensor:
    """Boolean image of the phantom's hull ellipsoid (stand-in for a detected hull)."""
    h = phantom.hull_ellipsoid()
    dev = torch.device(device)
    col = torch.arange(cfg.COLUMNS, device=dev, dtype=torch.float64)
    row = torch.arange(cfg.ROWS, device=dev, dtype=torch.float64)
    sl = torch.arange(cfg.SLICES, device=dev, dtype=torch.float64)
    x = -cfg.RECON_CYL_RADIUS + (col + 0.5) * cfg.VOXEL_WIDTH
    y = cfg.RECON_CYL_RADIUS - (row + 0.5) * cfg.VOXEL_HEIGHT
    z = cfg.RECON_CYL_HEIGHT / 2 - (sl + 0.5) * cfg.VOXEL_THICKNESS
    Z, Y, X = torch.meshgrid(z, y, x, indexing="ij")
    inside = ((X - h.cx) / h.ax) ** 2 + ((Y - h.cy) / h.ay) ** 2 + ((Z - h.cz) / h.az) ** 2 <= 1.0
    return inside.reshape(-1)
