"""Seeded synthetic workloads for the granular hot path.

The reference publishes no benchmark inputs, so these generators stand in for
them with the shapes, sizes and value distributions the benchmark
configurations name:

* ``sphere_pour``  -- monodisperse Hertz/history pour on a flat floor with
  periodic x/y (20,000 spheres, r = 1 mm, 40 x 40 x 200 mm box).
* ``drum``         -- rotating drum: spheres of radius U(0.8, 1.2) mm in a
  closed, triangulated cylinder (axis x) turned by ``fix move/mesh rotate``.
* ``hopper``       -- polydisperse spheres (lognormal radius, median 1 mm,
  sigma 0.25, clipped to 0.5-2 mm) with Hertz/history + rolling friction cdt
  in a procedurally triangulated conical hopper (60 deg half-angle, 30 mm
  outlet) discharging onto a flat catch floor; ``hopper_packed`` is the same
  hopper packed at the start of its discharge (configuration 2's state).
* ``drum_config3`` -- configuration 3: 8M spheres packed in the bottom of a
  0.5 m drum of 32,768 triangles turned by ``fix move/mesh rotate``.
* ``bed_config5``  -- configuration 5: 20M spheres of r = 0.5 mm in hexagonal
  close packing over a 65,536-triangle bumpy plate in a walled box.

A scenario is a plain dict (box, materials, atoms, ordered fix list) that the
engine wrapper and the tests both consume.  Units are SI throughout.
"""
import math

import numpy as np


def _materials(ntypes, E, nu, e, mu, mur=0.0):
    return {
        "ntypes": ntypes,
        "youngs": np.full(ntypes, E),
        "poisson": np.full(ntypes, nu),
        "restitution": np.full((ntypes, ntypes), e),
        "friction": np.full((ntypes, ntypes), mu),
        "rollfriction": np.full((ntypes, ntypes), mur),
    }


def _atoms(pos, radius, density, vel, seed_omega=None):
    n = len(radius)
    # the reference's read_data mass, in its evaluation order (src/atom_vec_sphere.cpp:1081)
    rmass = 4.0 * math.pi / 3.0 * radius * radius * radius * density
    return {
        "x": np.ascontiguousarray(pos, dtype=np.float64),
        "v": np.ascontiguousarray(vel, dtype=np.float64),
        "omega": np.zeros((n, 3)) if seed_omega is None else seed_omega,
        "radius": np.ascontiguousarray(radius, dtype=np.float64),
        "rmass": np.ascontiguousarray(rmass, dtype=np.float64),
        "density": np.ascontiguousarray(np.broadcast_to(np.asarray(density, dtype=np.float64), (n,))),
        "type": np.ones(n, dtype=np.int32),
        "tag": np.arange(1, n + 1, dtype=np.int32),
    }


def sphere_pour(n=20000, seed=12345, dt=1e-5, skin=0.5e-3, jitter=0.2e-3, vmax=0.1,
                box=(0.04, 0.04, 0.2), spacing=(2.5e-3, 2.5e-3, 2.4e-3), omega_max=0.0):
    """Monodisperse pour: jittered lattice (16 x 16 per layer at 2.5 mm, layers
    2.4 mm apart), uniform +-vmax velocities, flat z=0 floor, gravity -z."""
    rng = np.random.default_rng(seed)
    r = 1e-3
    nx = int(round(box[0] / spacing[0]))
    ny = int(round(box[1] / spacing[1]))
    per_layer = nx * ny
    nlayers = (n + per_layer - 1) // per_layer
    ii = np.arange(nlayers * per_layer)[:n]
    ix = ii % nx
    iy = (ii // nx) % ny
    iz = ii // per_layer
    pos = np.stack([(ix + 0.5) * spacing[0], (iy + 0.5) * spacing[1], 1.5e-3 + iz * spacing[2]], axis=1)
    pos = pos + rng.uniform(-jitter, jitter, size=pos.shape)
    vel = rng.uniform(-vmax, vmax, size=(n, 3))
    om = rng.uniform(-omega_max, omega_max, size=(n, 3)) if omega_max > 0 else None
    if pos[:, 2].max() + r >= box[2]:
        raise ValueError("lattice does not fit the box")
    sc = {
        "name": "sphere_pour",
        "dt": dt, "skin": skin,
        "boxlo": [0.0, 0.0, 0.0], "boxhi": list(box), "periodic": [1, 1, 0],
        "every": 1, "delay": 0, "check": 1, "sortfreq": 1000, "sortbinsize": 0.0,
        "rolling_cdt": 0, "tangential_damping": 1,
        "atoms": _atoms(pos, np.full(n, r), 2500.0, vel, om),
        "fixes": [
            {"kind": "gravity", "magnitude": 9.81, "vector": [0.0, 0.0, -1.0]},
            {"kind": "wall_plane", "dim": 2, "pos": 0.0, "wall_type": 1, "rolling_cdt": 0},
            {"kind": "nve_sphere"},
        ],
    }
    sc.update(_materials(1, 5e6, 0.45, 0.3, 0.5))
    return sc


def bidisperse_bed(nx=26, nlayers=12, r_small=0.3e-3, r_big=3e-3, n_big=2, seed=5, dt=2e-6, skin=0.5e-3,
                   vmax=0.3):
    """Small spheres on a jittered lattice (0.75 mm spacing) with a few large
    spheres buried in it (small ones overlapping them removed), periodic in
    x and y, floor at z = 0, gravity -z.  A large sphere has far more than 64
    neighbours within the cutoff, so its pairs take the serial path."""
    rng = np.random.default_rng(seed)
    sp = 0.75e-3
    L = nx * sp
    ii = np.arange(nx * nx * nlayers)
    pos = np.stack([(ii % nx + 0.5) * sp, ((ii // nx) % nx + 0.5) * sp, r_small + 0.05e-3 + (ii // (nx * nx)) * sp],
                   axis=1)
    pos = pos + rng.uniform(-0.05e-3, 0.05e-3, size=pos.shape)
    zmid = 0.5 * (pos[:, 2].min() + pos[:, 2].max())
    big = np.stack([np.array([(k + 0.5) * L / n_big, 0.5 * L, zmid]) for k in range(n_big)])
    keep = np.ones(len(pos), dtype=bool)
    for c in big:
        keep &= np.linalg.norm(pos - c, axis=1) > r_big + r_small + 0.05e-3
    pos = np.concatenate([big, pos[keep]])
    rad = np.concatenate([np.full(n_big, r_big), np.full(int(keep.sum()), r_small)])
    n = len(pos)
    vel = rng.uniform(-vmax, vmax, size=(n, 3))
    sc = {
        "name": "bidisperse_bed",
        "dt": dt, "skin": skin,
        "boxlo": [0.0, 0.0, 0.0], "boxhi": [L, L, pos[:, 2].max() + 2 * r_big + 5e-3], "periodic": [1, 1, 0],
        "every": 1, "delay": 0, "check": 1, "sortfreq": 1000, "sortbinsize": 0.0,
        "rolling_cdt": 1, "tangential_damping": 1,
        "atoms": _atoms(pos, rad, 2500.0, vel, None),
        "fixes": [
            {"kind": "gravity", "magnitude": 9.81, "vector": [0.0, 0.0, -1.0]},
            {"kind": "wall_plane", "dim": 2, "pos": 0.0, "wall_type": 1, "rolling_cdt": 1},
            {"kind": "nve_sphere"},
        ],
    }
    sc.update(_materials(1, 5e6, 0.45, 0.3, 0.5))
    sc["rollfriction"] = np.array([[0.1]])
    return sc


def cone_mesh(n_theta=128, n_z=32, r_out=0.015, half_angle_deg=60.0, height=0.17, z0=0.0):
    """Triangulated cone frustum (a hopper), ``2 * n_theta * n_z`` triangles.

    Rings are evenly spaced in z; every quad between two rings and two
    generators is planar and is split along one diagonal.  Returned as an
    (ntri, 3, 3) node array in STL facet order."""
    t = math.tan(math.radians(half_angle_deg))
    th = np.linspace(0.0, 2.0 * math.pi, n_theta + 1)[:-1]
    zs = z0 + np.linspace(0.0, height, n_z + 1)
    rs = r_out + (zs - z0) * t
    tris = []
    for l in range(n_z):
        for k in range(n_theta):
            k2 = (k + 1) % n_theta
            p00 = (rs[l] * math.cos(th[k]), rs[l] * math.sin(th[k]), zs[l])
            p01 = (rs[l] * math.cos(th[k2]), rs[l] * math.sin(th[k2]), zs[l])
            p10 = (rs[l + 1] * math.cos(th[k]), rs[l + 1] * math.sin(th[k]), zs[l + 1])
            p11 = (rs[l + 1] * math.cos(th[k2]), rs[l + 1] * math.sin(th[k2]), zs[l + 1])
            tris.append((p00, p01, p11))
            tris.append((p00, p11, p10))
    return np.asarray(tris, dtype=np.float64)


def hopper(n=1_000_000, seed=2024, dt=5e-6, skin=0.5e-3, n_theta=128, n_z=32, half_angle_deg=60.0,
           r_out=0.015, gap=0.05, vmax=0.0, floor_drop=0.08):
    """Polydisperse hopper discharge (Hertz/history + rolling friction cdt).

    Radii: lognormal, median 1 mm, sigma 0.25, clipped to [0.5, 2] mm.  The
    particles are sorted by radius (largest first) and stacked bottom-up in
    simple-cubic layers whose spacing is (2 + gap) x the largest radius in the
    layer, clipped to the cone interior, so the fill starts dense with small
    gaps and no overlaps.  A flat floor ``floor_drop`` below the outlet
    catches the discharge so no atom leaves the box."""
    rng = np.random.default_rng(seed)
    rad = np.exp(rng.normal(math.log(1e-3), 0.25, size=n))
    rad = np.clip(rad, 0.5e-3, 2e-3)
    rad = np.sort(rad)[::-1].copy()
    t = math.tan(math.radians(half_angle_deg))
    pos = np.zeros((n, 3))
    placed = 0
    z = 2.1e-3
    while placed < n:
        rmax = rad[placed]
        s = (2.0 + gap) * rmax
        zc = z + rmax
        # usable radius: cone wall distance >= radius (wall normal inclined)
        rcone = r_out + zc * t
        rin = rcone - rmax / math.cos(math.radians(half_angle_deg)) - 0.2e-3
        if rin <= 0:
            z += s
            continue
        m = int(rin // s)
        g = np.arange(-m, m + 1) * s
        gx, gy = np.meshgrid(g, g, indexing="ij")
        ok = gx ** 2 + gy ** 2 <= rin ** 2
        pts = np.stack([gx[ok], gy[ok]], axis=1)
        take = min(len(pts), n - placed)
        sl = slice(placed, placed + take)
        pos[sl, 0] = pts[:take, 0]
        pos[sl, 1] = pts[:take, 1]
        pos[sl, 2] = zc
        placed += take
        z = zc + rmax + gap * rmax
    height = pos[:, 2].max() + 0.01
    nodes = cone_mesh(n_theta, n_z, r_out, half_angle_deg, height)
    rtop = r_out + height * t
    lo = [-(rtop + 0.01), -(rtop + 0.01), -floor_drop - 0.01]
    hi = [rtop + 0.01, rtop + 0.01, height + 0.02]
    vel = rng.uniform(-vmax, vmax, size=(n, 3)) if vmax > 0 else np.zeros((n, 3))
    sc = {
        "name": "hopper",
        "dt": dt, "skin": skin,
        "boxlo": lo, "boxhi": hi, "periodic": [0, 0, 0],
        "every": 1, "delay": 0, "check": 1, "sortfreq": 1000, "sortbinsize": 0.0,
        "rolling_cdt": 1, "tangential_damping": 1,
        "atoms": _atoms(pos, rad, 2500.0, vel),
        "fixes": [
            {"kind": "gravity", "magnitude": 9.81, "vector": [0.0, 0.0, -1.0]},
            {"kind": "wall_mesh", "nodes": nodes, "wall_type": 1, "curvature": 0.0, "rolling_cdt": 1},
            {"kind": "wall_plane", "dim": 2, "pos": -floor_drop, "wall_type": 1, "rolling_cdt": 1},
            {"kind": "nve_sphere"},
        ],
    }
    sc.update(_materials(1, 5e6, 0.45, 0.3, 0.5, 0.1))
    return sc


def _hex_annulus(a, rho_in, rho_out):
    """Sites of a triangular lattice of spacing a (centred on the axis) with
    rho_in <= rho <= rho_out, innermost first (ties in lattice order)."""
    m = int(rho_out / a * 1.2) + 2
    i, j = np.meshgrid(np.arange(-m, m + 1), np.arange(-m, m + 1), indexing="ij")
    x = a * (i + 0.5 * j).ravel()
    y = a * (0.5 * math.sqrt(3.0) * j).ravel()
    r2 = x * x + y * y
    keep = (r2 <= rho_out * rho_out) & (r2 >= rho_in * rho_in)
    x, y, r2 = x[keep], y[keep], r2[keep]
    order = np.argsort(r2, kind="stable")
    return x[order], y[order]


def hopper_packed(n=1_000_000, seed=2024, dt=5e-6, skin=0.5e-3, n_theta=128, n_z=32, half_angle_deg=60.0,
                  r_out=0.015, floor_drop=0.08, overlap=1e-4, band=2e-3, wall_overlap=2e-3, sortfreq=1000):
    """Packed conical hopper at the start of its discharge (config 2's state).

    Radii as ``hopper`` (lognormal, median 1 mm, sigma 0.25, clipped to
    0.5-2 mm), sorted largest first and stacked bottom-up in horizontal
    layers.  A layer is filled from the axis outwards in annular patches,
    each a triangular lattice holding particles of one narrow radius band
    (at most ``band`` relative) whose spacing is (1 - overlap) x the
    smallest diameter in the patch, so every in-plane neighbour pair inside
    a patch touches (overlaps of 1e-4 to ~5e-3 of a diameter); patches are
    one diameter apart.  Layers are a sum of their largest radii apart, so
    layers do not overlap.  Every other angular bin
    of the outermost ring is pushed horizontally outwards until it overlaps
    the triangulated cone wall by ``wall_overlap`` of its radius (its facet
    plane), which gives tens of thousands of mesh contacts at 1M particles;
    a clear ring of one diameter separates those from the lattice.  The 30 mm
    outlet is open and the particles start at rest, so the bed starts to
    discharge onto the catch floor ``floor_drop`` below the outlet."""
    rng = np.random.default_rng(seed)
    rad = np.exp(rng.normal(math.log(1e-3), 0.25, size=n))
    rad = np.clip(rad, 0.5e-3, 2e-3)
    rad = np.sort(rad)[::-1].copy()
    neg_rad = -rad   # ascending, for the band searches
    th = math.radians(half_angle_deg)
    t = math.tan(th)
    # facet planes of the triangulated cone (a quad between two generators
    # is planar and contains the apex): inward unit normal and a point
    phis = np.linspace(0.0, 2.0 * math.pi, n_theta + 1)
    p0 = np.stack([r_out * np.cos(phis[:-1]), r_out * np.sin(phis[:-1]), np.zeros(n_theta)], axis=1)
    p1 = np.stack([r_out * np.cos(phis[1:]), r_out * np.sin(phis[1:]), np.zeros(n_theta)], axis=1)
    r1 = r_out + 1.0 * t
    p2 = np.stack([r1 * np.cos(phis[:-1]), r1 * np.sin(phis[:-1]), np.ones(n_theta)], axis=1)
    nrm = np.cross(p1 - p0, p2 - p0)
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    nrm *= np.where((nrm[:, 0] * np.cos(phis[:-1]) + nrm[:, 1] * np.sin(phis[:-1])) > 0, -1.0, 1.0)[:, None]
    pos = np.zeros((n, 3))
    chunk = max(200, n // 500)
    placed = 0
    zbot = 0.5e-3
    while placed < n:
        rmax = rad[placed]
        zc = zbot + rmax
        R = r_out + zc * t
        # a sphere of radius r touches the cone at rho = R - r / cos(half angle); keep one diameter clear
        rho_lim = R - rmax * (1.0 - wall_overlap) / math.cos(th) - 2.1 * rmax
        if rho_lim <= rmax:
            zbot += 2.0 * rmax
            continue
        # the layer is filled from the axis outwards in annular patches of at
        # most `chunk` particles, each a lattice whose spacing is the smallest
        # diameter of its particles (narrow radius band per patch); patches
        # are one diameter apart
        rho_in, last = 0.0, None
        while placed < n:
            r0 = rad[placed]
            x, y = _hex_annulus(2.0 * r0, rho_in, rho_lim)
            if len(x) == 0:
                break
            # at most `chunk` particles and a radius band of at most `band` (relative)
            j = int(np.searchsorted(neg_rad, -r0 / (1.0 + band), side="right"))
            take = max(1, min(len(x), chunk, n - placed, j - placed))
            a = 2.0 * rad[placed + take - 1] * (1.0 - overlap)
            x, y = _hex_annulus(a, rho_in, rho_lim)
            take = min(take, len(x))
            if take == 0:
                break
            x, y = x[:take], y[:take]
            sl = slice(placed, placed + take)
            pos[sl, 0], pos[sl, 1], pos[sl, 2] = x, y, zc
            last = (placed, take, a)
            placed += take
            rho_in = np.hypot(x, y).max() + 2.0 * r0 + 1e-7
        if last is not None and last[1] > 7:
            # outermost band of the outermost patch, in angular order: a
            # particle is pushed outwards onto the wall when it is at least
            # 2.05 rmax of arc from the last one pushed (and from the first)
            p0_, take, a = last
            idx = np.arange(p0_, p0_ + take)
            x, y = pos[idx, 0], pos[idx, 1]
            rho = np.hypot(x, y)
            phi = np.arctan2(y, x) % (2.0 * math.pi)
            dphi = 2.05 * rmax / max(R - rmax / math.cos(th), rmax)
            cand = np.flatnonzero(rho > rho.max() - a)
            cand = cand[np.argsort(phi[cand], kind="stable")]
            chosen = []
            for c in cand:
                if not chosen or phi[c] - phi[chosen[-1]] >= dphi:
                    if not chosen or phi[chosen[0]] + 2.0 * math.pi - phi[c] >= dphi:
                        chosen.append(c)
            sel = np.array(sorted(chosen), dtype=np.int64)
            if len(sel):
                k = np.minimum((phi[sel] / (2.0 * math.pi) * n_theta).astype(int), n_theta - 1)
                e = np.stack([np.cos(phi[sel]), np.sin(phi[sel]), np.zeros(len(sel))], axis=1)
                pts = np.stack([x[sel], y[sel], np.full(len(sel), zc)], axis=1)
                dist = np.einsum("ij,ij->i", pts - p0[k], nrm[k])
                en = np.einsum("ij,ij->i", e, nrm[k])
                dh = (dist - rad[idx[sel]] * (1.0 - wall_overlap)) / (-en)
                pos[idx[sel], 0] = x[sel] + dh * e[:, 0]
                pos[idx[sel], 1] = y[sel] + dh * e[:, 1]
        zbot = zc + rmax + 1e-7
    height = pos[:, 2].max() + 0.01
    nodes = cone_mesh(n_theta, n_z, r_out, half_angle_deg, height)
    rtop = r_out + height * t
    lo = [-(rtop + 0.01), -(rtop + 0.01), -floor_drop - 0.01]
    hi = [rtop + 0.01, rtop + 0.01, height + 0.02]
    sc = {
        "name": "hopper_packed",
        "dt": dt, "skin": skin,
        "boxlo": lo, "boxhi": hi, "periodic": [0, 0, 0],
        "every": 1, "delay": 0, "check": 1, "sortfreq": sortfreq, "sortbinsize": 0.0,
        "rolling_cdt": 1, "tangential_damping": 1,
        "atoms": _atoms(pos, rad, 2500.0, np.zeros((n, 3))),
        "fixes": [
            {"kind": "gravity", "magnitude": 9.81, "vector": [0.0, 0.0, -1.0]},
            {"kind": "wall_mesh", "nodes": nodes, "wall_type": 1, "curvature": 0.0, "rolling_cdt": 1},
            {"kind": "wall_plane", "dim": 2, "pos": -floor_drop, "wall_type": 1, "rolling_cdt": 1},
            {"kind": "nve_sphere"},
        ],
    }
    sc.update(_materials(1, 5e6, 0.45, 0.3, 0.5, 0.1))
    return sc


def plate_mesh(half=0.025, z=0.0, k=8):
    """Square plate at height z, side 2 * half, 2 * k * k triangles (normal +z)."""
    g = np.linspace(-half, half, k + 1)
    tris = []
    for a in range(k):
        for b in range(k):
            p00, p10 = (g[a], g[b], z), (g[a + 1], g[b], z)
            p01, p11 = (g[a], g[b + 1], z), (g[a + 1], g[b + 1], z)
            tris.append((p00, p10, p11))
            tris.append((p00, p11, p01))
    return np.asarray(tris, dtype=np.float64)


def silo(n=2000, seed=21, dt=5e-6, skin=0.5e-3, radius=0.02, piston_speed=1.0, vmax=0.1):
    """Spheres (r U(0.8, 1.2) mm) on a jittered lattice inside a vertical
    cylinder wall (primitive zcylinder, radius 20 mm, axis at x = y = 0) on a
    flat floor, pressed by a triangulated square piston that moves down at
    ``piston_speed`` (fix move/mesh linear)."""
    rng = np.random.default_rng(seed)
    rad = rng.uniform(0.8e-3, 1.2e-3, size=n)
    s = 2.6e-3
    m = int((radius - 1.5e-3) // s)
    g = np.arange(-m, m + 1) * s
    gx, gy = np.meshgrid(g, g, indexing="ij")
    ok = gx ** 2 + gy ** 2 <= (radius - 1.5e-3) ** 2
    layer = np.stack([gx[ok], gy[ok]], axis=1)
    nl = (n + len(layer) - 1) // len(layer)
    pos = np.zeros((n, 3))
    for l in range(nl):
        sl = slice(l * len(layer), min(n, (l + 1) * len(layer)))
        cnt = sl.stop - sl.start
        pos[sl, 0:2] = layer[:cnt]
        pos[sl, 2] = 1.5e-3 + l * s
    pos[:, :2] += rng.uniform(-0.1e-3, 0.1e-3, size=(n, 2))
    top = pos[:, 2].max() + 3e-3
    vel = rng.uniform(-vmax, vmax, size=(n, 3))
    box = 0.03
    sc = {
        "name": "silo", "dt": dt, "skin": skin,
        "boxlo": [-box, -box, -0.01], "boxhi": [box, box, top + 0.02], "periodic": [0, 0, 0],
        "every": 1, "delay": 0, "check": 1, "sortfreq": 500, "sortbinsize": 0.0,
        "rolling_cdt": 0, "tangential_damping": 1,
        "atoms": _atoms(pos, rad, 2500.0, vel),
        "fixes": [
            {"kind": "gravity", "magnitude": 9.81, "vector": [0.0, 0.0, -1.0]},
            {"kind": "wall_cylinder", "dim": 2, "radius": radius, "c1": 0.0, "c2": 0.0, "wall_type": 1},
            {"kind": "wall_plane", "dim": 2, "pos": 0.0, "wall_type": 1},
            {"kind": "wall_mesh", "nodes": plate_mesh(0.025, top, 8), "wall_type": 1, "curvature": 0.0},
            {"kind": "move_mesh_linear", "mesh": 3, "velocity": [0.0, 0.0, -piston_speed]},
            {"kind": "nve_sphere"},
        ],
    }
    sc.update(_materials(1, 5e6, 0.45, 0.3, 0.5))
    return sc


def drum_mesh(diameter=0.5, length=0.85, n_theta=128, n_ax=121, cap_rings=4):
    """Closed cylinder along x centred on the origin: a side of
    ``2 * n_theta * n_ax`` triangles (axial rings, so no triangle spans the
    drum) and two end caps on polar grids (a fan of ``n_theta`` triangles
    around the axis, then ``cap_rings - 1`` annuli of ``2 * n_theta``).
    The defaults give 32,768 triangles."""
    R = 0.5 * diameter
    th = np.linspace(0.0, 2.0 * math.pi, n_theta + 1)[:-1]
    cs, sn = np.cos(th), np.sin(th)
    xs = np.linspace(-0.5 * length, 0.5 * length, n_ax + 1)
    tris = []
    for l in range(n_ax):
        for k in range(n_theta):
            k2 = (k + 1) % n_theta
            p00 = (xs[l], R * cs[k], R * sn[k])
            p01 = (xs[l], R * cs[k2], R * sn[k2])
            p10 = (xs[l + 1], R * cs[k], R * sn[k])
            p11 = (xs[l + 1], R * cs[k2], R * sn[k2])
            tris.append((p00, p11, p01))
            tris.append((p00, p10, p11))
    radii = np.linspace(0.0, R, cap_rings + 1)
    for x0 in (-0.5 * length, 0.5 * length):
        for q in range(cap_rings):
            r0, r1 = radii[q], radii[q + 1]
            for k in range(n_theta):
                k2 = (k + 1) % n_theta
                a1 = (x0, r1 * cs[k], r1 * sn[k])
                b1 = (x0, r1 * cs[k2], r1 * sn[k2])
                if q == 0:
                    tris.append(((x0, 0.0, 0.0), a1, b1))
                else:
                    a0 = (x0, r0 * cs[k], r0 * sn[k])
                    b0 = (x0, r0 * cs[k2], r0 * sn[k2])
                    tris.append((a0, a1, b1))
                    tris.append((a0, b1, b0))
    return np.asarray(tris, dtype=np.float64)


def drum(n=8_000_000, seed=7, dt=5e-6, skin=0.5e-3, diameter=0.5, length=0.85, n_theta=128, n_ax=121,
         cap_rings=4, omega=2.0, gap=0.05, margin=0.01, clearance=1.5e-3, vmax=0.0):
    """Rotating drum (Hertz/history): radius U(0.8, 1.2) mm, density 2700,
    E 1e7, nu 0.45, e 0.5, mu 0.4; drum of ``diameter`` x ``length`` turning
    at ``omega`` rad/s about the x axis (fix move/mesh rotate).  Particles
    are sorted by radius and stacked bottom-up in simple-cubic layers of
    spacing (2 + gap) x the largest radius of the layer, inside the drum with
    ``clearance`` to its wall, with uniform +-vmax velocities; ``margin``
    keeps the box clear of the mesh by more than the neighbour cutoff."""
    rng = np.random.default_rng(seed)
    rad = np.sort(rng.uniform(0.8e-3, 1.2e-3, size=n))[::-1].copy()
    R = 0.5 * diameter
    pos = np.zeros((n, 3))
    placed = 0
    z = -R + clearance
    xlim = 0.5 * length - clearance
    while placed < n:
        rmax = rad[placed]
        s = (2.0 + gap) * rmax
        zc = z + rmax
        if zc + rmax > R - clearance:
            raise ValueError("drum too small for %d particles" % n)
        half = math.sqrt(max((R - clearance - rmax) ** 2 - zc ** 2, 0.0))
        ny = int(half // s)
        nx = int((xlim - rmax) // s)
        if ny < 0 or nx < 0:
            z += s
            continue
        gy = np.arange(-ny, ny + 1) * s
        gx = np.arange(-nx, nx + 1) * s
        gxx, gyy = np.meshgrid(gx, gy, indexing="ij")
        pts = np.stack([gxx.ravel(), gyy.ravel()], axis=1)
        take = min(len(pts), n - placed)
        sl = slice(placed, placed + take)
        pos[sl, 0] = pts[:take, 0]
        pos[sl, 1] = pts[:take, 1]
        pos[sl, 2] = zc
        placed += take
        z = zc + rmax + gap * rmax
    nodes = drum_mesh(diameter, length, n_theta, n_ax, cap_rings)
    lo = [-0.5 * length - margin, -R - margin, -R - margin]
    hi = [0.5 * length + margin, R + margin, R + margin]
    sc = {
        "name": "drum",
        "dt": dt, "skin": skin,
        "boxlo": lo, "boxhi": hi, "periodic": [0, 0, 0],
        "every": 1, "delay": 0, "check": 1, "sortfreq": 1000, "sortbinsize": 0.0,
        "rolling_cdt": 0, "tangential_damping": 1,
        "atoms": _atoms(pos, rad, 2700.0, rng.uniform(-vmax, vmax, size=(n, 3)) if vmax > 0 else np.zeros((n, 3))),
        "fixes": [
            {"kind": "gravity", "magnitude": 9.81, "vector": [0.0, 0.0, -1.0]},
            {"kind": "wall_mesh", "nodes": nodes, "wall_type": 1, "curvature": 0.0, "rolling_cdt": 0},
            {"kind": "move_mesh_rotate", "mesh": 1, "origin": [0.0, 0.0, 0.0], "axis": [1.0, 0.0, 0.0],
             "period": 2.0 * math.pi / omega},
            {"kind": "nve_sphere"},
        ],
    }
    sc.update(_materials(1, 1e7, 0.45, 0.5, 0.4))
    return sc


def _hex_rect(a, x0, x1, y0, y1):
    """Sites of a triangular lattice of spacing a (rows along x) inside the
    rectangle [x0, x1] x [y0, y1], ordered by x then y."""
    h = 0.5 * math.sqrt(3.0) * a
    j = np.arange(int(math.ceil(y0 / h)) - 1, int(math.floor(y1 / h)) + 2)
    y = j * h
    j = j[(y >= y0) & (y <= y1)]
    off = 0.5 * a * (j % 2)
    lo = np.ceil((x0 - off) / a).astype(np.int64)
    hi = np.floor((x1 - off) / a).astype(np.int64)
    cnt = np.maximum(hi - lo + 1, 0)
    total = int(cnt.sum())
    if total == 0:
        return np.zeros(0), np.zeros(0)
    start = np.repeat(np.cumsum(cnt) - cnt, cnt)
    i = np.repeat(lo, cnt) + (np.arange(total) - start)
    x = i * a + np.repeat(off, cnt)
    yy = np.repeat(j, cnt) * h
    order = np.lexsort((yy, x))
    return x[order], yy[order]


def drum_config3(n=8_000_000, seed=7, dt=5e-6, skin=0.5e-3, diameter=0.5, length=0.85, n_theta=128, n_ax=121,
                 cap_rings=4, omega=2.0, margin=0.01, clearance=1.5e-3, overlap=1e-4, band=2e-3,
                 wall_overlap=2e-3, sortfreq=1000):
    """Rotating drum of configuration 3, packed at the start of the run.

    Radii U(0.8, 1.2) mm sorted largest first, density 2700, E 1e7, nu 0.45,
    e 0.5, mu 0.4; drum ``diameter`` x ``length`` (0.85 m gives the 35 %% fill
    for 8M spheres) of 32,768 triangles turning at ``omega`` rad/s about x.
    Horizontal layers from the bottom of the drum, each filled along x with
    patches of a triangular lattice holding one narrow radius band (spacing
    (1 - overlap) x the smallest diameter of the patch, patches one diameter
    apart), so neighbours inside a patch touch; in every other lattice row
    the outermost particle of each column is pushed sideways onto the plane
    of the drum facet at that height (overlap ``wall_overlap`` of its
    radius), giving wall contacts all along the drum.  Layers where the wall
    is closer to horizontal than vertical (more than 60 degrees from the
    drum's horizontal diameter) are not pushed."""
    rng = np.random.default_rng(seed)
    rad = np.sort(rng.uniform(0.8e-3, 1.2e-3, size=n))[::-1].copy()
    neg_rad = -rad   # ascending, for the band searches
    R = 0.5 * diameter
    pos = np.zeros((n, 3))
    placed = 0
    z = -R + clearance
    xlo, xhi = -0.5 * length + clearance, 0.5 * length - clearance
    dth = 2.0 * math.pi / n_theta
    chunk = max(200, n // 4000)
    while placed < n:
        rmax = rad[placed]
        zc = z + rmax
        if zc + rmax > R - clearance:
            raise ValueError("drum too small for %d particles" % n)
        half = math.sqrt(max((R - clearance - rmax) ** 2 - zc ** 2, 0.0)) - 2.1 * rmax
        if half <= rmax:
            z += 2.0 * rmax
            continue
        x_in = xlo + rmax
        patches = []
        while placed < n and x_in < xhi - rmax:
            r0 = rad[placed]
            jb = int(np.searchsorted(neg_rad, -r0 / (1.0 + band), side="right"))
            want = max(1, min(n - placed, jb - placed, chunk))
            # a window along x long enough for `want` sites (the lattice holds
            # 2 half / (a h) sites per unit length), not the rest of the layer
            xw = min(xhi - r0, x_in + 1.5 * want * (2.0 * r0) ** 2 * 0.87 / (2.0 * half) + 8.0 * r0)
            x, y = _hex_rect(2.0 * r0, x_in, xw, -half, half)
            if len(x) < want and xw < xhi - r0:
                xw = xhi - r0
                x, y = _hex_rect(2.0 * r0, x_in, xw, -half, half)
            if len(x) == 0:
                break
            take = max(1, min(len(x), want))
            a = 2.0 * rad[placed + take - 1] * (1.0 - overlap)
            x, y = _hex_rect(a, x_in, xw, -half, half)
            take = min(take, len(x))
            if take == 0:
                break
            x, y = x[:take], y[:take]
            sl = slice(placed, placed + take)
            pos[sl, 0], pos[sl, 1], pos[sl, 2] = x, y, zc
            patches.append((placed, take, a))
            placed += take
            x_in = x.max() + 2.0 * r0 + 1e-7
        # in even lattice rows (columns one spacing apart) the outermost
        # particle of every column, at both ends in y, onto the side wall
        for p0, take, ap in patches:
            idx = np.arange(p0, p0 + take)
            row = np.rint(pos[idx, 1] / (0.5 * math.sqrt(3.0) * ap)).astype(np.int64)
            idx = idx[row % 2 == 0]
            if len(idx) == 0:
                continue
            xs = np.round(pos[idx, 0], 12)
            yw = math.sqrt(max(R * R - zc * zc, 0.0))   # the drum wall at this height: y = +-yw
            if yw < 0.5 * R:   # the wall is closer to horizontal than vertical here: no sideways push
                continue
            for side in (-1.0, 1.0):
                ys = side * pos[idx, 1]
                order = np.lexsort((-ys, xs))
                first = np.ones(len(order), dtype=bool)
                first[1:] = xs[order][1:] != xs[order][:-1]
                th = math.atan2(zc, side * yw) % (2.0 * math.pi)
                k = int(th / dth) % n_theta
                # facet plane through the drum nodes at angles k, k+1 (a chord)
                c1, s1 = math.cos(k * dth), math.sin(k * dth)
                c2, s2 = math.cos((k + 1) * dth), math.sin((k + 1) * dth)
                ny, nz = -(c1 + c2), -(s1 + s2)
                nn = math.hypot(ny, nz)
                ny, nz = ny / nn, nz / nn                  # inward unit normal in (y, z)
                if ny == 0.0:
                    continue
                d0 = (R * c1) * ny + (R * s1) * nz         # plane: (y, z).n = d0
                sel = idx[order[first]]
                dist = pos[sel, 1] * ny + zc * nz - d0       # distance inside the plane
                dy = (rad[sel] * (1.0 - wall_overlap) - dist) / ny
                mv = side * dy > 0
                pos[sel[mv], 1] += dy[mv]
        z = zc + rmax + 1e-7
    nodes = drum_mesh(diameter, length, n_theta, n_ax, cap_rings)
    lo = [-0.5 * length - margin, -R - margin, -R - margin]
    hi = [0.5 * length + margin, R + margin, R + margin]
    sc = {
        "name": "drum_config3",
        "dt": dt, "skin": skin,
        "boxlo": lo, "boxhi": hi, "periodic": [0, 0, 0],
        "every": 1, "delay": 0, "check": 1, "sortfreq": sortfreq, "sortbinsize": 0.0,
        "rolling_cdt": 0, "tangential_damping": 1,
        "atoms": _atoms(pos, rad, 2700.0, np.zeros((n, 3))),
        "fixes": [
            {"kind": "gravity", "magnitude": 9.81, "vector": [0.0, 0.0, -1.0]},
            {"kind": "wall_mesh", "nodes": nodes, "wall_type": 1, "curvature": 0.0, "rolling_cdt": 0},
            {"kind": "move_mesh_rotate", "mesh": 1, "origin": [0.0, 0.0, 0.0], "axis": [1.0, 0.0, 0.0],
             "period": 2.0 * math.pi / omega},
            {"kind": "nve_sphere"},
        ],
    }
    sc.update(_materials(1, 1e7, 0.45, 0.5, 0.4))
    return sc


def bumpy_plate_mesh(lx=0.2, ly=0.2, nx=128, ny=256, z0=1.5e-3, amp=1.0e-3, waves=(8, 8)):
    """Procedural bumpy plate over [0, lx] x [0, ly]: z = z0 + amp sin(2 pi kx x / lx)
    sin(2 pi ky y / ly) on an nx x ny grid, two triangles per cell
    (2 nx ny triangles; the defaults give 65,536)."""
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    Z = z0 + amp * np.sin(2.0 * math.pi * waves[0] * X / lx) * np.sin(2.0 * math.pi * waves[1] * Y / ly)
    P = np.stack([X, Y, Z], axis=-1)
    p00, p10, p01, p11 = P[:-1, :-1], P[1:, :-1], P[:-1, 1:], P[1:, 1:]
    t1 = np.stack([p00, p10, p11], axis=2).reshape(-1, 3, 3)
    t2 = np.stack([p00, p11, p01], axis=2).reshape(-1, 3, 3)
    return np.ascontiguousarray(np.stack([t1, t2], axis=1).reshape(-1, 3, 3))


def bed_config5(n=20_000_000, seed=5, dt=2e-6, skin=0.5e-3, r=0.5e-3, box=(0.2, 0.2, 0.5), overlap=1e-4,
                plate_nx=128, plate_ny=256, plate_z0=1.5e-3, plate_amp=1.0e-3, plate_waves=(8, 8), sortfreq=1000):
    """Large settled bed of configuration 5: n spheres of radius r (density
    2500, E 5e6, nu 0.45, e 0.3, mu 0.5) in a box walled by planes on all
    sides but the top, with a procedural bumpy-plate mesh of 65,536 triangles
    over the floor.  The spheres stand in hexagonal close packing (ABAB
    stacking, every neighbour at (1 - overlap) x the diameter, so each sphere
    touches its 12 neighbours), the lowest layer resting on the plate's
    crests, the sides against the walls."""
    a = 2.0 * r * (1.0 - overlap)
    cz = math.sqrt(2.0 / 3.0) * a
    lx, ly, lz = box
    m = r * (1.0 - overlap)
    xa, ya = _hex_rect(a, m, lx - m, m, ly - m)
    # the lowest layer rests on the plate's crests (overlap up to 2 % of r right above a crest node)
    z0 = plate_z0 + plate_amp + r * (1.0 - 2e-2)
    pos = np.zeros((n, 3))
    placed = 0
    layer = 0
    while placed < n:
        sx = 0.5 * a if layer % 2 else 0.0
        sy = a / (2.0 * math.sqrt(3.0)) if layer % 2 else 0.0
        x, y = xa + sx, ya + sy
        keep = (x <= lx - m) & (y <= ly - m)
        x, y = x[keep], y[keep]
        take = min(len(x), n - placed)
        zl = z0 + layer * cz
        if zl + r > lz:
            raise ValueError("box too small for %d spheres" % n)
        pos[placed:placed + take, 0] = x[:take]
        pos[placed:placed + take, 1] = y[:take]
        pos[placed:placed + take, 2] = zl
        placed += take
        layer += 1
    del seed   # the packing is fully determined; kept for the workload interface
    nodes = bumpy_plate_mesh(lx, ly, plate_nx, plate_ny, plate_z0, plate_amp, plate_waves)
    sc = {
        "name": "bed_config5",
        "dt": dt, "skin": skin,
        "boxlo": [-0.005, -0.005, -0.005], "boxhi": [lx + 0.005, ly + 0.005, lz], "periodic": [0, 0, 0],
        "every": 1, "delay": 0, "check": 1, "sortfreq": sortfreq, "sortbinsize": 0.0,
        "rolling_cdt": 0, "tangential_damping": 1,
        "atoms": _atoms(pos, np.full(n, r), 2500.0, np.zeros((n, 3))),
        "fixes": [
            {"kind": "gravity", "magnitude": 9.81, "vector": [0.0, 0.0, -1.0]},
            {"kind": "wall_mesh", "nodes": nodes, "wall_type": 1, "curvature": 0.0, "rolling_cdt": 0},
            {"kind": "wall_plane", "dim": 2, "pos": 0.0, "wall_type": 1},
            {"kind": "wall_plane", "dim": 0, "pos": 0.0, "wall_type": 1},
            {"kind": "wall_plane", "dim": 0, "pos": lx, "wall_type": 1},
            {"kind": "wall_plane", "dim": 1, "pos": 0.0, "wall_type": 1},
            {"kind": "wall_plane", "dim": 1, "pos": ly, "wall_type": 1},
            {"kind": "nve_sphere"},
        ],
    }
    sc.update(_materials(1, 5e6, 0.45, 0.3, 0.5))
    return sc


def sq_volume(shape, n):
    """Volume of a superquadric with n1 = n2 = n (Jaklic et al.,
    Segmentation and Recovery of Superquadrics, eq. 2.60; the reference's
    volume_superquadric)."""
    from scipy.special import beta
    e = 2.0 / np.asarray(n, dtype=np.float64)
    a, b, c = (np.asarray(shape)[..., k] for k in range(3))
    return 2.0 * a * b * c * e * e * beta(0.5 * e, e + 1.0) * beta(0.5 * e, 0.5 * e + 1.0)


def sq_inertia(shape, n, density):
    """Principal moments of inertia of a superquadric, n1 = n2 = n (the
    same published formulas as the reference's inertia_superquadric)."""
    from scipy.special import beta
    e = 2.0 / np.asarray(n, dtype=np.float64)
    a1, a2, a3 = (np.asarray(shape)[..., k] for k in range(3))
    pre = 0.5 * a1 * a2 * a3 * e * e * density
    t1 = beta(1.5 * e, 0.5 * e) * beta(0.5 * e, 2.0 * e + 1.0)
    t2 = 4.0 * beta(0.5 * e, 0.5 * e + 1.0) * beta(1.5 * e, e + 1.0)
    ixx = pre * (a2 * a2 * t1 + a3 * a3 * t2)
    iyy = pre * (a1 * a1 * t1 + a3 * a3 * t2)
    izz = pre * (a1 * a1 + a2 * a2) * t1
    return np.stack([ixx, iyy, izz], axis=-1)


def random_quaternions(rng, n):
    """Uniformly distributed unit quaternions (w, x, y, z) (Shoemake)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * math.pi * u2), np.sqrt(1 - u1) * np.cos(2 * math.pi * u2),
                  np.sqrt(u1) * np.sin(2 * math.pi * u3), np.sqrt(u1) * np.cos(2 * math.pi * u3)], axis=1)
    return q[:, [3, 0, 1, 2]].copy()


def sq_bounding_radius(shape, blk):
    """Bounding-sphere radius of superquadrics with n1 = n2 = blk (the closed
    form of Superquadric's bounding sphere, src/superquadric.cpp, with its
    1.0001 margin), vectorised over particles."""
    shape = np.asarray(shape, dtype=np.float64)
    blk = np.asarray(blk, dtype=np.float64)
    a = np.maximum(shape[:, 0], shape[:, 1])
    b = np.minimum(shape[:, 0], shape[:, 1])
    c = shape[:, 2]
    n = np.maximum(2.1, blk)
    with np.errstate(divide="ignore", invalid="ignore"):
        alpha = np.power(b / a, 2.0 / (n - 2.0))
        gamma = np.power(1.0 + np.power(alpha, n), 0.0)
        beta = np.power(c * c / (a * a) * gamma, 1.0 / (n - 2.0))
        x0 = 1.0 / np.power(1.0 + np.power(alpha, n) + np.power(beta, n), 1.0 / n)
    r = np.sqrt((x0 * a) ** 2 + (alpha * x0 * b) ** 2 + (beta * x0 * c) ** 2) * 1.0001
    ellipsoid = np.abs(blk - 2.0) < 1e-13
    return np.where(ellipsoid, shape.max(axis=1) * 1.0001, r)


def sq_packing(n=200_000, seed=11, dt=1e-5, skin=0.5e-3, vin=1.0, density=2500.0, fill=0.8):
    """Superquadric packing: half-axes U(1, 2) mm, blockiness U(2, 8) (one
    exponent per particle, n1 = n2), uniformly random orientations, Hertz
    contact with config-1 materials (E 5e6, nu 0.45, e 0.3, mu 0.5), on a
    cubic lattice of spacing ``fill`` x the largest bounding diameter, with
    uniform random velocities of +-``vin`` so contacts form and break."""
    rng = np.random.default_rng(seed)
    shape = rng.uniform(1e-3, 2e-3, size=(n, 3))
    blk = rng.uniform(2.0, 8.0, size=n)
    quat = random_quaternions(rng, n)
    if n <= 20000:
        rb = sq_bounding_radius(shape, blk)
    else:   # large packings: the corner of the box bounds every blockiness
        rb = np.linalg.norm(shape, axis=1) * 1.0001
    s = fill * 2.0 * rb.max()
    m = int(math.ceil(n ** (1.0 / 3.0)))
    idx = np.arange(n)
    pos = np.stack([idx % m, (idx // m) % m, idx // (m * m)], axis=1).astype(np.float64) * s
    pos -= pos.mean(axis=0)
    vel = rng.uniform(-vin, vin, size=(n, 3))
    vol = sq_volume(shape, blk)
    atoms = {"x": pos, "v": vel, "quat": quat, "angmom": np.zeros((n, 3)), "shape": shape, "blockiness": blk,
             "rmass": vol * density, "inertia": sq_inertia(shape, blk, density), "volume": vol}
    return {"name": "sq_packing", "dt": dt, "skin": skin, "atoms": atoms,
            "youngs": 5e6, "poisson": 0.45, "restitution": 0.3, "friction": 0.5}


def subset(sc, n):
    """First ``n`` atoms of a scenario (same box, fixes and materials)."""
    out = dict(sc)
    out["atoms"] = {k: np.ascontiguousarray(v[:n]) for k, v in sc["atoms"].items()}
    return out


def stream_pour(n_bed=400, seed=78, periodic=True, nparticles=300, particlerate=20000.0, insert_every=200,
                vel=(0.0, 0.0, -2.0), vel_style="uniform", exact_number=1, max_atoms=2000):
    """fix insert/stream above a bed: the 20 x 20 x 60 mm box of insert_pour
    (x/y periodic or walled, n_bed spheres of r = 1 mm at the bottom, dt
    1e-5), an insertion face of two triangles spanning x, y in 2-18 mm at
    z = 40 mm, the same two templates (r = 1.2 and 0.8 mm, mass fractions
    0.5 / 0.5), particles inserted every insert_every steps at particlerate
    per second up to nparticles, moving down at the insertion velocity's
    normal part until they cross the face, released there with the
    insertion velocity (+- 0.1 m/s per component for vel uniform)."""
    sc = sphere_pour(n=n_bed, seed=seed, box=(0.02, 0.02, 0.06), spacing=(2.5e-3, 2.5e-3, 2.4e-3), vmax=0.05)
    sc["name"] = "stream_pour"
    sc["periodic"] = [1, 1, 0] if periodic else [0, 0, 0]
    fixes = [sc["fixes"][0], sc["fixes"][1]]
    if not periodic:
        for dim in (0, 1):
            fixes.append({"kind": "wall_plane", "dim": dim, "pos": 0.0, "wall_type": 1, "rolling_cdt": 0})
            fixes.append({"kind": "wall_plane", "dim": dim, "pos": 0.02, "wall_type": 1, "rolling_cdt": 0})
    z = 0.04
    face = np.array([[0.002, 0.002, z, 0.018, 0.002, z, 0.018, 0.018, z],
                     [0.002, 0.002, z, 0.018, 0.018, z, 0.002, 0.018, z]])
    fx = {
        "kind": "insert_stream", "seed": 32452867, "dist_seed": 15485867, "face_nodes": face,
        "nparticles": nparticles, "particlerate": particlerate, "insert_every": insert_every,
        "exact_number": exact_number, "vel_style": vel_style, "vel": list(vel), "vel_fluct": [0.1, 0.1, 0.1],
        "templates": [{"type": 1, "radius": 1.2e-3, "density": 2500.0, "weight": 0.5, "seed": 67867979},
                      {"type": 1, "radius": 0.8e-3, "density": 2500.0, "weight": 0.5, "seed": 86028157}],
        "max_atoms": max_atoms,
    }
    fixes += [fx, {"kind": "nve_sphere"}]
    sc["fixes"] = fixes
    return sc


def insert_pour(n_bed=400, seed=77, periodic=True, dt=2e-6, vel_style="uniform", all_in=0, exact_number=1,
                target=("volumefraction_region", 0.25), insert_every=300, max_atoms=8000, polydisperse=False,
                cylinder=False):
    """fix insert/pack above a settled-looking bed: a 20 x 20 x 60 mm box (x/y
    periodic or walled), n_bed spheres of r = 1 mm at the bottom, and a region
    block 2-18 x 2-18 x 30-55 mm refilled every insert_every steps from two
    templates (r = 1.2 mm and 0.8 mm, 2500 kg/m^3, mass fractions 0.5 / 0.5)
    falling at -0.5 m/s (+- 0.1 m/s per component for vel uniform).
    polydisperse: radius uniform in 1.0-1.3 mm and gaussian 0.8 +- 0.05 mm
    instead of the two constants.  cylinder: a region cylinder z (axis at
    x = y = 10 mm, radius 8 mm, z 30-55 mm) instead of the block."""
    sc = sphere_pour(n=n_bed, seed=seed, dt=dt, box=(0.02, 0.02, 0.06), spacing=(2.5e-3, 2.5e-3, 2.4e-3), vmax=0.05)
    sc["name"] = "insert_pour"
    sc["periodic"] = [1, 1, 0] if periodic else [0, 0, 0]
    fixes = [sc["fixes"][0], sc["fixes"][1]]
    if not periodic:
        for dim in (0, 1):
            fixes.append({"kind": "wall_plane", "dim": dim, "pos": 0.0, "wall_type": 1, "rolling_cdt": 0})
            fixes.append({"kind": "wall_plane", "dim": dim, "pos": 0.02, "wall_type": 1, "rolling_cdt": 0})
    fx = {
        "kind": "insert_pack", "seed": 32452843, "dist_seed": 15485863,
        "region_lo": [0.002, 0.002, 0.03], "region_hi": [0.018, 0.018, 0.055],
        target[0]: target[1], "insert_every": insert_every, "all_in": all_in, "exact_number": exact_number,
        "vel_style": vel_style, "vel": [0.0, 0.0, -0.5], "vel_fluct": [0.1, 0.1, 0.1],
        "templates": [{"type": 1, "radius": 1.2e-3, "density": 2500.0, "weight": 0.5, "seed": 67867967},
                      {"type": 1, "radius": 0.8e-3, "density": 2500.0, "weight": 0.5, "seed": 67867979}],
        "max_atoms": max_atoms,
    }
    if cylinder:
        del fx["region_lo"], fx["region_hi"]
        fx["region_cylinder"] = {"axis": 2, "c1": 0.01, "c2": 0.01, "radius": 0.008, "lo": 0.03, "hi": 0.055}
    if polydisperse:
        fx["templates"][0].update(radius=1.0e-3, radius_style="uniform", radius2=1.3e-3, seed=86028121)
        fx["templates"][1].update(radius_style="gaussian", radius2=0.05e-3, seed=49979687)
    fixes += [fx, {"kind": "nve_sphere"}]
    sc["fixes"] = fixes
    return sc
