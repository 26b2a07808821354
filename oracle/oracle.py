"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this
module, and only as the checker.  The oracle restates the reference algorithm
(LIGGGHTS-PUBLIC 3.8.0); see gran_oracle.h for its parity status.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

D = ctypes.POINTER(ctypes.c_double)
I = ctypes.POINTER(ctypes.c_int)
U8 = ctypes.POINTER(ctypes.c_ubyte)


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("ntypes", ctypes.c_int),
        ("dt", ctypes.c_double),
        ("skin", ctypes.c_double),
        ("boxlo", ctypes.c_double * 3),
        ("boxhi", ctypes.c_double * 3),
        ("periodic", ctypes.c_int * 3),
        ("every", ctypes.c_int),
        ("delay", ctypes.c_int),
        ("check", ctypes.c_int),
        ("sortfreq", ctypes.c_int),
        ("sortbinsize", ctypes.c_double),
        ("rolling_cdt", ctypes.c_int),
        ("tangential_damping", ctypes.c_int),
        ("youngs", D),
        ("poisson", D),
        ("restitution", D),
        ("friction", D),
        ("rollfriction", D),
    ]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int, D, D, D, D, D, I, I]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_add_gravity.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 4
        L.orc_add_wall_plane.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.orc_add_wall_mesh.argtypes = [ctypes.c_void_p, ctypes.c_int, D, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_setup.argtypes = [ctypes.c_void_p]
        L.orc_run.argtypes = [ctypes.c_void_p, ctypes.c_int]
        for fn in ("orc_nlocal", "orc_nghost", "orc_nbuilds"):
            getattr(L, fn).argtypes = [ctypes.c_void_p]
        L.orc_ntimestep.restype = ctypes.c_long
        L.orc_ntimestep.argtypes = [ctypes.c_void_p]
        L.orc_get_atoms.argtypes = [ctypes.c_void_p, D, D, D, D, D, I]
        L.orc_get_pairs.argtypes = [ctypes.c_void_p, ctypes.c_int, I, I, I, D]
        L.orc_get_wall_hist.argtypes = [ctypes.c_void_p, ctypes.c_int, D]
        L.orc_get_mesh_contacts.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, I, I, D]
        L.orc_get_mesh_topology.argtypes = [ctypes.c_void_p, ctypes.c_int, U8, U8, I]
        L.orc_get_mesh_nneighs.argtypes = [ctypes.c_void_p, ctypes.c_int, I]
        L.orc_add_move_mesh_rotate.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 7
        L.orc_get_mesh_nodes.argtypes = [ctypes.c_void_p, ctypes.c_int, D, D]
        L.orc_get_mesh_geom.argtypes = [ctypes.c_void_p, ctypes.c_int, D]
        L.orc_add_move_mesh_linear.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 3
        L.orc_contact_atom.argtypes = [ctypes.c_void_p, D]
        L.orc_upload_history.argtypes = [ctypes.c_void_p, ctypes.c_int, I, I, D]
        L.orc_add_mesh_stress.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 3
        L.orc_get_mesh_stress.argtypes = [ctypes.c_void_p, ctypes.c_int, D, D]
        L.orc_get_mesh_sigma.argtypes = [ctypes.c_void_p, ctypes.c_int, D, D]
        L.orc_get_mesh_history.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, I, I, D]
        L.orc_upload_mesh_hist.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, I, I, D]
        L.orc_add_mesh_wear.argtypes = [ctypes.c_void_p, ctypes.c_int, D]
        L.orc_get_mesh_wear.argtypes = [ctypes.c_void_p, ctypes.c_int, D]
        L.orc_get_radius_mass.argtypes = [ctypes.c_void_p, D, D]
        L.orc_park_after.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_add_insert_pack.argtypes = [ctypes.c_void_p, ctypes.POINTER(OrcInsertPack)]
        L.orc_insert_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long), D,
                                       ctypes.POINTER(ctypes.c_long)]
        L.orc_pair_gran_local.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_int, D]
        L.orc_get_history.argtypes = [ctypes.c_void_p, I, I, D]
        L.orc_upload_wall_hist.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, D]
        L.orc_add_wall_cylinder.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 3 + [ctypes.c_int] * 2
        L.orc_error.restype = ctypes.c_char_p
        L.orc_error.argtypes = [ctypes.c_void_p]
        L.orc_pair_force.argtypes = [ctypes.POINTER(OrcParams), D, D, D, D, D, D, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, D, ctypes.c_int,
                                     D, D, D, D]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(D)


def _ip(a):
    return a.ctypes.data_as(I)


class OrcInsertPack(ctypes.Structure):
    """orc_insert_pack (fix insert/pack with its distribution and templates)."""
    _fields_ = [("seed", ctypes.c_int), ("region_lo", ctypes.c_double * 3), ("region_hi", ctypes.c_double * 3),
                ("volumefraction_region", ctypes.c_double), ("particles_in_region", ctypes.c_int),
                ("mass_in_region", ctypes.c_double), ("insert_every", ctypes.c_int), ("start", ctypes.c_int),
                ("maxattempt", ctypes.c_int), ("overlapcheck", ctypes.c_int), ("all_in", ctypes.c_int),
                ("exact_number", ctypes.c_int), ("vel_style", ctypes.c_int), ("vel", ctypes.c_double * 3),
                ("vel_fluct", ctypes.c_double * 3), ("omega", ctypes.c_double * 3), ("ntry_mc", ctypes.c_int),
                ("check_dist_from_subdomain_border", ctypes.c_int), ("dist_seed", ctypes.c_int),
                ("dist_mass_based", ctypes.c_int), ("ntemplates", ctypes.c_int), ("tmpl_type", ctypes.c_int * 8),
                ("tmpl_radius", ctypes.c_double * 8), ("tmpl_density", ctypes.c_double * 8),
                ("tmpl_weight", ctypes.c_double * 8), ("max_atoms", ctypes.c_int),
                ("tmpl_radius_style", ctypes.c_int * 8), ("tmpl_radius2", ctypes.c_double * 8),
                ("tmpl_seed", ctypes.c_int * 8), ("region_style", ctypes.c_int), ("cyl_axis", ctypes.c_int),
                ("cyl_c1", ctypes.c_double), ("cyl_c2", ctypes.c_double), ("cyl_radius", ctypes.c_double),
                ("cyl_lo", ctypes.c_double), ("cyl_hi", ctypes.c_double)]


def make_insert(fx):
    """OrcInsertPack from a scenario fix dict (kind "insert_pack"), keyword defaults as the reference's."""
    p = OrcInsertPack()
    p.seed = int(fx["seed"])
    cyl = fx.get("region_cylinder")
    if cyl is not None:
        p.region_style, p.cyl_axis = 1, int(cyl["axis"])
        p.cyl_c1, p.cyl_c2, p.cyl_radius = float(cyl["c1"]), float(cyl["c2"]), float(cyl["radius"])
        p.cyl_lo, p.cyl_hi = float(cyl["lo"]), float(cyl["hi"])
    for d in range(3):
        p.region_lo[d] = fx.get("region_lo", (0.0, 0.0, 0.0))[d]
        p.region_hi[d] = fx.get("region_hi", (0.0, 0.0, 0.0))[d]
        p.vel[d] = fx.get("vel", (0.0, 0.0, 0.0))[d]
        p.vel_fluct[d] = fx.get("vel_fluct", (0.0, 0.0, 0.0))[d]
        p.omega[d] = fx.get("omega", (0.0, 0.0, 0.0))[d]
    p.volumefraction_region = float(fx.get("volumefraction_region", 0.0))
    p.particles_in_region = int(fx.get("particles_in_region", 0))
    p.mass_in_region = float(fx.get("mass_in_region", 0.0))
    p.insert_every = int(fx["insert_every"])
    p.start = int(fx.get("start", 0))
    p.maxattempt = int(fx.get("maxattempt", 50))
    p.overlapcheck = int(fx.get("overlapcheck", 1))
    p.all_in = int(fx.get("all_in", 0))
    p.exact_number = int(fx.get("exact_number", 1))
    p.vel_style = {"constant": 0, "uniform": 1, "gaussian": 2}[fx.get("vel_style", "constant")]
    p.ntry_mc = int(fx.get("ntry_mc", 100000))
    p.check_dist_from_subdomain_border = int(fx.get("check_dist_from_subdomain_border", 1))
    p.dist_seed = int(fx["dist_seed"])
    p.dist_mass_based = int(fx.get("dist_mass_based", 1))
    p.ntemplates = len(fx["templates"])
    for i, t in enumerate(fx["templates"]):
        p.tmpl_type[i], p.tmpl_radius[i] = int(t["type"]), float(t["radius"])
        p.tmpl_density[i], p.tmpl_weight[i] = float(t["density"]), float(t["weight"])
        p.tmpl_radius_style[i] = {"constant": 0, "uniform": 1, "gaussian": 2}[t.get("radius_style", "constant")]
        p.tmpl_radius2[i] = float(t.get("radius2", 0.0))
        p.tmpl_seed[i] = int(t.get("seed", 67867967))
    p.max_atoms = int(fx.get("max_atoms", 0))
    return p


def make_params(sc):
    """OrcParams from a scenario dict (see the package's scenarios module)."""
    keep = []
    p = OrcParams()
    p.ntypes = sc["ntypes"]
    p.dt = sc["dt"]
    p.skin = sc["skin"]
    for d in range(3):
        p.boxlo[d] = sc["boxlo"][d]
        p.boxhi[d] = sc["boxhi"][d]
        p.periodic[d] = int(sc["periodic"][d])
    p.every, p.delay, p.check = sc.get("every", 1), sc.get("delay", 0), sc.get("check", 1)
    p.sortfreq = sc.get("sortfreq", 1000)
    p.sortbinsize = sc.get("sortbinsize", 0.0)
    p.rolling_cdt = int(sc.get("rolling_cdt", 0))
    p.tangential_damping = int(sc.get("tangential_damping", 1))
    for name in ("youngs", "poisson", "restitution", "friction", "rollfriction"):
        arr = np.ascontiguousarray(np.asarray(sc[name], dtype=np.float64).ravel())
        keep.append(arr)
        setattr(p, name, _dp(arr))
    return p, keep


class Oracle:
    """One oracle simulation built from a scenario dict."""

    def __init__(self, sc):
        L = lib()
        self.L = L
        self.p, self._keep = make_params(sc)
        a = sc["atoms"]
        self._arrs = {k: np.ascontiguousarray(a[k], dtype=np.float64) for k in ("x", "v", "omega", "radius", "rmass")}
        self._type = np.ascontiguousarray(a["type"], dtype=np.int32)
        self._tag = np.ascontiguousarray(a["tag"], dtype=np.int32)
        n = len(self._tag)
        self.h = L.orc_create(ctypes.byref(self.p), n, _dp(self._arrs["x"]), _dp(self._arrs["v"]),
                              _dp(self._arrs["omega"]), _dp(self._arrs["radius"]), _dp(self._arrs["rmass"]),
                              _ip(self._type), _ip(self._tag))
        self.fix_ids = []
        for fx in sc["fixes"]:
            kind = fx["kind"]
            if kind == "gravity":
                d = fx["vector"]
                k = L.orc_add_gravity(self.h, fx["magnitude"], d[0], d[1], d[2])
            elif kind == "wall_plane":
                k = L.orc_add_wall_plane(self.h, fx["dim"], fx["pos"], fx["wall_type"], int(fx.get("rolling_cdt", 0)))
            elif kind == "wall_cylinder":
                k = L.orc_add_wall_cylinder(self.h, fx["dim"], fx["radius"], fx["c1"], fx["c2"], fx["wall_type"],
                                            int(fx.get("rolling_cdt", 0)))
            elif kind == "wall_mesh":
                nodes = np.ascontiguousarray(fx["nodes"], dtype=np.float64)
                self._keep.append(nodes)
                k = L.orc_add_wall_mesh(self.h, nodes.shape[0], _dp(nodes), fx["wall_type"],
                                        fx.get("curvature", 0.0), int(fx.get("rolling_cdt", 0)))
            elif kind == "move_mesh_rotate":
                o, a = fx["origin"], fx["axis"]
                k = L.orc_add_move_mesh_rotate(self.h, self.fix_ids[fx["mesh"]], o[0], o[1], o[2], a[0], a[1], a[2],
                                               float(fx["period"]))
                if k < 0:
                    raise ValueError("oracle: bad move_mesh_rotate")
            elif kind == "move_mesh_linear":
                v = fx["velocity"]
                k = L.orc_add_move_mesh_linear(self.h, self.fix_ids[fx["mesh"]], v[0], v[1], v[2])
                if k < 0:
                    raise ValueError("oracle: bad move_mesh_linear")
            elif kind == "nve_sphere":
                k = None   # the oracle always integrates with fix nve/sphere
            elif kind == "insert_pack":
                ip = make_insert(fx)
                self._keep.append(ip)
                if L.orc_add_insert_pack(self.h, ctypes.byref(ip)) != 0:
                    raise ValueError("oracle: " + L.orc_error(self.h).decode())
                k = 0
            else:
                raise ValueError(kind)
            self.fix_ids.append(k)

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError("oracle: " + self.L.orc_error(self.h).decode())

    def setup(self):
        self._check(self.L.orc_setup(self.h))

    def run(self, n):
        self._check(self.L.orc_run(self.h, n))

    @property
    def nlocal(self):
        return self.L.orc_nlocal(self.h)

    @property
    def nbuilds(self):
        return self.L.orc_nbuilds(self.h)

    def atoms(self):
        n = self.nlocal
        out = {k: np.zeros((n, 3)) for k in ("x", "v", "omega", "f", "torque")}
        tag = np.zeros(n, dtype=np.int32)
        self.L.orc_get_atoms(self.h, _dp(out["x"]), _dp(out["v"]), _dp(out["omega"]), _dp(out["f"]),
                             _dp(out["torque"]), _ip(tag))
        out["tag"] = tag
        return out

    def insert_stats(self):
        n, nxt, m = ctypes.c_long(), ctypes.c_long(), np.zeros(1)
        if self.L.orc_insert_stats(self.h, ctypes.byref(n), _dp(m), ctypes.byref(nxt)) != 0:
            raise ValueError("no fix insert/pack")
        return {"ninserted": n.value, "massinserted": float(m[0]), "next_step": nxt.value}

    def pair_gran_local(self, keys=0x4 | 0x8 | 0x40 | 0x200):
        """compute pair/gran/local: (nrows, ncols) for a keyword bit mask
        (bit b: pos, vel, id, force, force_normal, force_tangential, torque,
        torque_normal, torque_tangential, history, contactArea, delta,
        contactPoint); the default is id force torque history, 12 columns."""
        width = (6, 6, 3, 3, 3, 3, 3, 3, 3, 3, 1, 1, 3)
        nc = sum(w for b, w in enumerate(width) if keys & (1 << b))
        n = self.L.orc_pair_gran_local(self.h, keys, 0, None)
        rows = np.zeros((n, nc))
        self.L.orc_pair_gran_local(self.h, keys, n, _dp(rows))
        return rows

    def add_mesh_stress(self, ifix, p_ref):
        if self.L.orc_add_mesh_stress(self.h, self.fix_ids[ifix], *[float(v) for v in p_ref]) != 0:
            raise RuntimeError("orc_add_mesh_stress failed")

    def mesh_stress(self, ifix):
        """Per-element force of the last step and f_total / torque_total."""
        n = self.L.orc_get_mesh_stress(self.h, self.fix_ids[ifix], None, None)
        f = np.zeros((n, 3))
        tot = np.zeros(6)
        self.L.orc_get_mesh_stress(self.h, self.fix_ids[ifix], _dp(f), _dp(tot))
        sn, st = np.zeros(n), np.zeros(n)
        self.L.orc_get_mesh_sigma(self.h, self.fix_ids[ifix], _dp(sn), _dp(st))
        return {"tri_f": f, "sigma_n": sn, "sigma_t": st, "f_total": tot[:3], "torque_total": tot[3:]}

    def upload_history(self, npartner, partner_tag, hist):
        """FixContactHistory restart data for the atoms as added (before setup)."""
        a = [np.ascontiguousarray(npartner, dtype=np.int32), np.ascontiguousarray(partner_tag, dtype=np.int32),
             np.ascontiguousarray(hist, dtype=np.float64)]
        if self.L.orc_upload_history(self.h, len(a[0]), _ip(a[0]), _ip(a[1]), _dp(a[2])) != 0:
            raise RuntimeError("orc_upload_history failed")

    def upload_wall_hist(self, ifix, hist):
        h = np.ascontiguousarray(hist, dtype=np.float64)
        if self.L.orc_upload_wall_hist(self.h, self.fix_ids[ifix], len(h), _dp(h)) != 0:
            raise RuntimeError("orc_upload_wall_hist failed")

    def history(self):
        """Current contact history in the partner layout: tag, npartner, partner_tag, hist."""
        npart = np.zeros(self.nlocal, dtype=np.int32)
        tot = self.L.orc_get_history(self.h, _ip(npart), None, None)
        pt = np.zeros(tot, dtype=np.int32)
        ph = np.zeros((tot, 3))
        self.L.orc_get_history(self.h, _ip(npart), _ip(pt), _dp(ph))
        return {"tag": self.atoms()["tag"], "npartner": npart, "partner_tag": pt, "hist": ph}

    def contact_atom(self):
        """compute contact/atom (skin 0): {tag, contact} per owned atom."""
        out = np.zeros(self.nlocal)
        self.L.orc_contact_atom(self.h, _dp(out))
        return {"tag": self.atoms()["tag"], "contact": out}

    def pairs(self):
        n = self.L.orc_get_pairs(self.h, 0, None, None, None, None)
        ti = np.zeros(n, dtype=np.int32)
        tj = np.zeros(n, dtype=np.int32)
        fl = np.zeros(n, dtype=np.int32)
        hi = np.zeros((n, 3))
        self.L.orc_get_pairs(self.h, n, _ip(ti), _ip(tj), _ip(fl), _dp(hi))
        return {"tag_i": ti, "tag_j": tj, "flag": fl, "hist": hi}

    def wall_hist(self, ifix):
        n = self.nlocal
        h = np.zeros((n, 3))
        self.L.orc_get_wall_hist(self.h, self.fix_ids[ifix], _dp(h))
        return h

    def mesh_contacts(self, ifix):
        k = self.fix_ids[ifix]
        n = self.L.orc_get_mesh_contacts(self.h, k, 0, None, None, None)
        tag = np.zeros(n, dtype=np.int32)
        tri = np.zeros(n, dtype=np.int32)
        h = np.zeros((n, 3))
        self.L.orc_get_mesh_contacts(self.h, k, n, _ip(tag), _ip(tri), _dp(h))
        return {"tag": tag, "tri": tri, "hist": h}

    def add_mesh_wear(self, ifix, k_finnie):
        kf = np.ascontiguousarray(k_finnie, dtype=np.float64).reshape(-1)
        self._keep.append(kf)
        if self.L.orc_add_mesh_wear(self.h, self.fix_ids[ifix], _dp(kf)) != 0:
            raise ValueError("orc_add_mesh_wear failed")

    def mesh_wear(self, ifix, ntri):
        w = np.zeros(ntri)
        if self.L.orc_get_mesh_wear(self.h, self.fix_ids[ifix], _dp(w)) != 0:
            raise ValueError("no wear on this mesh")
        return w

    def radius_mass(self):
        """Radius and mass of the owned atoms (current order)."""
        r, m = np.zeros(self.nlocal), np.zeros(self.nlocal)
        self.L.orc_get_radius_mass(self.h, _dp(r), _dp(m))
        return r, m

    def mesh_history(self, ifix):
        """Mesh contact history in the restart layout: {tag, npartner, tri, hist}."""
        k = self.fix_ids[ifix]
        tot = self.L.orc_get_mesh_history(self.h, k, 0, None, None, None)
        npart = np.zeros(self.nlocal, dtype=np.int32)
        tri = np.zeros(tot, dtype=np.int32)
        h = np.zeros((tot, 3))
        self.L.orc_get_mesh_history(self.h, k, tot, _ip(npart), _ip(tri), _dp(h))
        return {"tag": self.atoms()["tag"], "npartner": npart, "tri": tri, "hist": h}

    def upload_mesh_hist(self, ifix, npartner, tri, hist):
        npart = np.ascontiguousarray(npartner, dtype=np.int32)
        t = np.ascontiguousarray(tri, dtype=np.int32)
        h = np.ascontiguousarray(hist, dtype=np.float64).reshape(-1)
        self._keep += [npart, t, h]
        if self.L.orc_upload_mesh_hist(self.h, self.fix_ids[ifix], len(npart), _ip(npart), _ip(t), _dp(h)) != 0:
            raise ValueError("orc_upload_mesh_hist failed")

    def mesh_nodes(self, ifix):
        n = self.L.orc_get_mesh_nodes(self.h, self.fix_ids[ifix], None, None)
        nodes = np.zeros((n, 3, 3))
        vel = np.zeros((n, 3, 3))
        self.L.orc_get_mesh_nodes(self.h, self.fix_ids[ifix], _dp(nodes), _dp(vel))
        return nodes, vel

    def mesh_geom(self, ifix):
        """Per element: centre, bounding radius, edge vectors, edge lengths,
        edge normals, surface normal, precision (29 columns)."""
        n = self.L.orc_get_mesh_geom(self.h, self.fix_ids[ifix], None)
        g = np.zeros((n, 29))
        self.L.orc_get_mesh_geom(self.h, self.fix_ids[ifix], _dp(g))
        return g

    def mesh_topology(self, ifix, ntri_max):
        k = self.fix_ids[ifix]
        ea = np.zeros(3 * ntri_max, dtype=np.uint8)
        ca = np.zeros(3 * ntri_max, dtype=np.uint8)
        ob = np.zeros(ntri_max, dtype=np.int32)
        n = self.L.orc_get_mesh_topology(self.h, k, ea.ctypes.data_as(U8), ca.ctypes.data_as(U8), _ip(ob))
        return ea[:3 * n].reshape(n, 3), ca[:3 * n].reshape(n, 3), ob[:n]

    def mesh_nneighs(self, ifix):
        n = self.nlocal
        out = np.zeros(n, dtype=np.int32)
        self.L.orc_get_mesh_nneighs(self.h, self.fix_ids[ifix], _ip(out))
        return out


def pair_force(sc, xi, xj, vi, vj, wi, wj, ri, rj, mi, mj, ti=1, tj=1, shear=None, shearupdate=1):
    """Single-pair force through the oracle's contact chain (for known-answer tests)."""
    L = lib()
    p, keep = make_params(sc)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (xi, xj, vi, vj, wi, wj)]
    sh = np.zeros(3) if shear is None else np.ascontiguousarray(shear, dtype=np.float64)
    outs = [np.zeros(3) for _ in range(4)]
    L.orc_pair_force(ctypes.byref(p), *[_dp(a) for a in arrs], ri, rj, mi, mj, ti, tj, _dp(sh), shearupdate,
                     *[_dp(o) for o in outs])
    return outs[0], outs[1], outs[2], outs[3], sh


# ---------------------------------------------------------------- superquadrics

class SqParticle(ctypes.Structure):
    _fields_ = [("center", ctypes.c_double * 3), ("quat", ctypes.c_double * 4), ("shape", ctypes.c_double * 3),
                ("n", ctypes.c_double)]


class SqSolution(ctypes.Structure):
    _fields_ = [("point", ctypes.c_double * 3), ("mu", ctypes.c_double), ("fi", ctypes.c_double),
                ("fj", ctypes.c_double), ("gradi", ctypes.c_double * 3), ("gradj", ctypes.c_double * 3),
                ("merit", ctypes.c_double), ("iters", ctypes.c_int), ("solves", ctypes.c_int), ("fail", ctypes.c_int)]


class SqParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("skin", ctypes.c_double), ("youngs", ctypes.c_double),
                ("poisson", ctypes.c_double), ("restitution", ctypes.c_double), ("friction", ctypes.c_double)]


def _sq_lib():
    L = lib()
    if not hasattr(L, "_sq_ready"):
        L.orc_sq_contact_point.argtypes = [ctypes.POINTER(SqParticle), ctypes.POINTER(SqParticle), ctypes.c_int, D,
                                           ctypes.POINTER(SqSolution)]
        L.orc_sq_shape_props.argtypes = [ctypes.POINTER(SqParticle), D, D, D, D]
        L.orc_sq_bounding_radius.restype = ctypes.c_double
        L.orc_sq_bounding_radius.argtypes = [D, ctypes.c_double]
        L.orc_sq_create.restype = ctypes.c_void_p
        L.orc_sq_create.argtypes = [ctypes.POINTER(SqParams), ctypes.c_int] + [D] * 9
        L.orc_sq_destroy.argtypes = [ctypes.c_void_p]
        L.orc_sq_setup.argtypes = [ctypes.c_void_p]
        L.orc_sq_run.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_sq_get_atoms.argtypes = [ctypes.c_void_p] + [D] * 7
        L.orc_sq_get_pairs.argtypes = [ctypes.c_void_p, ctypes.c_int, I, I, I, D, D]
        LP = ctypes.POINTER(ctypes.c_long)
        L.orc_sq_counters.argtypes = [ctypes.c_void_p, LP, LP, LP, LP]
        L._sq_ready = True
    return L


def sq_particle(center, quat, shape, n):
    p = SqParticle()
    for k in range(3):
        p.center[k] = center[k]
        p.shape[k] = shape[k]
    for k in range(4):
        p.quat[k] = quat[k]
    p.n = n
    return p


def sq_contact_point(pa, pb, guess=None):
    """Contact-point solve for two superquadrics (dicts with center, quat,
    shape, n): homotopy from spheres when guess is None, else one Newton
    solve from guess.  Returns a dict of the solution."""
    L = _sq_lib()
    A = sq_particle(pa["center"], pa["quat"], pa["shape"], pa["n"])
    B = sq_particle(pb["center"], pb["quat"], pb["shape"], pb["n"])
    out = SqSolution()
    g = np.ascontiguousarray(guess if guess is not None else np.zeros(3), dtype=np.float64)
    L.orc_sq_contact_point(ctypes.byref(A), ctypes.byref(B), 0 if guess is None else 1, _dp(g), ctypes.byref(out))
    return {"point": np.array(out.point[:]), "mu": out.mu, "fi": out.fi, "fj": out.fj,
            "gradi": np.array(out.gradi[:]), "gradj": np.array(out.gradj[:]), "merit": out.merit,
            "iters": out.iters, "solves": out.solves, "fail": out.fail}


def sq_shape_props(p, x):
    L = _sq_lib()
    P = sq_particle(p["center"], p["quat"], p["shape"], p["n"])
    f = ctypes.c_double()
    g = np.zeros(3)
    h = np.zeros(9)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    L.orc_sq_shape_props(ctypes.byref(P), _dp(xx), ctypes.cast(ctypes.byref(f), D), _dp(g), _dp(h))
    return f.value, g, h.reshape(3, 3)


def sq_bounding_radius(shape, n):
    s = np.ascontiguousarray(shape, dtype=np.float64)
    return _sq_lib().orc_sq_bounding_radius(_dp(s), float(n))


class SqOracle:
    """Superquadric DEM run in the oracle (see sq_oracle.h)."""

    def __init__(self, sc):
        L = _sq_lib()
        self.L = L
        p = SqParams(sc["dt"], sc["skin"], sc["youngs"], sc["poisson"], sc["restitution"], sc["friction"])
        a = sc["atoms"]
        self._keep = [np.ascontiguousarray(a[k], dtype=np.float64) for k in
                      ("x", "v", "quat", "angmom", "shape", "blockiness", "rmass", "inertia", "volume")]
        self.n = len(a["rmass"])
        self.h = L.orc_sq_create(ctypes.byref(p), self.n, *[_dp(k) for k in self._keep])

    def close(self):
        if self.h:
            self.L.orc_sq_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup(self):
        self.L.orc_sq_setup(self.h)

    def run(self, n):
        self.L.orc_sq_run(self.h, n)

    def atoms(self):
        n = self.n
        out = {k: np.zeros((n, 3)) for k in ("x", "v", "angmom", "omega", "f", "torque")}
        out["quat"] = np.zeros((n, 4))
        self.L.orc_sq_get_atoms(self.h, _dp(out["x"]), _dp(out["v"]), _dp(out["quat"]), _dp(out["angmom"]),
                                _dp(out["omega"]), _dp(out["f"]), _dp(out["torque"]))
        return out

    def pairs(self):
        n = self.L.orc_sq_get_pairs(self.h, 0, None, None, None, None, None)
        ti, tj, st = (np.zeros(n, dtype=np.int32) for _ in range(3))
        cp, sh = np.zeros((n, 3)), np.zeros((n, 3))
        self.L.orc_sq_get_pairs(self.h, n, _ip(ti), _ip(tj), _ip(st), _dp(cp), _dp(sh))
        return {"tag_i": ti, "tag_j": tj, "state": st, "cp": cp, "shear": sh}

    def counters(self):
        v = [ctypes.c_long() for _ in range(4)]
        self.L.orc_sq_counters(self.h, *[ctypes.byref(x) for x in v])
        return {"iters": v[0].value, "solves": v[1].value, "pairs_solved": v[2].value, "nbuilds": v[3].value}
