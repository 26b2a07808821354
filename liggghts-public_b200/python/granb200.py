"""ctypes front end of libgranb200 (the C ABI in include/granb200.h).

``Engine(scenario)`` builds one device-resident simulation from a scenario
dict (see gb2_scenarios) and mirrors the reference's run sequence:
``setup()`` is Verlet::setup, ``run(n)`` is Verlet::run(n).  There is no CPU
fallback: constructing an Engine without the built library, or without a
CUDA device, raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libgranb200.so")
_LIB = None

D = ctypes.POINTER(ctypes.c_double)
I = ctypes.POINTER(ctypes.c_int)
U8 = ctypes.POINTER(ctypes.c_ubyte)

PREC_FP64 = 0
PREC_SPLIT = 1

EXPORTS = (
    "gb2_create", "gb2_destroy", "gb2_set_materials", "gb2_upload_atoms", "gb2_add_gravity",
    "gb2_add_wall_plane", "gb2_add_wall_mesh", "gb2_setup", "gb2_run", "gb2_sync", "gb2_download_atoms",
    "gb2_download_pairs", "gb2_download_wall_history", "gb2_download_mesh_contacts", "gb2_mesh_topology",
    "gb2_get_stats", "gb2_last_error", "gb2_version", "gb2_census", "gb2_set_profiling", "gb2_timer_start",
    "gb2_timer_stop", "gb2_census_noalloc", "gb2_add_move_mesh_rotate", "gb2_download_mesh_nodes",
    "gb2_add_move_mesh_linear", "gb2_add_wall_cylinder", "gb2_contact_atom",
    "gb2_upload_history", "gb2_download_history", "gb2_upload_wall_history", "gb2_add_mesh_stress",
    "gb2_download_mesh_stress", "gb2_pair_gran_local",
    "gb2_pair_gran_local_keys", "gb2_add_insert_pack", "gb2_add_insert_stream", "gb2_insert_stats", "gb2_download_mesh_history",
    "gb2_upload_mesh_history", "gb2_add_mesh_wear", "gb2_download_mesh_wear", "gb2_upload_mesh_wear", "gb2_host_alloc", "gb2_host_free", "gb2_set_timestep",
)

NOALLOC_MAX_ATOMS = 16384 * 128   # GB2_NOALLOC_MAX_ATOMS

# compute pair/gran/local keywords (GB2_PGL_*), in the reference's column order,
# with their column counts
PGL_KEYWORDS = (("pos", 6), ("vel", 6), ("id", 3), ("force", 3), ("force_normal", 3), ("force_tangential", 3),
                ("torque", 3), ("torque_normal", 3), ("torque_tangential", 3), ("history", 3), ("contactArea", 1),
                ("delta", 1), ("contactPoint", 3))
PGL_DEFAULT = ("pos", "vel", "id", "force", "torque", "history", "contactArea")


def pgl_keys(keywords):
    """Bit mask of a pair/gran/local keyword list; unknown names raise ValueError."""
    names = [k for k, _ in PGL_KEYWORDS]
    keys = 0
    for w in keywords:
        if w not in names:
            raise ValueError("compute pair/gran/local: unknown or unsupported keyword %r" % (w,))
        keys |= 1 << names.index(w)
    return keys


def pgl_columns(keys):
    """Column names of a pair/gran/local row for a keyword bit mask."""
    cols = []
    for b, (name, n) in enumerate(PGL_KEYWORDS):
        if keys & (1 << b):
            cols += [name] if n == 1 else ["%s[%d]" % (name, c) for c in range(n)]
    return cols


INSERT_MAX_TEMPLATES = 8   # GB2_INSERT_MAX_TEMPLATES


class InsertPackParams(ctypes.Structure):
    """gb2_insert_pack: fix insert/pack + particledistribution/discrete + particletemplate/sphere."""
    _fields_ = [
        ("seed", ctypes.c_int),
        ("region_lo", ctypes.c_double * 3),
        ("region_hi", ctypes.c_double * 3),
        ("volumefraction_region", ctypes.c_double),
        ("particles_in_region", ctypes.c_int),
        ("mass_in_region", ctypes.c_double),
        ("insert_every", ctypes.c_int),
        ("start", ctypes.c_int),
        ("maxattempt", ctypes.c_int),
        ("overlapcheck", ctypes.c_int),
        ("all_in", ctypes.c_int),
        ("exact_number", ctypes.c_int),
        ("vel_style", ctypes.c_int),
        ("vel", ctypes.c_double * 3),
        ("vel_fluct", ctypes.c_double * 3),
        ("omega", ctypes.c_double * 3),
        ("ntry_mc", ctypes.c_int),
        ("check_dist_from_subdomain_border", ctypes.c_int),
        ("dist_seed", ctypes.c_int),
        ("dist_mass_based", ctypes.c_int),
        ("ntemplates", ctypes.c_int),
        ("tmpl_type", ctypes.c_int * INSERT_MAX_TEMPLATES),
        ("tmpl_radius", ctypes.c_double * INSERT_MAX_TEMPLATES),
        ("tmpl_density", ctypes.c_double * INSERT_MAX_TEMPLATES),
        ("tmpl_weight", ctypes.c_double * INSERT_MAX_TEMPLATES),
        ("max_atoms", ctypes.c_int),
        ("tmpl_radius_style", ctypes.c_int * INSERT_MAX_TEMPLATES),
        ("tmpl_radius2", ctypes.c_double * INSERT_MAX_TEMPLATES),
        ("tmpl_seed", ctypes.c_int * INSERT_MAX_TEMPLATES),
        ("region_style", ctypes.c_int),
        ("cyl_axis", ctypes.c_int),
        ("cyl_c1", ctypes.c_double),
        ("cyl_c2", ctypes.c_double),
        ("cyl_radius", ctypes.c_double),
        ("cyl_lo", ctypes.c_double),
        ("cyl_hi", ctypes.c_double),
    ]


class InsertStreamParams(ctypes.Structure):
    """gb2_insert_stream: fix insert/stream + particledistribution/discrete + particletemplate/sphere."""
    _fields_ = [
        ("seed", ctypes.c_int),
        ("nface", ctypes.c_int),
        ("face_nodes", ctypes.POINTER(ctypes.c_double)),
        ("nparticles", ctypes.c_double),
        ("mass", ctypes.c_double),
        ("ninsert_inf", ctypes.c_int),
        ("particlerate", ctypes.c_double),
        ("massrate", ctypes.c_double),
        ("insert_every", ctypes.c_int),
        ("extrude_length", ctypes.c_double),
        ("duration", ctypes.c_int),
        ("start", ctypes.c_int),
        ("maxattempt", ctypes.c_int),
        ("overlapcheck", ctypes.c_int),
        ("exact_number", ctypes.c_int),
        ("vel_style", ctypes.c_int),
        ("vel", ctypes.c_double * 3),
        ("vel_fluct", ctypes.c_double * 3),
        ("omega", ctypes.c_double * 3),
        ("ntry_mc", ctypes.c_int),
        ("dist_seed", ctypes.c_int),
        ("dist_mass_based", ctypes.c_int),
        ("ntemplates", ctypes.c_int),
        ("tmpl_type", ctypes.c_int * INSERT_MAX_TEMPLATES),
        ("tmpl_radius", ctypes.c_double * INSERT_MAX_TEMPLATES),
        ("tmpl_density", ctypes.c_double * INSERT_MAX_TEMPLATES),
        ("tmpl_weight", ctypes.c_double * INSERT_MAX_TEMPLATES),
        ("tmpl_radius_style", ctypes.c_int * INSERT_MAX_TEMPLATES),
        ("tmpl_radius2", ctypes.c_double * INSERT_MAX_TEMPLATES),
        ("tmpl_seed", ctypes.c_int * INSERT_MAX_TEMPLATES),
        ("max_atoms", ctypes.c_int),
    ]


VEL_STYLES = {"constant": 0, "uniform": 1, "gaussian": 2}
RADIUS_STYLES = {"constant": 0, "uniform": 1, "gaussian": 2}


def insert_pack_params(fx, struct=InsertPackParams):
    """Fill the insertion parameter struct from a scenario fix dict (the
    reference's keyword defaults where a key is absent)."""
    p = struct()
    p.seed = int(fx["seed"])
    cyl = fx.get("region_cylinder")
    if cyl is not None:   # {"axis": 0|1|2, "c1", "c2", "radius", "lo", "hi"}
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
    p.vel_style = VEL_STYLES[fx.get("vel_style", "constant")]
    p.ntry_mc = int(fx.get("ntry_mc", 100000))
    p.check_dist_from_subdomain_border = int(fx.get("check_dist_from_subdomain_border", 1))
    p.dist_seed = int(fx["dist_seed"])
    p.dist_mass_based = int(fx.get("dist_mass_based", 1))
    tm = fx["templates"]
    if not 1 <= len(tm) <= INSERT_MAX_TEMPLATES:
        raise ValueError("1 to %d templates" % INSERT_MAX_TEMPLATES)
    p.ntemplates = len(tm)
    for i, t in enumerate(tm):
        p.tmpl_type[i] = int(t["type"])
        p.tmpl_radius[i] = float(t["radius"])
        p.tmpl_density[i] = float(t["density"])
        p.tmpl_weight[i] = float(t["weight"])
        p.tmpl_radius_style[i] = RADIUS_STYLES[t.get("radius_style", "constant")]
        p.tmpl_radius2[i] = float(t.get("radius2", 0.0))
        p.tmpl_seed[i] = int(t.get("seed", 67867967))
    p.max_atoms = int(fx.get("max_atoms", 0))
    return p


def insert_stream_params(fx):
    """(struct, face node array to keep alive) of a scenario's insert_stream fix."""
    p = InsertStreamParams()
    face = np.ascontiguousarray(np.asarray(fx["face_nodes"], dtype=np.float64).reshape(-1, 9))
    p.seed = int(fx["seed"])
    p.nface = len(face)
    p.face_nodes = face.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    p.nparticles = float(fx.get("nparticles", 0))
    p.mass = float(fx.get("mass", 0.0))
    p.ninsert_inf = int(fx.get("nparticles") == "INF" or fx.get("mass") == "INF")
    if p.ninsert_inf:
        p.nparticles = p.mass = 0.0
    p.particlerate = float(fx.get("particlerate", 0.0))
    p.massrate = float(fx.get("massrate", 0.0))
    p.insert_every = int(fx.get("insert_every", -1))
    p.extrude_length = float(fx.get("extrude_length", 0.0))
    p.duration = int(fx.get("duration", 0))
    p.start = int(fx.get("start", 0))
    p.maxattempt = int(fx.get("maxattempt", 50))
    p.overlapcheck = int(fx.get("overlapcheck", 1))
    p.exact_number = int(fx.get("exact_number", 1))
    p.vel_style = VEL_STYLES[fx.get("vel_style", "constant")]
    for d in range(3):
        p.vel[d] = fx.get("vel", (0.0, 0.0, 0.0))[d]
        p.vel_fluct[d] = fx.get("vel_fluct", (0.0, 0.0, 0.0))[d]
        p.omega[d] = fx.get("omega", (0.0, 0.0, 0.0))[d]
    p.ntry_mc = int(fx.get("ntry_mc", 100000))
    p.dist_seed = int(fx["dist_seed"])
    p.dist_mass_based = int(fx.get("dist_mass_based", 1))
    tm = fx["templates"]
    if not 1 <= len(tm) <= INSERT_MAX_TEMPLATES:
        raise ValueError("1 to %d templates" % INSERT_MAX_TEMPLATES)
    p.ntemplates = len(tm)
    for i, t in enumerate(tm):
        p.tmpl_type[i] = int(t["type"])
        p.tmpl_radius[i] = float(t["radius"])
        p.tmpl_density[i] = float(t["density"])
        p.tmpl_weight[i] = float(t["weight"])
        p.tmpl_radius_style[i] = RADIUS_STYLES[t.get("radius_style", "constant")]
        p.tmpl_radius2[i] = float(t.get("radius2", 0.0))
        p.tmpl_seed[i] = int(t.get("seed", 67867967))
    p.max_atoms = int(fx.get("max_atoms", 0))
    return p, face


class Params(ctypes.Structure):
    _fields_ = [
        ("ntypes", ctypes.c_int),
        ("dt", ctypes.c_double),
        ("skin", ctypes.c_double),
        ("boxlo", ctypes.c_double * 3),
        ("boxhi", ctypes.c_double * 3),
        ("periodic", ctypes.c_int * 3),
        ("neigh_every", ctypes.c_int),
        ("neigh_delay", ctypes.c_int),
        ("neigh_check", ctypes.c_int),
        ("sort_freq", ctypes.c_int),
        ("sort_binsize", ctypes.c_double),
        ("rolling_cdt", ctypes.c_int),
        ("tangential_damping", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("device", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("ntimestep", ctypes.c_long),
        ("nlocal", ctypes.c_int),
        ("nghost", ctypes.c_int),
        ("nbuilds", ctypes.c_int),
        ("npairs", ctypes.c_long),
        ("ntouch", ctypes.c_long),
        ("maxneigh", ctypes.c_int),
        ("maxpartner", ctypes.c_int),
        ("time_pair", ctypes.c_double),
        ("time_neigh", ctypes.c_double),
        ("time_other", ctypes.c_double),
        ("kernel_launches", ctypes.c_long),
        ("t_integrate", ctypes.c_double),
        ("t_pair_tail", ctypes.c_double),
        ("t_pair_main", ctypes.c_double),
        ("t_forward", ctypes.c_double),
        ("t_rebuild", ctypes.c_double),
        ("n_pair_main", ctypes.c_long),
        ("nsteps_rebuild", ctypes.c_long),
        ("maxrev", ctypes.c_int),
        ("maxmesh", ctypes.c_int),
        ("ngrow", ctypes.c_long),
        ("n_rebuild_timed", ctypes.c_long),
    ]


class Census(ctypes.Structure):
    _fields_ = [(f, ctypes.c_long) for f in
                ("nlist", "ntouch", "nrev", "nwall_list", "nwall_touch", "nmesh_cand", "nmesh_touch")]


def lib(path=LIB_PATH):
    """Load the in-tree shared library (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(path):
            raise RuntimeError("libgranb200.so not built: run __graft_entry__.build() (%s)" % path)
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.gb2_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(vp)]
        L.gb2_destroy.argtypes = [vp]
        L.gb2_set_materials.argtypes = [vp, D, D, D, D, D]
        L.gb2_upload_atoms.argtypes = [vp, ctypes.c_int, D, D, D, D, D, I, I]
        L.gb2_add_gravity.argtypes = [vp, ctypes.c_double, D]
        L.gb2_add_wall_plane.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.gb2_add_wall_mesh.argtypes = [vp, ctypes.c_int, D, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.gb2_setup.argtypes = [vp]
        L.gb2_run.argtypes = [vp, ctypes.c_int]
        L.gb2_sync.argtypes = [vp]
        L.gb2_download_atoms.argtypes = [vp, ctypes.c_int, I, D, D, D, D, D, I]
        L.gb2_download_pairs.argtypes = [vp, ctypes.c_int, I, I, I, I, D]
        L.gb2_download_wall_history.argtypes = [vp, ctypes.c_int, ctypes.c_int, D]
        L.gb2_contact_atom.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), I, D]
        L.gb2_upload_history.argtypes = [vp, ctypes.c_int, I, I, D]
        L.gb2_download_history.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_int), I, I, I, D]
        L.gb2_upload_wall_history.argtypes = [vp, ctypes.c_int, ctypes.c_int, D]
        L.gb2_add_mesh_stress.argtypes = [vp, ctypes.c_int, D]
        L.gb2_pair_gran_local.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), D]
        L.gb2_add_mesh_wear.argtypes = [vp, ctypes.c_int, D]
        L.gb2_download_mesh_wear.argtypes = [vp, ctypes.c_int, ctypes.c_int, D]
        L.gb2_upload_mesh_wear.argtypes = [vp, ctypes.c_int, ctypes.c_int, D]
        L.gb2_download_mesh_history.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, I, I, I, I, I, D]
        L.gb2_upload_mesh_history.argtypes = [vp, ctypes.c_int, ctypes.c_int, I, I, D]
        L.gb2_add_insert_pack.argtypes = [vp, ctypes.POINTER(InsertPackParams)]
        L.gb2_add_insert_stream.argtypes = [vp, ctypes.POINTER(InsertStreamParams)]
        L.gb2_insert_stats.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_long), D,
                                       ctypes.POINTER(ctypes.c_long)]
        L.gb2_pair_gran_local_keys.argtypes = [vp, ctypes.c_uint, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int), D]
        L.gb2_download_mesh_stress.argtypes = [vp, ctypes.c_int, ctypes.c_int, D, D, D, D]
        L.gb2_download_mesh_contacts.argtypes = [vp, ctypes.c_int, ctypes.c_int, I, I, I, D]
        L.gb2_mesh_topology.argtypes = [vp, ctypes.c_int, ctypes.c_int, I, U8, U8, I]
        L.gb2_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
        L.gb2_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        L.gb2_version.restype = ctypes.c_char_p
        L.gb2_census.argtypes = [vp, ctypes.POINTER(Census)]
        L.gb2_census_noalloc.argtypes = [vp, ctypes.POINTER(Census)]
        L.gb2_set_profiling.argtypes = [vp, ctypes.c_int]
        L.gb2_timer_start.argtypes = [vp]
        L.gb2_timer_stop.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.gb2_add_move_mesh_rotate.argtypes = [vp, ctypes.c_int, D, D, ctypes.c_double]
        L.gb2_add_move_mesh_linear.argtypes = [vp, ctypes.c_int, D]
        L.gb2_add_wall_cylinder.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_int, ctypes.c_int]
        L.gb2_download_mesh_nodes.argtypes = [vp, ctypes.c_int, ctypes.c_int, I, D, D]
        L.gb2_host_alloc.argtypes = [ctypes.c_size_t, ctypes.POINTER(vp)]
        L.gb2_host_free.argtypes = [vp]
        L.gb2_set_timestep.argtypes = [vp, ctypes.c_long]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(D)


def _ip(a):
    return a.ctypes.data_as(I)


class GB2Error(RuntimeError):
    pass


def pinned_empty(shape, dtype=np.float64):
    """A numpy array in page-locked host memory (gb2_host_alloc): the
    library's atom upload and download copy it with the device directly.
    The memory is released (gb2_host_free) when the array is collected."""
    import weakref
    L = lib()
    dt = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dt.itemsize
    ptr = ctypes.c_void_p()
    if L.gb2_host_alloc(max(nbytes, 1), ctypes.byref(ptr)) != 0:
        raise GB2Error("gb2_host_alloc of %d bytes failed" % nbytes)
    buf = (ctypes.c_char * max(nbytes, 1)).from_address(ptr.value)
    arr = np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)
    weakref.finalize(buf, L.gb2_host_free, ptr)
    return arr


def restart_scenario(sc, atoms, mesh_nodes=None, ntimestep=None):
    """The scenario with its atoms replaced by a run's current state (same
    tags, the run's atom order), as read_restart would bring them back;
    `mesh_nodes` maps a scenario fix index to that mesh's current nodes
    (ntri, 3, 3), for meshes that have moved; `ntimestep` is the step the
    restarted run starts from (the restart file's timestep)."""
    out = dict(sc)
    if ntimestep is not None:
        out["ntimestep"] = int(ntimestep)
    a = dict(sc["atoms"])
    tags = np.asarray(a["tag"])
    order = np.argsort(tags, kind="stable")
    idx = order[np.searchsorted(tags, atoms["tag"], sorter=order)]
    for k in a:
        a[k] = np.ascontiguousarray(np.asarray(a[k])[idx])
    for k in ("x", "v", "omega"):
        a[k] = np.ascontiguousarray(atoms[k])
    a["tag"] = np.ascontiguousarray(atoms["tag"])
    out["atoms"] = a
    if mesh_nodes:
        fixes = [dict(f) for f in sc["fixes"]]
        for i, nodes in mesh_nodes.items():
            fixes[i]["nodes"] = np.ascontiguousarray(np.asarray(nodes, dtype=np.float64).reshape(-1, 9))
        out["fixes"] = fixes
    return out


class Engine:
    """One device-resident granular simulation (one gb2_ctx)."""

    def __init__(self, sc, precision=PREC_FP64, device=0):
        L = lib()
        self.L = L
        p = Params()
        p.ntypes = sc["ntypes"]
        self.ntypes = int(sc["ntypes"])
        p.dt = sc["dt"]
        p.skin = sc["skin"]
        for d in range(3):
            p.boxlo[d] = sc["boxlo"][d]
            p.boxhi[d] = sc["boxhi"][d]
            p.periodic[d] = int(sc["periodic"][d])
        p.neigh_every = sc.get("every", 1)
        p.neigh_delay = sc.get("delay", 0)
        p.neigh_check = sc.get("check", 1)
        p.sort_freq = sc.get("sortfreq", 1000)
        p.sort_binsize = sc.get("sortbinsize", 0.0)
        p.rolling_cdt = int(sc.get("rolling_cdt", 0))
        p.tangential_damping = int(sc.get("tangential_damping", 1))
        p.precision = precision
        p.device = device
        self.h = ctypes.c_void_p()
        rc = L.gb2_create(ctypes.byref(p), ctypes.byref(self.h))
        if rc != 0:
            raise GB2Error("gb2_create failed (%d): no CUDA device or unsupported option" % rc)
        keep = []

        def arr(x, dt=np.float64):
            a = np.ascontiguousarray(np.asarray(x, dtype=dt).ravel())
            keep.append(a)
            return a

        self._check(L.gb2_set_materials(self.h, _dp(arr(sc["youngs"])), _dp(arr(sc["poisson"])),
                                        _dp(arr(sc["restitution"])), _dp(arr(sc["friction"])),
                                        _dp(arr(sc["rollfriction"]))))
        a = sc["atoms"]
        n = len(a["tag"])
        self._check(L.gb2_upload_atoms(self.h, n, _dp(arr(a["x"])), _dp(arr(a["v"])), _dp(arr(a["omega"])),
                                       _dp(arr(a["radius"])), _dp(arr(a["rmass"])), _ip(arr(a["type"], np.int32)),
                                       _ip(arr(a["tag"], np.int32))))
        self.fix_ids = []
        self.ntri = {}
        for fx in sc["fixes"]:
            kind = fx["kind"]
            if kind == "gravity":
                k = L.gb2_add_gravity(self.h, fx["magnitude"], _dp(arr(fx["vector"])))
            elif kind == "wall_plane":
                k = L.gb2_add_wall_plane(self.h, fx["dim"], fx["pos"], fx["wall_type"], int(fx.get("rolling_cdt", 0)))
            elif kind == "wall_cylinder":
                k = L.gb2_add_wall_cylinder(self.h, fx["dim"], fx["radius"], fx["c1"], fx["c2"], fx["wall_type"],
                                            int(fx.get("rolling_cdt", 0)))
            elif kind == "wall_mesh":
                nodes = arr(fx["nodes"])
                k = L.gb2_add_wall_mesh(self.h, len(nodes) // 9, _dp(nodes), fx["wall_type"], fx.get("curvature", 0.0),
                                        int(fx.get("rolling_cdt", 0)))
                if k >= 0:
                    self.ntri[len(self.fix_ids)] = len(nodes) // 9
            elif kind == "move_mesh_rotate":
                mesh_id = self.fix_ids[fx["mesh"]]
                self._check(L.gb2_add_move_mesh_rotate(self.h, mesh_id, _dp(arr(fx["origin"])), _dp(arr(fx["axis"])),
                                                       float(fx["period"])))
                k = None
            elif kind == "move_mesh_linear":
                self._check(L.gb2_add_move_mesh_linear(self.h, self.fix_ids[fx["mesh"]], _dp(arr(fx["velocity"]))))
                k = None
            elif kind == "nve_sphere":
                k = None
            elif kind == "insert_pack":
                ip = insert_pack_params(fx)
                keep.append(ip)
                self._check(L.gb2_add_insert_pack(self.h, ctypes.byref(ip)))
                k = 0
            elif kind == "insert_stream":
                ip, face = insert_stream_params(fx)
                keep += [ip, face]
                self._check(L.gb2_add_insert_stream(self.h, ctypes.byref(ip)))
                k = 0
            else:
                raise ValueError("unsupported fix kind " + kind)
            if k is not None and k < 0:
                self._check(k)
            self.fix_ids.append(k)
        self.n = n
        if int(sc.get("ntimestep", 0)):   # a restarted run keeps its step count (atom-sort schedule)
            self._check(L.gb2_set_timestep(self.h, int(sc["ntimestep"])))

    def _err(self):
        buf = ctypes.create_string_buffer(512)
        self.L.gb2_last_error(self.h, buf, 512)
        return buf.value.decode()

    def _check(self, rc):
        if rc != 0:
            raise GB2Error("granb200 error %d: %s" % (rc, self._err()))

    def close(self):
        if self.h:
            self.L.gb2_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup(self):
        self._check(self.L.gb2_setup(self.h))

    def run(self, n):
        self._check(self.L.gb2_run(self.h, n))

    def sync(self):
        self._check(self.L.gb2_sync(self.h))

    def stats(self):
        s = Stats()
        self._check(self.L.gb2_get_stats(self.h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in Stats._fields_}

    def census(self):
        c = Census()
        self._check(self.L.gb2_census(self.h, ctypes.byref(c)))
        return {f: getattr(c, f) for f, _ in Census._fields_}

    def census_noalloc(self):
        """gb2_census_noalloc: the census without any device allocation (static scratch)."""
        c = Census()
        self._check(self.L.gb2_census_noalloc(self.h, ctypes.byref(c)))
        return {f: getattr(c, f) for f, _ in Census._fields_}

    def set_profiling(self, on, every=1):
        """Per-kernel CUDA-event timing, on every `every`-th step."""
        self._check(self.L.gb2_set_profiling(self.h, max(1, int(every)) if on else 0))

    def timer_start(self):
        self._check(self.L.gb2_timer_start(self.h))

    def timer_stop(self):
        ms = ctypes.c_double()
        self._check(self.L.gb2_timer_stop(self.h, ctypes.byref(ms)))
        return ms.value

    def count(self):
        """Current number of owned atoms (fix insert/pack adds atoms)."""
        cnt0 = ctypes.c_int()
        self._check(self.L.gb2_download_atoms(self.h, 0, ctypes.byref(cnt0), None, None, None, None, None, None))
        self.n = cnt0.value
        return self.n

    def atoms(self, out=None):
        """x, v, omega, f, torque [n][3] and tag [n] of the owned atoms; `out`
        may hold preallocated arrays (e.g. pinned_empty) of the right shape."""
        n = self.count()
        if out is None or len(out["tag"]) != n:
            out = {k: np.zeros((n, 3)) for k in ("x", "v", "omega", "f", "torque")}
            out["tag"] = np.zeros(n, dtype=np.int32)
        tag = out["tag"]
        cnt = ctypes.c_int()
        self._check(self.L.gb2_download_atoms(self.h, n, ctypes.byref(cnt), _dp(out["x"]), _dp(out["v"]),
                                              _dp(out["omega"]), _dp(out["f"]), _dp(out["torque"]), _ip(tag)))
        out["tag"] = tag
        return out

    def pairs(self):
        cnt = ctypes.c_int()
        self._check(self.L.gb2_download_pairs(self.h, 0, ctypes.byref(cnt), None, None, None, None))
        n = cnt.value
        ti = np.zeros(n, dtype=np.int32)
        tj = np.zeros(n, dtype=np.int32)
        fl = np.zeros(n, dtype=np.int32)
        hi = np.zeros((n, 3))
        self._check(self.L.gb2_download_pairs(self.h, n, ctypes.byref(cnt), _ip(ti), _ip(tj), _ip(fl), _dp(hi)))
        return {"tag_i": ti, "tag_j": tj, "flag": fl, "hist": hi}

    def insert_stats(self):
        """fix insert/pack: particles and mass inserted so far, next insertion step."""
        n, nxt, m = ctypes.c_long(), ctypes.c_long(), np.zeros(1)
        self._check(self.L.gb2_insert_stats(self.h, 0, ctypes.byref(n), _dp(m), ctypes.byref(nxt)))
        return {"ninserted": n.value, "massinserted": float(m[0]), "next_step": nxt.value}

    def pair_gran_local(self, keywords=None):
        """compute pair/gran/local on the device: (nrows, ncols).  Without
        keywords the 12 columns id force torque history; a keyword list gives
        the columns in the reference's order (pgl_columns)."""
        n = ctypes.c_int()
        if keywords is None:
            self._check(self.L.gb2_pair_gran_local(self.h, 0, ctypes.byref(n), None))
            rows = np.zeros((n.value, 12))
            if n.value:
                self._check(self.L.gb2_pair_gran_local(self.h, n.value, ctypes.byref(n), _dp(rows)))
            return rows
        keys = pgl_keys(keywords)
        nc = ctypes.c_int()
        self._check(self.L.gb2_pair_gran_local_keys(self.h, keys, 0, ctypes.byref(n), ctypes.byref(nc), None))
        rows = np.zeros((n.value, nc.value))
        if n.value:
            self._check(self.L.gb2_pair_gran_local_keys(self.h, keys, n.value, ctypes.byref(n), ctypes.byref(nc),
                                                        _dp(rows)))
        return rows

    def add_mesh_stress(self, ifix, p_ref):
        """fix mesh/surface/stress on the mesh wall of scenario fix ifix (before setup)."""
        pr = np.ascontiguousarray(p_ref, dtype=np.float64)
        self._check(self.L.gb2_add_mesh_stress(self.h, self.fix_ids[ifix], _dp(pr)))

    def mesh_stress(self, ifix):
        """Per-triangle force of the last step and f_total / torque_total."""
        nt = self.ntri[ifix]
        f = np.zeros((nt, 3))
        sn, st = np.zeros(nt), np.zeros(nt)
        tot = np.zeros(6)
        self._check(self.L.gb2_download_mesh_stress(self.h, self.fix_ids[ifix], nt, _dp(f), _dp(sn), _dp(st), _dp(tot)))
        return {"tri_f": f, "sigma_n": sn, "sigma_t": st, "f_total": tot[:3], "torque_total": tot[3:]}

    def upload_history(self, npartner, partner_tag, hist):
        """FixContactHistory restart data (per atom: partner count, tags and
        shear) for the atoms as uploaded; before setup."""
        a = [np.ascontiguousarray(npartner, dtype=np.int32), np.ascontiguousarray(partner_tag, dtype=np.int32),
             np.ascontiguousarray(hist, dtype=np.float64)]
        self._check(self.L.gb2_upload_history(self.h, len(a[0]), _ip(a[0]), _ip(a[1]), _dp(a[2])))

    def upload_wall_hist(self, ifix, hist):
        h = np.ascontiguousarray(hist, dtype=np.float64)
        self._check(self.L.gb2_upload_wall_history(self.h, self.fix_ids[ifix], len(h), _dp(h)))

    def history(self):
        """Current contact history in the partner layout: tag, npartner, partner_tag, hist."""
        n, tot = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.gb2_download_history(self.h, 0, 0, ctypes.byref(n), ctypes.byref(tot), None, None, None,
                                                None))
        tag = np.zeros(n.value, dtype=np.int32)
        npart = np.zeros(n.value, dtype=np.int32)
        pt = np.zeros(tot.value, dtype=np.int32)
        ph = np.zeros((tot.value, 3))
        self._check(self.L.gb2_download_history(self.h, n.value, tot.value, ctypes.byref(n), ctypes.byref(tot),
                                                _ip(tag), _ip(npart), _ip(pt), _dp(ph)))
        return {"tag": tag, "npartner": npart, "partner_tag": pt, "hist": ph}

    def contact_atom(self):
        """compute contact/atom (skin 0) on the device: {tag, contact}."""
        n = ctypes.c_int()
        self.count()
        tag = np.zeros(self.n, dtype=np.int32)
        out = np.zeros(self.n)
        self._check(self.L.gb2_contact_atom(self.h, self.n, ctypes.byref(n), _ip(tag), _dp(out)))
        return {"tag": tag, "contact": out}

    def wall_hist(self, ifix):
        self.count()
        h = np.zeros((self.n, 3))
        self._check(self.L.gb2_download_wall_history(self.h, self.fix_ids[ifix], self.n, _dp(h)))
        return h

    def mesh_contacts(self, ifix):
        k = self.fix_ids[ifix]
        cnt = ctypes.c_int()
        self._check(self.L.gb2_download_mesh_contacts(self.h, k, 0, ctypes.byref(cnt), None, None, None))
        n = cnt.value
        tag = np.zeros(n, dtype=np.int32)
        tri = np.zeros(n, dtype=np.int32)
        h = np.zeros((n, 3))
        self._check(self.L.gb2_download_mesh_contacts(self.h, k, n, ctypes.byref(cnt), _ip(tag), _ip(tri), _dp(h)))
        return {"tag": tag, "tri": tri, "hist": h}

    def add_mesh_wear(self, ifix, k_finnie):
        """Finnie wear on the mesh of scenario fix ifix (after add_mesh_stress, before setup)."""
        kf = np.ascontiguousarray(k_finnie, dtype=np.float64)
        nt = self.ntypes
        if kf.shape != (nt, nt):
            raise ValueError("k_finnie must be an ntypes x ntypes array (%d x %d), got %s" % (nt, nt, kf.shape))
        kf = kf.reshape(-1)
        self._check(self.L.gb2_add_mesh_wear(self.h, self.fix_ids[ifix], _dp(kf)))

    def upload_mesh_wear(self, ifix, wear):
        """Cumulative wear per triangle of a restart (after add_mesh_wear, before setup)."""
        w = np.ascontiguousarray(wear, dtype=np.float64)
        self._check(self.L.gb2_upload_mesh_wear(self.h, self.fix_ids[ifix], len(w), _dp(w)))

    def mesh_wear(self, ifix):
        """Cumulative Finnie wear per triangle."""
        w = np.zeros(max(self.ntri.get(ifix, 0), 1))
        self._check(self.L.gb2_download_mesh_wear(self.h, self.fix_ids[ifix], len(w), _dp(w)))
        return w[:self.ntri.get(ifix, 0)]

    def mesh_history(self, ifix):
        """Mesh contact history in the restart layout: {tag, npartner, tri, hist}."""
        k = self.fix_ids[ifix]
        n, tot = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.gb2_download_mesh_history(self.h, k, 0, 0, ctypes.byref(n), ctypes.byref(tot), None, None,
                                                     None, None))
        tag = np.zeros(n.value, dtype=np.int32)
        npart = np.zeros(n.value, dtype=np.int32)
        tri = np.zeros(tot.value, dtype=np.int32)
        h = np.zeros((tot.value, 3))
        self._check(self.L.gb2_download_mesh_history(self.h, k, n.value, tot.value, ctypes.byref(n), ctypes.byref(tot),
                                                     _ip(tag), _ip(npart), _ip(tri), _dp(h)))
        return {"tag": tag, "npartner": npart, "tri": tri, "hist": h}

    def upload_mesh_hist(self, ifix, npartner, tri, hist):
        """Mesh contact history of the uploaded atoms (restart layout), before setup."""
        npart = np.ascontiguousarray(npartner, dtype=np.int32)
        t = np.ascontiguousarray(tri, dtype=np.int32)
        h = np.ascontiguousarray(hist, dtype=np.float64).reshape(-1)
        self._check(self.L.gb2_upload_mesh_history(self.h, self.fix_ids[ifix], len(npart), _ip(npart), _ip(t), _dp(h)))

    def mesh_nodes(self, ifix):
        """Current nodes (ntri, 3, 3) and node velocities of the mesh of fix ifix."""
        n = ctypes.c_int()
        self._check(self.L.gb2_download_mesh_nodes(self.h, self.fix_ids[ifix], 0, ctypes.byref(n), None, None))
        nodes = np.zeros((n.value, 3, 3))
        vel = np.zeros((n.value, 3, 3))
        self._check(self.L.gb2_download_mesh_nodes(self.h, self.fix_ids[ifix], n.value, ctypes.byref(n), _dp(nodes),
                                                   _dp(vel)))
        return nodes, vel

    def snapshot(self, sc):
        """What a restart of this run needs, downloaded: the timestep, the
        atoms, the pair contact history (partner layout), every primitive
        wall's history and every mesh's contact history (restart layout) and
        current nodes."""
        snap = {"atoms": self.atoms(), "history": self.history(), "walls": {}, "meshes": {},
                "ntimestep": int(self.stats()["ntimestep"])}
        for i, f in enumerate(sc["fixes"]):
            if f["kind"] in ("wall_plane", "wall_cylinder"):
                snap["walls"][i] = self.wall_hist(i)
            elif f["kind"] == "wall_mesh":
                nodes, _ = self.mesh_nodes(i)
                snap["meshes"][i] = {"history": self.mesh_history(i), "nodes": nodes}
        return snap

    def restore(self, snap):
        """Upload a snapshot's histories (the engine was built from
        restart_scenario(sc, snap["atoms"], ...)); before setup."""
        h = snap["history"]
        self.upload_history(h["npartner"], h["partner_tag"], h["hist"])
        for i, w in snap["walls"].items():
            self.upload_wall_hist(i, w)
        for i, m in snap["meshes"].items():
            mh = m["history"]
            self.upload_mesh_hist(i, mh["npartner"], mh["tri"], mh["hist"])

    def mesh_topology(self, ifix):
        k = self.fix_ids[ifix]
        nmax = self.ntri[ifix]
        ea = np.zeros(3 * nmax, dtype=np.uint8)
        ca = np.zeros(3 * nmax, dtype=np.uint8)
        ob = np.zeros(nmax, dtype=np.int32)
        nt = ctypes.c_int()
        self._check(self.L.gb2_mesh_topology(self.h, k, nmax, ctypes.byref(nt), ea.ctypes.data_as(U8),
                                             ca.ctypes.data_as(U8), _ip(ob)))
        n = nt.value
        return ea[:3 * n].reshape(n, 3), ca[:3 * n].reshape(n, 3), ob[:n]


# ---------------------------------------------------------------- superquadrics

SQ_MLP_SIZE = 9576   # GB2_SQ_MLP_SIZE


class SqParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("skin", ctypes.c_double), ("youngs", ctypes.c_double),
                ("poisson", ctypes.c_double), ("restitution", ctypes.c_double), ("friction", ctypes.c_double),
                ("device", ctypes.c_int)]


def _sq_lib():
    L = lib()
    if not getattr(L, "_sq_ready", False):
        vp = ctypes.c_void_p
        L.gb2_sq_create.argtypes = [ctypes.POINTER(SqParams), ctypes.POINTER(vp)]
        L.gb2_sq_destroy.argtypes = [vp]
        L.gb2_sq_upload.argtypes = [vp, ctypes.c_int] + [D] * 9
        L.gb2_sq_set_learned_guess.argtypes = [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int]
        L.gb2_sq_setup.argtypes = [vp]
        L.gb2_sq_run.argtypes = [vp, ctypes.c_int]
        L.gb2_sq_run_timed.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.gb2_sq_download.argtypes = [vp, ctypes.c_int] + [D] * 7
        L.gb2_sq_download_pairs.argtypes = [vp, ctypes.c_int, I, I, I, I, D, D]
        L.gb2_sq_counters.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.gb2_sq_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        L._sq_ready = True
    return L


class SqEngine:
    """Device-resident superquadric simulation (one gb2_sq_ctx)."""

    def __init__(self, sc, device=0, learned=None):
        L = _sq_lib()
        self.L = L
        p = SqParams(sc["dt"], sc["skin"], sc["youngs"], sc["poisson"], sc["restitution"], sc["friction"], device)
        self.h = ctypes.c_void_p()
        rc = L.gb2_sq_create(ctypes.byref(p), ctypes.byref(self.h))
        if rc != 0:
            raise GB2Error("gb2_sq_create failed (%d)" % rc)
        a = sc["atoms"]
        self.n = len(a["rmass"])
        keep = [np.ascontiguousarray(a[k], dtype=np.float64) for k in
                ("x", "v", "quat", "angmom", "shape", "blockiness", "rmass", "inertia", "volume")]
        self._check(L.gb2_sq_upload(self.h, self.n, *[_dp(k) for k in keep]))
        if learned is not None:
            self.set_learned_guess(learned)

    def _check(self, rc):
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            self.L.gb2_sq_last_error(self.h, buf, 512)
            raise GB2Error("granb200 sq error %d: %s" % (rc, buf.value.decode()))

    def close(self):
        if self.h:
            self.L.gb2_sq_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_learned_guess(self, params):
        if params is None:
            self._check(self.L.gb2_sq_set_learned_guess(self.h, None, 0))
            return
        self._w = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self.L.gb2_sq_set_learned_guess(self.h, self._w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                    len(self._w)))

    def setup(self):
        self._check(self.L.gb2_sq_setup(self.h))

    def run(self, n):
        self._check(self.L.gb2_sq_run(self.h, n))

    def run_timed(self, n):
        ms = ctypes.c_double()
        self._check(self.L.gb2_sq_run_timed(self.h, n, ctypes.byref(ms)))
        return ms.value

    def atoms(self):
        n = self.n
        out = {k: np.zeros((n, 3)) for k in ("x", "v", "angmom", "omega", "f", "torque")}
        out["quat"] = np.zeros((n, 4))
        self._check(self.L.gb2_sq_download(self.h, n, _dp(out["x"]), _dp(out["v"]), _dp(out["quat"]),
                                           _dp(out["angmom"]), _dp(out["omega"]), _dp(out["f"]), _dp(out["torque"])))
        return out

    def pairs(self):
        cnt = ctypes.c_int()
        self._check(self.L.gb2_sq_download_pairs(self.h, 0, ctypes.byref(cnt), None, None, None, None, None))
        n = cnt.value
        ti, tj, st = (np.zeros(n, dtype=np.int32) for _ in range(3))
        cp, sh = np.zeros((n, 3)), np.zeros((n, 3))
        self._check(self.L.gb2_sq_download_pairs(self.h, n, ctypes.byref(cnt), _ip(ti), _ip(tj), _ip(st), _dp(cp),
                                                 _dp(sh)))
        return {"tag_i": ti, "tag_j": tj, "state": st, "cp": cp, "shear": sh}

    def counters(self):
        out = (ctypes.c_longlong * 7)()
        self._check(self.L.gb2_sq_counters(self.h, out))
        keys = ("iters", "solves", "pairs_solved", "learned_used", "learned_rejected", "nbuilds", "npairs")
        return dict(zip(keys, [int(v) for v in out]))


class MlpTrainer:
    """Device-side training of the learned initial guess (one gb2_mlp_ctx)."""

    def __init__(self, device=0):
        L = lib()
        if not getattr(L, "_mlp_ready", False):
            vp = ctypes.c_void_p
            F = ctypes.POINTER(ctypes.c_float)
            L.gb2_mlp_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
            L.gb2_mlp_destroy.argtypes = [vp]
            L.gb2_mlp_make_data.argtypes = [vp, ctypes.c_long, ctypes.c_ulonglong, D]
            L.gb2_mlp_init.argtypes = [vp, ctypes.c_ulonglong]
            L.gb2_mlp_train.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, F]
            L.gb2_mlp_get_params.argtypes = [vp, F, ctypes.c_int]
            L.gb2_mlp_set_params.argtypes = [vp, F, ctypes.c_int]
            L.gb2_mlp_grad.argtypes = [vp, ctypes.c_int, F, F, F]
            L.gb2_mlp_evaluate.argtypes = [vp, ctypes.c_long, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_longlong), D]
            L.gb2_mlp_time_solves.argtypes = [vp, ctypes.c_long, ctypes.c_ulonglong, D, D,
                                              ctypes.POINTER(ctypes.c_longlong)]
            L.gb2_mlp_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
            L._mlp_ready = True
        self.L = L
        self.h = ctypes.c_void_p()
        rc = L.gb2_mlp_create(device, ctypes.byref(self.h))
        if rc != 0:
            raise GB2Error("gb2_mlp_create failed (%d)" % rc)

    def _check(self, rc):
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            self.L.gb2_mlp_last_error(self.h, buf, 512)
            raise GB2Error("granb200 mlp error %d: %s" % (rc, buf.value.decode()))

    def close(self):
        if self.h:
            self.L.gb2_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def make_data(self, n, seed):
        out = np.zeros(3)
        self._check(self.L.gb2_mlp_make_data(self.h, n, seed, _dp(out)))
        return {"valid": int(out[0]), "plain_iters": float(out[1]), "plain_solves": float(out[2])}

    def init(self, seed):
        self._check(self.L.gb2_mlp_init(self.h, seed))

    def train(self, epochs, batch, lr):
        loss = np.zeros(2, dtype=np.float32)
        self._check(self.L.gb2_mlp_train(self.h, epochs, batch, lr, loss.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return float(loss[0]), float(loss[1])

    def params(self):
        p = np.zeros(SQ_MLP_SIZE, dtype=np.float32)
        self._check(self.L.gb2_mlp_get_params(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), SQ_MLP_SIZE))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self.L.gb2_mlp_set_params(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), SQ_MLP_SIZE))

    def grad(self, samples):
        s = np.ascontiguousarray(samples, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        g = np.zeros(SQ_MLP_SIZE, dtype=np.float32)
        F = ctypes.POINTER(ctypes.c_float)
        self._check(self.L.gb2_mlp_grad(self.h, len(s), s.ctypes.data_as(F), loss.ctypes.data_as(F), g.ctypes.data_as(F)))
        return float(loss[0]), g

    def evaluate(self, n, seed):
        st = (ctypes.c_longlong * 9)()
        md = ctypes.c_double()
        self._check(self.L.gb2_mlp_evaluate(self.h, n, seed, st, ctypes.byref(md)))
        keys = ("pairs", "plain_iters", "plain_solves", "learned_iters", "learned_solves", "learned_accepted",
                "plain_fail", "learned_fail", "differ")
        out = dict(zip(keys, [int(v) for v in st]))
        out["maxdiff"] = md.value
        return out

    def time_solves(self, n, seed):
        """Device time of the first-contact solve of the same fresh pairs,
        plain homotopy against the learned guess (each launch timed alone)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        cnt = (ctypes.c_longlong * 3)()
        self._check(self.L.gb2_mlp_time_solves(self.h, n, seed, ctypes.byref(a), ctypes.byref(b), cnt))
        return {"pairs": int(cnt[0]), "plain_ms": a.value, "learned_ms": b.value,
                "plain_iters": int(cnt[1]), "learned_iters": int(cnt[2]),
                "speedup": a.value / b.value if b.value > 0 else None}
