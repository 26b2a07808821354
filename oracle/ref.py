"""Run a scenario through the reference itself (oracle/_ref/ref_harness).

TEST INFRASTRUCTURE ONLY: writes the scenario as LIGGGHTS input (a read_data
file, ASCII STL meshes and an input script in the reference's own grammar),
runs the harness built by Makefile.ref, and reads back its raw dumps.  Used by
tests/ to pin the oracle and the engine to the reference, and by bench.py's
reference arm (input writing only; that arm runs the stock lmp_ref binary).

Every number is written with %.17g, so the reference reads back the same
doubles.  The atom order is kept (atom_modify map array, sort as the scenario
says) and the data file lists atoms in the scenario's order, so the reference's
local indices equal the oracle's and the engine's.
"""
import math
import os
import shutil
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
HARNESS = os.path.join(REF_DIR, "ref_harness")
LMP = os.path.join(REF_DIR, "lmp_ref")
# the reference with the b200 suffix styles (Makefile.ref target b200)
HARNESS_B200 = os.path.join(REF_DIR, "ref_harness_b200")
LMP_B200 = os.path.join(REF_DIR, "lmp_b200")
REF_SRC = "/root/reference/src"


def available():
    return os.path.exists(HARNESS) and os.path.exists(LMP)


def build(jobs=8):
    """Build the reference (about 90 s on 8 cores) when its sources are present."""
    if available():
        return True
    if not os.path.isdir(REF_SRC):
        return False
    subprocess.run(["make", "-s", "-f", "Makefile.ref", "-j%d" % jobs, "REF=" + REF_SRC], cwd=_HERE, check=True)
    return available()


def _g(v):
    return "%.17g" % float(v)


def write_stl(path, nodes):
    """ASCII STL of (ntri, 3, 3) nodes; the reference recomputes the normals."""
    with open(path, "w") as f:
        f.write("solid b200\n")
        for t in np.asarray(nodes, dtype=np.float64):
            f.write("facet normal 0 0 0\nouter loop\n")
            for p in t:
                f.write("vertex %s %s %s\n" % (_g(p[0]), _g(p[1]), _g(p[2])))
            f.write("endloop\nendfacet\n")
        f.write("endsolid b200\n")


def write_data(path, sc, density=None):
    """read_data file (atom_style granular: id type diameter density x y z;
    Velocities: id vx vy vz wx wy wz), atoms in scenario order.  The density
    column is the scenario's per-atom density (else rmass / (4/3 pi r^3));
    the reference recomputes the mass from it, so callers compare against
    the mass it reports."""
    a = sc["atoms"]
    n = len(a["tag"])
    r = np.asarray(a["radius"], dtype=np.float64)
    if density is None:
        density = a.get("density")
    if density is None:
        density = np.asarray(a["rmass"], dtype=np.float64) / (4.0 * math.pi / 3.0 * r * r * r)
    density = np.broadcast_to(np.asarray(density, dtype=np.float64), (n,))
    lo, hi = sc["boxlo"], sc["boxhi"]
    with open(path, "w") as f:
        f.write("LIGGGHTS data file written for a parity check\n\n%d atoms\n%d atom types\n\n" % (n, sc["ntypes"]))
        for d, nm in enumerate("xyz"):
            f.write("%s %s %slo %shi\n" % (_g(lo[d]), _g(hi[d]), nm, nm))
        f.write("\nAtoms\n\n")
        x = a["x"]
        for i in range(n):
            f.write("%d %d %s %s %s %s %s\n" % (a["tag"][i], a["type"][i], _g(2.0 * r[i]), _g(density[i]),
                                                _g(x[i, 0]), _g(x[i, 1]), _g(x[i, 2])))
        f.write("\nVelocities\n\n")
        v, w = a["v"], a["omega"]
        for i in range(n):
            f.write("%d %s %s %s %s %s %s\n" % (a["tag"][i], _g(v[i, 0]), _g(v[i, 1]), _g(v[i, 2]),
                                               _g(w[i, 0]), _g(w[i, 1]), _g(w[i, 2])))


def _model(sc, rolling):
    m = "model hertz tangential history"
    if rolling:
        m += " rolling_friction cdt"
    return m


def _model_opts(sc):
    """Model keywords; a wall takes them after its geometry keywords."""
    return "" if int(sc.get("tangential_damping", 1)) else " tangential_damping off"


def _matrix(name, arr, nt):
    vals = " ".join(_g(v) for v in np.asarray(arr, dtype=np.float64).ravel())
    return "fix m_%s all property/global %s peratomtypepair %d %s" % (name, name, nt, vals)


def script(sc, workdir, segments, dump_names=None, thermo=0):
    """Input script lines for a scenario: setup plus runs of the given step
    counts.  segments[0] is the first run (0 = setup only); a "#@dump" line
    follows every segment when dump_names is given."""
    nt = sc["ntypes"]
    per = sc["periodic"]
    lines = [
        "atom_style granular",
        "atom_modify map array sort %d %s" % (int(sc.get("sortfreq", 1000)), _g(sc.get("sortbinsize", 0.0))),
        "boundary %s" % " ".join("p" if per[d] else "f" for d in range(3)),
        "newton off",
        "communicate single vel yes",
        "units si",
        "read_data %s" % os.path.join(workdir, "data.txt"),
        "neighbor %s bin" % _g(sc["skin"]),
        "neigh_modify every %d delay %d check %s" % (int(sc.get("every", 1)), int(sc.get("delay", 0)),
                                                      "yes" if int(sc.get("check", 1)) else "no"),
        "fix m_E all property/global youngsModulus peratomtype %s" % " ".join(_g(v) for v in sc["youngs"]),
        "fix m_nu all property/global poissonsRatio peratomtype %s" % " ".join(_g(v) for v in sc["poisson"]),
        _matrix("coefficientRestitution", sc["restitution"], nt),
        _matrix("coefficientFriction", sc["friction"], nt),
    ]
    rolling_any = int(sc.get("rolling_cdt", 0)) or any(int(f.get("rolling_cdt", 0)) for f in sc["fixes"])
    if rolling_any:
        lines.append(_matrix("coefficientRollingFriction", sc["rollfriction"], nt))
    lines += ["pair_style gran %s%s" % (_model(sc, int(sc.get("rolling_cdt", 0))), _model_opts(sc)), "pair_coeff * *",
              "timestep %s" % _g(sc["dt"])]
    mesh_ids = {}
    for k, fx in enumerate(sc["fixes"]):
        kind = fx["kind"]
        if kind == "gravity":
            v = fx["vector"]
            lines.append("fix f%d all gravity %s vector %s %s %s" % (k, _g(fx["magnitude"]), _g(v[0]), _g(v[1]),
                                                                     _g(v[2])))
        elif kind == "wall_plane":
            lines.append("fix f%d all wall/gran %s primitive type %d %splane %s%s" % (
                k, _model(sc, int(fx.get("rolling_cdt", 0))), fx["wall_type"], "xyz"[fx["dim"]], _g(fx["pos"]),
                _model_opts(sc)))
        elif kind == "wall_cylinder":
            lines.append("fix f%d all wall/gran %s primitive type %d %scylinder %s %s %s%s" % (
                k, _model(sc, int(fx.get("rolling_cdt", 0))), fx["wall_type"], "xyz"[fx["dim"]], _g(fx["radius"]),
                _g(fx["c1"]), _g(fx["c2"]), _model_opts(sc)))
        elif kind == "wall_mesh":
            stl = os.path.join(workdir, "mesh%d.stl" % k)
            write_stl(stl, fx["nodes"])
            cur = "" if not fx.get("curvature", 0.0) else " curvature %s" % _g(fx["curvature"])
            lines.append("fix cad%d all mesh/surface file %s type %d%s" % (k, stl, fx["wall_type"], cur))
            lines.append("fix f%d all wall/gran %s mesh n_meshes 1 meshes cad%d%s" % (
                k, _model(sc, int(fx.get("rolling_cdt", 0))), k, _model_opts(sc)))
            mesh_ids[k] = "cad%d" % k
        elif kind == "move_mesh_rotate":
            o, a = fx["origin"], fx["axis"]
            lines.append("fix f%d all move/mesh mesh %s rotate origin %s %s %s axis %s %s %s period %s" % (
                k, mesh_ids[fx["mesh"]], _g(o[0]), _g(o[1]), _g(o[2]), _g(a[0]), _g(a[1]), _g(a[2]),
                _g(fx["period"])))
        elif kind == "move_mesh_linear":
            v = fx["velocity"]
            lines.append("fix f%d all move/mesh mesh %s linear %s %s %s" % (k, mesh_ids[fx["mesh"]], _g(v[0]),
                                                                            _g(v[1]), _g(v[2])))
        elif kind == "nve_sphere":
            lines.append("fix f%d all nve/sphere" % k)
        elif kind == "insert_pack":
            lines += _insert_pack(fx, k)
        elif kind == "insert_stream":
            lines += _insert_stream(fx, k, workdir)
        else:
            raise ValueError("no reference input for fix kind %r" % kind)
    lines.append("thermo %d" % thermo)
    for s, nsteps in enumerate(segments):
        lines.append("run %d" % nsteps if s == 0 else "run %d pre no post no" % nsteps)
        if dump_names is not None:
            lines.append("#@dump %s" % dump_names[s])
    return lines


def _insert_pack(fx, k):
    """fix particletemplate/sphere (one per template), fix
    particledistribution/discrete, the region and fix insert/pack
    (src/fix_template_sphere.cpp, src/fix_particledistribution_discrete.cpp,
    src/fix_insert.cpp:118-290, src/fix_insert_pack.cpp).  The reference's
    template parses only 'radius constant' (src/fix_template_sphere.cpp:
    190-199), so scenarios with other radius styles have no reference input."""
    out = []
    names = []
    for t, tp in enumerate(fx["templates"]):
        if tp.get("radius_style", "constant") != "constant":
            raise ValueError("the reference's particletemplate/sphere takes only 'radius constant'")
        nm = "pts%d_%d" % (k, t)
        names.append(nm)
        out.append("fix %s all particletemplate/sphere %d atom_type %d density constant %s radius constant %s" % (
            nm, int(tp.get("seed", 67867967)), int(tp["type"]), _g(tp["density"]), _g(tp["radius"])))
    style = "particledistribution/discrete" if int(fx.get("dist_mass_based", 1)) else \
        "particledistribution/discrete/numberbased"
    out.append("fix pdd%d all %s %d %d %s" % (k, style, int(fx["dist_seed"]), len(names),
                                              " ".join("%s %s" % (nm, _g(tp["weight"]))
                                                       for nm, tp in zip(names, fx["templates"]))))
    cyl = fx.get("region_cylinder")
    if cyl is not None:
        out.append("region ins%d cylinder %s %s %s %s %s %s units box" % (
            k, "xyz"[int(cyl["axis"])], _g(cyl["c1"]), _g(cyl["c2"]), _g(cyl["radius"]), _g(cyl["lo"]),
            _g(cyl["hi"])))
    else:
        lo, hi = fx["region_lo"], fx["region_hi"]
        out.append("region ins%d block %s %s %s %s %s %s units box" % (
            k, _g(lo[0]), _g(hi[0]), _g(lo[1]), _g(hi[1]), _g(lo[2]), _g(hi[2])))
    yn = lambda v: "yes" if int(v) else "no"
    vs = fx.get("vel_style", "constant")
    v = fx.get("vel", (0.0, 0.0, 0.0))
    vel = "vel constant %s %s %s" % tuple(_g(c) for c in v) if vs == "constant" else \
        "vel %s %s %s %s %s %s %s" % ((vs,) + tuple(_g(c) for c in v) + tuple(_g(c) for c in fx["vel_fluct"]))
    w = fx.get("omega", (0.0, 0.0, 0.0))
    cmd = ("fix f%d all insert/pack seed %d distributiontemplate pdd%d insert_every %d maxattempt %d overlapcheck %s "
           "all_in %s random_distribute %s %s omega constant %s %s %s" % (
               k, int(fx["seed"]), k, int(fx["insert_every"]), int(fx.get("maxattempt", 50)),
               yn(fx.get("overlapcheck", 1)), yn(fx.get("all_in", 0)),
               "exact" if int(fx.get("exact_number", 1)) else "uncorrelated", vel, _g(w[0]), _g(w[1]), _g(w[2])))
    if int(fx.get("start", 0)):
        cmd += " start %d" % int(fx["start"])
    cmd += " check_dist_from_subdomain_border %s ntry_mc %d" % (yn(fx.get("check_dist_from_subdomain_border", 1)),
                                                               int(fx.get("ntry_mc", 100000)))
    for key in ("volumefraction_region", "particles_in_region", "mass_in_region"):
        if key in fx:
            cmd += " %s %s" % (key, _g(fx[key]) if key != "particles_in_region" else "%d" % int(fx[key]))
    cmd += " region ins%d" % k
    out.append(cmd)
    return out


def _distribution(fx, k):
    """fix particletemplate/sphere (one per template) and fix
    particledistribution/discrete for an insertion fix."""
    out, names = [], []
    for t, tp in enumerate(fx["templates"]):
        if tp.get("radius_style", "constant") != "constant":
            raise ValueError("the reference's particletemplate/sphere takes only 'radius constant'")
        nm = "pts%d_%d" % (k, t)
        names.append(nm)
        out.append("fix %s all particletemplate/sphere %d atom_type %d density constant %s radius constant %s" % (
            nm, int(tp.get("seed", 67867967)), int(tp["type"]), _g(tp["density"]), _g(tp["radius"])))
    style = "particledistribution/discrete" if int(fx.get("dist_mass_based", 1)) else \
        "particledistribution/discrete/numberbased"
    out.append("fix pdd%d all %s %d %d %s" % (k, style, int(fx["dist_seed"]), len(names),
                                              " ".join("%s %s" % (nm, _g(tp["weight"]))
                                                       for nm, tp in zip(names, fx["templates"]))))
    return out


def _insert_stream(fx, k, workdir):
    """The insertion face as fix mesh/surface (an STL) and fix insert/stream
    (src/fix_insert.cpp:118-290 keywords first, then
    src/fix_insert_stream.cpp:71-150's)."""
    out = _distribution(fx, k)
    stl = os.path.join(workdir, "face%d.stl" % k)
    write_stl(stl, np.asarray(fx["face_nodes"], dtype=np.float64).reshape(-1, 3, 3))
    out.append("fix face%d all mesh/surface file %s type 1" % (k, stl))
    vs = fx.get("vel_style", "constant")
    v = fx.get("vel", (0.0, 0.0, 0.0))
    vel = "vel constant %s %s %s" % tuple(_g(c) for c in v) if vs == "constant" else \
        "vel %s %s %s %s %s %s %s" % ((vs,) + tuple(_g(c) for c in v) + tuple(_g(c) for c in fx["vel_fluct"]))
    w = fx.get("omega", (0.0, 0.0, 0.0))
    yn = lambda v: "yes" if int(v) else "no"
    cmd = "fix f%d all insert/stream seed %d distributiontemplate pdd%d" % (k, int(fx["seed"]), k)
    if fx.get("nparticles") is not None:
        cmd += " nparticles %s" % ("INF" if fx["nparticles"] == "INF" else "%d" % int(fx["nparticles"]))
    if fx.get("mass") is not None:
        cmd += " mass %s" % ("INF" if fx["mass"] == "INF" else _g(fx["mass"]))
    if fx.get("particlerate"):
        cmd += " particlerate %s" % _g(fx["particlerate"])
    if fx.get("massrate"):
        cmd += " massrate %s" % _g(fx["massrate"])
    if int(fx.get("insert_every", -1)) > 0:
        cmd += " insert_every %d" % int(fx["insert_every"])
    if int(fx.get("start", 0)):
        cmd += " start %d" % int(fx["start"])
    cmd += " maxattempt %d overlapcheck %s all_in no random_distribute %s %s omega constant %s %s %s" % (
        int(fx.get("maxattempt", 50)), yn(fx.get("overlapcheck", 1)),
        "exact" if int(fx.get("exact_number", 1)) else "uncorrelated", vel, _g(w[0]), _g(w[1]), _g(w[2]))
    cmd += " insertion_face face%d" % k
    if float(fx.get("extrude_length", 0.0)) > 0:
        cmd += " extrude_length %s" % _g(fx["extrude_length"])
    if int(fx.get("duration", 0)):
        cmd += " duration %d" % int(fx["duration"])
    cmd += " ntry_mc %d" % int(fx.get("ntry_mc", 100000))
    out.append(cmd)
    return out


def read_dump(path):
    """Records of one harness dump as {name: array} (scalars as Python floats)."""
    out = {}
    with open(path, "rb") as f:
        buf = f.read()
    p = 0
    while p < len(buf):
        name = buf[p:p + 32].split(b"\0", 1)[0].decode()
        typ = chr(buf[p + 32])
        ncol = int(np.frombuffer(buf, np.int32, 1, p + 33)[0])
        nrow = int(np.frombuffer(buf, np.int64, 1, p + 37)[0])
        p += 45
        dt = np.float64 if typ == "d" else np.int32
        cnt = nrow * ncol
        arr = np.frombuffer(buf, dt, cnt, p).copy()
        p += cnt * np.dtype(dt).itemsize
        arr = arr.reshape(nrow, ncol) if ncol > 1 else arr
        out[name] = arr
    for k in ("ntimestep", "ncalls", "nlocal", "nghost"):
        if k in out:
            out[k] = float(out[k][0])
    return out


def available_b200():
    return os.path.exists(HARNESS_B200) and os.path.exists(LMP_B200)


def build_b200(jobs=8):
    """Build the reference with the b200 suffix styles (needs the built
    libgranb200.so and the reference sources)."""
    if available_b200():
        return True
    if not os.path.isdir(REF_SRC) or not build(jobs):
        return False
    subprocess.run(["make", "-s", "-f", "Makefile.ref", "-j%d" % jobs, "REF=" + REF_SRC, "b200"], cwd=_HERE,
                   check=True)
    return available_b200()


def restart_script(sc, workdir, n_before, segments):
    """A run of n_before steps that ends in write_restart, then clear and
    read_restart (src/write_restart.cpp, src/read_restart.cpp) and the given
    segments with a dump after each.  The restart file carries the box, the
    atoms with their per-atom fix data (pair contact history, primitive-wall
    history, mesh contact slots), the pair settings and the global fix state
    (mesh nodes, the mover's time); neighbour and communication settings,
    materials, the timestep, newton pair and every fix are given again,
    under the same fix ids, so their restart data is applied to them."""
    first = script(sc, workdir, [n_before])
    path = os.path.join(workdir, "phase1.restart")
    out = first + ["write_restart %s" % path, "clear"]
    second = script(sc, workdir, segments, ["s%d" % i for i in range(len(segments))])
    skip = ("atom_style", "boundary", "newton", "units", "communicate")
    for line in second:
        if line.startswith(skip):
            continue
        if line.startswith("read_data"):
            # newton pair follows the script, not the file (src/read_restart.cpp)
            out += ["read_restart %s" % path, "newton off", "communicate single vel yes"]
            continue
        out.append(line)
    return out


def run_restart(sc, n_before, segments, keep=None):
    """The scenario through a real restart file: one dump per segment after
    the restart (see restart_script)."""
    return run(sc, segments, keep=keep, script_lines=lambda wd: restart_script(sc, wd, n_before, segments))


def run(sc, segments, keep=None, harness=None, extra_args=(), script_lines=None):
    """Run the scenario in the reference: setup + segments[0] steps, then
    each further segment as a continued run; returns one dump per segment.
    harness/extra_args select another harness build and LAMMPS command-line
    arguments (e.g. HARNESS_B200 with "-sf b200"); script_lines replaces the
    generated input script (its "#@dump s<k>" lines name the dumps)."""
    harness = harness or HARNESS
    if not os.path.exists(harness):
        raise RuntimeError("reference harness not built (oracle/Makefile.ref)")
    wd = keep or tempfile.mkdtemp(prefix="gb2ref_")
    os.makedirs(wd, exist_ok=True)
    try:
        write_data(os.path.join(wd, "data.txt"), sc)
        names = ["s%d" % i for i in range(len(segments))]
        lines = script(sc, wd, segments, names) if script_lines is None else script_lines(wd)
        with open(os.path.join(wd, "in.case"), "w") as f:
            f.write("\n".join(lines) + "\n")
        # the reference's messages may hold stray non-UTF-8 bytes (an error
        # line printing an unterminated keyword buffer): decode leniently
        r = subprocess.run([harness, os.path.join(wd, "in.case"), wd] + list(extra_args), capture_output=True,
                           text=True, errors="replace")
        if r.returncode != 0 or not os.path.exists(os.path.join(wd, names[-1] + ".bin")):
            tail = ""
            for fn in ("screen.txt", "log.lammps"):
                p = os.path.join(wd, fn)
                if os.path.exists(p):
                    with open(p, errors="replace") as f:
                        tail += f.read()[-3000:]
            raise RuntimeError("reference run failed (rc %d): %s %s" % (r.returncode, r.stderr[-2000:], tail))
        return [read_dump(os.path.join(wd, n + ".bin")) for n in names]
    finally:
        if keep is None:
            shutil.rmtree(wd, ignore_errors=True)


def with_ref_mass(sc, dump):
    """The scenario with radius and mass as the reference read them (the
    reference derives the mass from diameter and density itself)."""
    out = dict(sc)
    a = dict(sc["atoms"])
    order = np.argsort(dump["tag"])
    idx = np.searchsorted(dump["tag"][order], a["tag"])
    a["radius"] = dump["radius"][order][idx].copy()
    a["rmass"] = dump["rmass"][order][idx].copy()
    out["atoms"] = a
    return out
