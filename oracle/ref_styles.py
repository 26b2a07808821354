"""Generate the style headers a LIGGGHTS build needs, into a directory of ours.

TEST INFRASTRUCTURE ONLY (part of the recipe that builds the reference as the
checker under oracle/_ref/).  The reference's own build writes these headers
into its source tree (src/Make.sh:12-100 `style`, :101-300 `models`); the
source tree here is read-only, so this script writes the same content into
the directory given on the command line and the compile puts that directory
on the include path.

* style_<prefix>.h: one `#include "<file>"` per header in src whose name
  starts with the class prefix and which contains the class macro, in glob
  (byte) order, as `grep -sl MACRO prefix*.h` lists them (src/Make.sh:34).
* version_liggghts.h: the LIGGGHTS_VERSION string (src/Make.sh:14-29).
* style_contact_model.h: the GRAN_MODEL whitelist.  With more than 1200
  model combinations the reference keeps a combination when the product of
  its (id + 1) values is below 30 and its tangential model is not "off"
  (src/Make.sh:213-252); the same rule is applied here, so the compiled set
  of template-optimised models is the stock one (Hertz/history with and
  without rolling cdt on the default surface among them; superquadric
  surfaces run through the runtime-dispatch path, as in a stock build).
"""
import glob
import os
import re
import sys

# (macro, header prefix, style file prefix) -- src/Make.sh:80-104
STYLES = [
    ("ANGLE_CLASS", "angle_", "angle"),
    ("ATOM_CLASS", "atom_vec_", "atom"),
    ("BODY_CLASS", "body_", "body"),
    ("BOND_CLASS", "bond_", "bond"),
    ("COMMAND_CLASS", "", "command"),
    ("COMPUTE_CLASS", "compute_", "compute"),
    ("DIHEDRAL_CLASS", "dihedral_", "dihedral"),
    ("DUMP_CLASS", "dump_", "dump"),
    ("FIX_CLASS", "fix_", "fix"),
    ("IMPROPER_CLASS", "improper_", "improper"),
    ("INTEGRATE_CLASS", "", "integrate"),
    ("KSPACE_CLASS", "", "kspace"),
    ("MINIMIZE_CLASS", "min_", "minimize"),
    ("PAIR_CLASS", "pair_", "pair"),
    ("SURFACE_MODEL", "surface_model_", "surface_model"),
    ("NORMAL_MODEL", "normal_model_", "normal_model"),
    ("TANGENTIAL_MODEL", "tangential_model_", "tangential_model"),
    ("COHESION_MODEL", "cohesion_model_", "cohesion_model"),
    ("ROLLING_MODEL", "rolling_model_", "rolling_model"),
    ("READER_CLASS", "reader_", "reader"),
    ("REGION_CLASS", "region_", "region"),
    ("CFD_DATACOUPLING_CLASS", "cfd_datacoupling_", "cfd_datacoupling"),
    ("CFD_REGIONMODEL_CLASS", "cfd_regionmodel_", "cfd_regionmodel"),
    ("LB_CLASS", "", "lb"),
    ("SPH_KERNEL_CLASS", "sph_kernel_", "sph_kernel"),
    ("MESHMODULE_CLASS", "mesh_module_", "mesh_module"),
    ("MESHMOVER_CLASS", "mesh_mover_", "mesh_mover"),
]


def _write(path, text):
    old = None
    if os.path.exists(path):
        with open(path) as f:
            old = f.read()
    if old != text:            # keep timestamps of unchanged headers (no needless recompiles)
        with open(path, "w") as f:
            f.write(text)


def _models(src, kind):
    """(name, id) of every <KIND>_MODEL(name, keyword, id) line, in glob order."""
    out = []
    pat = re.compile(r"^%s_MODEL\((.+),\s*(.+),\s*(.+)\)" % kind)
    for h in sorted(glob.glob(os.path.join(src, "%s_model_*.h" % kind.lower()))):
        with open(h, errors="replace") as f:
            for line in f:
                m = pat.match(line)
                if m:
                    out.append((m.group(1).strip(), int(m.group(3).strip())))
    return out


def contact_whitelist(src):
    surf = _models(src, "SURFACE")
    norm = _models(src, "NORMAL")
    tang = [("TANGENTIAL_OFF", 0)] + _models(src, "TANGENTIAL")
    coh = [("COHESION_OFF", 0)] + _models(src, "COHESION")
    roll = [("ROLLING_OFF", 0)] + _models(src, "ROLLING")
    # the "off" entries count as 1; the others as id + 1 (src/Make.sh:150-190)
    def val(lst):
        return [(n, 1 if n.endswith("_OFF") else i + 1) for n, i in lst]
    surf, norm, tang, coh, roll = val(surf), val(norm), val(tang), val(coh), val(roll)
    ncomb = len(surf) * len(norm) * len(tang) * len(coh) * len(roll)
    lines = []
    for s, v1 in surf:
        for nm, v2 in norm:
            for t, v3 in tang:
                for c, v4 in coh:
                    for r, v5 in roll:
                        res = v1 * v2 * v3 * v4 * v5
                        if (res < 30 and v3 > 1) or ncomb <= 1200:
                            lines.append("GRAN_MODEL(%s, %s, %s, %s, %s)\n" % (nm, t, c, r, s))
    return "".join(lines)


def main(src, out, extra=()):
    """Style headers for the sources in src plus the style files in the
    directories `extra` (the b200 suffix styles, as if dropped into src)."""
    os.makedirs(out, exist_ok=True)
    for macro, prefix, name in STYLES:
        files = []
        for d in (src,) + tuple(extra):
            for h in glob.glob(os.path.join(d, prefix + "*.h")):
                with open(h, errors="replace") as f:
                    if macro in f.read():
                        files.append(os.path.basename(h))
        files.sort()
        _write(os.path.join(out, "style_%s.h" % name), "".join('#include "%s"\n' % b for b in files))
    with open(os.path.join(src, "version_liggghts.txt")) as f:
        vers = f.read().strip()
    with open(os.path.join(src, "version_liggghts_branch.txt")) as f:
        bra = f.read().strip()
    _write(os.path.join(out, "version_liggghts.h"),
           '#define LIGGGHTS_VERSION "%s %s, reference build for parity checks"\n' % (bra, vers))
    _write(os.path.join(out, "style_contact_model.h"), contact_whitelist(src))


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2], tuple(sys.argv[3:]))
