/*
 * ref_harness.cpp -- runs an input script through the reference library
 * (LIGGGHTS-PUBLIC 3.8.0 built by Makefile.ref) and dumps its raw state.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that pins the oracle and the engine to
 * the reference itself.  Nothing in the product links or runs it.
 *
 *   ref_harness <script> <outdir> [lammps command-line arguments...]
 *
 * (e.g. "-sf b200" on the build that includes the b200 suffix styles).
 * Every script line goes to lammps_command (src/library.cpp:129) on an
 * instance made by lammps_open_no_mpi (src/library.cpp:88), except lines
 * "#@dump <name>", which write <outdir>/<name>.bin, and other comments.
 *
 * A dump is a sequence of records: a 32-byte zero-padded name, one type byte
 * ('d' double, 'i' int32), int32 columns, int64 rows, then rows*columns
 * values (little endian, no text rounding).  Records:
 *   scalars            ntimestep, ncalls (Neighbor::ncalls), nlocal, nghost
 *   per owned atom     tag type x v omega f torque radius rmass (local order)
 *   pair list          pair_i pair_j (tags), pair_flag, pair_hist, walking
 *                      PairGran::list and listgranhistory exactly as
 *                      Granular<>::compute_force does (src/pair_gran_base.h:
 *                      213-270): ilist order, then each atom's j order
 *   partners           cp_n, cp_tag, cp_hist: FixContactHistory::npartner_,
 *                      partner_, contacthistory_ (src/fix_contact_history.h:
 *                      122-124), i.e. the state of the last pre_exchange
 *   per wall/gran fix  w<k>_hist: primitive wall history per owned atom
 *                      (FixWallGran::fix_history_primitive_); for a mesh wall
 *                      w<k>_nn (FixContactHistoryMesh::nneighs), w<k>_tag,
 *                      w<k>_tri, w<k>_hist (occupied slots, i then slot
 *                      order, src/fix_contact_history_mesh.h), w<k>_nodes and
 *                      w<k>_vnode (TriMesh nodes, node velocity property "v"),
 *                      w<k>_geom (per element: centre 3, bounding radius,
 *                      unit edge vectors 9, edge lengths 3, edge normals 9,
 *                      surface normal 3, mesh precision)
 * The reference's classes keep these members protected; the harness is a
 * test tool, so it opens them by redefining the access keywords while it
 * includes the reference headers (the class layouts do not depend on them).
 */
#include <mpi.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <list>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#define protected public
#define private public
#include "lammps.h"
#include "library.h"
#include "atom.h"
#include "force.h"
#include "pair.h"
#include "pair_gran.h"
#include "neigh_list.h"
#include "neighbor.h"
#include "modify.h"
#include "fix.h"
#include "fix_contact_history.h"
#include "fix_contact_history_mesh.h"
#include "fix_wall_gran.h"
#include "fix_mesh_surface.h"
#include "fix_property_atom.h"
#include "tri_mesh.h"
#include "update.h"
#undef protected
#undef private

using namespace LAMMPS_NS;

namespace {

struct Dump {
    FILE *f;
    void rec(const char *name, char type, int ncol, int64_t nrow, const void *data)
    {
        char nm[32];
        memset(nm, 0, sizeof(nm));
        strncpy(nm, name, 31);
        fwrite(nm, 1, 32, f);
        fputc(type, f);
        int32_t c = ncol;
        fwrite(&c, 4, 1, f);
        fwrite(&nrow, 8, 1, f);
        size_t sz = (type == 'd' ? 8 : 4);
        if (nrow * ncol > 0) fwrite(data, sz, (size_t)(nrow * ncol), f);
    }
    void scalar(const char *name, double v) { rec(name, 'd', 1, 1, &v); }
};

void dump_state(LAMMPS *lmp, const std::string &path)
{
    Dump d;
    d.f = fopen(path.c_str(), "wb");
    if (!d.f) {
        fprintf(stderr, "ref_harness: cannot write %s\n", path.c_str());
        exit(2);
    }
    Atom *atom = lmp->atom;
    const int nlocal = atom->nlocal;
    d.scalar("ntimestep", (double)lmp->update->ntimestep);
    d.scalar("ncalls", (double)lmp->neighbor->ncalls);
    d.scalar("nlocal", (double)nlocal);
    d.scalar("nghost", (double)atom->nghost);
    d.rec("tag", 'i', 1, nlocal, atom->tag);
    d.rec("type", 'i', 1, nlocal, atom->type);
    d.rec("x", 'd', 3, nlocal, nlocal ? atom->x[0] : NULL);
    d.rec("v", 'd', 3, nlocal, nlocal ? atom->v[0] : NULL);
    d.rec("omega", 'd', 3, nlocal, nlocal ? atom->omega[0] : NULL);
    d.rec("f", 'd', 3, nlocal, nlocal ? atom->f[0] : NULL);
    d.rec("torque", 'd', 3, nlocal, nlocal ? atom->torque[0] : NULL);
    d.rec("radius", 'd', 1, nlocal, atom->radius);
    d.rec("rmass", 'd', 1, nlocal, atom->rmass);

    PairGran *pg = dynamic_cast<PairGran *>(lmp->force->pair);
    if (pg && pg->list) {
        NeighList *list = pg->list;
        NeighList *hl = pg->listgranhistory;
        const int dnum = hl ? hl->dnum : 0;
        std::vector<int> pi, pj, pf;
        std::vector<double> ph;
        for (int ii = 0; ii < list->inum; ii++) {
            const int i = list->ilist[ii];
            const int *jlist = list->firstneigh[i];
            for (int jj = 0; jj < list->numneigh[i]; jj++) {
                const int j = jlist[jj] & NEIGHMASK;
                pi.push_back(atom->tag[i]);
                pj.push_back(atom->tag[j]);
                pf.push_back(hl ? hl->firstneigh[i][jj] : 0);
                for (int k = 0; k < dnum; k++) ph.push_back(hl->firstdouble[i][dnum * jj + k]);
            }
        }
        d.rec("pair_i", 'i', 1, (int64_t)pi.size(), pi.data());
        d.rec("pair_j", 'i', 1, (int64_t)pj.size(), pj.data());
        d.rec("pair_flag", 'i', 1, (int64_t)pf.size(), pf.data());
        d.rec("pair_hist", 'd', dnum > 0 ? dnum : 1, dnum > 0 ? (int64_t)pi.size() : 0, ph.data());
        FixContactHistory *ch = pg->fix_history;
        if (ch && ch->npartner_) {
            std::vector<int> pt;
            std::vector<double> hh;
            const int dn = ch->dnum_;
            for (int i = 0; i < nlocal; i++)
                for (int k = 0; k < ch->npartner_[i]; k++) {
                    pt.push_back(ch->partner_[i][k]);
                    for (int q = 0; q < dn; q++) hh.push_back(ch->contacthistory_[i][k * dn + q]);
                }
            d.rec("cp_n", 'i', 1, nlocal, ch->npartner_);
            d.rec("cp_tag", 'i', 1, (int64_t)pt.size(), pt.data());
            d.rec("cp_hist", 'd', dn > 0 ? dn : 1, dn > 0 ? (int64_t)pt.size() : 0, hh.data());
        }
    }

    int k = 0;
    for (int ifix = 0; ifix < lmp->modify->nfix; ifix++) {
        Fix *fx = lmp->modify->fix[ifix];
        if (strncmp(fx->style, "wall/gran", 9) != 0) continue;   // wall/gran and its suffixed forms
        FixWallGran *fw = dynamic_cast<FixWallGran *>(fx);
        char nm[32];
        if (!fw->is_mesh_wall()) {
            FixPropertyAtom *h = fw->fix_history_primitive_;
            if (h && h->array_atom) {
                snprintf(nm, sizeof(nm), "w%d_hist", k);
                d.rec(nm, 'd', h->nvalues, nlocal, nlocal ? h->array_atom[0] : NULL);
            }
        } else {
            for (int im = 0; im < fw->n_meshes(); im++) {
                FixMeshSurface *fm = fw->mesh_list()[im];
                FixContactHistoryMesh *cm = fm->contactHistory();
                TriMesh *mesh = fm->triMesh();
                std::vector<int> nn(nlocal), tg, tr;
                std::vector<double> hh;
                const int dn = cm ? cm->dnum_ : 0;
                for (int i = 0; i < nlocal; i++) {
                    nn[i] = cm ? cm->nneighs(i) : 0;
                    for (int s = 0; s < nn[i]; s++) {
                        if (cm->partner_[i][s] < 0) continue;
                        tg.push_back(atom->tag[i]);
                        tr.push_back(cm->partner_[i][s]);
                        for (int q = 0; q < dn; q++) hh.push_back(cm->contacthistory_[i][s * dn + q]);
                    }
                }
                const char *suffix = im == 0 ? "" : "m";
                snprintf(nm, sizeof(nm), "w%d%s%d_nn", k, suffix, im);
                if (im == 0) snprintf(nm, sizeof(nm), "w%d_nn", k);
                d.rec(nm, 'i', 1, nlocal, nn.data());
                if (im == 0) snprintf(nm, sizeof(nm), "w%d_tag", k); else snprintf(nm, sizeof(nm), "w%dm%d_tag", k, im);
                d.rec(nm, 'i', 1, (int64_t)tg.size(), tg.data());
                if (im == 0) snprintf(nm, sizeof(nm), "w%d_tri", k); else snprintf(nm, sizeof(nm), "w%dm%d_tri", k, im);
                d.rec(nm, 'i', 1, (int64_t)tr.size(), tr.data());
                if (im == 0) snprintf(nm, sizeof(nm), "w%d_hist", k); else snprintf(nm, sizeof(nm), "w%dm%d_hist", k, im);
                d.rec(nm, 'd', dn > 0 ? dn : 1, dn > 0 ? (int64_t)tg.size() : 0, hh.data());
                const int nt = mesh->sizeLocal();
                std::vector<double> nodes(9 * (size_t)nt), vel(9 * (size_t)nt, 0.0);
                MultiVectorContainer<double, 3, 3> *v =
                    mesh->prop().getElementProperty<MultiVectorContainer<double, 3, 3> >("v");
                for (int t = 0; t < nt; t++)
                    for (int a = 0; a < 3; a++)
                        for (int c = 0; c < 3; c++) {
                            nodes[9 * t + 3 * a + c] = mesh->node_(t)[a][c];
                            if (v) vel[9 * t + 3 * a + c] = (*v)(t)[a][c];
                        }
                if (im == 0) snprintf(nm, sizeof(nm), "w%d_nodes", k); else snprintf(nm, sizeof(nm), "w%dm%d_nodes", k, im);
                d.rec(nm, 'd', 9, nt, nodes.data());
                if (im == 0) snprintf(nm, sizeof(nm), "w%d_vnode", k); else snprintf(nm, sizeof(nm), "w%dm%d_vnode", k, im);
                d.rec(nm, 'd', 9, nt, vel.data());
                // element geometry as the contact code reads it: centre, bounding
                // radius, unit edge vectors, edge lengths, edge normals, normal
                std::vector<double> geom(29 * (size_t)nt);
                for (int t = 0; t < nt; t++) {
                    double *g = &geom[29 * (size_t)t];
                    for (int c = 0; c < 3; c++) g[c] = mesh->center_(t)[c];
                    g[3] = mesh->rBound_(t);
                    for (int a = 0; a < 3; a++)
                        for (int c = 0; c < 3; c++) {
                            g[4 + 3 * a + c] = mesh->edgeVec(t)[a][c];
                            g[16 + 3 * a + c] = mesh->edgeNorm(t)[a][c];
                        }
                    for (int a = 0; a < 3; a++) g[13 + a] = mesh->edgeLen(t)[a];
                    for (int c = 0; c < 3; c++) g[25 + c] = mesh->surfaceNorm(t)[c];
                    g[28] = mesh->precision_trimesh();
                }
                if (im == 0) snprintf(nm, sizeof(nm), "w%d_geom", k); else snprintf(nm, sizeof(nm), "w%dm%d_geom", k, im);
                d.rec(nm, 'd', 29, nt, geom.data());
            }
        }
        k++;
    }
    fclose(d.f);
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: ref_harness <script> <outdir> [lammps arguments...]\n");
        return 2;
    }
    std::ifstream in(argv[1]);
    if (!in) {
        fprintf(stderr, "ref_harness: cannot read %s\n", argv[1]);
        return 2;
    }
    const std::string out = argv[2];
    const std::string logf = out + "/log.lammps", scr = out + "/screen.txt";
    std::vector<char *> args = {(char *)"ref_harness", (char *)"-log", (char *)logf.c_str(), (char *)"-screen",
                                (char *)scr.c_str(), (char *)"-echo", (char *)"log"};
    for (int a = 3; a < argc; a++) args.push_back(argv[a]);
    args.push_back(NULL);
    void *handle = NULL;
    lammps_open_no_mpi((int)args.size() - 1, args.data(), &handle);
    LAMMPS *lmp = (LAMMPS *)handle;
    std::string line;
    while (std::getline(in, line)) {
        size_t a = line.find_first_not_of(" \t\r");
        if (a == std::string::npos) continue;
        line = line.substr(a);
        if (line.compare(0, 7, "#@dump ") == 0) {
            std::string name = line.substr(7);
            name.erase(name.find_last_not_of(" \t\r") + 1);
            dump_state(lmp, out + "/" + name + ".bin");
            continue;
        }
        if (line[0] == '#') continue;
        lammps_command(lmp, (char *)line.c_str());
    }
    lammps_close(handle);
    return 0;
}
