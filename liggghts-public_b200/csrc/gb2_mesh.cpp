// gb2_mesh.cpp -- host-side triangle-mesh import and topology.
//
// Reproduces what FixMeshSurface does once at load (LIGGGHTS-PUBLIC 3.8.0):
//   * MultiNodeMesh::addElement (src/multi_node_mesh_I.h:139): drop elements
//     with coincident nodes, centre = node mean, rBound = max centre-node
//     distance;
//   * SurfaceMesh::calcSurfPropertiesOfNewElement (src/surface_mesh_I.h:282):
//     unit edge vectors and lengths, surface normal, in-plane edge normals,
//     obtuse-angle index (each per-node call overwrites the element's index,
//     so the last node decides, as in the reference);
//   * SurfaceMesh::buildNeighbours / handleSharedEdge / handleCorner
//     (src/surface_mesh_I.h:453-555, 1035-1152): an edge shared by two
//     non-coplanar (or overlapping coplanar) elements stays active only on
//     the element with the larger id, a coplanar shared edge is inactive on
//     both; a corner is active only on the largest-id element around the
//     node, and only if some edge there is active and no two edges through
//     the node are colinear;
//   * SurfaceMesh::areCoplanarNodeNeighs (src/surface_mesh_I.h:892), which
//     the mesh contact history uses for face contacts.
//
// The reference finds candidate element pairs with a bounding-sphere search
// and walks node neighbourhoods recursively.  Here candidate pairs come from
// a hash grid over node coordinates and the node neighbourhood is a
// breadth-first search over edge neighbours; both enumerate the same sets.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "gb2_internal.h"

namespace gb2 {

namespace {

inline bool comp_double(double a, double b, double prec)
{
    if (a == b) return true;
    if (b == 0) return a < prec && a > -prec;
    const double x = (a - b);
    return x < prec && x > -prec;
}

inline bool nodes_equal(const double *a, const double *b, double prec)
{
    return comp_double(a[0], b[0], prec) && comp_double(a[1], b[1], prec) && comp_double(a[2], b[2], prec);
}

inline double dotv(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double magv(const double *v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
inline void crossv(const double *a, const double *b, double *r)
{
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
inline void scale_inv(double *v, double s)
{
    const double sinv = 1. / s;
    v[0] = sinv * v[0];
    v[1] = sinv * v[1];
    v[2] = sinv * v[2];
}

struct CellKey {
    int64_t x, y, z;
    bool operator==(const CellKey &o) const { return x == o.x && y == o.y && z == o.z; }
};
struct CellHash {
    size_t operator()(const CellKey &k) const
    {
        return (size_t)(k.x * 73856093ll) ^ (size_t)(k.y * 19349663ll) ^ (size_t)(k.z * 83492791ll);
    }
};

}  // namespace

bool build_mesh_topology(const double *nodes, int ntri_in, double curvature, double precision, MeshTopo &out,
                         std::string &err)
{
    out.tri.clear();
    std::vector<TriGeom> &T = out.tri;
    T.reserve(ntri_in);
    for (int t = 0; t < ntri_in; t++) {
        const double *nd = nodes + 9 * t;
        if (nodes_equal(nd, nd + 3, precision) || nodes_equal(nd + 3, nd + 6, precision) ||
            nodes_equal(nd, nd + 6, precision))
            continue;
        TriGeom g;
        std::memset(&g, 0, sizeof g);
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++) g.node[k][c] = nd[3 * k + c];
        double avg[3] = {0., 0., 0.};
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++) avg[c] = g.node[k][c] + avg[c];
        scale_inv(avg, 3.0);
        std::memcpy(g.center, avg, sizeof avg);
        double rb = 0.;
        for (int k = 0; k < 3; k++) {
            double vec[3] = {g.center[0] - g.node[k][0], g.center[1] - g.node[k][1], g.center[2] - g.node[k][2]};
            rb = std::max(rb, magv(vec));
        }
        g.rbound = rb;
        for (int k = 0; k < 3; k++) {
            for (int c = 0; c < 3; c++) g.edgevec[k][c] = g.node[(k + 1) % 3][c] - g.node[k][c];
            g.edgelen[k] = magv(g.edgevec[k]);
            scale_inv(g.edgevec[k], g.edgelen[k]);
        }
        crossv(g.edgevec[0], g.edgevec[1], g.surfnorm);
        if (magv(g.surfnorm) < 1e-15) crossv(g.edgevec[1], g.edgevec[2], g.surfnorm);
        if (magv(g.surfnorm) < 1e-15) crossv(g.edgevec[2], g.edgevec[0], g.surfnorm);
        if (magv(g.surfnorm) < 1e-15) {
            err = "mesh element " + std::to_string(t) + " is degenerate (no surface normal)";
            return false;
        }
        scale_inv(g.surfnorm, magv(g.surfnorm));
        for (int k = 0; k < 3; k++) {
            crossv(g.edgevec[k], g.surfnorm, g.edgenorm[k]);
            if (magv(g.edgenorm[k]) < 1e-15)
                std::memcpy(g.edgenorm[k], g.edgevec[(k + 1) % 3], sizeof(double) * 3);
            else
                scale_inv(g.edgenorm[k], magv(g.edgenorm[k]));
        }
        g.obtuse = -1;
        for (int k = 0; k < 3; k++) g.obtuse = dotv(g.edgevec[k], g.edgevec[(k + 2) % 3]) > 0. ? k : -1;
        g.active = 0x3f;   // all edges and corners active until topology says otherwise
        T.push_back(g);
    }
    const int n = (int)T.size();

    // candidate pairs: elements owning a node equal (within `precision`) to
    // one of the element's nodes.  Node entries are sorted by their hash cell
    // (side 1000 x precision); equal nodes share a cell unless they sit within
    // `precision` of a cell face, so a node looks into a neighbouring cell
    // only along the axes where it is that close to a face.
    const double cell = std::max(1e3 * precision, 1e-9);
    const double near_face = 2.0 * precision / cell;   // in cell units, with a margin for rounding
    struct NodeEnt {
        int64_t x, y, z;
        int t;
        bool operator<(const NodeEnt &o) const
        {
            return x != o.x ? x < o.x : (y != o.y ? y < o.y : (z != o.z ? z < o.z : t < o.t));
        }
    };
    std::vector<NodeEnt> ents;
    ents.reserve((size_t)3 * n);
    for (int t = 0; t < n; t++)
        for (int k = 0; k < 3; k++) {
            const double *p = T[t].node[k];
            ents.push_back(NodeEnt{(int64_t)std::floor(p[0] / cell), (int64_t)std::floor(p[1] / cell),
                                   (int64_t)std::floor(p[2] / cell), t});
        }
    std::sort(ents.begin(), ents.end());
    std::vector<std::vector<int>> cand(n);
    for (int t = 0; t < n; t++) {
        for (int k = 0; k < 3; k++) {
            const double *p = T[t].node[k];
            int64_t c[3];
            int lo[3], hi[3];
            for (int d = 0; d < 3; d++) {
                const double q = p[d] / cell;
                c[d] = (int64_t)std::floor(q);
                const double fr = q - (double)c[d];
                lo[d] = fr < near_face ? -1 : 0;
                hi[d] = 1.0 - fr < near_face ? 1 : 0;
            }
            for (int dx = lo[0]; dx <= hi[0]; dx++)
                for (int dy = lo[1]; dy <= hi[1]; dy++)
                    for (int dz = lo[2]; dz <= hi[2]; dz++) {
                        const NodeEnt key{c[0] + dx, c[1] + dy, c[2] + dz, -1};
                        for (auto it = std::lower_bound(ents.begin(), ents.end(), key);
                             it != ents.end() && it->x == key.x && it->y == key.y && it->z == key.z; ++it)
                            if (it->t != t) cand[t].push_back(it->t);
                    }
        }
        std::sort(cand[t].begin(), cand[t].end());
        cand[t].erase(std::unique(cand[t].begin(), cand[t].end()), cand[t].end());
    }

    auto bsphere_overlap = [&](int a, int b) {
        const double d[3] = {T[a].center[0] - T[b].center[0], T[a].center[1] - T[b].center[1],
                             T[a].center[2] - T[b].center[2]};
        const double rs = T[a].rbound + T[b].rbound;
        return !(d[0] * d[0] + d[1] * d[1] + d[2] * d[2] > rs * rs);
    };
    auto n_shared = [&](int a, int b) {
        if (!bsphere_overlap(a, b)) return 0;
        int ns = 0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                if (nodes_equal(T[a].node[i], T[b].node[j], precision)) ns++;
        return ns;
    };

    // shared edges
    out.edge_neigh.assign(n, {});
    std::vector<uint8_t> edge_active((size_t)3 * n, 1);
    for (int a = 0; a < n; a++)
        for (int b : cand[a]) {
            if (b >= a) continue;
            if (!bsphere_overlap(a, b)) continue;
            int ia[2], jb[2], ns = 0;
            for (int i = 0; i < 3 && ns < 2; i++)
                for (int j = 0; j < 3 && ns < 2; j++)
                    if (nodes_equal(T[a].node[i], T[b].node[j], precision)) {
                        ia[ns] = i;
                        jb[ns] = j;
                        ns++;
                    }
            if (ns < 2) continue;
            const int ea = (2 == ia[0] + ia[1]) ? 2 : std::min(ia[0], ia[1]);
            const int eb = (2 == jb[0] + jb[1]) ? 2 : std::min(jb[0], jb[1]);
            out.edge_neigh[a].push_back(b);
            out.edge_neigh[b].push_back(a);
            const bool coplanar = std::fabs(dotv(T[a].surfnorm, T[b].surfnorm)) >= curvature;
            bool overlap = false;
            if (coplanar) {
                const double *pRef = T[a].node[ea];
                const double *eN = T[a].edgenorm[ea];
                const double *na = T[a].node[(ea + 2) % 3];
                const double *nb = T[b].node[(eb + 2) % 3];
                const double vI[3] = {na[0] - pRef[0], na[1] - pRef[1], na[2] - pRef[2]};
                const double vJ[3] = {nb[0] - pRef[0], nb[1] - pRef[1], nb[2] - pRef[2]};
                overlap = dotv(vI, eN) * dotv(vJ, eN) > 0.;
            }
            if (!coplanar || overlap) {
                // the element with the larger id keeps the edge
                edge_active[3 * a + ea] = (a < b) ? 0 : 1;
                edge_active[3 * b + eb] = (a < b) ? 1 : 0;
            } else {
                edge_active[3 * a + ea] = 0;
                edge_active[3 * b + eb] = 0;
            }
        }

    // corners.  The walk from corner (t, k) over edge neighbours that hold a
    // copy of the node reaches the same elements from any of them, so it runs
    // once per such group and settles every member's corner: active only at
    // the group's largest element id, when an edge at the node is active and
    // no two of its edges are colinear.
    std::vector<uint8_t> corner_active((size_t)3 * n, 1), corner_done((size_t)3 * n, 0);
    std::vector<int> mark(n, -1), queue, members;
    std::vector<const double *> evec, eend;
    int stamp = 0;
    for (int t = 0; t < n; t++)
        for (int k = 0; k < 3; k++) {
            if (corner_done[3 * t + k]) continue;
            const double *nc = T[t].node[k];
            stamp++;
            queue.clear();
            members.clear();
            evec.clear();
            eend.clear();
            queue.push_back(t);
            mark[t] = stamp;
            bool any_active = false;
            int maxid = -1;
            for (size_t qi = 0; qi < queue.size(); qi++) {
                const int e = queue[qi];
                int in = -1;
                for (int q = 0; q < 3; q++)
                    if (nodes_equal(T[e].node[q], nc, precision)) {
                        in = q;
                        break;
                    }
                if (in < 0) continue;   // visited but holds no copy of the node: not expanded
                members.push_back(3 * e + in);
                maxid = std::max(maxid, e);
                const int prev = (in + 2) % 3;
                evec.push_back(T[e].edgevec[in]);
                eend.push_back(T[e].node[(in + 1) % 3]);
                evec.push_back(T[e].edgevec[prev]);
                eend.push_back(T[e].node[prev]);
                if (edge_active[3 * e + in] || edge_active[3 * e + prev]) any_active = true;
                for (int nb : out.edge_neigh[e])
                    if (mark[nb] != stamp) {
                        mark[nb] = stamp;
                        queue.push_back(nb);
                    }
            }
            bool colinear = false;
            for (size_t a = 0; a < evec.size() && !colinear; a++)
                for (size_t b = a + 1; b < evec.size(); b++)
                    if (std::fabs(dotv(evec[a], evec[b])) > curvature && !nodes_equal(eend[a], eend[b], precision)) {
                        colinear = true;
                        break;
                    }
            for (int m : members) {
                corner_active[m] = (!colinear && any_active && m / 3 == maxid) ? 1 : 0;
                corner_done[m] = 1;
            }
        }
    for (int t = 0; t < n; t++) {
        int bits = 0;
        for (int k = 0; k < 3; k++) {
            if (edge_active[3 * t + k]) bits |= 1 << k;
            if (corner_active[3 * t + k]) bits |= 1 << (3 + k);
        }
        T[t].active = bits;
    }

    // coplanar node neighbours: edge neighbour or shared node, and |n_a.n_b| > curvature
    out.cnn_start.assign(n + 1, 0);
    out.cnn_list.clear();
    for (int a = 0; a < n; a++) {
        out.cnn_start[a] = (int)out.cnn_list.size();
        for (int b : cand[a]) {
            const bool neigh = std::find(out.edge_neigh[a].begin(), out.edge_neigh[a].end(), b) != out.edge_neigh[a].end();
            if (!neigh && n_shared(a, b) == 0) continue;
            if (std::fabs(dotv(T[a].surfnorm, T[b].surfnorm)) > curvature) out.cnn_list.push_back(b);
        }
    }
    out.cnn_start[n] = (int)out.cnn_list.size();
    return true;
}

// TriMesh::resolveTriSphereNeighbuild on the host (bin pre-selection)
bool tri_neighbuild_host(const TriGeom &T, double rSphere, const double *c, double treshold)
{
    const double maxDist = rSphere + treshold;
    const double v[3] = {c[0] - T.center[0], c[1] - T.center[1], c[2] - T.center[2]};
    const double dNorm = std::fabs(dotv(T.surfnorm, v));
    if (dNorm > maxDist) return false;
    const double dParaMax = maxDist * maxDist;
    for (int k = 0; k < 3; k++) {
        const double w[3] = {c[0] - T.node[k][0], c[1] - T.node[k][1], c[2] - T.node[k][2]};
        const double d = dotv(T.edgenorm[k], w);
        if (d > 0 && d * d > dParaMax) return false;
    }
    return true;
}

}  // namespace gb2
