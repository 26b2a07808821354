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

namespace {

struct NodeEnt {
    int64_t x, y, z;
    int t;
    bool operator<(const NodeEnt &o) const
    {
        return x != o.x ? x < o.x : (y != o.y ? y < o.y : (z != o.z ? z < o.z : t < o.t));
    }
    bool same_cell(const NodeEnt &o) const { return x == o.x && y == o.y && z == o.z; }
};

// Node entries in (cell x, y, z, element) order.  They are created in
// element order, so a stable sort by the packed cell key gives that order;
// an LSD radix sort on 16-bit digits does it in four passes when every axis
// spans fewer than 2^21 cells, the comparison sort otherwise.
void sort_node_entries(std::vector<NodeEnt> &e)
{
    const size_t n = e.size();
    if (n < 2) return;
    int64_t lo[3] = {e[0].x, e[0].y, e[0].z}, hi[3] = {e[0].x, e[0].y, e[0].z};
    for (const NodeEnt &q : e) {
        const int64_t v[3] = {q.x, q.y, q.z};
        for (int d = 0; d < 3; d++) {
            lo[d] = std::min(lo[d], v[d]);
            hi[d] = std::max(hi[d], v[d]);
        }
    }
    for (int d = 0; d < 3; d++)
        if (hi[d] - lo[d] >= (int64_t(1) << 21)) {
            std::stable_sort(e.begin(), e.end());
            return;
        }
    std::vector<uint64_t> key(n), key2(n);
    std::vector<uint32_t> idx(n), idx2(n);
    for (size_t i = 0; i < n; i++) {
        key[i] = (uint64_t(e[i].x - lo[0]) << 42) | (uint64_t(e[i].y - lo[1]) << 21) | uint64_t(e[i].z - lo[2]);
        idx[i] = (uint32_t)i;
    }
    std::vector<uint32_t> cnt(65536);
    for (int pass = 0; pass < 4; pass++) {
        const int sh = 16 * pass;
        std::fill(cnt.begin(), cnt.end(), 0u);
        for (size_t i = 0; i < n; i++) cnt[(key[i] >> sh) & 0xffff]++;
        uint32_t sum = 0;
        for (uint32_t &c : cnt) {
            const uint32_t v = c;
            c = sum;
            sum += v;
        }
        for (size_t i = 0; i < n; i++) {
            const uint32_t dst = cnt[(key[i] >> sh) & 0xffff]++;
            key2[dst] = key[i];
            idx2[dst] = idx[i];
        }
        key.swap(key2);
        idx.swap(idx2);
    }
    std::vector<NodeEnt> out(n);
    for (size_t i = 0; i < n; i++) out[i] = e[idx[i]];
    e.swap(out);
}

}  // namespace

bool build_mesh_topology(const double *nodes, int ntri_in, double curvature, double precision, MeshTopo &out,
                         std::string &err)
{
    out.tri.clear();
    std::vector<TriGeom> &T = out.tri;
    // elements with three distinct nodes, in input order
    std::vector<int> keep;
    keep.reserve(ntri_in);
    for (int t = 0; t < ntri_in; t++) {
        const double *nd = nodes + 9 * t;
        if (nodes_equal(nd, nd + 3, precision) || nodes_equal(nd + 3, nd + 6, precision) ||
            nodes_equal(nd, nd + 6, precision))
            continue;
        keep.push_back(t);
    }
    T.resize(keep.size());
    int degenerate = ntri_in;   // smallest input index without a surface normal
#pragma omp parallel for schedule(static) reduction(min : degenerate) if (keep.size() > 2048)
    for (int q = 0; q < (int)keep.size(); q++) {
        const int t = keep[q];
        const double *nd = nodes + 9 * t;
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
            degenerate = std::min(degenerate, t);
            continue;
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
        T[q] = g;
    }
    if (degenerate < ntri_in) {
        err = "mesh element " + std::to_string(degenerate) + " is degenerate (no surface normal)";
        return false;
    }
    const int n = (int)T.size();

    // Node entries are sorted by their hash cell (side 1000 x precision);
    // equal nodes share a cell unless they sit within `precision` of a cell
    // face, so a node looks into a neighbouring cell only along the axes where
    // it is that close to a face.
    const double cell = std::max(1e3 * precision, 1e-9);
    const double near_face = 2.0 * precision / cell;   // in cell units, with a margin for rounding
    std::vector<NodeEnt> ents;
    ents.reserve((size_t)3 * n);
    for (int t = 0; t < n; t++)
        for (int k = 0; k < 3; k++) {
            const double *p = T[t].node[k];
            ents.push_back(NodeEnt{(int64_t)std::floor(p[0] / cell), (int64_t)std::floor(p[1] / cell),
                                   (int64_t)std::floor(p[2] / cell), t});
        }
    sort_node_entries(ents);
    // runs of one cell in the sorted entries
    const int ne = (int)ents.size();
    std::vector<int> run_lo(ne), run_hi(ne);
    for (int i = 0; i < ne;) {
        int j = i;
        while (j < ne && ents[j].same_cell(ents[i])) j++;
        for (int q = i; q < j; q++) {
            run_lo[q] = i;
            run_hi[q] = j;
        }
        i = j;
    }
    // the cells a node looks into: its own, plus the neighbours along the
    // axes where it lies within `precision` of a face (rare)
    auto for_each_cell_run = [&](const double *p, int self_run, auto &&fn) {
        int64_t c[3];
        int lo[3], hi[3];
        for (int d = 0; d < 3; d++) {
            const double q = p[d] / cell;
            c[d] = (int64_t)std::floor(q);
            const double fr = q - (double)c[d];
            lo[d] = fr < near_face ? -1 : 0;
            hi[d] = 1.0 - fr < near_face ? 1 : 0;
        }
        fn(run_lo[self_run], run_hi[self_run]);
        for (int dx = lo[0]; dx <= hi[0]; dx++)
            for (int dy = lo[1]; dy <= hi[1]; dy++)
                for (int dz = lo[2]; dz <= hi[2]; dz++) {
                    if (dx == 0 && dy == 0 && dz == 0) continue;
                    const NodeEnt key{c[0] + dx, c[1] + dy, c[2] + dz, -1};
                    auto it = std::lower_bound(ents.begin(), ents.end(), key);
                    if (it != ents.end() && it->same_cell(key)) {
                        const int q = (int)(it - ents.begin());
                        fn(run_lo[q], run_hi[q]);
                    }
                }
    };
    // each element's node entries (position in the sorted list)
    std::vector<int> ent_of((size_t)3 * n);
    {
        std::vector<int> seen(n, 0);
        for (int i = 0; i < ne; i++) ent_of[3 * ents[i].t + seen[ents[i].t]++] = i;
    }
    // candidate pairs: elements owning a node equal (within `precision`) to
    // one of the element's nodes, as a CSR (two passes: count, fill), each
    // row sorted with duplicates and the element itself removed
    std::vector<int> cand_start(n + 1, 0);
#pragma omp parallel for schedule(static) if (n > 2048)
    for (int t = 0; t < n; t++) {
        int m = 0;
        for (int k = 0; k < 3; k++) {
            const int e = ent_of[3 * t + k];
            for_each_cell_run(T[t].node[k], e, [&](int lo, int hi) { m += hi - lo; });
        }
        cand_start[t + 1] = m;
    }
    for (int t = 0; t < n; t++) cand_start[t + 1] += cand_start[t];
    std::vector<int> cand_all(cand_start[n]);
#pragma omp parallel for schedule(static) if (n > 2048)
    for (int t = 0; t < n; t++) {
        int w = cand_start[t];
        for (int k = 0; k < 3; k++) {
            const int e = ent_of[3 * t + k];
            for_each_cell_run(T[t].node[k], e, [&](int lo, int hi) {
                for (int q = lo; q < hi; q++) cand_all[w++] = ents[q].t;
            });
        }
    }
    std::vector<std::vector<int>> cand(n);
#pragma omp parallel for schedule(static) if (n > 2048)
    for (int t = 0; t < n; t++) {
        int *b0 = cand_all.data() + cand_start[t], *b1 = cand_all.data() + cand_start[t + 1];
        std::sort(b0, b1);
        int *e1 = std::unique(b0, b1);
        std::vector<int> &row = cand[t];
        row.reserve(e1 - b0);
        for (int *q = b0; q != e1; q++)
            if (*q != t) row.push_back(*q);
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

    // shared edges.  Element a settles its own edges and lists its edge
    // neighbours in ascending order; a pair is examined from its larger
    // element x (nodes of x matched against those of the smaller y, x's edge
    // normal as reference), and where several neighbours share an edge of a
    // the one with the largest id decides, as if the pairs were visited in
    // ascending (x, y) order with the later one overwriting
    out.edge_neigh.assign(n, {});
    std::vector<uint8_t> edge_active((size_t)3 * n, 1);
#pragma omp parallel for schedule(dynamic, 64) if (n > 2048)
    for (int a = 0; a < n; a++)
        for (int b : cand[a]) {
            if (!bsphere_overlap(a, b)) continue;
            const int x = std::max(a, b), y = std::min(a, b);
            int ix[2], jy[2], ns = 0;
            for (int i = 0; i < 3 && ns < 2; i++)
                for (int j = 0; j < 3 && ns < 2; j++)
                    if (nodes_equal(T[x].node[i], T[y].node[j], precision)) {
                        ix[ns] = i;
                        jy[ns] = j;
                        ns++;
                    }
            if (ns < 2) continue;
            const int ex = (2 == ix[0] + ix[1]) ? 2 : std::min(ix[0], ix[1]);
            const int ey = (2 == jy[0] + jy[1]) ? 2 : std::min(jy[0], jy[1]);
            out.edge_neigh[a].push_back(b);
            const bool coplanar = std::fabs(dotv(T[x].surfnorm, T[y].surfnorm)) >= curvature;
            bool overlap = false;
            if (coplanar) {
                const double *pRef = T[x].node[ex];
                const double *eN = T[x].edgenorm[ex];
                const double *nx = T[x].node[(ex + 2) % 3];
                const double *ny = T[y].node[(ey + 2) % 3];
                const double vI[3] = {nx[0] - pRef[0], nx[1] - pRef[1], nx[2] - pRef[2]};
                const double vJ[3] = {ny[0] - pRef[0], ny[1] - pRef[1], ny[2] - pRef[2]};
                overlap = dotv(vI, eN) * dotv(vJ, eN) > 0.;
            }
            // the element with the larger id keeps a non-coplanar or folded edge
            const uint8_t keep_edge = (!coplanar || overlap) ? (a == x ? 1 : 0) : 0;
            edge_active[3 * a + (a == x ? ex : ey)] = keep_edge;
        }

    // corners.  The walk from corner (t, k) over edge neighbours that hold a
    // copy of the node reaches the same group of corners from any of its
    // members (the connected holders of the node), so every corner walks its
    // own group, in parallel, and settles only itself: active only at the
    // group's largest element id, when an edge at the node is active and no
    // two of the group's edges are colinear.
    std::vector<uint8_t> corner_active((size_t)3 * n, 1);
#pragma omp parallel if (n > 2048)
    {
        std::vector<int> mark(n, -1), queue;
        std::vector<const double *> evec, eend;
        int stamp = 0;
#pragma omp for schedule(dynamic, 64)
        for (int t = 0; t < n; t++)
            for (int k = 0; k < 3; k++) {
                const double *nc = T[t].node[k];
                stamp++;
                queue.clear();
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
                corner_active[3 * t + k] = (!colinear && any_active && t == maxid) ? 1 : 0;
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
    std::vector<std::vector<int>> cnn(n);
#pragma omp parallel for schedule(dynamic, 64) if (n > 2048)
    for (int a = 0; a < n; a++)
        for (int b : cand[a]) {
            const bool neigh = std::find(out.edge_neigh[a].begin(), out.edge_neigh[a].end(), b) != out.edge_neigh[a].end();
            if (!neigh && n_shared(a, b) == 0) continue;
            if (std::fabs(dotv(T[a].surfnorm, T[b].surfnorm)) > curvature) cnn[a].push_back(b);
        }
    out.cnn_start.assign(n + 1, 0);
    out.cnn_list.clear();
    for (int a = 0; a < n; a++) {
        out.cnn_start[a] = (int)out.cnn_list.size();
        out.cnn_list.insert(out.cnn_list.end(), cnn[a].begin(), cnn[a].end());
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
