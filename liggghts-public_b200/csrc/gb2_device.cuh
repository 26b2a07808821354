// gb2_device.cuh -- device helpers shared by every kernel of the granular
// step: bin arithmetic, material lookup, the triangle-sphere narrow phase,
// neighbour-record gathers, warp item enumeration and the wall contacts of
// one atom.  Included by both compiled units (the bit-exact FP64 unit built
// with --fmad=false and the split-precision unit), so everything here is a
// header-only __device__ function.
#pragma once

#include "gb2_internal.h"

namespace gb2 {
__device__ __forceinline__ dbl4 ld4(const dbl4 *p) { return *p; }

__device__ __forceinline__ flt8 make_kin(const dbl4 &v, const dbl4 &w)
{
    flt8 k;
    k.vx = (float)v.x;
    k.vy = (float)v.y;
    k.vz = (float)v.z;
    k.m = (float)v.w;
    k.wx = (float)w.x;
    k.wy = (float)w.y;
    k.wz = (float)w.z;
    k.pad = 0.0f;
    return k;
}

__device__ __forceinline__ int coord2bin3(const Dev &D, double x0, double x1, double x2, int &ix, int &iy, int &iz)
{
    // Neighbor::coord2bin src/neighbor.cpp:2112
    const double x[3] = {x0, x1, x2};
    int idx[3];
    for (int d = 0; d < 3; d++) {
        int v;
        if (x[d] >= D.bboxhi[d])
            v = static_cast<int>((x[d] - D.bboxhi[d]) * D.bininv[d]) + D.nbin[d];
        else if (x[d] >= D.bboxlo[d]) {
            v = static_cast<int>((x[d] - D.bboxlo[d]) * D.bininv[d]);
            v = min(v, D.nbin[d] - 1);
        } else
            v = static_cast<int>((x[d] - D.bboxlo[d]) * D.bininv[d]) - 1;
        idx[d] = v - D.mbinlo[d];
    }
    ix = idx[0];
    iy = idx[1];
    iz = idx[2];
    return iz * D.mbin[1] * D.mbin[0] + iy * D.mbin[0] + ix;
}

__device__ __forceinline__ int coord2bin(const Dev &D, double x0, double x1, double x2)
{
    int a, b, c;
    return coord2bin3(D, x0, x1, x2, a, b, c);
}

__device__ __forceinline__ const MatPair &mat(const Dev &D, int ti, int tj)
{
    return D.mat[ti * (kMaxTypes + 1) + tj];
}


// ------------------------------------------------------------------
// mesh support

__device__ __forceinline__ double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// TriMesh::resolveTriSphereNeighbuild (src/tri_mesh_I.h:255)
__device__ __forceinline__ bool tri_neighbuild(const TriGeom &T, double rSphere, const double c[3], double treshold)
{
    const double maxDist = rSphere + treshold;
    double v[3] = {c[0] - T.center[0], c[1] - T.center[1], c[2] - T.center[2]};
    const double dNorm = fabs(dot3(T.surfnorm, v));
    if (dNorm > maxDist) return false;
    const double dParaMax = maxDist * maxDist;
    for (int k = 0; k < 3; k++) {
        double w[3] = {c[0] - T.node[k][0], c[1] - T.node[k][1], c[2] - T.node[k][2]};
        const double d = dot3(T.edgenorm[k], w);
        if (d > 0 && d * d > dParaMax) return false;
    }
    return true;
}


// TriMesh::resolveTriSphereContactBary and its edge/corner/face helpers
// (src/tri_mesh_I.h:65-251).  Returns distance - radius; LARGE (1e6) for an
// inactive feature.
__device__ __forceinline__ double calc_dist(const double *cs, const double *cp, double *delta)
{
    delta[0] = cp[0] - cs[0];
    delta[1] = cp[1] - cs[1];
    delta[2] = cp[2] - cs[2];
    const double d2 = (cs[0] - cp[0]) * (cs[0] - cp[0]) + (cs[1] - cp[1]) * (cs[1] - cp[1]) +
                      (cs[2] - cp[2]) * (cs[2] - cp[2]);
    return sqrt(d2);
}

#define GB2_SMALL_TRIMESH 1.e-10
#define GB2_LARGE_TRIMESH 1000000
#define GB2_EDGE_ACTIVE(T, k) (((T).active >> (k)) & 1)
#define GB2_CORNER_ACTIVE(T, k) (((T).active >> (3 + (k))) & 1)

static __device__ double tri_edge(const TriGeom &T, int iEdge, const double *p, double *delta, double *bary)
{
    const int ip = (iEdge + 1) % 3, ipp = (iEdge + 2) % 3;
    double nodeToP[3] = {p[0] - T.node[iEdge][0], p[1] - T.node[iEdge][1], p[2] - T.node[iEdge][2]};
    const double distFromNode = dot3(nodeToP, T.edgevec[iEdge]);
    if (distFromNode < -GB2_SMALL_TRIMESH) {
        if (!GB2_CORNER_ACTIVE(T, iEdge)) return GB2_LARGE_TRIMESH;
        bary[iEdge] = 1.;
        bary[ip] = 0.;
        bary[ipp] = 0.;
        return calc_dist(p, T.node[iEdge], delta);
    } else if (distFromNode > T.edgelen[iEdge] + GB2_SMALL_TRIMESH) {
        if (!GB2_CORNER_ACTIVE(T, ip)) return GB2_LARGE_TRIMESH;
        bary[iEdge] = 0.;
        bary[ip] = 1.;
        bary[ipp] = 0.;
        return calc_dist(p, T.node[ip], delta);
    }
    if (!GB2_EDGE_ACTIVE(T, iEdge)) return GB2_LARGE_TRIMESH;
    double cp[3];
    cp[0] = T.node[iEdge][0] + distFromNode * T.edgevec[iEdge][0];
    cp[1] = T.node[iEdge][1] + distFromNode * T.edgevec[iEdge][1];
    cp[2] = T.node[iEdge][2] + distFromNode * T.edgevec[iEdge][2];
    const double d = calc_dist(p, cp, delta);
    bary[ipp] = 0.;
    bary[iEdge] = 1. - distFromNode / T.edgelen[iEdge];
    bary[ip] = 1. - bary[iEdge];
    return d;
}

static __device__ double tri_corner(const TriGeom &T, int iNode, bool obtuse, const double *p, double *delta,
                                    double *bary)
{
    const int ip = (iNode + 1) % 3, ipp = (iNode + 2) % 3;
    const double *n = T.node[iNode];
    if (obtuse) {
        double nodeToP[3] = {p[0] - n[0], p[1] - n[1], p[2] - n[2]};
        double cp[3];
        double distFromNode = dot3(nodeToP, T.edgevec[ipp]);
        if (distFromNode < GB2_SMALL_TRIMESH) {
            if (distFromNode > -T.edgelen[ipp]) {
                if (!GB2_EDGE_ACTIVE(T, ipp)) return GB2_LARGE_TRIMESH;
                cp[0] = n[0] + distFromNode * T.edgevec[ipp][0];
                cp[1] = n[1] + distFromNode * T.edgevec[ipp][1];
                cp[2] = n[2] + distFromNode * T.edgevec[ipp][2];
                bary[ip] = 0.;
                bary[iNode] = 1. + distFromNode / T.edgelen[ipp];
                bary[ipp] = 1. - bary[iNode];
                return calc_dist(p, cp, delta);
            }
            if (!GB2_CORNER_ACTIVE(T, ipp)) return GB2_LARGE_TRIMESH;
            bary[ipp] = 1.;
            bary[iNode] = bary[ip] = 0.;
            return calc_dist(p, T.node[ipp], delta);
        }
        distFromNode = dot3(nodeToP, T.edgevec[iNode]);
        if (distFromNode > -GB2_SMALL_TRIMESH) {
            if (distFromNode < T.edgelen[iNode]) {
                if (!GB2_EDGE_ACTIVE(T, iNode)) return GB2_LARGE_TRIMESH;
                cp[0] = n[0] + distFromNode * T.edgevec[iNode][0];
                cp[1] = n[1] + distFromNode * T.edgevec[iNode][1];
                cp[2] = n[2] + distFromNode * T.edgevec[iNode][2];
                bary[ipp] = 0.;
                bary[iNode] = 1. - distFromNode / T.edgelen[iNode];
                bary[ip] = 1. - bary[iNode];
                return calc_dist(p, cp, delta);
            }
            if (!GB2_CORNER_ACTIVE(T, ip)) return GB2_LARGE_TRIMESH;
            bary[ip] = 1.;
            bary[iNode] = bary[ipp] = 0.;
            return calc_dist(p, T.node[ip], delta);
        }
    }
    if (!GB2_CORNER_ACTIVE(T, iNode)) return GB2_LARGE_TRIMESH;
    bary[iNode] = 1.;
    bary[ip] = bary[ipp] = 0.;
    return calc_dist(p, T.node[iNode], delta);
}

// bary: barycentric coordinates of the contact point as the reference's
// resolveTriSphereContactBary leaves them (the moving-wall velocity is
// interpolated with them)
static __device__ double tri_sphere(const TriGeom &T, double rSphere, const double *cs, double *delta, int &barySign,
                                    double precision, double *bary)
{
    double n0ToC[3] = {cs[0] - T.node[0][0], cs[1] - T.node[0][1], cs[2] - T.node[0][2]};
    // MathExtraLiggghts::calcBaryTriCoords (src/math_extra_liggghts.h:559)
    const double a = dot3(n0ToC, T.edgevec[0]);
    const double b = dot3(n0ToC, T.edgevec[2]);
    const double c = dot3(T.edgevec[0], T.edgevec[2]);
    const double oneMinCSqr = 1 - c * c;
    bary[1] = (a - b * c) / (T.edgelen[0] * oneMinCSqr);
    bary[2] = (a * c - b) / (T.edgelen[2] * oneMinCSqr);
    bary[0] = 1. - bary[1] - bary[2];
    const double invlen = 1. / (2. * T.rbound);
    barySign = (bary[0] > -precision * invlen) + 2 * (bary[1] > -precision * invlen) +
               4 * (bary[2] > -precision * invlen);
    double d;
    switch (barySign) {
    case 1: d = tri_corner(T, 0, T.obtuse == 0, cs, delta, bary); break;
    case 2: d = tri_corner(T, 1, T.obtuse == 1, cs, delta, bary); break;
    case 3: d = tri_edge(T, 0, cs, delta, bary); break;
    case 4: d = tri_corner(T, 2, T.obtuse == 2, cs, delta, bary); break;
    case 5: d = tri_edge(T, 2, cs, delta, bary); break;
    case 6: d = tri_edge(T, 1, cs, delta, bary); break;
    case 7: {
        const double dNorm = dot3(T.surfnorm, n0ToC);
        const double tmp[3] = {T.surfnorm[0] * dNorm, T.surfnorm[1] * dNorm, T.surfnorm[2] * dNorm};
        const double csPlane[3] = {cs[0] - tmp[0], cs[1] - tmp[1], cs[2] - tmp[2]};
        d = calc_dist(cs, csPlane, delta);
        break;
    }
    default: d = 1.; break;
    }
    return d - rSphere;
}

__device__ __forceinline__ bool coplanar_node_neighs(const MeshDev &M, int a, int b)
{
    for (int q = M.cnn_start[a]; q < M.cnn_start[a + 1]; q++)
        if (M.cnn_list[q] == b) return true;
    return false;
}

// ------------------------------------------------------------------
// pair passes.  Both walk a per-atom list in two phases: a screening phase
// issues the neighbour-position gathers of all entries independently (so
// many loads are in flight per thread) and records which entries touch in a
// bit mask; the compute phase then evaluates only touching entries, in list
// order, so the per-atom sums keep the reference's order.

// One 32-byte record through the read-only path as a single 256-bit load
// (sm_100 vector width): a scattered warp-wide gather then needs one L1
// wavefront per lane's line instead of two.  Records are 32-byte aligned.
__device__ __forceinline__ dbl4 ldg4(const dbl4 *p)
{
    dbl4 r;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
    return r;
}

// One split-precision kinematics record (eight FP32 values) as one 256-bit
// read-only load.
__device__ __forceinline__ flt8 ldg8f(const flt8 *p)
{
    flt8 r;
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(r.vx), "=f"(r.vy), "=f"(r.vz), "=f"(r.m), "=f"(r.wx), "=f"(r.wy), "=f"(r.wz), "=f"(r.pad)
        : "l"(p));
    return r;
}

// A 32-byte record copied to shared memory without passing through
// registers (two 16-byte cp.async, L2 only); complete after cp_async_wait().
// Each thread reads back only what it copied itself, so no barrier is needed.
__device__ __forceinline__ void stage4(dbl4 *dst, const dbl4 *src)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n\t"
                 "cp.async.cg.shared.global [%2], [%3], 16;" ::"r"(s),
                 "l"(src), "r"(s + 16u), "l"((const char *)src + 16)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ bool touching(const dbl4 &a, const dbl4 &b)
{
    const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    const double rs = a.w + b.w;
    return dx * dx + dy * dy + dz * dz < rs * rs;
}

// Warp-cooperative evaluation of the touching entries found by screening.
// The warp's touching entries are enumerated owner-lane-major (each owner's
// entries in list order); in rounds of 32, lane t evaluates item base+t and
// leaves the pair's raw contribution in shared memory, then every owner lane
// adds the items it owns in order.  The per-atom sums therefore keep the
// reference's order while the FP64 contact arithmetic runs on full warps.
struct WarpItems {
    int cnt, excl, total;
};

__device__ __forceinline__ WarpItems warp_items(unsigned long long mask)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    WarpItems it;
    it.cnt = __popcll(mask);
    int x = it.cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    it.excl = x - it.cnt;
    it.total = __shfl_sync(FULL, x, 31);
    return it;
}

// Index stream loads: read once per step, evict-first so they do not push
// the neighbour records out of L2
__device__ __forceinline__ int ld_stream(const int *p) { return __ldcs(p); }

// Screening of the j-side (rev) and own (nbr) entries of one atom in one
// loop: per round two indices of each list, then four independent record
// gathers, then the distance tests.  Both lists are <= 64 entries here.
__device__ __forceinline__ void screen_both(const Dev &D, int k, int nr, int nn, const dbl4 &pk,
                                            unsigned long long &mrev, unsigned long long &mown)
{
    const int cap = D.cap;
    const int n = max(nr, nn);
    // the indices of the next pair of entries are requested while this
    // pair's records are in flight (one dependent round trip per pair)
    int a0 = (0 < nr) ? ld_stream(&D.rev[k]) : k;
    int a1 = (1 < nr) ? ld_stream(&D.rev[cap + k]) : k;
    int b0 = (0 < nn) ? ld_stream(&D.nbr[k]) : k;
    int b1 = (1 < nn) ? ld_stream(&D.nbr[cap + k]) : k;
    for (int t = 0; t < n; t += 2) {
        const dbl4 qa0 = ldg4(&D.pos[a0]);
        const dbl4 qa1 = ldg4(&D.pos[a1]);
        const dbl4 qb0 = ldg4(&D.pos[b0]);
        const dbl4 qb1 = ldg4(&D.pos[b1]);
        const int u = t + 2;
        a0 = (u < nr) ? ld_stream(&D.rev[u * cap + k]) : k;
        a1 = (u + 1 < nr) ? ld_stream(&D.rev[(u + 1) * cap + k]) : k;
        b0 = (u < nn) ? ld_stream(&D.nbr[u * cap + k]) : k;
        b1 = (u + 1 < nn) ? ld_stream(&D.nbr[(u + 1) * cap + k]) : k;
        if (t < nr && touching(pk, qa0)) mrev |= 1ull << t;
        if (t + 1 < nr && touching(pk, qa1)) mrev |= 1ull << (t + 1);
        if (t < nn && touching(pk, qb0)) mown |= 1ull << t;
        if (t + 1 < nn && touching(pk, qb1)) mown |= 1ull << (t + 1);
    }
}

// Screening that also lists the warp's touching entries in shared memory,
// so the contact rounds read each item's partner and slot there instead of
// gathering the list index again: lrev holds the j-side entries, lown the
// own entries, each as {other atom, owner lane | slot << 8} in the order the
// owner's sum takes them (every atom's rev entries by r, then its own entries
// by s; the rev list is evaluated first).  Entries are appended per loop
// step with ballots; the loop runs to the warp's longest list so every lane
// takes part.  Inactive lanes (invalid or serial atoms) pass nr = nn = 0.
// Returns false when a list outgrew D.item_cap (the lists' size in the
// kernel's dynamic shared memory, at most kItemCap; the bitmasks are
// complete either way, and the caller falls back to enumerating them).
constexpr int kItemCap = 256;

__device__ __forceinline__ void list_append(int2 *list, int cap, int &n, bool take, int other, int code)
{
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int pos = n + __popc(m & ((1u << lane) - 1u));
    if (take && pos < cap) list[pos] = make_int2(other, code);
    n += __popc(m);
}

__device__ __forceinline__ bool screen_list(const Dev &D, int k, int nr, int nn, const dbl4 &pk,
                                            unsigned long long &mrev, unsigned long long &mown, int2 *lrev,
                                            int2 *lown, int &nlrev, int &nlown)
{
    const int cap = D.cap, lane = threadIdx.x & 31;
    const int nw = __reduce_max_sync(0xffffffffu, max(nr, nn));
    nlrev = nlown = 0;
    int a0 = (0 < nr) ? ld_stream(&D.rev[k]) : 0;
    int a1 = (1 < nr) ? ld_stream(&D.rev[cap + k]) : 0;
    int s0 = (0 < nr) ? (int)D.revs[k] : 0;
    int s1 = (1 < nr) ? (int)D.revs[cap + k] : 0;
    int b0 = (0 < nn) ? ld_stream(&D.nbr[k]) : 0;
    int b1 = (1 < nn) ? ld_stream(&D.nbr[cap + k]) : 0;
    for (int t = 0; t < nw; t += 2) {
        const dbl4 qa0 = ldg4(&D.pos[a0]);
        const dbl4 qa1 = ldg4(&D.pos[a1]);
        const dbl4 qb0 = ldg4(&D.pos[b0]);
        const dbl4 qb1 = ldg4(&D.pos[b1]);
        const int ca0 = a0, ca1 = a1, cs0 = s0, cs1 = s1, cb0 = b0, cb1 = b1;
        const int u = t + 2;
        a0 = (u < nr) ? ld_stream(&D.rev[u * cap + k]) : 0;
        a1 = (u + 1 < nr) ? ld_stream(&D.rev[(u + 1) * cap + k]) : 0;
        s0 = (u < nr) ? (int)D.revs[u * cap + k] : 0;
        s1 = (u + 1 < nr) ? (int)D.revs[(u + 1) * cap + k] : 0;
        b0 = (u < nn) ? ld_stream(&D.nbr[u * cap + k]) : 0;
        b1 = (u + 1 < nn) ? ld_stream(&D.nbr[(u + 1) * cap + k]) : 0;
        const bool ta0 = t < nr && touching(pk, qa0), ta1 = t + 1 < nr && touching(pk, qa1);
        const bool tb0 = t < nn && touching(pk, qb0), tb1 = t + 1 < nn && touching(pk, qb1);
        if (ta0) mrev |= 1ull << t;
        if (ta1) mrev |= 1ull << (t + 1);
        if (tb0) mown |= 1ull << t;
        if (tb1) mown |= 1ull << (t + 1);
        list_append(lrev, D.item_cap, nlrev, ta0, ca0, lane | (cs0 << 8));
        list_append(lrev, D.item_cap, nlrev, ta1, ca1, lane | (cs1 << 8));
        list_append(lown, D.item_cap, nlown, tb0, cb0, lane | (t << 8));
        list_append(lown, D.item_cap, nlown, tb1, cb1, lane | ((t + 1) << 8));
    }
    return nlrev <= D.item_cap && nlown <= D.item_cap;
}

__device__ __forceinline__ WarpItems warp_items_cnt(int cnt)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    WarpItems it;
    it.cnt = cnt;
    int x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    it.excl = x - cnt;
    it.total = __shfl_sync(FULL, x, 31);
    return it;
}

// owner lane of item w: the largest lane whose exclusive prefix is <= w
__device__ __forceinline__ int item_owner(int w, int excl)
{
    const unsigned FULL = 0xffffffffu;
    int L = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
        const int cand = L + step;
        const int ex = __shfl_sync(FULL, excl, cand & 31);
        if (cand < 32 && ex <= w) L = cand;
    }
    return L;
}

__device__ __forceinline__ int nth_set_bit(unsigned long long m, int rank)
{
    for (int q = 0; q < rank; q++) m &= m - 1ull;
    return __ffsll((long long)m) - 1;
}

__device__ __forceinline__ unsigned long long shfl64(unsigned long long v, int src)
{
    const unsigned FULL = 0xffffffffu;
    const unsigned lo = __shfl_sync(FULL, (unsigned)(v & 0xffffffffull), src);
    const unsigned hi = __shfl_sync(FULL, (unsigned)(v >> 32), src);
    return ((unsigned long long)hi << 32) | lo;
}

// Wall-contact records: the force and torque one wall contact adds to its
// atom, kept (shared memory) until the pair sums they must follow are
// available.  A record starts from negative zeros, so -0.0 + x == x for
// every x (signed zeros included) and adding the record later is the same
// operation as adding the contact force in place.
constexpr int kWallRec = 4;   // records per atom
typedef double WallRec[6];

__device__ __forceinline__ ContactOut wall_record_zero()
{
    ContactOut o;
    for (int c = 0; c < 3; c++) o.F[c] = o.T[c] = -0.0;
    return o;
}

__device__ __forceinline__ void wall_record_put(WallRec *rec, int &n, const ContactOut &o)
{
    for (int c = 0; c < 3; c++) {
        rec[n][c] = o.F[c];
        rec[n][3 + c] = o.T[c];
    }
    n++;
}

// One candidate triangle t in contact with atom i (deltan <= 0): the body of
// FixWallGran::post_force_mesh's loop -- FixContactHistoryMesh::handleContact
// (slot lookup, new slot with the shear of a coplanar neighbour for face
// contacts, or skip when a coplanar neighbour already holds the contact) and
// the wall contact force.  keep/np: markAllContacts mask and npartner; sp:
// the atom's slot partners (a shared-memory copy of spartner, kept in step).
// Returns true when the contact force was added to acc.
static __device__ bool mesh_contact(const Dev &D, const MeshDev &M, int i, int t, const dbl4 &p, const double v[3],
                                    const double w[3], double mass, int itype, bool upd, int nn, int *sp,
                                    unsigned long long &keep, int &np, ContactOut &acc)
{
    const int cap = D.cap;
    const double cs[3] = {p.x, p.y, p.z};
    const TriGeom &T = M.tri[t];
    double delta[3], bary[3] = {0., 0., 0.};
    int barysign = -1;
    const double deltan = tri_sphere(T, p.w, cs, delta, barysign, 1e-8, bary);
    const bool faceflag = (7 == barysign);
    int slot = -1;
    for (int k = 0; k < nn; k++)
        if (sp[k] == t) {
            slot = k;
            break;
        }
    if (slot >= 0) {
        keep |= 1ull << slot;
    } else {
        if (faceflag) {
            for (int k = 0; k < nn; k++) {
                const int idp = sp[k];
                if (idp >= 0 && idp != t && coplanar_node_neighs(M, idp, t) && ((keep >> k) & 1ull)) return false;
            }
        }
        int ic = -1;
        for (int k = 0; k < nn; k++)
            if (-1 == sp[k]) {
                ic = k;
                break;
            }
        if (ic < 0 || np >= nn) {
            atomicOr(D.status, ST_MESH_INTERNAL);
            return false;
        }
        sp[ic] = t;
        M.spartner[ic * cap + i] = t;
        keep |= 1ull << ic;
        double h0 = 0.0, h1 = 0.0, h2 = 0.0;
        np++;
        if (faceflag) {
            for (int k = 0; k < nn; k++) {
                const int tri = sp[k];
                if (tri >= 0 && tri != t && coplanar_node_neighs(M, tri, t)) {
                    h0 = M.shist[(3 * k + 0) * cap + i];
                    h1 = M.shist[(3 * k + 1) * cap + i];
                    h2 = M.shist[(3 * k + 2) * cap + i];
                }
            }
        }
        M.shist[(3 * ic + 0) * cap + i] = h0;
        M.shist[(3 * ic + 1) * cap + i] = h1;
        M.shist[(3 * ic + 2) * cap + i] = h2;
        slot = ic;
    }
    double sh[3] = {M.shist[(3 * slot + 0) * cap + i], M.shist[(3 * slot + 1) * cap + i],
                    M.shist[(3 * slot + 2) * cap + i]};
    const double dvec[3] = {-delta[0], -delta[1], -delta[2]};
    double vwall[3] = {0.0, 0.0, 0.0};
    if (M.vnode) {   // moving mesh: barycentric node velocity (src/fix_wall_gran.cpp:992-996)
        const double *vn = M.vnode + 9 * t;
        for (int c = 0; c < 3; c++) vwall[c] = (bary[0] * vn[c] + bary[1] * vn[3 + c] + bary[2] * vn[6 + c]);
    }
    // the contact's own force first (-0.0 + x == x), then added to acc: the
    // same IEEE additions as accumulating in place
    ContactOut wc;
    for (int c = 0; c < 3; c++) wc.F[c] = wc.T[c] = -0.0;
    wall_contact(mat(D, itype, M.wtype), dvec, -deltan, p.w, v, w, vwall, mass, sh, upd, D.dt, M.rolling != 0,
                 D.tdamp != 0, wc);
    for (int c = 0; c < 3; c++) {
        acc.F[c] += wc.F[c];
        acc.T[c] += wc.T[c];
    }
    M.shist[(3 * slot + 0) * cap + i] = sh[0];
    M.shist[(3 * slot + 1) * cap + i] = sh[1];
    M.shist[(3 * slot + 2) * cap + i] = sh[2];
    if (M.trif) {   // MeshModuleStress::add_particle_contribution (src/mesh_module_stress.cpp:276-304)
        const double frc[3] = {-wc.F[0], -wc.F[1], -wc.F[2]};
        const double tmp[3] = {p.x + delta[0] - M.pref[0], p.y + delta[1] - M.pref[1], p.z + delta[2] - M.pref[2]};
        const double tq[3] = {tmp[1] * frc[2] - tmp[2] * frc[1], tmp[2] * frc[0] - tmp[0] * frc[2],
                              tmp[0] * frc[1] - tmp[1] * frc[0]};
        for (int c = 0; c < 3; c++) {
            atomicAdd(&M.trif[3 * t + c], frc[c]);
            atomicAdd(&M.ftot[c], frc[c]);
            atomicAdd(&M.ftot[3 + c], tq[c]);
        }
        if (M.wear) {   // Finnie wear (src/mesh_module_stress.cpp:306-352), summed straight into the total
            const double vr[3] = {v[0] - vwall[0], v[1] - vwall[1], v[2] - vwall[2]};
            const double vm = sqrt(vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]);
            if (!(delta[0] * vr[0] + delta[1] * vr[1] + delta[2] * vr[2] < 0.) && !(0.0000001 > vm)) {
                const double *sn = M.tri[t].surfnorm;
                const double cr[3] = {vr[1] * sn[2] - vr[2] * sn[1], vr[2] * sn[0] - vr[0] * sn[2],
                                      vr[0] * sn[1] - vr[1] * sn[0]};
                double sg = fabs(vr[0] * sn[0] + vr[1] * sn[1] + vr[2] * sn[2]) / vm;
                double cg = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]) / vm;
                cg = cg > 1. ? 1. : cg;
                sg = sg > 1. ? 1. : sg;
                double E = (cg < 0.0001 || 3. * sg > cg) ? 0.33333 * cg * cg : 2. * sg * cg - 3. * sg * sg;
                E *= 2. * M.kfin[itype] * vm * sqrt(frc[0] * frc[0] + frc[1] * frc[1] + frc[2] * frc[2]);
                atomicAdd(&M.wear[t], E * D.dt / M.tarea[t]);
            }
        }
    }
    return true;
}

// FixWallGran::post_force_mesh for the atoms owned by the lanes of a warp
// (own: lane holds atom i; acc is the owner's).  The sphere-triangle
// distances of all candidates of the warp's atoms are independent of one
// another and of the contact history, so they are evaluated one candidate
// per lane (owner-major items, rounds of 32); each owner then handles its
// candidates in contact (deltan <= 0) in ascending order with mesh_contact,
// exactly as the sequential loop, and FixContactHistoryMesh::cleanUpContacts
// clears the slots that lost their contact.  At most 64 candidates per atom.
//
// sp: shared-memory scratch of the warp (at least kTailAtoms * 64 ints) for
// the slot partners of its atoms, loaded with the candidates (one slot per
// candidate item) so the slot searches of mesh_contact read shared memory.
//
// REC: each contact's force goes to the owner's records (rec, nrec) instead
// of acc; an owner with more candidates in contact than records left is
// dropped before anything of it changes (recok cleared) and is handled
// later with REC=false.
template <bool REC>
__device__ __forceinline__ void mesh_wall_items(const Dev &D, const MeshDev &M, bool own, int i, const dbl4 &p,
                                                const double v[3], const double w[3], double mass, int itype,
                                                bool upd, int *sp, ContactOut &acc, WallRec *rec = nullptr,
                                                int *nrec = nullptr, bool *recok = nullptr)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int cap = D.cap;
    const int nn = own ? M.tcnt[i] : 0;
    int np = own ? M.snp[i] : 0;
    const WarpItems it = warp_items_cnt(nn);
    if (it.total == 0) return;
    unsigned long long touch = 0ull;
    for (int base = 0; base < it.total; base += 32) {
        const int wq = base + lane;
        const int L = item_owner(min(wq, it.total - 1), it.excl);
        const int iL = __shfl_sync(FULL, i, L);
        const int exL = __shfl_sync(FULL, it.excl, L);
        const double px = __shfl_sync(FULL, p.x, L), py = __shfl_sync(FULL, p.y, L);
        const double pz = __shfl_sync(FULL, p.z, L), pr = __shfl_sync(FULL, p.w, L);
        bool hit = false;
        if (wq < it.total) {
            const double cs[3] = {px, py, pz};
            double delta[3], bary[3] = {0., 0., 0.};
            int barysign = -1;
            const int t = M.tlist[(wq - exL) * cap + iL];
            sp[wq] = M.spartner[(wq - exL) * cap + iL];
            const double deltan = tri_sphere(M.tri[t], pr, cs, delta, barysign, 1e-8, bary);
            hit = !(deltan > D.cutneighmax) && (deltan <= 0);
        }
        const unsigned bal = __ballot_sync(FULL, hit);
        const int lo = max(it.excl, base), hi = min(it.excl + nn, base + 32);
        if (lo < hi) {
            const unsigned long long bits = (unsigned long long)(bal >> (lo - base)) & ((1ull << (hi - lo)) - 1ull);
            touch |= bits << (lo - it.excl);
        }
    }
    __syncwarp();
    bool act = nn > 0;
    if constexpr (REC) {
        if (act && *nrec + __popcll(touch) > kWallRec) {
            act = false;
            *recok = false;
        }
    }
    unsigned long long keep = act ? 0ull : ~0ull;   // an owner left for later keeps every slot here
    if (act) {
        for (unsigned long long m = touch; m; m &= m - 1ull) {
            const int q = __ffsll((long long)m) - 1;
            const int t = M.tlist[q * cap + i];
            if constexpr (REC) {
                ContactOut o = wall_record_zero();
                if (mesh_contact(D, M, i, t, p, v, w, mass, itype, upd, nn, sp + it.excl, keep, np, o))
                    wall_record_put(rec, *nrec, o);
            } else {
                mesh_contact(D, M, i, t, p, v, w, mass, itype, upd, nn, sp + it.excl, keep, np, acc);
            }
        }
    }
    __syncwarp();
    // cleanUpContacts, one slot per lane (the slots of one atom are
    // independent; npartner drops by the cleared slots that held a partner)
    for (int base = 0; base < it.total; base += 32) {
        const int wq = base + lane;
        const int L = item_owner(min(wq, it.total - 1), it.excl);
        const int iL = __shfl_sync(FULL, i, L);
        const int exL = __shfl_sync(FULL, it.excl, L);
        const unsigned long long keepL = shfl64(keep, L);
        bool held = false;
        if (wq < it.total) {
            const int k = wq - exL;
            if (!((keepL >> k) & 1ull)) {
                held = sp[wq] > -1;
                M.spartner[k * cap + iL] = -1;
                M.shist[(3 * k + 0) * cap + iL] = 0.0;
                M.shist[(3 * k + 1) * cap + iL] = 0.0;
                M.shist[(3 * k + 2) * cap + iL] = 0.0;
            }
        }
        const unsigned bal = __ballot_sync(FULL, held);
        const int lo = max(it.excl, base), hi = min(it.excl + nn, base + 32);
        if (lo < hi) np -= __popc((bal >> (lo - base)) & (unsigned)((1ull << (hi - lo)) - 1ull));
    }
    if (act) M.snp[i] = np;
}

// True when the atom's step is finished by the tail kernel: more than 64
// entries on a side, a primitive wall that lists it, or mesh candidate
// triangles.  The inputs change only at a neighbour build.
__device__ __forceinline__ bool tail_atom(const Dev &D, int k, int nr, int nn)
{
    if (nr > 64 || nn > 64) return true;
    for (int q = 0; q < D.nfix; q++) {
        const FixDev &F = D.fix[q];
        if (F.kind == FIX_WALL_PLANE && F.inlist[k]) return true;
        if (F.kind == FIX_WALL_MESH && F.mesh.tcnt[k] != 0) return true;
    }
    return false;
}

// Cylinder<dim>::calcRadialDistance (src/primitive_wall_definitions.h:165)
__device__ __forceinline__ double cyl_radial(const FixDev &F, const dbl4 &p, double &dy, double &dz)
{
    const double c[3] = {p.x, p.y, p.z};
    const int y = F.dim == 0 ? 1 : (F.dim == 1 ? 2 : 0), z = F.dim == 0 ? 2 : (F.dim == 1 ? 0 : 1);
    dy = (y == 0 ? c[0] : (y == 1 ? c[1] : c[2])) - F.cc1;
    dz = (z == 0 ? c[0] : (z == 1 ? c[1] : c[2])) - F.cc2;
    return sqrt(dy * dy + dz * dz);
}

// FixWallGran::post_force_primitive for one atom in the plane's neighbour
// list (src/fix_wall_gran.cpp:1024-1148, Plane<dim>::resolveContact
// src/primitive_wall_definitions.h:133)
// Returns true when the contact force was added to acc.
__device__ __forceinline__ bool plane_wall_atom(const Dev &D, const FixDev &F, int i, const dbl4 &pi, const double *vi,
                                             const double *wi, double mass, int ti, bool upd, ContactOut &acc)
{
    const int cap = D.cap;
    double deltan;
    double d[3];   // -delta, with constant indices only (keeps d in registers)
    if (F.cyl) {   // Cylinder<dim>::resolveContact (src/primitive_wall_definitions.h:172-197)
        double dy, dz, ey = 0.0, ez = 0.0;
        const double dist = cyl_radial(F, pi, dy, dz);
        if (dist < 1e-13 && dist > -1e-13) {   // compDouble(dist, 0.0): zero delta, zero distance
            deltan = 0.0;
        } else if (dist > F.cr) {
            deltan = dist - F.cr - pi.w;
            const double fact = (dist - F.cr) / dist;
            ey = -dy * fact;
            ez = -dz * fact;
        } else {
            deltan = F.cr - dist - pi.w;
            const double fact = (F.cr - dist) / dist;
            ey = +dy * fact;
            ez = +dz * fact;
        }
        // delta[dim] = 0, delta[(dim+1)%3] = ey, delta[(dim+2)%3] = ez
        const int y = F.dim == 0 ? 1 : (F.dim == 1 ? 2 : 0);
        d[0] = -(y == 0 ? ey : (F.dim == 0 ? 0. : ez));
        d[1] = -(y == 1 ? ey : (F.dim == 1 ? 0. : ez));
        d[2] = -(y == 2 ? ey : (F.dim == 2 ? 0. : ez));
    } else {
        const double x = F.dim == 0 ? pi.x : (F.dim == 1 ? pi.y : pi.z);
        const double delta_d = F.pos - x;
        if (x > F.pos)
            deltan = x - F.pos - pi.w;
        else
            deltan = F.pos - x - pi.w;
        d[0] = F.dim == 0 ? -delta_d : -0.;
        d[1] = F.dim == 1 ? -delta_d : -0.;
        d[2] = F.dim == 2 ? -delta_d : -0.;
    }
    if (deltan > D.cutneighmax) return false;
    if (deltan <= 0) {
        double sh[3] = {F.whist[0 * cap + i], F.whist[1 * cap + i], F.whist[2 * cap + i]};
        const double vwall[3] = {0., 0., 0.};
        wall_contact(mat(D, ti, F.wtype), d, -deltan, pi.w, vi, wi, vwall, mass, sh, upd, D.dt, F.rolling != 0,
                     D.tdamp != 0, acc);
        F.whist[0 * cap + i] = sh[0];
        F.whist[1 * cap + i] = sh[1];
        F.whist[2 * cap + i] = sh[2];
        return true;
    }
    F.whist[0 * cap + i] = 0.0;
    F.whist[1 * cap + i] = 0.0;
    F.whist[2 * cap + i] = 0.0;
    return false;
}

}  // namespace gb2
