// gb2_kernels.cuh -- device kernels of one granular time step (FP64 path).
//
// Included by gb2_engine.cu only.  One thread owns one particle in every
// per-particle kernel: the reference's force sums are sequential per
// particle (src/pair_gran_base.h:255-430), and a per-particle owner thread
// reproduces their order exactly without atomics:
//   f[k] = sum over reverse entries (pairs (i,k), i < k, ascending i)
//        + sum over k's own half-list entries (list order)
//        + post_force fixes in definition order.
// A reverse entry is evaluated from k's side with the pair's shear negated.
// Negation commutes with IEEE rounding and every symmetric expression in the
// model chain (sums, products, sqrt) is evaluated with the same operands, so
// the result is bit-identical to the reference's j_forces for that pair.
#pragma once

#include "gb2_internal.h"

namespace gb2 {

__device__ __forceinline__ dbl4 ld4(const dbl4 *p) { return *p; }

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
// FixNVESphere::initial_integrate (src/fix_nve_sphere.cpp:138-206) and the
// displacement part of Neighbor::check_distance (src/neighbor.cpp:1438)

__global__ void k_initial_integrate(Dev D, int check)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const double dtv = D.dt, dtf = 0.5 * D.dt * 1.0;
    const double dtfrotate = dtf / 0.4;
    dbl4 p = D.pos[i], v = D.vel[i], w = D.omg[i];
    const dbl4 f = D.f[i], t = D.tq[i];
    const double dtfm = dtf / (v.w * 1.0);
    v.x += dtfm * f.x;
    v.y += dtfm * f.y;
    v.z += dtfm * f.z;
    p.x += dtv * v.x;
    p.y += dtv * v.y;
    p.z += dtv * v.z;
    const double dtirotate = dtfrotate / (p.w * p.w * v.w);
    w.x += dtirotate * t.x;
    w.y += dtirotate * t.y;
    w.z += dtirotate * t.z;
    D.pos[i] = p;
    D.vel[i] = v;
    D.omg[i] = w;
    if (check) {
        const dbl4 h = D.xhold[i];
        const double delx = p.x - h.x, dely = p.y - h.y, delz = p.z - h.z;
        const double rsq = delx * delx + dely * dely + delz * delz;
        if (rsq > D.triggersq) *D.dflag = 1;
    }
}

// Comm::forward_comm with AtomVecSphere::pack_comm_vel (src/comm.cpp:773):
// ghost = owned source + accumulated periodic shift
__global__ void k_forward_comm(Dev D)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= D.nghost) return;
    const int src = D.gsrc[g];
    const dbl4 s = D.gshift[g];
    const dbl4 p = D.pos[src];
    dbl4 q;
    q.x = p.x + s.x;
    q.y = p.y + s.y;
    q.z = p.z + s.z;
    q.w = p.w;
    const int gi = D.nlocal + g;
    D.pos[gi] = q;
    D.vel[gi] = D.vel[src];
    D.omg[gi] = D.omg[src];
}

// ------------------------------------------------------------------
// rebuild: FixContactHistory::pre_exchange (src/fix_contact_history.cpp:305)
// converts the half list's flagged slots into per-atom (partner tag, shear)
// records; the j side receives the negated shear (newtonflag = 1).

__global__ void k_partners(Dev D)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.nlocal) return;
    const int cap = D.cap;
    int np = 0;
    // entries where k is the j side
    const int nr = D.rnum[k];
    for (int r = 0; r < nr; r++) {
        const int e = D.rev[r * cap + k];
        if (!D.flag[e]) continue;
        const int s = e / cap, i = e - s * cap;
        if (np < D.maxp) {
            D.ptag[np * cap + k] = D.tag[i];
            for (int c = 0; c < 3; c++) D.phist[(3 * np + c) * cap + k] = -D.hist[(3 * s + c) * cap + i];
        }
        np++;
    }
    const int nn = D.nnum[k];
    for (int s = 0; s < nn; s++) {
        const int e = s * cap + k;
        if (!D.flag[e]) continue;
        if (np < D.maxp) {
            D.ptag[np * cap + k] = D.tag[D.nbr[e]];
            for (int c = 0; c < 3; c++) D.phist[(3 * np + c) * cap + k] = D.hist[(3 * s + c) * cap + k];
        }
        np++;
    }
    if (np > D.maxp) atomicOr(D.status, ST_PARTNER_OVERFLOW);
    D.pnum[k] = min(np, D.maxp);
}

// Domain::pbc (src/domain.cpp:530) and the serial Comm::exchange check
__global__ void k_pbc(Dev D, double lo0, double lo1, double lo2, double hi0, double hi1, double hi2, int p0, int p1,
                      int p2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    dbl4 p = D.pos[i];
    const double lo[3] = {lo0, lo1, lo2}, hi[3] = {hi0, hi1, hi2};
    const int per[3] = {p0, p1, p2};
    double x[3] = {p.x, p.y, p.z};
    for (int d = 0; d < 3; d++) {
        if (per[d]) {
            const double prd = hi[d] - lo[d];
            if (x[d] < lo[d]) x[d] += prd;
            if (x[d] >= hi[d]) {
                x[d] -= prd;
                x[d] = fmax(x[d], lo[d]);
            }
        }
        if (x[d] < lo[d] || x[d] >= hi[d]) atomicOr(D.status, ST_LOST_ATOM);
    }
    p.x = x[0];
    p.y = x[1];
    p.z = x[2];
    D.pos[i] = p;
}

// Atom::sort keys (src/atom.cpp:1343-1354)
__global__ void k_sort_keys(Dev D, double lo0, double lo1, double lo2, double inv0, double inv1, double inv2, int nb0,
                            int nb1, int nb2, unsigned *keys, int *vals)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const dbl4 p = D.pos[i];
    int ix = static_cast<int>((p.x - lo0) * inv0);
    int iy = static_cast<int>((p.y - lo1) * inv1);
    int iz = static_cast<int>((p.z - lo2) * inv2);
    ix = max(ix, 0);
    iy = max(iy, 0);
    iz = max(iz, 0);
    ix = min(ix, nb0 - 1);
    iy = min(iy, nb1 - 1);
    iz = min(iz, nb2 - 1);
    keys[i] = static_cast<unsigned>(iz * nb1 * nb0 + iy * nb0 + ix);
    vals[i] = i;
}

template <typename T>
__global__ void k_gather(const T *__restrict__ src, T *__restrict__ dst, const int *__restrict__ perm, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[perm[i]];
}

// slot-major gather: dst[s*cap + i] = src[s*cap + perm[i]] for s < nslot
template <typename T>
__global__ void k_gather_slots(const T *__restrict__ src, T *__restrict__ dst, const int *__restrict__ perm, int n,
                               int cap, int nslot)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (i < n && s < nslot) dst[(size_t)s * cap + i] = src[(size_t)s * cap + perm[i]];
}

// Comm::borders swap selection (src/comm.cpp:1028, Comm::decide src/comm_I.h:66)
__global__ void k_border_flags(Dev D, int nlast, int dim, int lowside, double bound, uint8_t *flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nlast) return;
    const dbl4 p = D.pos[i];
    const double x = dim == 0 ? p.x : (dim == 1 ? p.y : p.z);
    bool send;
    if (lowside)
        send = x >= -1.0e20 && x <= (bound + p.w);
    else
        send = x >= (bound - p.w) && x <= 1.0e20;
    flags[i] = send ? 1 : 0;
}

__global__ void k_border_fill(Dev D, const int *sel, int nsel, int first, int dim, double shift)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsel) return;
    const int src = sel[k];
    const int g = first + k;                 // absolute index of the new ghost
    const int gi = g - D.nlocal;
    dbl4 sh;
    int root;
    if (src < D.nlocal) {
        root = src;
        sh.x = 0.0;
        sh.y = 0.0;
        sh.z = 0.0;
    } else {
        root = D.gsrc[src - D.nlocal];
        sh = D.gshift[src - D.nlocal];
    }
    // pack_border_vel: x + pbc*prd with the swap's dimension shifted
    if (dim == 0) sh.x = shift;
    if (dim == 1) sh.y = shift;
    if (dim == 2) sh.z = shift;
    sh.w = 0.0;
    D.gsrc[gi] = root;
    D.gshift[gi] = sh;
    const dbl4 p = D.pos[src];
    dbl4 q;
    q.x = p.x + (dim == 0 ? shift : 0.0);
    q.y = p.y + (dim == 1 ? shift : 0.0);
    q.z = p.z + (dim == 2 ? shift : 0.0);
    q.w = p.w;
    D.pos[g] = q;
    D.vel[g] = D.vel[src];
    D.omg[g] = D.omg[src];
    D.type[g] = D.type[src];
    D.tag[g] = D.tag[src];
}

// Neighbor::bin_atoms keys (src/neighbor.cpp:2027)
__global__ void k_bin_keys(Dev D, int nall, unsigned *keys, int *vals, int *counts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nall) return;
    const dbl4 p = D.pos[i];
    int b = coord2bin(D, p.x, p.y, p.z);
    if (b < 0 || b >= D.mbins) {
        atomicOr(D.status, ST_LOST_ATOM);
        b = b < 0 ? 0 : D.mbins - 1;
    }
    keys[i] = static_cast<unsigned>(b);
    vals[i] = i;
    atomicAdd(&counts[b], 1);
}

// Neighbor::granular_bin_no_newton (src/neigh_gran.cpp:485-639): half list
// j > i in stencil order, ascending index within each bin, with the shear
// history restored from the partner records of pairs touching now.
__global__ void k_build_list(Dev D)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const int cap = D.cap;
    const dbl4 pi = D.pos[i];
    const double xtmp = pi.x, ytmp = pi.y, ztmp = pi.z, radi = pi.w;
    const int ibin = coord2bin(D, xtmp, ytmp, ztmp);
    const double skin = D.skin;
    const int np = D.pnum[i];
    int n = 0;
    for (int k = 0; k < D.nstencil; k++) {
        const int b = ibin + D.stencil[k];
        if (b < 0 || b >= D.mbins) continue;
        const int e0 = D.bin_start[b], e1 = D.bin_start[b + 1];
        for (int q = e0; q < e1; q++) {
            const int j = D.bin_atoms[q];
            if (j <= i) continue;
            const dbl4 pj = D.pos[j];
            const double delx = xtmp - pj.x;
            const double dely = ytmp - pj.y;
            const double delz = ztmp - pj.z;
            const double rsq = delx * delx + dely * dely + delz * delz;
            const double radsum = (radi + pj.w) * 1.0;
            const double cutsq = (radsum + skin) * (radsum + skin);
            if (rsq <= cutsq) {
                if (n < D.maxn) {
                    const int e = n * cap + i;
                    D.nbr[e] = j;
                    int fl = 0;
                    double h0 = 0.0, h1 = 0.0, h2 = 0.0;
                    if (rsq < radsum * radsum) {
                        const int tj = D.tag[j];
                        for (int m = 0; m < np; m++)
                            if (D.ptag[m * cap + i] == tj) {
                                fl = 1;
                                h0 = D.phist[(3 * m + 0) * cap + i];
                                h1 = D.phist[(3 * m + 1) * cap + i];
                                h2 = D.phist[(3 * m + 2) * cap + i];
                                break;
                            }
                    }
                    D.flag[e] = fl;
                    D.hist[(3 * n + 0) * cap + i] = h0;
                    D.hist[(3 * n + 1) * cap + i] = h1;
                    D.hist[(3 * n + 2) * cap + i] = h2;
                }
                n++;
            }
        }
    }
    if (n > D.maxn) atomicOr(D.status, ST_NEIGH_OVERFLOW);
    D.nnum[i] = min(n, D.maxn);
    dbl4 h;
    h.x = xtmp;
    h.y = ytmp;
    h.z = ztmp;
    h.w = 0.0;
    D.xhold[i] = h;
}

// reverse list: every local j collects the slots (i, s) with nbr == j
__global__ void k_rev_fill(Dev D)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const int cap = D.cap;
    const int nn = D.nnum[i];
    for (int s = 0; s < nn; s++) {
        const int e = s * cap + i;
        const int j = D.nbr[e];
        if (j >= D.nlocal) continue;
        const int r = atomicAdd(&D.rnum[j], 1);
        if (r < D.maxr)
            D.rev[r * cap + j] = e;
        else
            atomicOr(D.status, ST_REV_OVERFLOW);
    }
}

// order each reverse segment by owner index (the reference loop order)
__global__ void k_rev_sort(Dev D)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.nlocal) return;
    const int cap = D.cap;
    int n = D.rnum[k];
    if (n > D.maxr) n = D.maxr;
    D.rnum[k] = n;
    for (int a = 1; a < n; a++) {
        const int ea = D.rev[a * cap + k];
        const int ia = ea % cap;
        int b = a - 1;
        while (b >= 0 && D.rev[b * cap + k] % cap > ia) {
            D.rev[(b + 1) * cap + k] = D.rev[b * cap + k];
            b--;
        }
        D.rev[(b + 1) * cap + k] = ea;
    }
}

// PrimitiveWall::buildNeighList (src/primitive_wall.h:129) for a plane
__global__ void k_plane_neighlist(Dev D, int ifix)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const FixDev &F = D.fix[ifix];
    const dbl4 p = D.pos[i];
    const double x = F.dim == 0 ? p.x : (F.dim == 1 ? p.y : p.z);
    const double dMax = p.w + D.skin;
    const double dist = x - F.pos;
    const double absdist = (dist > 0.0) ? dist : -dist;
    F.inlist[i] = (absdist <= dMax) ? 1 : 0;
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

// FixNeighlistMesh::pre_force per owned atom: triangles (ascending) whose
// bin list holds the atom's bin and that pass the neighbour-build test
__global__ void k_mesh_candidates(Dev D, int ifix)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const MeshDev &M = D.fix[ifix].mesh;
    const int cap = D.cap;
    const dbl4 p = D.pos[i];
    const int b = coord2bin(D, p.x, p.y, p.z);
    const double c[3] = {p.x, p.y, p.z};
    int n = 0;
    if (b >= 0 && b < D.mbins) {
        const int t0 = M.bin_tri_start[b], t1 = M.bin_tri_start[b + 1];
        for (int q = t0; q < t1; q++) {
            const int t = M.bin_tri_list[q];
            if (tri_neighbuild(M.tri[t], p.w * 1.0, c, M.nl_skin)) {
                if (n < M.maxt) M.tlist[n * cap + i] = t;
                n++;
            }
        }
    }
    if (n > M.maxt) atomicOr(D.status, ST_MESHSLOT_OVERFLOW);
    M.tcnt[i] = min(n, M.maxt);
}

__device__ __forceinline__ void mesh_swap_slot(const MeshDev &M, int cap, int i, int a, int b)
{
    const int t = M.spartner[a * cap + i];
    M.spartner[a * cap + i] = M.spartner[b * cap + i];
    M.spartner[b * cap + i] = t;
    for (int c = 0; c < 3; c++) {
        const double h = M.shist[(3 * a + c) * cap + i];
        M.shist[(3 * a + c) * cap + i] = M.shist[(3 * b + c) * cap + i];
        M.shist[(3 * b + c) * cap + i] = h;
    }
}

// FixContactHistoryMesh::sort_contacts (src/fix_contact_history_mesh.cpp:375)
__global__ void k_mesh_sort_contacts(Dev D, int ifix)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const MeshDev &M = D.fix[ifix].mesh;
    const int cap = D.cap;
    const int nn = M.tcnt[i];
    if (nn == 0) return;
    int fe, lf;
    do {
        fe = lf = -1;
        for (int j = 0; j < nn; j++) {
            if (-1 == fe && -1 == M.spartner[j * cap + i]) fe = j;
            if (M.spartner[j * cap + i] >= 0) lf = j;
        }
        if (fe > -1 && lf > -1 && fe < lf) mesh_swap_slot(M, cap, i, fe, lf);
    } while (fe > -1 && lf > -1 && fe < lf);
}

// FixContactHistoryMesh::pre_force with cleanUpContactJumps
// (src/fix_contact_history_mesh.cpp:315-373, :466-508).  Reads the old slot
// arrays (oldM) and writes re-paged slots sized to the new candidate count.
__global__ void k_mesh_repage(Dev D, int ifix, int *old_snp, int *old_spartner, double *old_shist, int old_maxt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const MeshDev &M = D.fix[ifix].mesh;
    const int cap = D.cap;
    int np = old_snp[i];
    const int nn = M.tcnt[i];
    int ip = 0;
    while (ip < np) {
        const int tri = old_spartner[ip * cap + i];
        bool inlist = false;
        for (int q = 0; q < nn; q++)
            if (M.tlist[q * cap + i] == tri) {
                inlist = true;
                break;
            }
        if (tri < 0) atomicOr(D.status, ST_MESH_INTERNAL);
        if (!inlist) {
            old_spartner[ip * cap + i] = -1;
            for (int c = 0; c < 3; c++) old_shist[(3 * ip + c) * cap + i] = 0.0;
            // swap(i, ipartner, npartner-1)
            const int last = np - 1;
            const int t = old_spartner[ip * cap + i];
            old_spartner[ip * cap + i] = old_spartner[last * cap + i];
            old_spartner[last * cap + i] = t;
            for (int c = 0; c < 3; c++) {
                const double h = old_shist[(3 * ip + c) * cap + i];
                old_shist[(3 * ip + c) * cap + i] = old_shist[(3 * last + c) * cap + i];
                old_shist[(3 * last + c) * cap + i] = h;
            }
            np--;
        } else
            ip++;
    }
    (void)old_maxt;
    if (np > nn) atomicOr(D.status, ST_MESH_INTERNAL);
    for (int k = 0; k < nn; k++) {
        int t = -1;
        double h0 = 0.0, h1 = 0.0, h2 = 0.0;
        if (k < np) {
            t = old_spartner[k * cap + i];
            h0 = old_shist[(3 * k + 0) * cap + i];
            h1 = old_shist[(3 * k + 1) * cap + i];
            h2 = old_shist[(3 * k + 2) * cap + i];
        }
        M.spartner[k * cap + i] = t;
        M.shist[(3 * k + 0) * cap + i] = h0;
        M.shist[(3 * k + 1) * cap + i] = h1;
        M.shist[(3 * k + 2) * cap + i] = h2;
    }
    M.snp[i] = min(np, nn);
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

__device__ double tri_edge(const TriGeom &T, int iEdge, const double *p, double *delta)
{
    const int ip = (iEdge + 1) % 3;
    double nodeToP[3] = {p[0] - T.node[iEdge][0], p[1] - T.node[iEdge][1], p[2] - T.node[iEdge][2]};
    const double distFromNode = dot3(nodeToP, T.edgevec[iEdge]);
    if (distFromNode < -GB2_SMALL_TRIMESH) {
        if (!GB2_CORNER_ACTIVE(T, iEdge)) return GB2_LARGE_TRIMESH;
        return calc_dist(p, T.node[iEdge], delta);
    } else if (distFromNode > T.edgelen[iEdge] + GB2_SMALL_TRIMESH) {
        if (!GB2_CORNER_ACTIVE(T, ip)) return GB2_LARGE_TRIMESH;
        return calc_dist(p, T.node[ip], delta);
    }
    if (!GB2_EDGE_ACTIVE(T, iEdge)) return GB2_LARGE_TRIMESH;
    double cp[3];
    cp[0] = T.node[iEdge][0] + distFromNode * T.edgevec[iEdge][0];
    cp[1] = T.node[iEdge][1] + distFromNode * T.edgevec[iEdge][1];
    cp[2] = T.node[iEdge][2] + distFromNode * T.edgevec[iEdge][2];
    return calc_dist(p, cp, delta);
}

__device__ double tri_corner(const TriGeom &T, int iNode, bool obtuse, const double *p, double *delta)
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
                return calc_dist(p, cp, delta);
            }
            if (!GB2_CORNER_ACTIVE(T, ipp)) return GB2_LARGE_TRIMESH;
            return calc_dist(p, T.node[ipp], delta);
        }
        distFromNode = dot3(nodeToP, T.edgevec[iNode]);
        if (distFromNode > -GB2_SMALL_TRIMESH) {
            if (distFromNode < T.edgelen[iNode]) {
                if (!GB2_EDGE_ACTIVE(T, iNode)) return GB2_LARGE_TRIMESH;
                cp[0] = n[0] + distFromNode * T.edgevec[iNode][0];
                cp[1] = n[1] + distFromNode * T.edgevec[iNode][1];
                cp[2] = n[2] + distFromNode * T.edgevec[iNode][2];
                return calc_dist(p, cp, delta);
            }
            if (!GB2_CORNER_ACTIVE(T, ip)) return GB2_LARGE_TRIMESH;
            return calc_dist(p, T.node[ip], delta);
        }
    }
    if (!GB2_CORNER_ACTIVE(T, iNode)) return GB2_LARGE_TRIMESH;
    return calc_dist(p, T.node[iNode], delta);
}

__device__ double tri_sphere(const TriGeom &T, double rSphere, const double *cs, double *delta, int &barySign,
                             double precision)
{
    double n0ToC[3] = {cs[0] - T.node[0][0], cs[1] - T.node[0][1], cs[2] - T.node[0][2]};
    // MathExtraLiggghts::calcBaryTriCoords (src/math_extra_liggghts.h:559)
    const double a = dot3(n0ToC, T.edgevec[0]);
    const double b = dot3(n0ToC, T.edgevec[2]);
    const double c = dot3(T.edgevec[0], T.edgevec[2]);
    const double oneMinCSqr = 1 - c * c;
    double bary[3];
    bary[1] = (a - b * c) / (T.edgelen[0] * oneMinCSqr);
    bary[2] = (a * c - b) / (T.edgelen[2] * oneMinCSqr);
    bary[0] = 1. - bary[1] - bary[2];
    const double invlen = 1. / (2. * T.rbound);
    barySign = (bary[0] > -precision * invlen) + 2 * (bary[1] > -precision * invlen) +
               4 * (bary[2] > -precision * invlen);
    double d;
    switch (barySign) {
    case 1: d = tri_corner(T, 0, T.obtuse == 0, cs, delta); break;
    case 2: d = tri_corner(T, 1, T.obtuse == 1, cs, delta); break;
    case 3: d = tri_edge(T, 0, cs, delta); break;
    case 4: d = tri_corner(T, 2, T.obtuse == 2, cs, delta); break;
    case 5: d = tri_edge(T, 2, cs, delta); break;
    case 6: d = tri_edge(T, 1, cs, delta); break;
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
// pair pass A: contributions of the entries where k is the j side,
// evaluated from k's side (see file header), in ascending owner order

template <bool ROLLING>
__global__ void __launch_bounds__(128) k_pair_reverse(Dev D, int shearupdate)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.nlocal) return;
    const int cap = D.cap;
    const dbl4 pk = D.pos[k], vk4 = D.vel[k], wk4 = D.omg[k];
    const int tk = D.type[k];
    const double vk[3] = {vk4.x, vk4.y, vk4.z}, wk[3] = {wk4.x, wk4.y, wk4.z};
    ContactOut acc;
    acc.F[0] = acc.F[1] = acc.F[2] = 0.0;
    acc.T[0] = acc.T[1] = acc.T[2] = 0.0;
    const int nr = D.rnum[k];
    for (int r = 0; r < nr; r++) {
        const int e = D.rev[r * cap + k];
        const int s = e / cap, i = e - s * cap;
        const dbl4 pi = D.pos[i];
        const double delx = pk.x - pi.x;
        const double dely = pk.y - pi.y;
        const double delz = pk.z - pi.z;
        const double rsq = delx * delx + dely * dely + delz * delz;
        const double radsum = pk.w + pi.w;
        if (!(rsq < radsum * radsum)) continue;
        const dbl4 vi4 = D.vel[i], wi4 = D.omg[i];
        const double vi[3] = {vi4.x, vi4.y, vi4.z}, wi[3] = {wi4.x, wi4.y, wi4.z};
        double sh[3];
        sh[0] = -D.hist[(3 * s + 0) * cap + i];
        sh[1] = -D.hist[(3 * s + 1) * cap + i];
        sh[2] = -D.hist[(3 * s + 2) * cap + i];
        // material lookup in the reference's (owner, neighbour) order
        pair_contact(mat(D, D.type[i], tk), delx, dely, delz, rsq, pk.w, pi.w, vk, vi, wk, wi, vk4.w, vi4.w, sh,
                     shearupdate != 0, D.dt, ROLLING, D.tdamp != 0, acc);
    }
    dbl4 F, T;
    F.x = acc.F[0];
    F.y = acc.F[1];
    F.z = acc.F[2];
    F.w = 0.0;
    T.x = acc.T[0];
    T.y = acc.T[1];
    T.z = acc.T[2];
    T.w = 0.0;
    D.fpart[k] = F;
    D.tpart[k] = T;
}

// ------------------------------------------------------------------
// pair pass B + post_force fixes + FixNVESphere::final_integrate

__device__ void mesh_wall_atom(const Dev &D, const MeshDev &M, int i, const dbl4 &p, const double v[3],
                               const double w[3], double mass, int itype, bool upd, ContactOut &acc)
{
    const int cap = D.cap;
    const int nn = M.tcnt[i];
    if (nn == 0) return;
    unsigned long long keep = 0ull;   // markAllContacts
    const double cs[3] = {p.x, p.y, p.z};
    const double vwall[3] = {0.0, 0.0, 0.0};
    int np = M.snp[i];
    for (int q = 0; q < nn; q++) {
        const int t = M.tlist[q * cap + i];
        const TriGeom &T = M.tri[t];
        double delta[3];
        int barysign = -1;
        const double deltan = tri_sphere(T, p.w, cs, delta, barysign, 1e-8);
        if (deltan > D.cutneighmax) continue;
        if (!(deltan <= 0)) continue;
        const bool faceflag = (7 == barysign);
        // FixContactHistoryMesh::handleContact
        int slot = -1;
        for (int k = 0; k < nn; k++)
            if (M.spartner[k * cap + i] == t) {
                slot = k;
                break;
            }
        if (slot >= 0) {
            keep |= 1ull << slot;
        } else {
            bool skip = false;
            if (faceflag) {
                for (int k = 0; k < nn; k++) {
                    const int idp = M.spartner[k * cap + i];
                    if (idp >= 0 && idp != t && coplanar_node_neighs(M, idp, t) && ((keep >> k) & 1ull)) {
                        skip = true;
                        break;
                    }
                }
            }
            if (skip) continue;
            int ic = -1;
            for (int k = 0; k < nn; k++)
                if (-1 == M.spartner[k * cap + i]) {
                    ic = k;
                    break;
                }
            if (ic < 0 || np >= nn) {
                atomicOr(D.status, ST_MESH_INTERNAL);
                continue;
            }
            M.spartner[ic * cap + i] = t;
            keep |= 1ull << ic;
            double h0 = 0.0, h1 = 0.0, h2 = 0.0;
            np++;
            if (faceflag) {
                for (int k = 0; k < nn; k++) {
                    const int tri = M.spartner[k * cap + i];
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
        wall_contact(mat(D, itype, M.wtype), dvec, -deltan, p.w, v, w, vwall, mass, sh, upd, D.dt, M.rolling != 0,
                     D.tdamp != 0, acc);
        M.shist[(3 * slot + 0) * cap + i] = sh[0];
        M.shist[(3 * slot + 1) * cap + i] = sh[1];
        M.shist[(3 * slot + 2) * cap + i] = sh[2];
    }
    // cleanUpContacts
    for (int k = 0; k < nn; k++)
        if (!((keep >> k) & 1ull)) {
            if (M.spartner[k * cap + i] > -1) np--;
            M.spartner[k * cap + i] = -1;
            M.shist[(3 * k + 0) * cap + i] = 0.0;
            M.shist[(3 * k + 1) * cap + i] = 0.0;
            M.shist[(3 * k + 2) * cap + i] = 0.0;
        }
    M.snp[i] = np;
}

template <bool ROLLING>
__global__ void __launch_bounds__(128) k_pair_main(Dev D, int shearupdate, int integrate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const int cap = D.cap;
    const dbl4 pi = D.pos[i];
    dbl4 vi4 = D.vel[i], wi4 = D.omg[i];
    const int ti = D.type[i];
    const double vi[3] = {vi4.x, vi4.y, vi4.z}, wi[3] = {wi4.x, wi4.y, wi4.z};
    const bool upd = shearupdate != 0;
    ContactOut acc;
    {
        const dbl4 F = D.fpart[i], T = D.tpart[i];
        acc.F[0] = F.x;
        acc.F[1] = F.y;
        acc.F[2] = F.z;
        acc.T[0] = T.x;
        acc.T[1] = T.y;
        acc.T[2] = T.z;
    }
    const int nn = D.nnum[i];
    for (int s = 0; s < nn; s++) {
        const int e = s * cap + i;
        const int j = D.nbr[e];
        const dbl4 pj = D.pos[j];
        const double delx = pi.x - pj.x;
        const double dely = pi.y - pj.y;
        const double delz = pi.z - pj.z;
        const double rsq = delx * delx + dely * dely + delz * delz;
        const double radsum = pi.w + pj.w;
        if (!(rsq < radsum * radsum)) continue;
        const dbl4 vj4 = D.vel[j], wj4 = D.omg[j];
        const double vj[3] = {vj4.x, vj4.y, vj4.z}, wj[3] = {wj4.x, wj4.y, wj4.z};
        const int fl = D.flag[e];
        if ((fl | 5) != fl) D.flag[e] = fl | 5;   // CONTACT_NORMAL_MODEL | CONTACT_TANGENTIAL_MODEL
        double sh[3] = {D.hist[(3 * s + 0) * cap + i], D.hist[(3 * s + 1) * cap + i], D.hist[(3 * s + 2) * cap + i]};
        pair_contact(mat(D, ti, D.type[j]), delx, dely, delz, rsq, pi.w, pj.w, vi, vj, wi, wj, vi4.w, vj4.w, sh, upd,
                     D.dt, ROLLING, D.tdamp != 0, acc);
        if (upd) {
            D.hist[(3 * s + 0) * cap + i] = sh[0];
            D.hist[(3 * s + 1) * cap + i] = sh[1];
            D.hist[(3 * s + 2) * cap + i] = sh[2];
        }
    }
    // post_force fixes in definition order
    for (int k = 0; k < D.nfix; k++) {
        const FixDev &F = D.fix[k];
        if (F.kind == FIX_GRAVITY) {
            const double massone = vi4.w * 1.;
            acc.F[0] += massone * F.acc[0];
            acc.F[1] += massone * F.acc[1];
            acc.F[2] += massone * F.acc[2];
        } else if (F.kind == FIX_WALL_PLANE) {
            if (!F.inlist[i]) continue;
            const double x = F.dim == 0 ? pi.x : (F.dim == 1 ? pi.y : pi.z);
            double delta_d, deltan;
            delta_d = F.pos - x;
            if (x > F.pos)
                deltan = x - F.pos - pi.w;
            else
                deltan = F.pos - x - pi.w;
            if (deltan > D.cutneighmax) continue;
            if (deltan <= 0) {
                double d[3] = {-0., -0., -0.};
                d[F.dim] = -delta_d;
                double sh[3] = {F.whist[0 * cap + i], F.whist[1 * cap + i], F.whist[2 * cap + i]};
                const double vwall[3] = {0., 0., 0.};
                wall_contact(mat(D, ti, F.wtype), d, -deltan, pi.w, vi, wi, vwall, vi4.w, sh, upd, D.dt,
                             F.rolling != 0, D.tdamp != 0, acc);
                F.whist[0 * cap + i] = sh[0];
                F.whist[1 * cap + i] = sh[1];
                F.whist[2 * cap + i] = sh[2];
            } else {
                F.whist[0 * cap + i] = 0.0;
                F.whist[1 * cap + i] = 0.0;
                F.whist[2 * cap + i] = 0.0;
            }
        } else if (F.kind == FIX_WALL_MESH) {
            mesh_wall_atom(D, F.mesh, i, pi, vi, wi, vi4.w, ti, upd, acc);
        }
    }
    dbl4 Fo, To;
    Fo.x = acc.F[0];
    Fo.y = acc.F[1];
    Fo.z = acc.F[2];
    Fo.w = 0.0;
    To.x = acc.T[0];
    To.y = acc.T[1];
    To.z = acc.T[2];
    To.w = 0.0;
    D.f[i] = Fo;
    D.tq[i] = To;
    if (integrate) {
        // FixNVESphere::final_integrate (src/fix_nve_sphere.cpp:208-246)
        const double dtf = 0.5 * D.dt * 1.0;
        const double dtfrotate = dtf / 0.4;
        const double dtfm = dtf / (vi4.w * 1.0);
        vi4.x += dtfm * Fo.x;
        vi4.y += dtfm * Fo.y;
        vi4.z += dtfm * Fo.z;
        const double dtirotate = dtfrotate / (pi.w * pi.w * vi4.w);
        wi4.x += dtirotate * To.x;
        wi4.y += dtirotate * To.y;
        wi4.z += dtirotate * To.z;
        // written to the second buffer: other threads of this pass still
        // read vel/omg of this atom as neighbour state
        D.vel_out[i] = vi4;
        D.omg_out[i] = wi4;
    }
}

// contact census (diagnostics and the bench's byte model)
__global__ void k_census(Dev D, unsigned long long *cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const int cap = D.cap;
    const dbl4 pi = D.pos[i];
    const int nn = D.nnum[i];
    unsigned long long touch = 0;
    for (int s = 0; s < nn; s++) {
        const dbl4 pj = D.pos[D.nbr[s * cap + i]];
        const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const double rs = pi.w + pj.w;
        if (dx * dx + dy * dy + dz * dz < rs * rs) touch++;
    }
    unsigned long long wl = 0, wt = 0, mc = 0, mt = 0;
    for (int k = 0; k < D.nfix; k++) {
        const FixDev &F = D.fix[k];
        if (F.kind == FIX_WALL_PLANE && F.inlist[i]) {
            wl++;
            const double x = F.dim == 0 ? pi.x : (F.dim == 1 ? pi.y : pi.z);
            const double dist = x > F.pos ? x - F.pos - pi.w : F.pos - x - pi.w;
            if (dist <= 0) wt++;
        } else if (F.kind == FIX_WALL_MESH) {
            const int tc = F.mesh.tcnt[i];
            mc += tc;
            for (int q = 0; q < tc; q++)
                if (F.mesh.spartner[q * cap + i] >= 0) mt++;
        }
    }
    atomicAdd(&cnt[0], (unsigned long long)nn);
    if (touch) atomicAdd(&cnt[1], touch);
    atomicAdd(&cnt[2], (unsigned long long)D.rnum[i]);
    if (wl) atomicAdd(&cnt[3], wl);
    if (wt) atomicAdd(&cnt[4], wt);
    if (mc) atomicAdd(&cnt[5], mc);
    if (mt) atomicAdd(&cnt[6], mt);
}

}  // namespace gb2
