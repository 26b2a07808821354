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
        const int i = D.rev[r * cap + k];
        const int s = D.revs[r * cap + k];
        if (!D.flag[s * cap + i]) continue;
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

// slot-major gather of the slots an atom uses: dst[s*cap+i] = src[s*cap+perm[i]]
// for s / div < cnt_old[perm[i]] (all slots when cnt_old is null)
template <typename T>
__global__ void k_gather_slots_cnt(const T *__restrict__ src, T *__restrict__ dst, const int *__restrict__ perm, int n,
                                   int cap, int nslot, const int *__restrict__ cnt_old, int div)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (i >= n || s >= nslot) return;
    const int o = perm[i];
    if (cnt_old && s / div >= cnt_old[o]) return;
    dst[(size_t)s * cap + i] = src[(size_t)s * cap + o];
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
                    // both history buffers, so either can serve as the next read buffer
                    D.hist[(3 * n + 0) * cap + i] = h0;
                    D.hist[(3 * n + 1) * cap + i] = h1;
                    D.hist[(3 * n + 2) * cap + i] = h2;
                    D.hist_out[(3 * n + 0) * cap + i] = h0;
                    D.hist_out[(3 * n + 1) * cap + i] = h1;
                    D.hist_out[(3 * n + 2) * cap + i] = h2;
                }
                n++;
            }
        }
    }
    if (n > D.maxn) atomicOr(D.status, ST_NEIGH_OVERFLOW);
    D.nnum[i] = min(n, D.maxn);
    D.prevmask[i] = 0ull;
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
        if (r < D.maxr) {
            D.rev[r * cap + j] = i;
            D.revs[r * cap + j] = (uint8_t)s;
        } else
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
        const int ia = D.rev[a * cap + k];
        const uint8_t sa = D.revs[a * cap + k];
        int b = a - 1;
        while (b >= 0 && D.rev[b * cap + k] > ia) {
            D.rev[(b + 1) * cap + k] = D.rev[b * cap + k];
            D.revs[(b + 1) * cap + k] = D.revs[b * cap + k];
            b--;
        }
        D.rev[(b + 1) * cap + k] = ia;
        D.revs[(b + 1) * cap + k] = sa;
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
    for (int t = 0; t < n; t += 2) {
        const int a0 = (t < nr) ? ld_stream(&D.rev[t * cap + k]) : k;
        const int a1 = (t + 1 < nr) ? ld_stream(&D.rev[(t + 1) * cap + k]) : k;
        const int b0 = (t < nn) ? ld_stream(&D.nbr[t * cap + k]) : k;
        const int b1 = (t + 1 < nn) ? ld_stream(&D.nbr[(t + 1) * cap + k]) : k;
        const dbl4 qa0 = ldg4(&D.pos[a0]);
        const dbl4 qa1 = ldg4(&D.pos[a1]);
        const dbl4 qb0 = ldg4(&D.pos[b0]);
        const dbl4 qb1 = ldg4(&D.pos[b1]);
        if (t < nr && touching(pk, qa0)) mrev |= 1ull << t;
        if (t + 1 < nr && touching(pk, qa1)) mrev |= 1ull << (t + 1);
        if (t < nn && touching(pk, qb0)) mown |= 1ull << t;
        if (t + 1 < nn && touching(pk, qb1)) mown |= 1ull << (t + 1);
    }
}

// Screening of n <= 64 list entries idx[r*cap + k]: four index loads, then
// four independent neighbour-record gathers, then the four distance tests,
// so a thread keeps several loads in flight.  Returns the touching mask.
__device__ __forceinline__ unsigned long long screen_entries(const int *__restrict__ idx, int cap, int k, int n,
                                                            const dbl4 &pk, const dbl4 *__restrict__ pos)
{
    unsigned long long m = 0ull;
    for (int r0 = 0; r0 < n; r0 += 4) {
        const int j0 = __ldg(&idx[min(r0 + 0, n - 1) * cap + k]);
        const int j1 = __ldg(&idx[min(r0 + 1, n - 1) * cap + k]);
        const int j2 = __ldg(&idx[min(r0 + 2, n - 1) * cap + k]);
        const int j3 = __ldg(&idx[min(r0 + 3, n - 1) * cap + k]);
        const dbl4 q0 = ldg4(&pos[j0]);
        const dbl4 q1 = ldg4(&pos[j1]);
        const dbl4 q2 = ldg4(&pos[j2]);
        const dbl4 q3 = ldg4(&pos[j3]);
        if (touching(pk, q0)) m |= 1ull << r0;
        if (r0 + 1 < n && touching(pk, q1)) m |= 1ull << (r0 + 1);
        if (r0 + 2 < n && touching(pk, q2)) m |= 1ull << (r0 + 2);
        if (r0 + 3 < n && touching(pk, q3)) m |= 1ull << (r0 + 3);
    }
    return m;
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

__device__ __forceinline__ void mesh_wall_atom(const Dev &D, const MeshDev &M, int i, const dbl4 &p, const double v[3],
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

// An atom with more than 64 reverse or own entries, evaluated serially in
// the reference order (rare; kept out of line so the hot loop stays small).
template <bool ROLLING>
__device__ __forceinline__ void serial_atom(const Dev &D, int k, const dbl4 &pk, const dbl4 &vi4, const dbl4 &wi4, int tk,
                                         int nr, int nn, bool upd, ContactOut &acc)
{
    const int cap = D.cap;
    const double vk[3] = {vi4.x, vi4.y, vi4.z}, wk[3] = {wi4.x, wi4.y, wi4.z};
    // more than 64 entries on one side: every entry in order on this lane
    for (int r = 0; r < nr; r++) {
        const int i = __ldg(&D.rev[r * cap + k]);
        const dbl4 pi = ldg4(&D.pos[i]);
        const double delx = pk.x - pi.x;
        const double dely = pk.y - pi.y;
        const double delz = pk.z - pi.z;
        const double rsq = delx * delx + dely * dely + delz * delz;
        const double radsum = pk.w + pi.w;
        if (!(rsq < radsum * radsum)) continue;
        const int s = D.revs[r * cap + k];
        const dbl4 v4 = ldg4(&D.vel[i]), w4 = ldg4(&D.omg[i]);
        const double vi[3] = {v4.x, v4.y, v4.z}, wi[3] = {w4.x, w4.y, w4.z};
        double sh[3];
        sh[0] = -D.hist[(3 * s + 0) * cap + i];
        sh[1] = -D.hist[(3 * s + 1) * cap + i];
        sh[2] = -D.hist[(3 * s + 2) * cap + i];
        pair_contact(mat(D, D.type[i], tk), delx, dely, delz, rsq, pk.w, pi.w, vk, vi, wk, wi, vi4.w, v4.w, sh,
                     upd, D.dt, ROLLING, D.tdamp != 0, acc);
    }
    for (int s = 0; s < nn; s++) {
        const int e = s * cap + k;
        const int j = __ldg(&D.nbr[e]);
        const dbl4 pj = ldg4(&D.pos[j]);
        const double delx = pk.x - pj.x;
        const double dely = pk.y - pj.y;
        const double delz = pk.z - pj.z;
        const double rsq = delx * delx + dely * dely + delz * delz;
        const double radsum = pk.w + pj.w;
        double sh[3] = {D.hist[(3 * s + 0) * cap + k], D.hist[(3 * s + 1) * cap + k],
                        D.hist[(3 * s + 2) * cap + k]};
        if (rsq < radsum * radsum) {
            const dbl4 v4 = ldg4(&D.vel[j]), w4 = ldg4(&D.omg[j]);
            const double vj[3] = {v4.x, v4.y, v4.z}, wj[3] = {w4.x, w4.y, w4.z};
            const int fl = D.flag[e];
            if ((fl | 5) != fl) D.flag[e] = fl | 5;
            pair_contact(mat(D, tk, D.type[j]), delx, dely, delz, rsq, pk.w, pj.w, vk, vj, wk, wj, vi4.w, v4.w,
                         sh, upd, D.dt, ROLLING, D.tdamp != 0, acc);
        }
        if (upd) {   // serial atoms write every slot
            D.hist_out[(3 * s + 0) * cap + k] = sh[0];
            D.hist_out[(3 * s + 1) * cap + k] = sh[1];
            D.hist_out[(3 * s + 2) * cap + k] = sh[2];
        }
    }
}

// FixWallGran::post_force_primitive for one atom in the plane's neighbour
// list (src/fix_wall_gran.cpp:1024-1148, Plane<dim>::resolveContact
// src/primitive_wall_definitions.h:133)
__device__ __forceinline__ void plane_wall_atom(const Dev &D, const FixDev &F, int i, const dbl4 &pi, const double *vi,
                                             const double *wi, double mass, int ti, bool upd, ContactOut &acc)
{
    const int cap = D.cap;
    const double x = F.dim == 0 ? pi.x : (F.dim == 1 ? pi.y : pi.z);
    double delta_d, deltan;
    delta_d = F.pos - x;
    if (x > F.pos)
        deltan = x - F.pos - pi.w;
    else
        deltan = F.pos - x - pi.w;
    if (deltan > D.cutneighmax) return;
    if (deltan <= 0) {
        // -delta with constant indices only (keeps d in registers)
        const double d[3] = {F.dim == 0 ? -delta_d : -0., F.dim == 1 ? -delta_d : -0., F.dim == 2 ? -delta_d : -0.};
        double sh[3] = {F.whist[0 * cap + i], F.whist[1 * cap + i], F.whist[2 * cap + i]};
        const double vwall[3] = {0., 0., 0.};
        wall_contact(mat(D, ti, F.wtype), d, -deltan, pi.w, vi, wi, vwall, mass, sh, upd, D.dt, F.rolling != 0,
                     D.tdamp != 0, acc);
        F.whist[0 * cap + i] = sh[0];
        F.whist[1 * cap + i] = sh[1];
        F.whist[2 * cap + i] = sh[2];
    } else {
        F.whist[0 * cap + i] = 0.0;
        F.whist[1 * cap + i] = 0.0;
        F.whist[2 * cap + i] = 0.0;
    }
}

// The pair step: PairGran::compute for one owned atom k with its j-side
// (reverse) entries and its own half-list entries, the post_force fixes,
// FixNVESphere::final_integrate and -- when the run continues -- the next
// step's initial_integrate with the displacement check.
//
// Shear history is double-buffered.  Invariant: when a step starts, every
// slot's current shear is in `hist` (the read buffer); the step writes the
// write buffer `hist_out`, which becomes the read buffer of the next step.
// A touching slot is read from hist and its update written to hist_out; a
// slot that stopped touching this step is copied once (after that both
// buffers agree); a rebuild writes both buffers.  Reverse entries therefore
// read the pre-update shear without racing the owner's update, exactly as
// the reference evaluates the pair once before the owner's shear changes.
//
// Per warp, the touching entries of its 32 atoms are enumerated owner-major
// (reverse entries in ascending owner order, then own entries in list
// order), evaluated one per lane in rounds of 32 with results staged in
// shared memory, and summed by each owner lane in that order.  Atoms with
// more than 64 reverse or own entries are evaluated serially by their owner
// lane after the rounds, in the same order.
template <bool ROLLING, int MINB>
__global__ void __launch_bounds__(128, MINB) k_pair_step(Dev D, int shearupdate, int integrate, int fuse_next,
                                                         int store_f)
{
    __shared__ double sres[4][32][6];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int wbase = blockIdx.x * blockDim.x + wid * 32;
    const bool valid = k < D.nlocal;
    const int cap = D.cap;
    const bool upd = shearupdate != 0;
    dbl4 pk, vi4, wi4, hold;
    unsigned long long prevm = 0ull;
    int nr = 0, nn = 0, tk = 0;
    unsigned long long mrev = 0ull, mown = 0ull;
    bool serial = false;
    if (valid) {
        // the atom's own records, including those only the tail needs, are
        // requested first so their latency overlaps the screening
        pk = D.pos[k];
        nr = D.rnum[k];
        nn = D.nnum[k];
        vi4 = D.vel[k];
        wi4 = D.omg[k];
        tk = D.type[k];
        if (fuse_next) hold = D.xhold[k];
        if (upd) prevm = D.prevmask[k];
        serial = nr > 64 || nn > 64;
        if (!serial) screen_both(D, k, nr, nn, pk, mrev, mown);
    }
    ContactOut acc;
    acc.F[0] = acc.F[1] = acc.F[2] = 0.0;
    acc.T[0] = acc.T[1] = acc.T[2] = 0.0;
    const int crev = __popcll(mrev);
    {
        const WarpItems it = warp_items_cnt(crev + __popcll(mown));
        for (int base = 0; base < it.total; base += 32) {
            const int w = base + lane;
            const int L = item_owner(w, it.excl);
            const int exL = __shfl_sync(0xffffffffu, it.excl, L);
            const unsigned long long mrL = shfl64(mrev, L);
            const unsigned long long moL = shfl64(mown, L);
            if (w < it.total) {
                const int kk = wbase + L;
                const int q = w - exL;
                const int qr = __popcll(mrL);
                const dbl4 pkk = ldg4(&D.pos[kk]), vk4 = ldg4(&D.vel[kk]), wk4 = ldg4(&D.omg[kk]);
                const double vk[3] = {vk4.x, vk4.y, vk4.z}, wk[3] = {wk4.x, wk4.y, wk4.z};
                // operands of one pair: j-side entries are evaluated from kk's side
                // with the shear negated, own entries update kk's slot
                int other, s, e = -1;
                double sgn;
                bool own;
                if (q < qr) {
                    const int r = nth_set_bit(mrL, q);
                    other = __ldg(&D.rev[r * cap + kk]);
                    s = D.revs[r * cap + kk];
                    sgn = -1.0;
                    own = false;
                } else {
                    s = nth_set_bit(moL, q - qr);
                    e = s * cap + kk;
                    other = __ldg(&D.nbr[e]);
                    sgn = 1.0;
                    own = true;
                }
                const int hrow = own ? kk : other;
                const dbl4 po = ldg4(&D.pos[other]), vo4 = ldg4(&D.vel[other]), wo4 = ldg4(&D.omg[other]);
                const double delx = pkk.x - po.x;
                const double dely = pkk.y - po.y;
                const double delz = pkk.z - po.z;
                const double rsq = delx * delx + dely * dely + delz * delz;
                const double vo[3] = {vo4.x, vo4.y, vo4.z}, wo[3] = {wo4.x, wo4.y, wo4.z};
                double sh[3];
                sh[0] = sgn * D.hist[(3 * s + 0) * cap + hrow];   // exact: multiplying by +-1 only flips the sign
                sh[1] = sgn * D.hist[(3 * s + 1) * cap + hrow];
                sh[2] = sgn * D.hist[(3 * s + 2) * cap + hrow];
                const int tkk = D.type[kk], to = D.type[other];
                // material lookup in the reference's (owner, neighbour) order
                const MatPair &M = own ? mat(D, tkk, to) : mat(D, to, tkk);
                if (own) {
                    const int fl = D.flag[e];
                    if ((fl | 5) != fl) D.flag[e] = fl | 5;   // CONTACT_NORMAL_MODEL | CONTACT_TANGENTIAL_MODEL
                }
                ContactOut res;
                pair_contact<false>(M, delx, dely, delz, rsq, pkk.w, po.w, vk, vo, wk, wo, vk4.w, vo4.w, sh, upd,
                                    D.dt, ROLLING, D.tdamp != 0, res);
                if (own && upd) {
                    D.hist_out[(3 * s + 0) * cap + kk] = sh[0];
                    D.hist_out[(3 * s + 1) * cap + kk] = sh[1];
                    D.hist_out[(3 * s + 2) * cap + kk] = sh[2];
                }
                for (int c = 0; c < 3; c++) {
                    sres[wid][lane][c] = res.F[c];
                    sres[wid][lane][3 + c] = res.T[c];
                }
            }
            __syncwarp();
            const int lo = max(it.excl, base), hi = min(it.excl + it.cnt, base + 32);
            for (int q = lo; q < hi; q++) {
                acc.F[0] += sres[wid][q - base][0];
                acc.F[1] += sres[wid][q - base][1];
                acc.F[2] += sres[wid][q - base][2];
                acc.T[0] += sres[wid][q - base][3];
                acc.T[1] += sres[wid][q - base][4];
                acc.T[2] += sres[wid][q - base][5];
            }
            __syncwarp();
        }
    }
    if (!valid) return;
    const double vk[3] = {vi4.x, vi4.y, vi4.z}, wk[3] = {wi4.x, wi4.y, wi4.z};
    if (serial) {
        serial_atom<ROLLING>(D, k, pk, vi4, wi4, tk, nr, nn, upd, acc);
    } else if (upd) {
        // slots that stopped touching this step: carry their shear into the write buffer
        unsigned long long stopped = prevm & ~mown;
        while (stopped) {
            const int s = __ffsll((long long)stopped) - 1;
            stopped &= stopped - 1ull;
            D.hist_out[(3 * s + 0) * cap + k] = D.hist[(3 * s + 0) * cap + k];
            D.hist_out[(3 * s + 1) * cap + k] = D.hist[(3 * s + 1) * cap + k];
            D.hist_out[(3 * s + 2) * cap + k] = D.hist[(3 * s + 2) * cap + k];
        }
    }
    if (upd) D.prevmask[k] = serial ? ~0ull : mown;
    const int i = k;
    const dbl4 pi = pk;
    const int ti = tk;
    const double *vi = vk, *wi = wk;
    // post_force fixes in definition order
    for (int k = 0; k < D.nfix; k++) {
        const FixDev &F = D.fix[k];
        if (F.kind == FIX_GRAVITY) {
            const double massone = vi4.w * 1.;
            acc.F[0] += massone * F.acc[0];
            acc.F[1] += massone * F.acc[1];
            acc.F[2] += massone * F.acc[2];
        } else if (F.kind == FIX_WALL_PLANE) {
            if (F.inlist[i]) plane_wall_atom(D, F, i, pi, vi, wi, vi4.w, ti, upd, acc);
        } else if (F.kind == FIX_WALL_MESH) {
            mesh_wall_atom(D, F.mesh, i, pi, vi, wi, vi4.w, ti, upd, acc);
        }
    }
    if (store_f) {
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
    }
    if (integrate) {
        // FixNVESphere::final_integrate (src/fix_nve_sphere.cpp:208-246)
        const double dtf = 0.5 * D.dt * 1.0;
        const double dtfrotate = dtf / 0.4;
        const double dtfm = dtf / (vi4.w * 1.0);
        vi4.x += dtfm * acc.F[0];
        vi4.y += dtfm * acc.F[1];
        vi4.z += dtfm * acc.F[2];
        const double dtirotate = dtfrotate / (pi.w * pi.w * vi4.w);
        wi4.x += dtirotate * acc.T[0];
        wi4.y += dtirotate * acc.T[1];
        wi4.z += dtirotate * acc.T[2];
        if (fuse_next) {
            // next step's FixNVESphere::initial_integrate with the same force,
            // then Neighbor::check_distance's displacement test
            const double dtv = D.dt;
            vi4.x += dtfm * acc.F[0];
            vi4.y += dtfm * acc.F[1];
            vi4.z += dtfm * acc.F[2];
            dbl4 p = pi;
            p.x += dtv * vi4.x;
            p.y += dtv * vi4.y;
            p.z += dtv * vi4.z;
            wi4.x += dtirotate * acc.T[0];
            wi4.y += dtirotate * acc.T[1];
            wi4.z += dtirotate * acc.T[2];
            D.pos_out[i] = p;
            const dbl4 h = hold;
            const double delx = p.x - h.x, dely = p.y - h.y, delz = p.z - h.z;
            if (delx * delx + dely * dely + delz * delz > D.triggersq) *D.dflag = 1;
        }
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
