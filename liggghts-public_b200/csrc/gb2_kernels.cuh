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

#include "../../include/granb200.h"
#include "gb2_device.cuh"
#include "gb2_insert.h"

namespace gb2 {

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
    if (D.kin) D.kin[i] = make_kin(v, w);
    if (check) {
        const dbl4 h = D.xhold[i];
        const double delx = p.x - h.x, dely = p.y - h.y, delz = p.z - h.z;
        const double rsq = delx * delx + dely * dely + delz * delz;
        if (rsq > D.triggersq) *D.dflag = 1;
    }
}

// Atom upload: the caller's [n][3] arrays (x, v, omega) and per-atom radius
// and mass, staged contiguously in `in` (x | v | omega | radius | rmass), packed
// into the 32-byte records; the values are checked as the host used to
// (finite state, positive radius and mass), the first bad atom recorded in
// bad[0] (and its kind in bad[1]: 1 non-finite, 2 radius, 3 mass).
__global__ void k_pack_atoms(const double *__restrict__ in, int n, dbl4 *pos, dbl4 *vel, dbl4 *omg, int *bad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *x = in, *v = in + 3 * (size_t)n, *w = in + 6 * (size_t)n, *r = in + 9 * (size_t)n,
                 *m = in + 10 * (size_t)n;
    const double xi0 = x[3 * i], xi1 = x[3 * i + 1], xi2 = x[3 * i + 2];
    const double vi0 = v[3 * i], vi1 = v[3 * i + 1], vi2 = v[3 * i + 2];
    const double wi0 = w[3 * i], wi1 = w[3 * i + 1], wi2 = w[3 * i + 2];
    const double ri = r[i], mi = m[i];
    int kind = 0;
    if (!(ri > 0.0)) kind = 2;
    else if (!(mi > 0.0)) kind = 3;
    else if (!isfinite(xi0) || !isfinite(xi1) || !isfinite(xi2) || !isfinite(vi0) || !isfinite(vi1) ||
             !isfinite(vi2) || !isfinite(wi0) || !isfinite(wi1) || !isfinite(wi2))
        kind = 1;
    if (kind) {
        atomicMin(&bad[0], i);
        atomicMax(&bad[1], kind);
    }
    pos[i] = dbl4{xi0, xi1, xi2, ri};
    vel[i] = dbl4{vi0, vi1, vi2, mi};
    omg[i] = dbl4{wi0, wi1, wi2, 0.0};
}

// Atom download: x, v, omega, f, torque of atoms [0, n) as five [n][3]
// planes of `out` (one contiguous block for one device-to-host copy)
__global__ void k_unpack_atoms(const dbl4 *__restrict__ pos, const dbl4 *__restrict__ vel,
                               const dbl4 *__restrict__ omg, const dbl4 *__restrict__ f, const dbl4 *__restrict__ tq,
                               int n, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const dbl4 *src[5] = {pos, vel, omg, f, tq};
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const dbl4 a = src[k][i];
        double *o = out + (size_t)k * 3 * n + 3 * (size_t)i;
        o[0] = a.x;
        o[1] = a.y;
        o[2] = a.z;
    }
}

// Comm::forward_comm with AtomVecSphere::pack_comm_vel (src/comm.cpp:773):
// ghost = owned source + accumulated periodic shift
__global__ void k_forward_comm(Dev D)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= D.nghost) return;
    if (D.dstop && *(volatile int *)D.dstop < D.step) return;   // queued step after a rebuild request
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
    if (D.kin) D.kin[gi] = D.kin[src];
}

// split precision: FP32 kinematics records of atoms [0, n) from the FP64 state
__global__ void k_make_kin(Dev D, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    D.kin[i] = make_kin(D.vel[i], D.omg[i]);
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
    if (np > D.maxp) {
        atomicOr(D.status, ST_PARTNER_OVERFLOW);
        atomicMax(&D.need[1], np);
    }
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

// slot-major gather of the slots an atom uses: dst[s*cap+i] = src[s*cap+perm[i]]
// for s / div < cnt_old[perm[i]] (all slots when cnt_old is null)
// (one thread per atom: it reads its source index and count once and copies
// only the occupied slots, so empty histories cost one thread per atom)
template <typename T>
__global__ void k_gather_slots_cnt(const T *__restrict__ src, T *__restrict__ dst, const int *__restrict__ perm, int n,
                                   int cap, int nslot, const int *__restrict__ cnt_old, int div)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int o = perm[i];
    const int m = cnt_old ? min(nslot, cnt_old[o] * div) : nslot;
    for (int s = 0; s < m; s++) dst[(size_t)s * cap + i] = src[(size_t)s * cap + o];
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
    // stencil runs: the bins of a run are consecutive, so their atoms are one
    // range of the bin-sorted array (bins outside the grid are skipped)
    for (int k = 0; k < D.nsrow; k++) {
        const int2 run = D.srow[k];
        const int b0 = max(ibin + run.x, 0), b1 = min(ibin + run.x + run.y, D.mbins);
        if (b0 >= b1) continue;
        const int e0 = D.bin_start[b0], e1 = D.bin_start[b1];
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
    if (n > D.maxn) {
        atomicOr(D.status, ST_NEIGH_OVERFLOW);
        atomicMax(&D.need[0], n);
    }
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
        } else {
            atomicOr(D.status, ST_REV_OVERFLOW);
            atomicMax(&D.need[2], r + 1);
        }
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
    const double dMax = p.w + D.skin;
    if (F.cyl) {   // Cylinder<dim>::resolveNeighlist (src/primitive_wall_definitions.h:199-205), as written
        double dy, dz;
        const double dist = cyl_radial(F, p, dy, dz) - F.cr;
        F.inlist[i] = (dMax < dist || -dMax < dist) ? 1 : 0;
        return;
    }
    const double x = F.dim == 0 ? p.x : (F.dim == 1 ? p.y : p.z);
    const double dist = x - F.pos;
    const double absdist = (dist > 0.0) ? dist : -dist;
    F.inlist[i] = (absdist <= dMax) ? 1 : 0;
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
    if (n > M.maxt) {
        atomicOr(D.status, ST_MESHSLOT_OVERFLOW);
        atomicMax(&D.need[3], n);
    }
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

// ------------------------------------------------------------------
// moving mesh (fix move/mesh rotate)

// MathExtraLiggghts::vec_quat_rotate (src/math_extra_liggghts.h:451-468):
// q * (0, v) * conj(q) with MathExtra::quatquat's operation order
// (src/math_extra.h:596), the zero scalar part included so signed zeros match
__device__ __forceinline__ void vec_quat_rotate(double *vec, const double *q)
{
    const double vq[4] = {0., vec[0], vec[1], vec[2]};
    const double qc[4] = {q[0], -q[1], -q[2], -q[3]};
    double t[4], r[4];
    t[0] = q[0] * vq[0] - q[1] * vq[1] - q[2] * vq[2] - q[3] * vq[3];
    t[1] = q[0] * vq[1] + vq[0] * q[1] + q[2] * vq[3] - q[3] * vq[2];
    t[2] = q[0] * vq[2] + vq[0] * q[2] + q[3] * vq[1] - q[1] * vq[3];
    t[3] = q[0] * vq[3] + vq[0] * q[3] + q[1] * vq[2] - q[2] * vq[1];
    r[0] = t[0] * qc[0] - t[1] * qc[1] - t[2] * qc[2] - t[3] * qc[3];
    r[1] = t[0] * qc[1] + qc[0] * t[1] + t[2] * qc[3] - t[3] * qc[2];
    r[2] = t[0] * qc[2] + qc[0] * t[2] + t[3] * qc[1] - t[1] * qc[3];
    r[3] = t[0] * qc[3] + qc[0] * t[3] + t[1] * qc[2] - t[2] * qc[1];
    vec[0] = r[1];
    vec[1] = r[2];
    vec[2] = r[3];
}

struct MeshRotate {
    double dQ[4];          // rotation of one step
    double origin[3];      // axis point
    int trans;             // origin != 0
    double omegaVec[3];    // axis * omega
    double triggersq;      // (skin/2)^2
};

// One step of MeshMoverRotate::initial_integrate (src/mesh_mover_rotation.cpp:110-138)
// per triangle: nodes and centre (MultiNodeMesh::rotate src/multi_node_mesh_I.h:643-660),
// edge vectors, edge normals and the surface normal (rotated element
// properties, src/surface_mesh_I.h:75-77, src/general_container_I.h:642),
// node velocities omega x (node - origin); and MultiNodeMesh::decideRebuild's
// displacement test against the nodes of the last rebuild (src/multi_node_mesh_I.h:791)
__global__ void k_mesh_rotate(TriGeom *tri, int ntri, double *vnode, const double *node_last, MeshRotate mv, int *flag)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntri) return;
    TriGeom &T = tri[t];
    double ctr[3] = {0., 0., 0.};
    for (int j = 0; j < 3; j++) {
        double nd[3] = {T.node[j][0], T.node[j][1], T.node[j][2]};
        if (mv.trans)
            for (int c = 0; c < 3; c++) nd[c] = nd[c] - mv.origin[c];
        vec_quat_rotate(nd, mv.dQ);
        if (mv.trans)
            for (int c = 0; c < 3; c++) nd[c] = nd[c] + mv.origin[c];
        for (int c = 0; c < 3; c++) {
            T.node[j][c] = nd[c];
            ctr[c] = nd[c] + ctr[c];
        }
    }
    const double sinv = 1. / 3.0;
    for (int c = 0; c < 3; c++) T.center[c] = sinv * ctr[c];
    for (int j = 0; j < 3; j++) {
        vec_quat_rotate(T.edgevec[j], mv.dQ);
        vec_quat_rotate(T.edgenorm[j], mv.dQ);
    }
    vec_quat_rotate(T.surfnorm, mv.dQ);
    bool far = false;
    for (int j = 0; j < 3; j++) {
        const double r0 = T.node[j][0] - mv.origin[0], r1 = T.node[j][1] - mv.origin[1],
                     r2 = T.node[j][2] - mv.origin[2];
        const double w0 = mv.omegaVec[0], w1 = mv.omegaVec[1], w2 = mv.omegaVec[2];
        double *vn = vnode + 9 * t + 3 * j;
        vn[0] = 0. + (w1 * r2 - w2 * r1);
        vn[1] = 0. + (w2 * r0 - w0 * r2);
        vn[2] = 0. + (w0 * r1 - w1 * r0);
        const double *o = node_last + 9 * t + 3 * j;
        const double d0 = T.node[j][0] - o[0], d1 = T.node[j][1] - o[1], d2 = T.node[j][2] - o[2];
        if (d0 * d0 + d1 * d1 + d2 * d2 > mv.triggersq) far = true;
    }
    if (far) *flag = 1;
}

// One step of MeshMoverLinear::initial_integrate (src/mesh_mover_linear.cpp:94-112)
// per triangle: nodes and centre shifted by v dt (MultiNodeMesh::move
// src/multi_node_mesh_I.h:502-513), node velocities 0 + v, and the
// displacement test of MultiNodeMesh::decideRebuild
__global__ void k_mesh_translate(TriGeom *tri, int ntri, double *vnode, const double *node_last, double dx0,
                                 double dx1, double dx2, double v0, double v1, double v2, double triggersq, int *flag)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntri) return;
    TriGeom &T = tri[t];
    const double dx[3] = {dx0, dx1, dx2}, v[3] = {v0, v1, v2};
    bool far = false;
    for (int j = 0; j < 3; j++) {
        double *vn = vnode + 9 * t + 3 * j;
        const double *o = node_last + 9 * t + 3 * j;
        for (int c = 0; c < 3; c++) {
            T.node[j][c] = T.node[j][c] + dx[c];
            vn[c] = 0. + v[c];
        }
        const double d0 = T.node[j][0] - o[0], d1 = T.node[j][1] - o[1], d2 = T.node[j][2] - o[2];
        if (d0 * d0 + d1 * d1 + d2 * d2 > triggersq) far = true;
    }
    for (int c = 0; c < 3; c++) T.center[c] = T.center[c] + dx[c];
    if (far) *flag = 1;
}

// A moving mesh on a rebuild step (FixMesh::pre_force -> pbcExchangeBorders,
// src/fix_mesh.cpp:564-574, src/multi_node_mesh_parallel_I.h:652-700):
// refreshOwned stores the nodes (MultiNodeMesh::storeNodePosRebuild,
// src/multi_node_mesh_I.h:212-225) and recomputes the element's unit edge
// vectors and lengths, surface normal, edge normals and obtuse-angle index
// from its current nodes (SurfaceMesh::recalcLocalSurfProperties,
// src/surface_mesh_I.h:163-200, with calcEdgeVecLen :361, calcSurfaceNorm
// :374, calcEdgeNormals :417, calcObtuseAngleIndex :435), in the order and
// arithmetic the mesh import uses, and with mesh/surface/stress the element
// area (TriMesh::calcArea, src/tri_mesh_I.h:305).  Centre and bounding radius
// stay: the reference updates them only for deforming meshes.
__global__ void k_mesh_refresh(TriGeom *tri, int ntri, double *node_last, double *area)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntri) return;
    TriGeom &T = tri[t];
    for (int j = 0; j < 3; j++)
        for (int c = 0; c < 3; c++) node_last[9 * t + 3 * j + c] = T.node[j][c];
    auto mag = [](const double *v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); };
    auto cross = [](const double *a, const double *b, double *r) {
        r[0] = a[1] * b[2] - a[2] * b[1];
        r[1] = a[2] * b[0] - a[0] * b[2];
        r[2] = a[0] * b[1] - a[1] * b[0];
    };
    auto scale_inv = [](double *v, double s) {
        const double sinv = 1. / s;
        v[0] = sinv * v[0];
        v[1] = sinv * v[1];
        v[2] = sinv * v[2];
    };
    for (int k = 0; k < 3; k++) {
        for (int c = 0; c < 3; c++) T.edgevec[k][c] = T.node[(k + 1) % 3][c] - T.node[k][c];
        T.edgelen[k] = mag(T.edgevec[k]);
        scale_inv(T.edgevec[k], T.edgelen[k]);
    }
    cross(T.edgevec[0], T.edgevec[1], T.surfnorm);
    if (mag(T.surfnorm) < 1e-15) cross(T.edgevec[1], T.edgevec[2], T.surfnorm);
    if (mag(T.surfnorm) < 1e-15) cross(T.edgevec[2], T.edgevec[0], T.surfnorm);
    scale_inv(T.surfnorm, mag(T.surfnorm));
    for (int k = 0; k < 3; k++) {
        cross(T.edgevec[k], T.surfnorm, T.edgenorm[k]);
        if (mag(T.edgenorm[k]) < 1e-15)
            for (int c = 0; c < 3; c++) T.edgenorm[k][c] = T.edgevec[(k + 1) % 3][c];
        else
            scale_inv(T.edgenorm[k], mag(T.edgenorm[k]));
    }
    int ob = -1;
    for (int k = 0; k < 3; k++) ob = dot3(T.edgevec[k], T.edgevec[(k + 2) % 3]) > 0. ? k : -1;
    T.obtuse = ob;
    if (area) {
        double cr[3];
        cross(T.edgevec[0], T.edgevec[1], cr);
        area[t] = 0.5 * mag(cr) * T.edgelen[0] * T.edgelen[1];
    }
}

// FixNeighlistMesh with a moving mesh (src/fix_neighlist_mesh.cpp:383-395,
// :411-424): every bin of the triangle's bounding box (shrunk to the box)
// extended by distmax.  Pass 1: per-axis bin ranges and their pair count.
// A range that leaves the bin grid is rejected (the reference would alias it
// to a neighbouring row of bins).
__global__ void k_tri_bin_range(Dev D, const TriGeom *tri, int ntri, double distmax, double lo0, double lo1,
                                double lo2, double hi0, double hi1, double hi2, int *range, int *count)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntri) return;
    const TriGeom &T = tri[t];
    double blo[3] = {1e300, 1e300, 1e300}, bhi[3] = {-1e300, -1e300, -1e300};
    for (int k = 0; k < 3; k++)
        for (int d = 0; d < 3; d++) {
            blo[d] = fmin(blo[d], T.node[k][d]);
            bhi[d] = fmax(bhi[d], T.node[k][d]);
        }
    const double boxlo[3] = {lo0, lo1, lo2}, boxhi[3] = {hi0, hi1, hi2};
    for (int d = 0; d < 3; d++) {   // BoundingBox::shrinkToSubbox
        if (blo[d] < boxlo[d]) blo[d] = boxlo[d];
        if (bhi[d] > boxhi[d]) bhi[d] = boxhi[d];
    }
    int l[3], h[3];
    coord2bin3(D, blo[0] - distmax, blo[1] - distmax, blo[2] - distmax, l[0], l[1], l[2]);
    coord2bin3(D, bhi[0] + distmax, bhi[1] + distmax, bhi[2] + distmax, h[0], h[1], h[2]);
    long n = 1;
    for (int d = 0; d < 3; d++) {
        if (l[d] < 0 || h[d] >= D.mbin[d] || h[d] < l[d]) {
            atomicOr(D.status, ST_MESH_OUTSIDE_GRID);
            n = 0;
        }
        range[6 * t + d] = l[d];
        range[6 * t + 3 + d] = h[d];
    }
    if (n) n = (long)(h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1);
    count[t] = (int)n;
}

// The bin lists' (triangle, bin) pairs: one block per triangle, its threads
// striding over the triangle's bin box (the q-th bin takes slot off[t] + q
// of the triangle's range in the exclusive scan of the per-triangle bin
// counts).  A large triangle spans hundreds of bins, so a block per triangle
// keeps the whole GPU busy where one thread per triangle left most SMs idle.
// Which slot of its triangle's range a bin takes does not matter: the stable
// sort by bin that follows orders each bin's triangles by slot, and so by
// triangle.
__device__ __forceinline__ int pair_bin(const Dev &D, const int *r, int q, int &ix, int &iy, int &iz)
{
    const int nz = r[5] - r[2] + 1, ny = r[4] - r[1] + 1;
    iz = r[2] + q % nz;
    iy = r[1] + (q / nz) % ny;
    ix = r[0] + q / (nz * ny);
    return iz * D.mbin[1] * D.mbin[0] + iy * D.mbin[0] + ix;
}

// Static mesh (FixNeighlistMesh::generate_bin_list, src/fix_neighlist_mesh.cpp:456-490):
// the same pairs, but a bin is kept only when a sphere of the bin's half
// diagonal at the bin centre passes the neighbour-build test against the
// triangle with threshold distmax + skin; dropped pairs get key 0xffffffff
// and sort to the end.
__global__ void k_tri_bin_fill_cull(Dev D, const TriGeom *tri, const int *range, const int *off, unsigned *keys,
                                    int *vals, int *bincnt, double maxdiag, double thresh)
{
    const int t = blockIdx.x;
    const int p0 = off[t], cnt = off[t + 1] - p0;
    const int *r = range + 6 * t;
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
        int ix, iy, iz;
        const int b = pair_bin(D, r, q, ix, iy, iz);
        double center[3];
        center[0] = (D.mbinlo[0] + ix + 0.5) * D.binsize[0] + D.bboxlo[0];
        center[1] = (D.mbinlo[1] + iy + 0.5) * D.binsize[1] + D.bboxlo[1];
        center[2] = (D.mbinlo[2] + iz + 0.5) * D.binsize[2] + D.bboxlo[2];
        const bool keep = tri_neighbuild(tri[t], maxdiag, center, thresh);
        keys[p0 + q] = keep ? (unsigned)b : 0xffffffffu;
        vals[p0 + q] = t;
        if (keep) atomicAdd(&bincnt[b], 1);
    }
}

// Moving mesh, at every rebuild: (bin, triangle) pairs and per-bin counts
__global__ void k_tri_bin_fill(Dev D, const int *range, const int *off, unsigned *keys, int *vals, int *bincnt)
{
    const int t = blockIdx.x;
    const int p0 = off[t], cnt = off[t + 1] - p0;
    const int *r = range + 6 * t;
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
        int ix, iy, iz;
        const int b = pair_bin(D, r, q, ix, iy, iz);
        keys[p0 + q] = (unsigned)b;
        vals[p0 + q] = t;
        atomicAdd(&bincnt[b], 1);
    }
}

// contact census (diagnostics and the bench's byte model)
__global__ void __launch_bounds__(128) k_census(Dev D, unsigned long long *cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long c[7] = {0, 0, 0, 0, 0, 0, 0};
    if (i < D.nlocal) {
        const int cap = D.cap;
        const dbl4 pi = D.pos[i];
        const int nn = D.nnum[i];
        c[0] = nn;
        for (int s = 0; s < nn; s++) {
            const dbl4 pj = D.pos[D.nbr[s * cap + i]];
            const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const double rs = pi.w + pj.w;
            if (dx * dx + dy * dy + dz * dz < rs * rs) c[1]++;
        }
        c[2] = D.rnum[i];
        for (int k = 0; k < D.nfix; k++) {
            const FixDev &F = D.fix[k];
            if (F.kind == FIX_WALL_PLANE && F.inlist[i]) {
                c[3]++;
                const double x = F.dim == 0 ? pi.x : (F.dim == 1 ? pi.y : pi.z);
                const double dist = x > F.pos ? x - F.pos - pi.w : F.pos - x - pi.w;
                if (dist <= 0) c[4]++;
            } else if (F.kind == FIX_WALL_MESH) {
                const int tc = F.mesh.tcnt[i];
                c[5] += tc;
                for (int q = 0; q < tc; q++)
                    if (F.mesh.spartner[q * cap + i] >= 0) c[6]++;
            }
        }
    }
    // warp sums, then one atomic per warp and counter (no contention on 7 words)
#pragma unroll
    for (int k = 0; k < 7; k++) {
        unsigned long long v = c[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&cnt[k], v);
    }
}

// The tail kernel's atom list, after each neighbour build (count zeroed
// before the launch; the order of the list does not affect any result).
__global__ void k_tail_list(Dev D)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.nlocal) return;
    if (tail_atom(D, k, D.rnum[k], D.nnum[k])) D.tail[atomicAdd(D.tailcnt, 1)] = k;
}

// Start of a queue of steps: the step just run (not queued) may already
// have asked for a rebuild of the next one through the displacement flag.
__global__ void k_queue_start(int *dstop, const int *dflag, int step) { *dstop = *dflag ? step : 0x7f7f7f7f; }

// ComputeContactAtom::compute_peratom with skin 0 (src/compute_contact_atom.cpp):
// contact if rsq <= (radi + radj)^2; an owned atom counts its own half-list
// entries and the entries where it is the j side (newton off: an image pair
// across a periodic boundary is in both owners' lists).
__global__ void k_contact_atom(Dev D, double *out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.nlocal) return;
    const int cap = D.cap;
    const dbl4 pk = D.pos[k];
    int cnt = 0;
    for (int s = 0; s < D.nnum[k]; s++) {
        const dbl4 pj = D.pos[D.nbr[s * cap + k]];
        const double delx = pk.x - pj.x, dely = pk.y - pj.y, delz = pk.z - pj.z;
        const double rsq = delx * delx + dely * dely + delz * delz;
        const double radsum = pk.w + pj.w + 0.0;
        if (rsq <= radsum * radsum) cnt++;
    }
    for (int r = 0; r < D.rnum[k]; r++) {
        const dbl4 pi = D.pos[D.rev[r * cap + k]];
        const double delx = pi.x - pk.x, dely = pi.y - pk.y, delz = pi.z - pk.z;
        const double rsq = delx * delx + dely * dely + delz * delz;
        const double radsum = pi.w + pk.w + 0.0;
        if (rsq <= radsum * radsum) cnt++;
    }
    out[k] = (double)cnt;
}

// fix insert/pack selections (FixInsertPack::calc_ninsert_this counts owned
// particles inside the region; FixInsert::load_xnear loads owned and ghost
// particles near it).  Ghost positions are those of the previous step's
// forward communication (gpos); owned ones the current ones.
__global__ void k_ins_flags(const dbl4 *pos, const dbl4 *gpos, int nlocal, int nall, InsertRegion R, uint8_t *freg,
                            uint8_t *fnear)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nall) return;
    const dbl4 p = i < nlocal ? pos[i] : gpos[i];
    const double x[3] = {p.x, p.y, p.z};
    freg[i] = (i < nlocal && R.inside(x)) ? 1 : 0;
    fnear[i] = R.near(x, p.w) ? 1 : 0;
}

// fix insert/stream's near list (FixInsertStream::is_nearby with the list's
// bounding box, src/fix_insert_stream.cpp:573-615): inside the box, within
// maxrad in front of the face plane and extrude_length + 3 maxrad behind it,
// and the point x + n d (d = the signed distance to the plane, as the
// reference forms it) inside one of the face's triangles
struct StreamNear {
    double p_ref[3], n[3], bblo[3], bbhi[3];
    double maxrad, extrude_length;
    int nface;
};

__global__ void k_ins_near_stream(const dbl4 *pos, const dbl4 *gpos, int nlocal, int nall, StreamNear S,
                                  const TriGeom *face, uint8_t *fnear)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nall) return;
    const dbl4 p = i < nlocal ? pos[i] : gpos[i];
    const double x[3] = {p.x, p.y, p.z};
    uint8_t near = 0;
    if (x[0] >= S.bblo[0] && x[0] <= S.bbhi[0] && x[1] >= S.bblo[1] && x[1] <= S.bbhi[1] && x[2] >= S.bblo[2] &&
        x[2] <= S.bbhi[2]) {
        const double rel[3] = {x[0] - S.p_ref[0], x[1] - S.p_ref[1], x[2] - S.p_ref[2]};
        const double d = rel[0] * S.n[0] + rel[1] * S.n[1] + rel[2] * S.n[2];
        if (!(d > S.maxrad) && !(d < -(S.extrude_length + 3. * S.maxrad))) {
            double pp[3];
            for (int c = 0; c < 3; c++) pp[c] = x[c] + S.n[c] * d;
            for (int t = 0; t < S.nface && !near; t++) {   // TriMesh::isInElement
                const TriGeom &T = face[t];
                double v0[3], v1[3], v2[3];
                for (int c = 0; c < 3; c++) {
                    v0[c] = T.node[2][c] - T.node[0][c];
                    v1[c] = T.node[1][c] - T.node[0][c];
                    v2[c] = pp[c] - T.node[0][c];
                }
                const double dot00 = v0[0] * v0[0] + v0[1] * v0[1] + v0[2] * v0[2];
                const double dot01 = v0[0] * v1[0] + v0[1] * v1[1] + v0[2] * v1[2];
                const double dot02 = v0[0] * v2[0] + v0[1] * v2[1] + v0[2] * v2[2];
                const double dot11 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
                const double dot12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
                const double invDenom = 1. / (dot00 * dot11 - dot01 * dot01);
                const double u = (dot11 * dot02 - dot01 * dot12) * invDenom;
                const double v = (dot00 * dot12 - dot01 * dot02) * invDenom;
                if ((u > -1e-10) && (v > -1e-10) && (u + v < 1. + 1e-10)) near = 1;
            }
        }
    }
    fnear[i] = near;
}

// records of the selected particles: region ones (radius, mass) first, then
// near ones (x, y, z, radius)
__global__ void k_ins_gather(const dbl4 *pos, const dbl4 *vel, const dbl4 *gpos, int nlocal, const int *ireg, int nreg,
                             const int *inear, int nnear, dbl4 *out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nreg) {
        const int i = ireg[k];
        out[k] = dbl4{pos[i].w, vel[i].w, 0.0, 0.0};
    } else if (k < nreg + nnear) {
        const int i = inear[k - nreg];
        out[k] = i < nlocal ? pos[i] : gpos[i];
    }
}

// compute pair/gran/local id force torque history (src/compute_pair_gran_local.cpp
// add_pair via PairGran::compute_pgl, src/pair_gran.cpp:676-707): every touching
// own-list pair (a pair with a ghost only when tag_i > tag_j), its force and
// torque on i evaluated with shearupdate 0 from the current state.  Count pass
// and row pass (rows in list order: per-atom offsets from a scan of the counts).
struct PglBox {
    double lo[3], hi[3];
    int periodic[3];
};

__device__ __forceinline__ bool pgl_pair(const Dev &D, int i, int s, const dbl4 &pi, int &j, double &delx,
                                         double &dely, double &delz, double &rsq)
{
    j = D.nbr[s * D.cap + i];
    const dbl4 pj = D.pos[j];
    delx = pi.x - pj.x;
    dely = pi.y - pj.y;
    delz = pi.z - pj.z;
    rsq = delx * delx + dely * dely + delz * delz;
    const double radsum = pi.w + pj.w;
    if (!(rsq < radsum * radsum)) return false;
    return !(j >= D.nlocal && D.tag[i] <= D.tag[j]);
}

__global__ void k_pgl_count(Dev D, int *cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const dbl4 pi = D.pos[i];
    int n = 0;
    for (int s = 0; s < D.nnum[i]; s++) {
        int j;
        double dx, dy, dz, rsq;
        if (pgl_pair(D, i, s, pi, j, dx, dy, dz, rsq)) n++;
    }
    cnt[i] = n;
}

// Domain::remap (src/domain.cpp:1136-1173) for an orthogonal box: the
// periodic image inside [lo, hi).  Ghost images lie within the ghost cutoff of
// the box, so a few shifts always suffice for finite coordinates.
__device__ __forceinline__ double pgl_remap(double x, double lo, double hi, int periodic)
{
    if (!periodic) return x;
    const double prd = hi - lo;
    for (int it = 0; it < 64 && x < lo; it++) x += prd;
    for (int it = 0; it < 64 && x >= hi; it++) x -= prd;
    return x > lo ? x : lo;
}

// the component of c along the unit vector from x_i to x_j
// (vectorSubtract3D / vectorNormalize3D, src/vector_liggghts.h:62-69)
__device__ __forceinline__ void pgl_along(const dbl4 &pi, const dbl4 &pj, const double c[3], double out[3])
{
    double n[3] = {pj.x - pi.x, pj.y - pi.y, pj.z - pi.z};
    const double norm = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    const double inv = (norm == 0.) ? 0. : 1. / norm;
    n[0] *= inv;
    n[1] *= inv;
    n[2] *= inv;
    const double mag = c[0] * n[0] + c[1] * n[1] + c[2] * n[2];
    out[0] = n[0] * mag;
    out[1] = n[1] * mag;
    out[2] = n[2] * mag;
}

// one row per touching pair with the columns the keyword mask selects, in
// the order ComputePairGranLocal::add_pair writes them
// (src/compute_pair_gran_local.cpp:445-606)
__global__ void k_pgl_rows(Dev D, const int *off, double *rows, PglBox B, unsigned keys, int ncols)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    const int cap = D.cap;
    const dbl4 pi = D.pos[i], vi4 = D.vel[i], wi4 = D.omg[i];
    const double vi[3] = {vi4.x, vi4.y, vi4.z}, wi[3] = {wi4.x, wi4.y, wi4.z};
    const int ti = D.type[i];
    int k = off[i];
    for (int s = 0; s < D.nnum[i]; s++) {
        int j;
        double delx, dely, delz, rsq;
        if (!pgl_pair(D, i, s, pi, j, delx, dely, delz, rsq)) continue;
        const dbl4 pj = D.pos[j], vj4 = D.vel[j], wj4 = D.omg[j];
        const double vj[3] = {vj4.x, vj4.y, vj4.z}, wj[3] = {wj4.x, wj4.y, wj4.z};
        double sh[3] = {D.hist[(3 * s + 0) * cap + i], D.hist[(3 * s + 1) * cap + i], D.hist[(3 * s + 2) * cap + i]};
        const double h0[3] = {sh[0], sh[1], sh[2]};
        ContactOut o;
        pair_contact<false>(mat(D, ti, D.type[j]), delx, dely, delz, rsq, pi.w, pj.w, vi, vj, wi, wj, vi4.w, vj4.w,
                            sh, false, D.dt, D.rolling != 0, D.tdamp != 0, o);
        double *row = rows + (size_t)ncols * k;
        int n = 0;
        if (keys & GB2_PGL_POS) {
            const double xi[3] = {pi.x, pi.y, pi.z}, xj[3] = {pj.x, pj.y, pj.z};
            for (int d = 0; d < 3; d++) row[n++] = pgl_remap(xi[d], B.lo[d], B.hi[d], B.periodic[d]);
            for (int d = 0; d < 3; d++) row[n++] = pgl_remap(xj[d], B.lo[d], B.hi[d], B.periodic[d]);
        }
        if (keys & GB2_PGL_VEL) {
            for (int d = 0; d < 3; d++) row[n++] = vi[d];
            for (int d = 0; d < 3; d++) row[n++] = vj[d];
        }
        if (keys & GB2_PGL_ID) {
            row[n++] = (double)D.tag[i];
            row[n++] = (double)D.tag[j];
            row[n++] = j < D.nlocal ? 0. : 1.;
        }
        if (keys & GB2_PGL_FORCE)
            for (int d = 0; d < 3; d++) row[n++] = o.F[d];
        if (keys & (GB2_PGL_FORCE_NORMAL | GB2_PGL_FORCE_TANGENTIAL)) {
            double fn[3];
            pgl_along(pi, pj, o.F, fn);
            if (keys & GB2_PGL_FORCE_NORMAL)
                for (int d = 0; d < 3; d++) row[n++] = fn[d];
            if (keys & GB2_PGL_FORCE_TANGENTIAL)
                for (int d = 0; d < 3; d++) row[n++] = o.F[d] - fn[d];
        }
        if (keys & GB2_PGL_TORQUE)
            for (int d = 0; d < 3; d++) row[n++] = o.T[d];
        if (keys & (GB2_PGL_TORQUE_NORMAL | GB2_PGL_TORQUE_TANGENTIAL)) {
            double tn[3];
            pgl_along(pi, pj, o.T, tn);
            if (keys & GB2_PGL_TORQUE_NORMAL)
                for (int d = 0; d < 3; d++) row[n++] = tn[d];
            if (keys & GB2_PGL_TORQUE_TANGENTIAL)
                for (int d = 0; d < 3; d++) row[n++] = o.T[d] - tn[d];
        }
        if (keys & GB2_PGL_HISTORY)
            for (int d = 0; d < 3; d++) row[n++] = h0[d];
        if (keys & (GB2_PGL_CONTACT_AREA | GB2_PGL_DELTA)) {
            // del = x_i - x_j as recomputed by add_pair (the same rsq as the pair test)
            const double r = sqrt(rsq);
            const double radi = pi.w, radj = pj.w;
            if (keys & GB2_PGL_CONTACT_AREA)
                row[n++] = -M_PI / 4 * ((r - radi - radj) * (r + radi - radj) * (r - radi + radj) * (r + radi + radj)) /
                           rsq;
            if (keys & GB2_PGL_DELTA) row[n++] = radi + radj - r;
        }
        if (keys & GB2_PGL_CONTACT_POINT) {
            const double xi[3] = {pi.x, pi.y, pi.z}, xj[3] = {pj.x, pj.y, pj.z};
            for (int d = 0; d < 3; d++) row[n++] = (xi[d] * pj.w + xj[d] * pi.w) / (pi.w + pj.w);
        }
        k++;
    }
}

}  // namespace gb2

