// gb2_step.cuh -- the fused pair-step kernel (one full time step per owned
// atom).  Instantiated with SPLIT=false by the bit-exact FP64 unit and with
// SPLIT=true by the split-precision unit (gb2_split.cu).
#pragma once

#include <type_traits>

#include "gb2_device.cuh"

namespace gb2 {
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

// Programmatic dependent launch: the pair step lets the tail kernel be
// scheduled as soon as all of its blocks are running; the tail kernel does
// what does not need the pair sums first and then waits for the pair step
// to complete (all its memory operations visible).
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// A kernel of a step queued ahead returns at once when an earlier step has
// asked for a neighbour rebuild (that step's successors are redone after it).
__device__ __forceinline__ bool step_cancelled(const Dev &D) { return D.dstop && *(volatile int *)D.dstop < D.step; }

// One touching pair of the warp-compacted evaluation: owner kk, the other
// atom, the half-list slot s of the pair (in kk's list when own, in other's
// list otherwise).  A j-side entry is evaluated from kk's side with the
// shear negated; an own entry updates kk's shear slot in the write buffer
// and sets the contact flag.  res receives the pair's force and torque on kk.
template <bool ROLLING, bool SPLIT, typename Real>
__device__ __forceinline__ void eval_item(const Dev &D, int kk, int other, int s, bool own, bool upd, Real *res)
{
    const int cap = D.cap;
    const int e = s * cap + kk;
    const double sgn = own ? 1.0 : -1.0;
    const int hrow = own ? kk : other;
    const dbl4 pkk = ldg4(&D.pos[kk]);
    const dbl4 po = ldg4(&D.pos[other]);
    const double delx = pkk.x - po.x;
    const double dely = pkk.y - po.y;
    const double delz = pkk.z - po.z;
    const double rsq = delx * delx + dely * dely + delz * delz;
    const int tkk = D.type[kk], to = D.type[other];
    // material lookup in the reference's (owner, neighbour) order
    const MatPair &M = own ? mat(D, tkk, to) : mat(D, to, tkk);
    if (own) {
        const int fl = D.flag[e];
        if ((fl | 5) != fl) D.flag[e] = fl | 5;   // CONTACT_NORMAL_MODEL | CONTACT_TANGENTIAL_MODEL
    }
    if constexpr (SPLIT) {
        const flt8 a = ldg8f(&D.kin[kk]), b = ldg8f(&D.kin[other]);
        const double r = sqrt(rsq);
        const double deltan = (pkk.w + po.w) - r;   // FP64 overlap
        const float va[3] = {a.vx, a.vy, a.vz}, wa[3] = {a.wx, a.wy, a.wz};
        const float vb[3] = {b.vx, b.vy, b.vz}, wb[3] = {b.wx, b.wy, b.wz};
        const float fs = (float)sgn;
        float sh[3];
        sh[0] = fs * (float)D.hist[(3 * s + 0) * cap + hrow];
        sh[1] = fs * (float)D.hist[(3 * s + 1) * cap + hrow];
        sh[2] = fs * (float)D.hist[(3 * s + 2) * cap + hrow];
        ContactOutF o;
        pair_contact_f32(M, (float)delx, (float)dely, (float)delz, (float)r, (float)deltan, (float)pkk.w,
                         (float)po.w, va, vb, wa, wb, a.m, b.m, sh, upd, (float)D.dt, ROLLING, D.tdamp != 0, o);
        if (own && upd) {
            D.hist_out[(3 * s + 0) * cap + kk] = sh[0];
            D.hist_out[(3 * s + 1) * cap + kk] = sh[1];
            D.hist_out[(3 * s + 2) * cap + kk] = sh[2];
        }
        for (int c = 0; c < 3; c++) {
            res[c] = o.F[c];
            res[3 + c] = o.T[c];
        }
    } else {
        const dbl4 vk4 = ldg4(&D.vel[kk]), wk4 = ldg4(&D.omg[kk]);
        const dbl4 vo4 = ldg4(&D.vel[other]), wo4 = ldg4(&D.omg[other]);
        const double vk[3] = {vk4.x, vk4.y, vk4.z}, wk[3] = {wk4.x, wk4.y, wk4.z};
        const double vo[3] = {vo4.x, vo4.y, vo4.z}, wo[3] = {wo4.x, wo4.y, wo4.z};
        double sh[3];
        sh[0] = sgn * D.hist[(3 * s + 0) * cap + hrow];   // exact: multiplying by +-1 only flips the sign
        sh[1] = sgn * D.hist[(3 * s + 1) * cap + hrow];
        sh[2] = sgn * D.hist[(3 * s + 2) * cap + hrow];
        ContactOut o;
        pair_contact<false>(M, delx, dely, delz, rsq, pkk.w, po.w, vk, vo, wk, wo, vk4.w, vo4.w, sh, upd, D.dt,
                            ROLLING, D.tdamp != 0, o);
        if (own && upd) {
            D.hist_out[(3 * s + 0) * cap + kk] = sh[0];
            D.hist_out[(3 * s + 1) * cap + kk] = sh[1];
            D.hist_out[(3 * s + 2) * cap + kk] = sh[2];
        }
        for (int c = 0; c < 3; c++) {
            res[c] = o.F[c];
            res[3 + c] = o.T[c];
        }
    }
}

// FP64: plain in-order sum.  Split: FP32 sum with Kahan compensation kc.
template <bool SPLIT, typename Real>
__device__ __forceinline__ void sum_item(Real *as, Real *kc, const Real *v)
{
#pragma unroll
    for (int c = 0; c < 6; c++) {
        if constexpr (SPLIT) {
            const float y = v[c] - kc[c];
            const float t = as[c] + y;
            kc[c] = (t - as[c]) - y;
            as[c] = t;
        } else {
            as[c] += v[c];
        }
    }
}

template <bool SPLIT, typename Real>
__device__ __forceinline__ void pair_total(const Real *as, const Real *kc, ContactOut &acc)
{
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if constexpr (SPLIT) {
            acc.F[c] = (double)as[c] - (double)kc[c];
            acc.T[c] = (double)as[3 + c] - (double)kc[3 + c];
        } else {
            acc.F[c] = as[c];
            acc.T[c] = as[3 + c];
        }
    }
}

// store_f / FixNVESphere::final_integrate / the next step's initial_integrate
// with the displacement test, for one atom whose total force is in acc
// FixInsertStream::end_of_step (src/fix_insert_stream.cpp:868-935) for atom
// i: a particle the stream inserted and has not released moves with its
// integration velocity from its insertion position (x = x_ins + v_int
// (step - i_step) dt, v = v_int, omega = 0); at its release step it gets the
// release velocity and omega.  Returns true when it applies; the atom's
// force and torque then read zero.
__device__ __forceinline__ bool stream_hold(const Dev &D, int i, dbl4 &x, dbl4 &v, dbl4 &w)
{
    const dbl4 r0 = D.rel[i];
    if (r0.w < 1e-13 && r0.w > -1e-13) return false;   // never inserted by the stream
    const dbl4 r1 = D.rel[D.cap + i];
    const int i_step = static_cast<int>(r0.w + 1e-14);
    const int r_step = static_cast<int>(r1.w + 1e-14);
    if (D.step > r_step) return false;
    const double time_elapsed = (D.step - i_step) * D.dt;
    x.x = r0.x + r1.x * time_elapsed;
    x.y = r0.y + r1.y * time_elapsed;
    x.z = r0.z + r1.z * time_elapsed;
    if (D.step == r_step) {
        const dbl4 r2 = D.rel[2 * D.cap + i], r3 = D.rel[3 * D.cap + i];
        v.x = r2.x, v.y = r2.y, v.z = r2.z;
        w.x = r3.x, w.y = r3.y, w.z = r3.z;
    } else {
        v.x = r1.x, v.y = r1.y, v.z = r1.z;
        w.x = 0.0, w.y = 0.0, w.z = 0.0;
    }
    return true;
}

template <bool SPLIT>
__device__ __forceinline__ void atom_store_integrate(const Dev &D, int i, const dbl4 &pi, dbl4 vi4, dbl4 wi4,
                                                     const dbl4 &hold, int integrate, int fuse_next, int store_f,
                                                     const ContactOut &acc_in)
{
    // an atom held by fix insert/stream ends the step where end_of_step puts
    // it, with zero force and torque (the next initial_integrate reads them)
    ContactOut acc = acc_in;
    dbl4 pcur = pi;
    if (D.rel && integrate && stream_hold(D, i, pcur, vi4, wi4)) {
        for (int c = 0; c < 3; c++) acc.F[c] = acc.T[c] = 0.0;
        integrate = 2;   // final_integrate's result is replaced
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
        const double dtirotate = dtfrotate / (pi.w * pi.w * vi4.w);
        if (integrate == 1) {
            vi4.x += dtfm * acc.F[0];
            vi4.y += dtfm * acc.F[1];
            vi4.z += dtfm * acc.F[2];
            wi4.x += dtirotate * acc.T[0];
            wi4.y += dtirotate * acc.T[1];
            wi4.z += dtirotate * acc.T[2];
        }
        if (fuse_next) {
            // next step's FixNVESphere::initial_integrate with the same force,
            // then Neighbor::check_distance's displacement test
            const double dtv = D.dt;
            vi4.x += dtfm * acc.F[0];
            vi4.y += dtfm * acc.F[1];
            vi4.z += dtfm * acc.F[2];
            dbl4 p = pcur;
            p.x += dtv * vi4.x;
            p.y += dtv * vi4.y;
            p.z += dtv * vi4.z;
            wi4.x += dtirotate * acc.T[0];
            wi4.y += dtirotate * acc.T[1];
            wi4.z += dtirotate * acc.T[2];
            D.pos_out[i] = p;
            const dbl4 h = hold;
            const double delx = p.x - h.x, dely = p.y - h.y, delz = p.z - h.z;
            if (delx * delx + dely * dely + delz * delz > D.triggersq) {
                *D.dflag = 1;
                if (D.dstop) atomicMin(D.dstop, D.step);
            }
        }
        D.vel_out[i] = vi4;
        D.omg_out[i] = wi4;
        if constexpr (SPLIT) D.kin_out[i] = make_kin(vi4, wi4);
    }
}

// The last step of a run (no fused initial_integrate): positions of the atoms
// fix insert/stream holds, set in place once the step's kernels are done.
static __global__ void k_stream_positions(Dev D)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nlocal) return;
    dbl4 x = D.pos[i], v, w;
    if (stream_hold(D, i, x, v, w)) D.pos[i] = x;
}

// Shear of own slots that stopped touching this step is carried into the
// write buffer, and the touching mask is kept for the next step.
__device__ __forceinline__ void atom_hist_tail(const Dev &D, int k, unsigned long long prevm,
                                               unsigned long long mown, bool upd)
{
    if (!upd) return;
    const int cap = D.cap;
    unsigned long long stopped = prevm & ~mown;
    while (stopped) {
        const int s = __ffsll((long long)stopped) - 1;
        stopped &= stopped - 1ull;
        D.hist_out[(3 * s + 0) * cap + k] = D.hist[(3 * s + 0) * cap + k];
        D.hist_out[(3 * s + 1) * cap + k] = D.hist[(3 * s + 1) * cap + k];
        D.hist_out[(3 * s + 2) * cap + k] = D.hist[(3 * s + 2) * cap + k];
    }
    D.prevmask[k] = mown;
}

// The per-atom end of the step once the pair sums are in acc, for an atom
// without wall or serial work (tail_atom is false): of the post_force
// fixes only gravity acts, then FixNVESphere::final_integrate and -- when
// the run continues -- the next step's initial_integrate with the
// displacement test.
template <bool SPLIT>
__device__ __forceinline__ void atom_fix_tail(const Dev &D, int k, const dbl4 &pk, dbl4 vi4, dbl4 wi4,
                                              const dbl4 &hold, int integrate, int fuse_next, int store_f,
                                              ContactOut &acc)
{
    for (int q = 0; q < D.nfix; q++) {
        const FixDev &F = D.fix[q];
        if (F.kind == FIX_GRAVITY) {
            const double massone = vi4.w * 1.;
            acc.F[0] += massone * F.acc[0];
            acc.F[1] += massone * F.acc[1];
            acc.F[2] += massone * F.acc[2];
        }
    }
    atom_store_integrate<SPLIT>(D, k, pk, vi4, wi4, hold, integrate, fuse_next, store_f, acc);
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
template <bool ROLLING, int MINB, bool SPLIT>
__global__ void __launch_bounds__(128, MINB) k_pair_step(Dev D, int shearupdate, int integrate, int fuse_next,
                                                         int store_f)
{
    using Real = typename std::conditional<SPLIT, float, double>::type;
    __shared__ Real sres[4][32][6];
    // the atom's records that only the tail needs (velocity, angular
    // velocity, position at the last rebuild) wait here, not in registers,
    // while the screening and the contact rounds run
    __shared__ __align__(16) dbl4 stail[3][128];
    // per warp: the touching entries listed by the screening (rev, own; the
    // launch gives 4 x 2 x D.item_cap of them in dynamic shared memory) and
    // each round's owner-lane masks, tagged with the round
    extern __shared__ __align__(16) unsigned char pair_dyn[];
    __shared__ unsigned long long sgrp[4][32];
    grid_dep_launch();   // the tail kernel may be scheduled once every block of this grid runs
    if (step_cancelled(D)) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int wbase = blockIdx.x * blockDim.x + wid * 32;
    const bool valid = k < D.nlocal;
    const int cap = D.cap;
    const bool upd = shearupdate != 0;
    dbl4 pk;
    unsigned long long prevm = 0ull;
    int nr = 0, nn = 0, tk = 0;
    unsigned long long mrev = 0ull, mown = 0ull;
    bool serial = false, tail = false;
    if (valid) {
        // the atom's own records, including those only the tail needs, are
        // requested first so their latency overlaps the screening
        stage4(&stail[0][threadIdx.x], &D.vel[k]);
        stage4(&stail[1][threadIdx.x], &D.omg[k]);
        if (fuse_next) stage4(&stail[2][threadIdx.x], &D.xhold[k]);
        pk = D.pos[k];
        nr = D.rnum[k];
        nn = D.nnum[k];
        tk = D.type[k];
        serial = nr > 64 || nn > 64;
        tail = tail_atom(D, k, nr, nn);
        if (!serial && upd) prevm = D.prevmask[k];
    }
    // screening of every non-serial atom of the warp, listing its touching
    // entries (all lanes take part in the list ballots)
    int nlrev = 0, nlown = 0;
    int2 *lrev = reinterpret_cast<int2 *>(pair_dyn) + (size_t)wid * 2 * D.item_cap, *lown = lrev + D.item_cap;
    const bool listed = screen_list(D, k, (valid && !serial) ? nr : 0, (valid && !serial) ? nn : 0, pk, mrev, mown,
                                    lrev, lown, nlrev, nlown);
    if (!listed && lane == 0 && D.item_cap > 0) atomicAdd(&D.need[4], 1);   // lists too short: counted for the host
    // FP64 path: plain in-order sums (bit-exact).  Split path: FP32 sums of
    // the FP32 pair contributions with Kahan compensation kc.
    Real as[6], kc[6];
#pragma unroll
    for (int c = 0; c < 6; c++) as[c] = kc[c] = Real(0);
    if (listed) {
        // rounds over the listed items, rev list first: lane t evaluates item
        // base + t; the lanes holding one owner's items find each other with
        // a match, the first of them publishes the group to the owner, and
        // the owner adds its items in list order
        sgrp[wid][lane] = ~0ull;
        __syncwarp();
        int round = 0;
        for (int li = 0; li < 2; li++) {
            const int tot = li ? nlown : nlrev;
            for (int base = 0; base < tot; base += 32, round++) {
                const int w = base + lane;
                int L = -1 - lane;   // lanes without an item match nobody
                if (w < tot) {
                    const int2 item = (li ? lown : lrev)[w];
                    L = item.y & 31;
                    Real res[6];
                    eval_item<ROLLING, SPLIT>(D, wbase + L, item.x, item.y >> 8, li == 1, upd, res);
#pragma unroll
                    for (int c = 0; c < 6; c++) sres[wid][lane][c] = res[c];
                }
                const unsigned grp = __match_any_sync(0xffffffffu, L);
                if (w < tot && (grp & ((1u << lane) - 1u)) == 0u)
                    sgrp[wid][L] = ((unsigned long long)(unsigned)round << 32) | grp;
                __syncwarp();
                const unsigned long long g = sgrp[wid][lane];
                unsigned mine = (unsigned)(g >> 32) == (unsigned)round ? (unsigned)g : 0u;
                while (mine) {
                    const int q = __ffs(mine) - 1;
                    mine &= mine - 1u;
                    sum_item<SPLIT>(as, kc, &sres[wid][q][0]);
                }
                __syncwarp();
            }
        }
    } else {   // a list outgrew its capacity: enumerate the bitmasks
        const int crev = __popcll(mrev);
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
                int other, s;
                bool own;
                if (q < qr) {
                    const int r = nth_set_bit(mrL, q);
                    other = __ldg(&D.rev[r * cap + kk]);
                    s = D.revs[r * cap + kk];
                    own = false;
                } else {
                    s = nth_set_bit(moL, q - qr);
                    other = __ldg(&D.nbr[s * cap + kk]);
                    own = true;
                }
                Real res[6];
                eval_item<ROLLING, SPLIT>(D, kk, other, s, own, upd, res);
#pragma unroll
                for (int c = 0; c < 6; c++) sres[wid][lane][c] = res[c];
            }
            __syncwarp();
            const int lo = max(it.excl, base), hi = min(it.excl + it.cnt, base + 32);
            for (int q = lo; q < hi; q++) sum_item<SPLIT>(as, kc, &sres[wid][q - base][0]);
            __syncwarp();
        }
    }
    ContactOut acc;
    pair_total<SPLIT>(as, kc, acc);
    if (!valid) return;
    cp_async_wait();
    if (!serial) atom_hist_tail(D, k, prevm, mown, upd);
    if (tail) {   // finished by k_pair_tail from these pair sums
        D.tailf[k] = dbl4{acc.F[0], acc.F[1], acc.F[2], 0.0};
        D.tailt[k] = dbl4{acc.T[0], acc.T[1], acc.T[2], 0.0};
        return;
    }
    const dbl4 vi4 = stail[0][threadIdx.x], wi4 = stail[1][threadIdx.x];
    dbl4 hold;
    if (fuse_next) hold = stail[2][threadIdx.x];
    atom_fix_tail<SPLIT>(D, k, pk, vi4, wi4, hold, integrate, fuse_next, store_f, acc);
}

// Atoms per warp of the tail kernel: lanes 0..kTailAtoms-1 own one atom
// each, all 32 lanes share the evaluation of their mesh candidates.
#ifndef GB2_TAIL_ATOMS
#define GB2_TAIL_ATOMS 8
#endif
constexpr int kTailAtoms = GB2_TAIL_ATOMS;

// Second kernel of the step: the atoms listed at the last neighbour build
// as having wall candidates or more than 64 entries on a side, kTailAtoms
// per warp.  Launched as a programmatic dependent of k_pair_step, it starts
// while the pair step's last blocks run: the wall contacts of an atom with
// one wall fix at work depend only on the step's input state and that
// wall's contact history, so they are evaluated first (mesh candidates
// spread over the lanes, slot partners staged in shared memory) and their
// forces kept as records.  After the wait, each atom is finished from the
// pair sums k_pair_step left in tailf/tailt (an atom with more than 64
// entries on a side evaluates its pairs here in the reference order): the
// post_force fixes in definition order with the records added at their
// fix, walls not yet done evaluated now, then final_integrate and the
// fused next initial_integrate.  Every atom's end of step touches only that
// atom's records, so the result is bit for bit that of one kernel.
template <bool ROLLING, bool SPLIT>
__global__ void __launch_bounds__(128, 4) k_pair_tail(Dev D, int shearupdate, int integrate, int fuse_next,
                                                      int store_f)
{
    __shared__ int s_sp[4][kTailAtoms * 64];            // slot partners of the warp's atoms (mesh walls)
    __shared__ WallRec s_rec[4][kTailAtoms][kWallRec];  // wall-contact records of the warp's atoms
    // every thread waits for the pair step before it exits, so this grid's
    // completion implies the pair step's for the launches after it
    if (step_cancelled(D)) {
        grid_dep_wait();
        return;
    }
    const int n = *D.tailcnt;
    const bool upd = shearupdate != 0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nwarp = gridDim.x * (blockDim.x >> 5);
    WallRec *rec = s_rec[wid][lane < kTailAtoms ? lane : 0];
    for (int base = (blockIdx.x * (blockDim.x >> 5) + wid) * kTailAtoms; base < n; base += nwarp * kTailAtoms) {
        const bool own = lane < kTailAtoms && base + lane < n;
        int i = 0, ti = 0, nr = 0, nn = 0, qw = -1, nwork = 0;
        dbl4 pi, vi4, wi4, hold;
        pi = vi4 = wi4 = hold = dbl4{0.0, 0.0, 0.0, 0.0};
        if (own) {
            i = D.tail[base + lane];
            pi = D.pos[i];
            vi4 = D.vel[i];
            wi4 = D.omg[i];
            if (fuse_next) hold = D.xhold[i];
            ti = D.type[i];
            nr = D.rnum[i];
            nn = D.nnum[i];
            for (int q = 0; q < D.nfix; q++) {
                const FixDev &F = D.fix[q];
                if ((F.kind == FIX_WALL_PLANE && F.inlist[i]) || (F.kind == FIX_WALL_MESH && F.mesh.tcnt[i] != 0)) {
                    qw = q;
                    nwork++;
                }
            }
        }
        const bool serial = nr > 64 || nn > 64;
        const double vi[3] = {vi4.x, vi4.y, vi4.z}, wi[3] = {wi4.x, wi4.y, wi4.z};
        // walls before the wait: atoms with one wall fix at work
        bool early = own && !serial && nwork == 1;
        int nrec = 0;
        ContactOut unused;
        for (int q = 0; q < D.nfix; q++) {
            const FixDev &F = D.fix[q];
            if (F.kind == FIX_WALL_PLANE) {
                if (early && qw == q) {
                    ContactOut o = wall_record_zero();
                    if (plane_wall_atom(D, F, i, pi, vi, wi, vi4.w, ti, upd, o)) wall_record_put(rec, nrec, o);
                }
            } else if (F.kind == FIX_WALL_MESH && __any_sync(0xffffffffu, early && qw == q)) {
                mesh_wall_items<true>(D, F.mesh, early && qw == q, i, pi, vi, wi, vi4.w, ti, upd, s_sp[wid], unused,
                                      rec, &nrec, &early);
            }
        }
        grid_dep_wait();
        ContactOut acc;
        for (int c = 0; c < 3; c++) acc.F[c] = acc.T[c] = 0.0;
        if (own) {
            if (serial) {
                serial_atom<ROLLING>(D, i, pi, vi4, wi4, ti, nr, nn, upd, acc);
                if (upd) D.prevmask[i] = ~0ull;   // every own slot written this step
            } else {
                const dbl4 F4 = D.tailf[i], T4 = D.tailt[i];
                acc.F[0] = F4.x;
                acc.F[1] = F4.y;
                acc.F[2] = F4.z;
                acc.T[0] = T4.x;
                acc.T[1] = T4.y;
                acc.T[2] = T4.z;
            }
        }
        const bool late = own && !early;   // walls evaluated after the wait
        for (int q = 0; q < D.nfix; q++) {
            const FixDev &F = D.fix[q];
            if (F.kind == FIX_GRAVITY) {
                const double massone = vi4.w * 1.;
                acc.F[0] += massone * F.acc[0];
                acc.F[1] += massone * F.acc[1];
                acc.F[2] += massone * F.acc[2];
            } else if (F.kind == FIX_WALL_PLANE || F.kind == FIX_WALL_MESH) {
                if (early && qw == q) {   // this fix's records, in the order they were made
                    for (int r = 0; r < nrec; r++) {
                        acc.F[0] += rec[r][0];
                        acc.F[1] += rec[r][1];
                        acc.F[2] += rec[r][2];
                        acc.T[0] += rec[r][3];
                        acc.T[1] += rec[r][4];
                        acc.T[2] += rec[r][5];
                    }
                }
                // walls left for now; the mesh routine is warp-collective, so
                // every lane calls it (owners without work pass own = false)
                if (F.kind == FIX_WALL_PLANE) {
                    if (late && F.inlist[i]) plane_wall_atom(D, F, i, pi, vi, wi, vi4.w, ti, upd, acc);
                } else if (__any_sync(0xffffffffu, late)) {
                    mesh_wall_items<false>(D, F.mesh, late, i, pi, vi, wi, vi4.w, ti, upd, s_sp[wid], acc);
                }
            }
        }
        if (own) atom_store_integrate<SPLIT>(D, i, pi, vi4, wi4, hold, integrate, fuse_next, store_f, acc);
    }
    grid_dep_wait();
}

// Host side: the tail kernel launched as a programmatic dependent of the
// pair step launched just before it on the same stream.
template <bool ROLLING, bool SPLIT>
inline cudaError_t launch_pair_tail(const Dev &D, int nblocks, cudaStream_t st, int shearupdate, int integrate,
                                    int fuse_next, int store_f)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_pair_tail<ROLLING, SPLIT>, D, shearupdate, integrate, fuse_next, store_f);
}

}  // namespace gb2
