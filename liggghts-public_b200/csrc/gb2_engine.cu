// gb2_engine.cu -- libgranb200: host orchestration of the device-resident
// granular time step and the C ABI declared in include/granb200.h.
//
// Step structure (Verlet::run, src/verlet.cpp:264-388, one GPU):
//   initial_integrate (+ displacement check)  -> one kernel
//   Neighbor::decide                           -> host reads one flag
//   rebuild (pre_exchange partners, pbc, sort, borders, bins, half list,
//            reverse list)  or  forward_comm   -> kernels + CUB
//   pre_force (wall neighbour lists, mesh history re-paging, rebuild only)
//   pair pass A (reverse entries) + pass B (own entries, post_force fixes,
//   final_integrate)                           -> two kernels
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/granb200.h"
#include "gb2_internal.h"
#include "gb2_insert.h"
#include "gb2_kernels.cuh"
#include "gb2_step.cuh"

using namespace gb2;

namespace {

constexpr int kBlock = 128;

inline int nblk(long n, int b = kBlock) { return (int)((n + b - 1) / b); }

// Device memory comes from the device's stream-ordered pool (the context
// creation keeps freed blocks in it for reuse within the process), so a
// context created after another was destroyed allocates without new page
// mappings.  Allocation completes before it returns, and a release first
// waits for the device, as cudaMalloc / cudaFree do.
inline cudaError_t dev_alloc(void **p, size_t bytes)
{
    cudaError_t e = cudaMallocAsync(p, bytes, cudaStreamLegacy);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
    return e;
}
inline void dev_free(void *p)
{
    cudaDeviceSynchronize();
    cudaFreeAsync(p, cudaStreamLegacy);
}

// device buffer with explicit growth
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release()
    {
        if (p) dev_free(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t m)   // discards contents
    {
        if (m <= n && p) return cudaSuccess;
        release();
        cudaError_t e = dev_alloc(reinterpret_cast<void **>(&p), std::max<size_t>(m, 1) * sizeof(T));
        if (e == cudaSuccess) n = m;
        else p = nullptr;
        return e;
    }
    cudaError_t grow_keep(size_t m, size_t keep, cudaStream_t s)   // keeps the first `keep` elements
    {
        if (m <= n && p) return cudaSuccess;
        T *q = nullptr;
        cudaError_t e = dev_alloc(reinterpret_cast<void **>(&q), std::max<size_t>(m, 1) * sizeof(T));
        if (e != cudaSuccess) return e;
        if (p && keep) cudaMemcpyAsync(q, p, std::min(keep, n) * sizeof(T), cudaMemcpyDeviceToDevice, s);
        cudaStreamSynchronize(s);
        release();
        p = q;
        n = m;
        return cudaSuccess;
    }
    void swap(DBuf &o)
    {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
};

struct MeshFix {
    MeshTopo topo;
    DBuf<TriGeom> tri;
    DBuf<int> cnn_start, cnn_list, bin_tri_start, bin_tri_list;
    int maxt = 32;   // candidate-triangle slots per atom (grown on demand up to 64)
    DBuf<int> tcnt, tlist, snp, spartner;
    DBuf<double> shist;
    DBuf<int> snp2, spartner2;   // re-paging target
    DBuf<double> shist2;
    DBuf<int> tcnt2, tcnt_s, snp_s, spartner_s;   // candidate-count double buffer, atom-sort shadows
    DBuf<double> shist_s;
    bool bins_valid = false;
    double nl_skin = 0, distmax = 0;
    // fix move/mesh rotate
    bool moving = false;
    int mover = 0;   // 1 rotate, 2 linear
    double mv_point[3] = {0, 0, 0}, mv_axis[3] = {0, 0, 1}, mv_omega = 0, mv_vel[3] = {0, 0, 0};
    DBuf<double> vnode, node_last;
    DBuf<int> trange, tcount, toff, bincnt, pvals;
    DBuf<unsigned> pkeys, pkeys2;
    long next_reneighbor = -1;   // FixMesh::next_reneighbor
    // fix mesh/surface/stress
    bool stress = false;
    double pref[3] = {0, 0, 0};
    DBuf<double> trif, ftot;
    DBuf<double> wear, tarea, kfin;   // Finnie wear
};

struct HostFix {
    int kind = FIX_NONE;
    double acc[3] = {0, 0, 0};
    int dim = 2;
    double pos = 0;
    int cyl = 0;
    double cr = 0, cc1 = 0, cc2 = 0;
    int wtype = 1;
    int rolling = 0;
    DBuf<uint8_t> inlist;
    DBuf<double> whist, whist_s;
    MeshFix *mesh = nullptr;
};

}  // namespace

struct gb2_ctx {
    gb2_params P{};
    std::string err;
    cudaStream_t st = nullptr;
    bool have_mat = false, have_atoms = false, setup_done = false, computeflag = false;
    // after an integrating step the ghost slots of vel/omg are two swaps old;
    // the values forwarded at that step's start are in vel2/omg2
    bool ghost_v_prev = false;
    MatPair hmat[(kMaxTypes + 1) * (kMaxTypes + 1)];
    DBuf<MatPair> dmat;

    int nlocal = 0, nghost = 0, nmax = 0, cap = 0;
    // per type, the largest radius of the atoms uploaded or inserted (the
    // neighbour cutoff at setup)
    double h_maxrad[kMaxTypes + 1] = {};
    DBuf<dbl4> pos, vel, omg, pos2, vel2, omg2, f, tq, tailf, tailt, xhold;
    bool split = false;           // GB2_PREC_SPLIT
    DBuf<flt8> kin, kin2;         // split precision: FP32 kinematics records (double-buffered like vel)
    DBuf<uint8_t> revs;
    int minb = 0;                 // register-allocation target of the pair step kernel (blocks/SM; 0: default)
    int nsm = 148;                // SMs of the device
    int tail_per_sm = 8;          // blocks of the tail kernel per SM (kTailAtoms atoms per warp)
    int item_cap = 160;           // listed-round capacity per warp and side (grown on demand up to kItemCap)
    bool item_cap_fixed = false;  // GB2_ITEM_CAP sets it and stops the growth (0: masks only)
    int item_cap_grown = 0;
    bool fused_pending = false;   // the previous pass B already ran this step's initial_integrate
    // steps queued ahead of the rebuild decision (see gb2_run)
    bool queue_ok = true;         // GB2_QUEUE_DEPTH=0 turns it off
    int queue_depth = 4;
    bool queue_active = false;
    DBuf<int> dstop;
    int *h_stop = nullptr;        // pinned ring of stop words read back per queued step
    cudaEvent_t qev[16] = {};
    DBuf<int> type, tag;
    int maxn = 16, maxr = 16, maxp = 16;
    DBuf<int> nnum, nbr, flag, rnum, rev, pnum, ptag, tail;
    DBuf<int> type_s, tag_s, pnum_s, ptag_s;   // atom-sort shadows
    DBuf<double> phist_s;
    DBuf<double> hist, hist2, phist;
    DBuf<unsigned long long> prevmask;
    DBuf<int> gsrc;
    DBuf<dbl4> gshift;
    // bins
    double bboxlo[3], bboxhi[3], bininv[3], binsize[3];
    int nbin[3], mbinlo[3], mbin[3], mbins = 0;
    std::vector<int> h_stencil;
    std::vector<int2> h_srow;   // stencil runs {first offset, bins}
    DBuf<int2> srow;
    DBuf<int> stencil, bin_start, bin_atoms, counts, vals, vals2, sel, nsel;
    DBuf<unsigned> keys, keys2;
    DBuf<uint8_t> bflags;
    DBuf<char> cubtmp;
    DBuf<int> dstatus, ddflag, dneed, dtailcnt;
    long ngrow = 0;
    int *h_pinned = nullptr;   // [0] status, [1] dflag, [2] nsel, [6] short item lists, [8..9] upload checks
    // neighbor
    double cutneighmax = 0, triggersq = 0;
    int ago = 0, nbuilds = 0;
    long ntimestep = 0, nextsort = 0;
    int snb[3] = {1, 1, 1};
    double sinv[3] = {0, 0, 0}, slo[3] = {0, 0, 0};
    // fixes
    int nfix = 0;
    HostFix fix[kMaxFix];
    // stats
    long npairs_last = 0;
    long launches = 0;
    long nsteps_rebuild = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // per-kernel event timing (gb2_set_profiling): every prof_every-th step
    bool prof = false;
    int prof_every = 1;
    struct EvPair {
        cudaEvent_t a, b;
        int cls;
    };
    std::vector<EvPair> ev_free, ev_pending;
    double prof_ms[5] = {0, 0, 0, 0, 0};
    long n_pair_main = 0;
    long n_rebuild_timed = 0;
    // fix insert/pack (at most one)
    InsertPack *ins = nullptr;
    // fix insert/stream (at most one insertion fix per context): release
    // data of the owned atoms [4][cap] and the face elements on the device
    InsertStream *stream = nullptr;
    DBuf<dbl4> rel, rel_s;
    DBuf<TriGeom> sface;
    long maxtag = 0;
    DBuf<uint8_t> insflag;
    DBuf<int> insidx;
    DBuf<dbl4> insrec;
    // atom upload / download: pinned host staging and packed [n][3] planes on the device
    void *hstage = nullptr;
    size_t hstage_bytes = 0;
    DBuf<double> iostage;
    DBuf<int> iocheck;
    ~gb2_ctx()
    {
        delete ins;
        delete stream;
        if (hstage) cudaFreeHost(hstage);
    }
};

namespace {

// host copy of large blocks split over a few threads (a single core copies
// ~10 GB/s; the staging copies of a 1M-atom state are ~100 MB)
void host_copy(void *dst, const void *src, size_t bytes)
{
    const size_t kChunk = size_t(8) << 20;
    unsigned nt = std::min<unsigned>(8, std::max(1u, std::thread::hardware_concurrency()));
    if (bytes < 2 * kChunk || nt < 2) {
        std::memcpy(dst, src, bytes);
        return;
    }
    nt = (unsigned)std::min<size_t>(nt, bytes / kChunk);
    std::vector<std::thread> th;
    const size_t per = (bytes + nt - 1) / nt;
    for (unsigned k = 0; k < nt; k++) {
        const size_t a = k * per, b = std::min(bytes, a + per);
        if (a >= b) break;
        th.emplace_back([=] { std::memcpy((char *)dst + a, (const char *)src + a, b - a); });
    }
    for (auto &t : th) t.join();
}

// true when p is page-locked host memory the device can copy to or from directly
bool host_pinned(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

// The pinned-slot arena: 64 KiB page-locked blocks (portable, so contexts on
// every device can copy through them) cut into kPinnedSlot-byte slots, handed
// out and taken back under a mutex; blocks are never unlocked.
namespace {
std::mutex g_pinned_mu;
std::vector<int *> g_pinned_free;
constexpr size_t kPinnedBlock = 64 * 1024;
}  // namespace

int gb2::pinned_slot_get(int **slot)
{
    *slot = nullptr;
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    if (g_pinned_free.empty()) {
        char *blk = nullptr;
        if (cudaHostAlloc((void **)&blk, kPinnedBlock, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return GB2_ERR_CUDA;
        }
        for (size_t o = kPinnedBlock; o >= kPinnedSlot; o -= kPinnedSlot)
            g_pinned_free.push_back(reinterpret_cast<int *>(blk + o - kPinnedSlot));
    }
    *slot = g_pinned_free.back();
    g_pinned_free.pop_back();
    std::memset(*slot, 0, kPinnedSlot);
    return 0;
}

void gb2::pinned_slot_put(int *slot)
{
    if (!slot) return;
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned_free.push_back(slot);
}

// insertion fixes (defined below, in the C-linkage block), called inside a rebuild
extern "C" {
static int do_insert(gb2_ctx *c, bool ghosts_prev);
static int do_insert_stream(gb2_ctx *c, bool ghosts_prev);
}

namespace {

int set_err(gb2_ctx *c, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
    return code;
}

#define CK(call)                                                                                                  \
    do {                                                                                                          \
        cudaError_t e_ = (call);                                                                                  \
        if (e_ != cudaSuccess) return set_err(c, GB2_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                                              __FILE__, __LINE__);                                                \
    } while (0)

#define CKL()                                                                                                     \
    do {                                                                                                          \
        c->launches++;                                                                                            \
        cudaError_t e_ = cudaGetLastError();                                                                      \
        if (e_ != cudaSuccess)                                                                                    \
            return set_err(c, GB2_ERR_CUDA, "kernel launch: %s (%s:%d)", cudaGetErrorString(e_), __FILE__,       \
                           __LINE__);                                                                             \
    } while (0)

// pinned host staging of at least `bytes` (grown, never shrunk)
int host_stage(gb2_ctx *c, size_t bytes)
{
    if (bytes <= c->hstage_bytes) return 0;
    if (c->hstage) cudaFreeHost(c->hstage);
    c->hstage = nullptr;
    c->hstage_bytes = 0;
    CK(cudaHostAlloc(&c->hstage, bytes, cudaHostAllocDefault));
    c->hstage_bytes = bytes;
    return 0;
}

Dev make_dev(gb2_ctx *c)
{
    Dev D;
    std::memset(&D, 0, sizeof D);
    D.nlocal = c->nlocal;
    D.nghost = c->nghost;
    D.nmax = c->nmax;
    D.cap = c->cap;
    D.pos = c->pos.p;
    D.vel = c->vel.p;
    D.omg = c->omg.p;
    D.pos_out = c->pos2.p;
    D.vel_out = c->vel2.p;
    D.omg_out = c->omg2.p;
    D.kin = c->split ? c->kin.p : nullptr;
    D.kin_out = c->split ? c->kin2.p : nullptr;
    D.type = c->type.p;
    D.tag = c->tag.p;
    D.f = c->f.p;
    D.tq = c->tq.p;
    D.tailf = c->tailf.p;
    D.tailt = c->tailt.p;
    D.tail = c->tail.p;
    D.tailcnt = c->dtailcnt.p;
    D.xhold = c->xhold.p;
    D.maxn = c->maxn;
    D.item_cap = c->item_cap;
    D.nnum = c->nnum.p;
    D.nbr = c->nbr.p;
    D.flag = c->flag.p;
    D.hist = c->hist.p;
    D.hist_out = c->hist2.p;
    D.prevmask = c->prevmask.p;
    D.maxr = c->maxr;
    D.rnum = c->rnum.p;
    D.rev = c->rev.p;
    D.revs = c->revs.p;
    D.rel = c->stream ? c->rel.p : nullptr;
    D.maxp = c->maxp;
    D.pnum = c->pnum.p;
    D.ptag = c->ptag.p;
    D.phist = c->phist.p;
    D.gsrc = c->gsrc.p;
    D.gshift = c->gshift.p;
    for (int d = 0; d < 3; d++) {
        D.bboxlo[d] = c->bboxlo[d];
        D.bboxhi[d] = c->bboxhi[d];
        D.bininv[d] = c->bininv[d];
        D.binsize[d] = c->binsize[d];
        D.nbin[d] = c->nbin[d];
        D.mbinlo[d] = c->mbinlo[d];
        D.mbin[d] = c->mbin[d];
    }
    D.mbins = c->mbins;
    D.nstencil = (int)c->h_stencil.size();
    D.stencil = c->stencil.p;
    D.nsrow = (int)c->h_srow.size();
    D.srow = c->srow.p;
    D.bin_start = c->bin_start.p;
    D.bin_atoms = c->bin_atoms.p;
    D.mat = c->dmat.p;
    D.ntypes = c->P.ntypes;
    D.dt = c->P.dt;
    D.skin = c->P.skin;
    D.cutneighmax = c->cutneighmax;
    D.triggersq = c->triggersq;
    D.rolling = c->P.rolling_cdt;
    D.tdamp = c->P.tangential_damping;
    D.nfix = c->nfix;
    for (int k = 0; k < c->nfix; k++) {
        const HostFix &H = c->fix[k];
        FixDev &F = D.fix[k];
        F.kind = H.kind;
        for (int q = 0; q < 3; q++) F.acc[q] = H.acc[q];
        F.dim = H.dim;
        F.pos = H.pos;
        F.cyl = H.cyl;
        F.cr = H.cr;
        F.cc1 = H.cc1;
        F.cc2 = H.cc2;
        F.wtype = H.wtype;
        F.rolling = H.rolling;
        F.inlist = H.inlist.p;
        F.whist = H.whist.p;
        if (H.mesh) {
            MeshFix &M = *H.mesh;
            MeshDev &m = F.mesh;
            m.ntri = (int)M.topo.tri.size();
            m.tri = M.tri.p;
            m.cnn_start = M.cnn_start.p;
            m.cnn_list = M.cnn_list.p;
            m.bin_tri_start = M.bin_tri_start.p;
            m.bin_tri_list = M.bin_tri_list.p;
            m.nl_skin = M.nl_skin;
            m.wtype = H.wtype;
            m.rolling = H.rolling;
            m.maxt = M.maxt;
            m.tcnt = M.tcnt.p;
            m.tlist = M.tlist.p;
            m.snp = M.snp.p;
            m.spartner = M.spartner.p;
            m.shist = M.shist.p;
            m.vnode = M.moving ? M.vnode.p : nullptr;
            m.trif = M.stress ? M.trif.p : nullptr;
            m.ftot = M.stress ? M.ftot.p : nullptr;
            m.wear = M.stress && M.wear.p ? M.wear.p : nullptr;
            m.tarea = M.tarea.p;
            m.kfin = M.kfin.p;
            for (int d = 0; d < 3; d++) m.pref[d] = M.pref[d];
        }
    }
    D.status = c->dstatus.p;
    D.dflag = c->ddflag.p;
    D.need = c->dneed.p;
    D.dstop = c->queue_active ? c->dstop.p : nullptr;
    D.step = (int)c->ntimestep;
    return D;
}

int read_status(gb2_ctx *c, int *st)
{
    CK(cudaMemcpyAsync(&c->h_pinned[0], c->dstatus.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    *st = c->h_pinned[0];
    return 0;
}

int clear_status(gb2_ctx *c)
{
    CK(cudaMemsetAsync(c->dstatus.p, 0, sizeof(int), c->st));
    return 0;
}

// ---------------------------------------------------------------- profiling
enum { PROF_INTEGRATE = 0, PROF_PAIR_TAIL = 1, PROF_PAIR_MAIN = 2, PROF_FORWARD = 3, PROF_REBUILD = 4 };

int prof_begin(gb2_ctx *c, int cls, gb2_ctx::EvPair *out)
{
    out->cls = -1;
    // rebuilds are timed whenever profiling is on (they are rare, and no
    // dependent launch follows them); the other kinds on sampled steps
    if (!c->prof || (cls != PROF_REBUILD && c->prof_every > 1 && c->ntimestep % c->prof_every != 0)) return 0;
    if (c->ev_free.empty()) {
        gb2_ctx::EvPair e;
        CK(cudaEventCreate(&e.a));
        CK(cudaEventCreate(&e.b));
        c->ev_free.push_back(e);
    }
    *out = c->ev_free.back();
    c->ev_free.pop_back();
    out->cls = cls;
    CK(cudaEventRecord(out->a, c->st));
    return 0;
}

int prof_end(gb2_ctx *c, gb2_ctx::EvPair *e)
{
    if (!c->prof || e->cls < 0) return 0;
    CK(cudaEventRecord(e->b, c->st));
    c->ev_pending.push_back(*e);
    return 0;
}

// accumulate every finished pair (called after stream synchronisation points)
void prof_resolve(gb2_ctx *c)
{
    size_t keep = 0;
    for (size_t k = 0; k < c->ev_pending.size(); k++) {
        gb2_ctx::EvPair &e = c->ev_pending[k];
        if (cudaEventQuery(e.b) == cudaSuccess) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) c->prof_ms[e.cls] += ms;
            if (e.cls == PROF_PAIR_MAIN) c->n_pair_main++;
            if (e.cls == PROF_REBUILD) c->n_rebuild_timed++;
            c->ev_free.push_back(e);
        } else
            c->ev_pending[keep++] = e;
    }
    c->ev_pending.resize(keep);
}

int cub_tmp(gb2_ctx *c, size_t bytes)
{
    if (bytes > c->cubtmp.n) CK(c->cubtmp.alloc(bytes + bytes / 4 + 1024));
    return 0;
}

// ---------------------------------------------------------------- capacity

int ensure_nmax(gb2_ctx *c, int need)
{
    if (need <= c->nmax) return 0;
    const int nm = std::max(need + need / 4, c->nmax + 1024);
    const size_t keep = (size_t)(c->nlocal + c->nghost);
    CK(c->pos.grow_keep(nm, keep, c->st));
    CK(c->vel.grow_keep(nm, keep, c->st));
    CK(c->omg.grow_keep(nm, keep, c->st));
    CK(c->pos2.grow_keep(nm, 0, c->st));
    CK(c->vel2.grow_keep(nm, 0, c->st));
    CK(c->omg2.grow_keep(nm, 0, c->st));
    if (c->split) {
        CK(c->kin.grow_keep(nm, keep, c->st));
        CK(c->kin2.grow_keep(nm, 0, c->st));
    }
    CK(c->type.grow_keep(nm, keep, c->st));
    CK(c->tag.grow_keep(nm, keep, c->st));
    CK(c->gsrc.grow_keep(nm, (size_t)c->nghost, c->st));
    CK(c->gshift.grow_keep(nm, (size_t)c->nghost, c->st));
    c->nmax = nm;
    return 0;
}

// ---------------------------------------------------------------- neighbor

void neighbor_init(gb2_ctx *c)
{
    // Neighbor::init cutoffs (src/neighbor.cpp:292-332) with
    // PairGran::init_one (src/pair_gran.cpp:623): cut = maxrad_i + maxrad_j
    const int nt = c->P.ntypes;
    std::vector<double> maxrad(nt + 1, 0.0);
    // future particles of an insertion fix count as dynamic (src/pair_gran.cpp:540-554)
    if (c->ins)
        for (int t = 1; t <= nt; t++) maxrad[t] = std::max(maxrad[t], c->ins->max_rad(t));
    if (c->stream)
        for (int t = 1; t <= nt; t++) maxrad[t] = std::max(maxrad[t], c->stream->max_rad(t));
    for (int t = 1; t <= nt; t++) maxrad[t] = std::max(maxrad[t], c->h_maxrad[t]);
    c->triggersq = 0.25 * c->P.skin * c->P.skin;
    c->cutneighmax = 0.0;
    for (int i = 1; i <= nt; i++)
        for (int j = 1; j <= nt; j++) {
            const double cut = (maxrad[i] + maxrad[j]) * 1.0;
            const double cutoff = std::sqrt(cut * cut);
            const double c2 = cutoff + (cutoff > 0.0 ? c->P.skin : 0.0);
            c->cutneighmax = std::max(c->cutneighmax, c2);
        }
}

int setup_bins(gb2_ctx *c)
{
    // Neighbor::setup_bins (src/neighbor.cpp:1642-1808), orthogonal box, one proc
    const double SMALL = 1.0e-6;
    const double cutghost = c->cutneighmax;
    double bbox[3], bsublo[3], bsubhi[3];
    for (int d = 0; d < 3; d++) {
        c->bboxlo[d] = c->P.boxlo[d];
        c->bboxhi[d] = c->P.boxhi[d];
        bsublo[d] = c->P.boxlo[d] - cutghost;
        bsubhi[d] = c->P.boxhi[d] + cutghost;
        bbox[d] = c->bboxhi[d] - c->bboxlo[d];
    }
    double binsize_optimal = 0.5 * c->cutneighmax;
    if (binsize_optimal == 0.0) binsize_optimal = bbox[0];
    const double binsizeinv = 1.0 / binsize_optimal;
    for (int d = 0; d < 3; d++) {
        c->nbin[d] = static_cast<int>(bbox[d] * binsizeinv);
        if (c->nbin[d] == 0) c->nbin[d] = 1;
        c->binsize[d] = bbox[d] / c->nbin[d];
        c->bininv[d] = 1.0 / c->binsize[d];
        if (binsize_optimal * c->bininv[d] > 100)
            return set_err(c, GB2_ERR_ARG, "Cannot use neighbor bins - box size << cutoff");
    }
    for (int d = 0; d < 3; d++) {
        double coord = bsublo[d] - SMALL * bbox[d];
        int lo = static_cast<int>((coord - c->bboxlo[d]) * c->bininv[d]);
        if (coord < c->bboxlo[d]) lo = lo - 1;
        coord = bsubhi[d] + SMALL * bbox[d];
        int hi = static_cast<int>((coord - c->bboxlo[d]) * c->bininv[d]);
        lo -= 1;
        hi += 1;
        c->mbinlo[d] = lo;
        c->mbin[d] = hi - lo + 1;
    }
    const long mb = (long)c->mbin[0] * c->mbin[1] * c->mbin[2];
    if (mb > (1l << 30)) return set_err(c, GB2_ERR_CAPACITY, "Too many neighbor bins");
    c->mbins = (int)mb;
    int s[3];
    for (int d = 0; d < 3; d++) {
        s[d] = static_cast<int>(c->cutneighmax * c->bininv[d]);
        if (s[d] * c->binsize[d] < c->cutneighmax) s[d]++;
    }
    const double cutsq = c->cutneighmax * c->cutneighmax;
    auto bin_distance = [&](int i, int j, int k) {
        double dx, dy, dz;
        if (i > 0) dx = (i - 1) * c->binsize[0];
        else if (i == 0) dx = 0.0;
        else dx = (i + 1) * c->binsize[0];
        if (j > 0) dy = (j - 1) * c->binsize[1];
        else if (j == 0) dy = 0.0;
        else dy = (j + 1) * c->binsize[1];
        if (k > 0) dz = (k - 1) * c->binsize[2];
        else if (k == 0) dz = 0.0;
        else dz = (k + 1) * c->binsize[2];
        return dx * dx + dy * dy + dz * dz;
    };
    c->h_stencil.clear();
    for (int k = -s[2]; k <= s[2]; k++)
        for (int j = -s[1]; j <= s[1]; j++)
            for (int i = -s[0]; i <= s[0]; i++)
                if (bin_distance(i, j, k) < cutsq) c->h_stencil.push_back(k * c->mbin[1] * c->mbin[0] + j * c->mbin[0] + i);
    CK(c->stencil.alloc(c->h_stencil.size()));
    CK(cudaMemcpyAsync(c->stencil.p, c->h_stencil.data(), c->h_stencil.size() * sizeof(int), cudaMemcpyHostToDevice,
                       c->st));
    // the stencil as runs of consecutive bins (x innermost: one run per (y, z)
    // offset), in stencil order: a run's atoms are one contiguous range of the
    // bin-sorted atom array, in the order the per-bin loop visits them
    c->h_srow.clear();
    for (size_t q = 0; q < c->h_stencil.size(); q++) {
        if (!c->h_srow.empty() && c->h_srow.back().x + c->h_srow.back().y == c->h_stencil[q])
            c->h_srow.back().y++;
        else
            c->h_srow.push_back(make_int2(c->h_stencil[q], 1));
    }
    CK(c->srow.alloc(std::max<size_t>(c->h_srow.size(), 1)));
    CK(cudaMemcpyAsync(c->srow.p, c->h_srow.data(), c->h_srow.size() * sizeof(int2), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    CK(c->bin_start.alloc((size_t)c->mbins + 1));
    CK(c->counts.alloc((size_t)c->mbins + 1));
    for (int k = 0; k < c->nfix; k++)
        if (c->fix[k].mesh) c->fix[k].mesh->bins_valid = false;
    return 0;
}

int coord2bin3_host(const gb2_ctx *c, const double *x, int *idx)
{
    for (int d = 0; d < 3; d++) {
        int v;
        if (x[d] >= c->bboxhi[d])
            v = static_cast<int>((x[d] - c->bboxhi[d]) * c->bininv[d]) + c->nbin[d];
        else if (x[d] >= c->bboxlo[d]) {
            v = static_cast<int>((x[d] - c->bboxlo[d]) * c->bininv[d]);
            v = std::min(v, c->nbin[d] - 1);
        } else
            v = static_cast<int>((x[d] - c->bboxlo[d]) * c->bininv[d]) - 1;
        idx[d] = v - c->mbinlo[d];
    }
    return idx[2] * c->mbin[1] * c->mbin[0] + idx[1] * c->mbin[0] + idx[0];
}

// FixNeighlistMesh::generate_bin_list (src/fix_neighlist_mesh.cpp:456) for a
// static mesh, inverted into bin -> ascending triangle list
int mesh_bins(gb2_ctx *c, MeshFix &M)
{
    const double skin = 0.5 * c->P.skin;
    const double rmax = 0.5 * (c->cutneighmax - c->P.skin);
    const double distmax = c->cutneighmax - rmax + skin / (70. * M_PI);
    M.nl_skin = skin;
    M.distmax = distmax;
    const double dx = c->binsize[0] / 2.0, dy = c->binsize[1] / 2.0, dz = c->binsize[2] / 2.0;
    const double maxdiag = std::sqrt(dx * dx + dy * dy + dz * dz);
    const int n = (int)M.topo.tri.size();
    std::vector<int> cnt((size_t)c->mbins + 1, 0);
    std::vector<std::pair<int, int>> entries;   // (bin, tri)
    for (int t = 0; t < n; t++) {
        const TriGeom &T = M.topo.tri[t];
        double blo[3], bhi[3];
        for (int d = 0; d < 3; d++) {
            blo[d] = 1e300;
            bhi[d] = -1e300;
        }
        for (int k = 0; k < 3; k++)
            for (int d = 0; d < 3; d++) {
                blo[d] = std::min(blo[d], T.node[k][d]);
                bhi[d] = std::max(bhi[d], T.node[k][d]);
            }
        for (int d = 0; d < 3; d++) {   // BoundingBox::shrinkToSubbox
            if (blo[d] < c->P.boxlo[d]) blo[d] = c->P.boxlo[d];
            if (bhi[d] > c->P.boxhi[d]) bhi[d] = c->P.boxhi[d];
        }
        double tmin[3] = {blo[0] - distmax, blo[1] - distmax, blo[2] - distmax};
        double tmax[3] = {bhi[0] + distmax, bhi[1] + distmax, bhi[2] + distmax};
        int lo[3], hi[3];
        coord2bin3_host(c, tmin, lo);
        coord2bin3_host(c, tmax, hi);
        for (int ix = lo[0]; ix <= hi[0]; ix++)
            for (int iy = lo[1]; iy <= hi[1]; iy++)
                for (int iz = lo[2]; iz <= hi[2]; iz++) {
                    const int b = iz * c->mbin[1] * c->mbin[0] + iy * c->mbin[0] + ix;
                    if (b < 0 || b >= c->mbins) continue;
                    double center[3];
                    center[0] = (c->mbinlo[0] + ix + 0.5) * c->binsize[0] + c->bboxlo[0];
                    center[1] = (c->mbinlo[1] + iy + 0.5) * c->binsize[1] + c->bboxlo[1];
                    center[2] = (c->mbinlo[2] + iz + 0.5) * c->binsize[2] + c->bboxlo[2];
                    if (tri_neighbuild_host(T, maxdiag, center, distmax + skin)) {
                        entries.emplace_back(b, t);
                        cnt[b]++;
                    }
                }
    }
    std::vector<int> start((size_t)c->mbins + 1, 0);
    for (int b = 0; b < c->mbins; b++) start[b + 1] = start[b] + cnt[b];
    std::vector<int> list(entries.size());
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (auto &e : entries) list[fill[e.first]++] = e.second;   // triangles visited in ascending order
    CK(M.bin_tri_start.alloc(start.size()));
    CK(M.bin_tri_list.alloc(std::max<size_t>(list.size(), 1)));
    CK(cudaMemcpyAsync(M.bin_tri_start.p, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice, c->st));
    if (!list.empty())
        CK(cudaMemcpyAsync(M.bin_tri_list.p, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    M.bins_valid = true;
    return 0;
}

// ---------------------------------------------------------------- rebuild parts

// Rotation of one step as MultiNodeMesh::rotate(dAngle, axis, p) builds it
// (src/multi_node_mesh_I.h:620-640): the axis normalised again, the
// quaternion from the host's cos/sin of half the increment omega*dt.
void mesh_rotation(const gb2_ctx *c, const MeshFix &M, MeshRotate &mv)
{
    const double dAngle = M.mv_omega * c->P.dt;
    double an[3] = {M.mv_axis[0], M.mv_axis[1], M.mv_axis[2]};
    const double mag = std::sqrt(an[0] * an[0] + an[1] * an[1] + an[2] * an[2]);
    const double sinv = 1. / mag;
    for (int d = 0; d < 3; d++) an[d] = sinv * an[d];
    mv.dQ[0] = std::cos(dAngle * 0.5);
    for (int d = 0; d < 3; d++) mv.dQ[d + 1] = an[d] * std::sin(dAngle * 0.5);
    for (int d = 0; d < 3; d++) {
        mv.origin[d] = M.mv_point[d];
        mv.omegaVec[d] = M.mv_axis[d] * M.mv_omega;
    }
    mv.trans = (M.mv_point[0] * M.mv_point[0] + M.mv_point[1] * M.mv_point[1] + M.mv_point[2] * M.mv_point[2]) > 0.;
    mv.triggersq = 0.25 * c->P.skin * c->P.skin;
}

// New capacity after an overflow: at least double, and half again the
// largest demand the overflowing kernel recorded in need[which], so a
// growing bed reallocates rarely (each reallocation synchronises the device).
int grown_capacity(gb2_ctx *c, int which, int old, int limit)
{
    int need = 0;
    if (cudaMemcpy(&need, c->dneed.p + which, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) need = 0;
    const long cap = std::max<long>(2l * old, (3l * need + 1) / 2);
    c->ngrow++;
    return (int)std::min<long>(cap, limit);
}

// Bin -> triangle lists of a moving mesh from its current nodes, on the
// device: per-triangle bin ranges, pairs in triangle order, a stable sort by
// bin (so each bin lists its triangles in ascending order) and a scan of the
// per-bin counts.
int mesh_bins_device(gb2_ctx *c, MeshFix &M, bool moving)
{
    if (moving) {   // changingMesh: full skin, distmax = cutneighmax + SMALL_DELTA
        M.nl_skin = c->P.skin;
        M.distmax = c->cutneighmax + M.nl_skin / (70. * M_PI);
    } else {        // static mesh: half skin, distmax = cutneighmax - rmax + SMALL_DELTA
        const double rmax = 0.5 * (c->cutneighmax - c->P.skin);
        M.nl_skin = 0.5 * c->P.skin;
        M.distmax = c->cutneighmax - rmax + M.nl_skin / (70. * M_PI);
    }
    const int n = (int)M.topo.tri.size();
    CK(M.trange.alloc((size_t)6 * n));
    CK(M.tcount.alloc((size_t)n + 1));
    CK(M.toff.alloc((size_t)n + 1));
    CK(M.bincnt.alloc((size_t)c->mbins + 1));
    CK(M.bin_tri_start.alloc((size_t)c->mbins + 1));
    if (clear_status(c)) return GB2_ERR_CUDA;
    Dev D = make_dev(c);
    k_tri_bin_range<<<nblk(n), kBlock, 0, c->st>>>(D, M.tri.p, n, M.distmax, c->P.boxlo[0], c->P.boxlo[1],
                                                   c->P.boxlo[2], c->P.boxhi[0], c->P.boxhi[1], c->P.boxhi[2],
                                                   M.trange.p, M.tcount.p);
    CKL();
    CK(cudaMemsetAsync(M.tcount.p + n, 0, sizeof(int), c->st));
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, M.tcount.p, M.toff.p, n + 1, c->st);
    if (cub_tmp(c, bytes)) return GB2_ERR_CUDA;
    bytes = c->cubtmp.n;
    CK(cub::DeviceScan::ExclusiveSum(c->cubtmp.p, bytes, M.tcount.p, M.toff.p, n + 1, c->st));
    int npairs = 0, st = 0;
    CK(cudaMemcpyAsync(&c->h_pinned[3], M.toff.p + n, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    if (read_status(c, &st)) return GB2_ERR_CUDA;
    npairs = c->h_pinned[3];
    if (st & ST_MESH_OUTSIDE_GRID) {
        if (!moving) return GB2_ERR_CAPACITY;   // static: the host list (exact bin aliasing) takes over
        return set_err(c, GB2_ERR_UNSUPPORTED, "moving mesh within the neighbour cutoff of the box boundary");
    }
    const size_t np = std::max(npairs, 1);
    if (M.pkeys.n < np) {   // headroom: the mesh turns, its bounding boxes change size
        CK(M.pkeys.alloc(np + np / 2));
        CK(M.pkeys2.alloc(np + np / 2));
        CK(M.pvals.alloc(np + np / 2));
        CK(M.bin_tri_list.alloc(np + np / 2));
    }
    CK(cudaMemsetAsync(M.bincnt.p, 0, sizeof(int) * ((size_t)c->mbins + 1), c->st));
    int endbit = 1;
    if (moving) {
        if (npairs > 0)
            k_tri_bin_fill<<<n, kBlock, 0, c->st>>>(D, M.trange.p, M.toff.p, M.pkeys.p, M.pvals.p, M.bincnt.p);
        while ((1l << endbit) < (long)c->mbins + 1) endbit++;
    } else {
        const double dx = c->binsize[0] / 2.0, dy = c->binsize[1] / 2.0, dz = c->binsize[2] / 2.0;
        const double maxdiag = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (npairs > 0)
            k_tri_bin_fill_cull<<<n, kBlock, 0, c->st>>>(D, M.tri.p, M.trange.p, M.toff.p, M.pkeys.p, M.pvals.p,
                                                          M.bincnt.p, maxdiag, M.distmax + M.nl_skin);
        endbit = 32;   // dropped pairs carry key 0xffffffff
    }
    CKL();
    size_t b1 = 0, b2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b1, M.pkeys.p, M.pkeys2.p, M.pvals.p, M.bin_tri_list.p, npairs, 0,
                                    endbit, c->st);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, M.bincnt.p, M.bin_tri_start.p, c->mbins + 1, c->st);
    if (cub_tmp(c, std::max(b1, b2))) return GB2_ERR_CUDA;
    bytes = c->cubtmp.n;
    if (npairs > 0)
        CK(cub::DeviceRadixSort::SortPairs(c->cubtmp.p, bytes, M.pkeys.p, M.pkeys2.p, M.pvals.p, M.bin_tri_list.p,
                                           npairs, 0, endbit, c->st));
    bytes = c->cubtmp.n;
    CK(cub::DeviceScan::ExclusiveSum(c->cubtmp.p, bytes, M.bincnt.p, M.bin_tri_start.p, c->mbins + 1, c->st));
    return 0;
}

int do_partners(gb2_ctx *c)
{
    for (int attempt = 0; attempt < 8; attempt++) {
        if (clear_status(c)) return GB2_ERR_CUDA;
        Dev D = make_dev(c);
        k_partners<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D);
        CKL();
        int st;
        if (read_status(c, &st)) return GB2_ERR_CUDA;
        if (!(st & ST_PARTNER_OVERFLOW)) return 0;
        c->maxp = grown_capacity(c, 1, c->maxp, 1 << 20);
        CK(c->ptag.alloc((size_t)c->maxp * c->cap));
        CK(c->phist.alloc((size_t)3 * c->maxp * c->cap));
    }
    return set_err(c, GB2_ERR_CAPACITY, "contact history partner capacity could not be grown");
}

int do_atom_sort(gb2_ctx *c)
{
    // Atom::sort (src/atom.cpp:1309): stable order by spatial sort bin
    c->nextsort = (c->ntimestep / c->P.sort_freq) * c->P.sort_freq + c->P.sort_freq;
    if ((long)c->snb[0] * c->snb[1] * c->snb[2] == 1) return 0;
    const int n = c->nlocal;
    Dev D = make_dev(c);
    CK(c->keys.alloc(std::max(c->nmax, 1)));
    CK(c->keys2.alloc(std::max(c->nmax, 1)));
    CK(c->vals.alloc(std::max(c->nmax, 1)));
    CK(c->vals2.alloc(std::max(c->nmax, 1)));
    k_sort_keys<<<nblk(n), kBlock, 0, c->st>>>(D, c->slo[0], c->slo[1], c->slo[2], c->sinv[0], c->sinv[1], c->sinv[2],
                                                c->snb[0], c->snb[1], c->snb[2], c->keys.p, c->vals.p);
    CKL();
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, c->keys.p, c->keys2.p, c->vals.p, c->vals2.p, n, 0, 32, c->st);
    if (cub_tmp(c, bytes)) return GB2_ERR_CUDA;
    bytes = c->cubtmp.n;
    CK(cub::DeviceRadixSort::SortPairs(c->cubtmp.p, bytes, c->keys.p, c->keys2.p, c->vals.p, c->vals2.p, n, 0, 32,
                                       c->st));
    const int *perm = c->vals2.p;
    // every per-atom array moves with its atom: gather into a persistent
    // shadow buffer and swap (no allocation once the shadows exist)
    {
        DBuf<dbl4> *arrs[][2] = {{&c->pos, &c->pos2}, {&c->vel, &c->vel2}, {&c->omg, &c->omg2}};
        for (auto &a : arrs) {
            k_gather<<<nblk(n), kBlock, 0, c->st>>>(a[0]->p, a[1]->p, perm, n);
            CKL();
            a[0]->swap(*a[1]);
        }
        auto gather_i = [&](DBuf<int> &a, DBuf<int> &sh) -> int {
            CK(sh.alloc(std::max<size_t>(a.n, 1)));
            k_gather<<<nblk(n), kBlock, 0, c->st>>>(a.p, sh.p, perm, n);
            CKL();
            a.swap(sh);
            return 0;
        };
        // slot-major arrays; only the slots an atom uses (s / div < cnt_old[atom]) are copied
        auto gather_slots = [&](auto &a, auto &sh, int nslot, const int *cnt_old, int div) -> int {
            if (nslot <= 0) return 0;
            CK(sh.alloc((size_t)nslot * c->cap));
            if (n > 0) k_gather_slots_cnt<<<nblk(n), kBlock, 0, c->st>>>(a.p, sh.p, perm, n, c->cap, nslot, cnt_old, div);
            CKL();
            a.swap(sh);
            return 0;
        };
        if (gather_i(c->type, c->type_s) || gather_i(c->tag, c->tag_s)) return GB2_ERR_CUDA;
        // partners: slots gathered against the pre-permutation counts, then the counts
        if (gather_slots(c->ptag, c->ptag_s, c->maxp, c->pnum.p, 1)) return GB2_ERR_CUDA;
        if (gather_slots(c->phist, c->phist_s, 3 * c->maxp, c->pnum.p, 3)) return GB2_ERR_CUDA;
        if (gather_i(c->pnum, c->pnum_s)) return GB2_ERR_CUDA;
        if (c->stream)
            if (gather_slots(c->rel, c->rel_s, 4, nullptr, 1)) return GB2_ERR_CUDA;
        for (int k = 0; k < c->nfix; k++) {
            HostFix &H = c->fix[k];
            if (H.kind == FIX_WALL_PLANE)
                if (gather_slots(H.whist, H.whist_s, 3, nullptr, 1)) return GB2_ERR_CUDA;
            if (H.mesh) {
                MeshFix &M = *H.mesh;
                if (gather_slots(M.spartner, M.spartner_s, M.maxt, M.tcnt.p, 1)) return GB2_ERR_CUDA;
                if (gather_slots(M.shist, M.shist_s, 3 * M.maxt, M.tcnt.p, 3)) return GB2_ERR_CUDA;
                if (gather_i(M.snp, M.snp_s) || gather_i(M.tcnt, M.tcnt_s)) return GB2_ERR_CUDA;
            }
        }
    }
    return 0;
}

int do_borders(gb2_ctx *c)
{
    // Comm::borders (src/comm.cpp:1028) with the granular slab widths of
    // Comm::setup (src/comm.cpp:670-695), one proc, periodic dims only
    c->nghost = 0;
    const double cg = c->cutneighmax / 2. + c->P.skin / 2.;
    for (int dim = 0; dim < 3; dim++) {
        if (!c->P.periodic[dim]) continue;
        const int nlast = c->nlocal + c->nghost;   // both swaps of a dim scan the same range
        for (int ineed = 0; ineed < 2; ineed++) {
            const bool low = (ineed % 2 == 0);
            const double prd = c->P.boxhi[dim] - c->P.boxlo[dim];
            const double bound = low ? c->P.boxlo[dim] + cg : c->P.boxhi[dim] - cg;
            const double shift = low ? 1 * prd : -1 * prd;
            CK(c->bflags.alloc(std::max(nlast, 1)));
            CK(c->sel.alloc(std::max(nlast, 1)));
            CK(c->nsel.alloc(1));
            Dev D = make_dev(c);
            k_border_flags<<<nblk(nlast), kBlock, 0, c->st>>>(D, nlast, dim, low ? 1 : 0, bound, c->bflags.p);
            CKL();
            size_t bytes = 0;
            thrust::counting_iterator<int> it(0);
            cub::DeviceSelect::Flagged(nullptr, bytes, it, c->bflags.p, c->sel.p, c->nsel.p, nlast, c->st);
            if (cub_tmp(c, bytes)) return GB2_ERR_CUDA;
            bytes = c->cubtmp.n;
            CK(cub::DeviceSelect::Flagged(c->cubtmp.p, bytes, it, c->bflags.p, c->sel.p, c->nsel.p, nlast, c->st));
            CK(cudaMemcpyAsync(&c->h_pinned[2], c->nsel.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
            CK(cudaStreamSynchronize(c->st));
            const int ns = c->h_pinned[2];
            const int first = c->nlocal + c->nghost;
            if (ensure_nmax(c, first + ns)) return GB2_ERR_CUDA;
            D = make_dev(c);
            if (ns > 0) {
                k_border_fill<<<nblk(ns), kBlock, 0, c->st>>>(D, c->sel.p, ns, first, dim, shift);
                CKL();
            }
            c->nghost += ns;
        }
    }
    return 0;
}

int do_build(gb2_ctx *c)
{
    const int nall = c->nlocal + c->nghost;
    CK(c->keys.alloc(std::max(c->nmax, 1)));
    CK(c->keys2.alloc(std::max(c->nmax, 1)));
    CK(c->vals.alloc(std::max(c->nmax, 1)));
    CK(c->bin_atoms.alloc(std::max(c->nmax, 1)));
    CK(cudaMemsetAsync(c->counts.p, 0, sizeof(int) * ((size_t)c->mbins + 1), c->st));
    if (clear_status(c)) return GB2_ERR_CUDA;
    Dev D = make_dev(c);
    k_bin_keys<<<nblk(nall), kBlock, 0, c->st>>>(D, nall, c->keys.p, c->vals.p, c->counts.p);
    CKL();
    size_t bytes = 0, b2 = 0;
    int endbit = 1;
    while ((1l << endbit) < (long)c->mbins + 1) endbit++;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, c->keys.p, c->keys2.p, c->vals.p, c->bin_atoms.p, nall, 0, endbit,
                                    c->st);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, c->counts.p, c->bin_start.p, c->mbins + 1, c->st);
    if (cub_tmp(c, std::max(bytes, b2))) return GB2_ERR_CUDA;
    bytes = c->cubtmp.n;
    CK(cub::DeviceRadixSort::SortPairs(c->cubtmp.p, bytes, c->keys.p, c->keys2.p, c->vals.p, c->bin_atoms.p, nall, 0,
                                       endbit, c->st));
    bytes = c->cubtmp.n;
    CK(cub::DeviceScan::ExclusiveSum(c->cubtmp.p, bytes, c->counts.p, c->bin_start.p, c->mbins + 1, c->st));
    for (int attempt = 0; attempt < 8; attempt++) {
        if (clear_status(c)) return GB2_ERR_CUDA;
        D = make_dev(c);
        k_build_list<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D);
        CKL();
        int st;
        if (read_status(c, &st)) return GB2_ERR_CUDA;
        if (st & ST_LOST_ATOM) return set_err(c, GB2_ERR_LOST, "an atom is outside the binned domain");
        if (!(st & ST_NEIGH_OVERFLOW)) break;
        if (c->maxn >= 256) return set_err(c, GB2_ERR_CAPACITY, "more than 256 neighbours per atom");
        c->maxn = grown_capacity(c, 0, c->maxn, 256);
        CK(c->nbr.alloc((size_t)c->maxn * c->cap));
        CK(c->flag.alloc((size_t)c->maxn * c->cap));
        CK(c->hist.alloc((size_t)3 * c->maxn * c->cap));
        CK(c->hist2.alloc((size_t)3 * c->maxn * c->cap));
        if (attempt == 7) return set_err(c, GB2_ERR_CAPACITY, "neighbor list capacity could not be grown");
    }
    for (int attempt = 0; attempt < 8; attempt++) {
        if (clear_status(c)) return GB2_ERR_CUDA;
        CK(cudaMemsetAsync(c->rnum.p, 0, sizeof(int) * c->cap, c->st));
        D = make_dev(c);
        k_rev_fill<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D);
        CKL();
        int st;
        if (read_status(c, &st)) return GB2_ERR_CUDA;
        if (!(st & ST_REV_OVERFLOW)) break;
        c->maxr = grown_capacity(c, 2, c->maxr, 1 << 20);
        CK(c->rev.alloc((size_t)c->maxr * c->cap));
        CK(c->revs.alloc((size_t)c->maxr * c->cap));
        if (attempt == 7) return set_err(c, GB2_ERR_CAPACITY, "reverse list capacity could not be grown");
    }
    D = make_dev(c);
    k_rev_sort<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D);
    CKL();
    c->ago = 0;
    c->nbuilds++;
    return 0;
}

int do_pre_force(gb2_ctx *c)
{
    // FixWallGran::pre_force, FixNeighlistMesh::pre_force,
    // FixContactHistoryMesh::pre_force (rebuild steps only)
    for (int k = 0; k < c->nfix; k++) {
        HostFix &H = c->fix[k];
        if (H.kind == FIX_WALL_PLANE) {
            Dev D = make_dev(c);
            k_plane_neighlist<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D, k);
            CKL();
        } else if (H.kind == FIX_WALL_MESH) {
            MeshFix &M = *H.mesh;
            if (M.moving) {
                // FixMesh::pre_force on a rebuild step: store the nodes and
                // recompute the element geometry (src/fix_mesh.cpp:567-572)
                const int nt = (int)M.topo.tri.size();
                k_mesh_refresh<<<nblk(nt), kBlock, 0, c->st>>>(M.tri.p, nt, M.node_last.p, M.tarea.p);
                CKL();
                int rc = mesh_bins_device(c, M, true);
                if (rc) return rc;
            } else if (!M.bins_valid) {
                const int rc = mesh_bins_device(c, M, false);
                if (rc == GB2_ERR_CAPACITY) {   // bins outside the grid: host list with the reference's aliasing
                    if (mesh_bins(c, M)) return GB2_ERR_CUDA;
                } else if (rc) {
                    return rc;
                }
                M.bins_valid = true;
            }
            // candidates into fresh buffers (old slots are still needed)
            const int old_maxt = M.maxt;
            CK(M.tcnt2.alloc(c->cap));
            M.tcnt.swap(M.tcnt2);   // the old counts are not needed by the re-paging
            for (int attempt = 0; attempt < 8; attempt++) {
                CK(M.tlist.alloc((size_t)M.maxt * c->cap));
                if (clear_status(c)) return GB2_ERR_CUDA;
                Dev D = make_dev(c);
                k_mesh_candidates<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D, k);
                CKL();
                int st;
                if (read_status(c, &st)) return GB2_ERR_CUDA;
                if (!(st & ST_MESHSLOT_OVERFLOW)) break;
                if (M.maxt >= 64) return set_err(c, GB2_ERR_CAPACITY, "more than 64 candidate triangles per atom");
                M.maxt = grown_capacity(c, 3, M.maxt, 64);
                M.tlist.release();
            }
            // re-page history into buffers sized for the new capacity
            CK(M.snp2.alloc(c->cap));
            CK(M.spartner2.alloc((size_t)M.maxt * c->cap));
            CK(M.shist2.alloc((size_t)3 * M.maxt * c->cap));
            M.snp.swap(M.snp2);
            M.spartner.swap(M.spartner2);
            M.shist.swap(M.shist2);
            if (clear_status(c)) return GB2_ERR_CUDA;
            Dev D = make_dev(c);
            // old slots now live in *2 buffers
            k_mesh_repage<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D, k, M.snp2.p, M.spartner2.p, M.shist2.p, old_maxt);
            CKL();
            int st;
            if (read_status(c, &st)) return GB2_ERR_CUDA;
            if (st & ST_MESH_INTERNAL) return set_err(c, GB2_ERR_STATE, "mesh contact history inconsistent");
        }
    }
    return 0;
}

// insert: an insertion fix adds atoms on this step.  Modify::
// list_init_pre_exchange (src/modify.cpp:1342-1367) calls the contact-history
// fixes first, so the pair and mesh histories are packed with the last
// build's ghost tags before the new atoms take the first ghost slots.
int do_rebuild(gb2_ctx *c, bool pre_exchange, bool sort_now, bool insert, bool ghosts_prev)
{
    if (pre_exchange)
        if (do_partners(c)) return GB2_ERR_CUDA;
    Dev D = make_dev(c);
    for (int k = 0; k < c->nfix; k++)
        if (c->fix[k].kind == FIX_WALL_MESH) {
            k_mesh_sort_contacts<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D, k);
            CKL();
        }
    if (insert) {
        const int rci = c->stream ? do_insert_stream(c, ghosts_prev) : do_insert(c, ghosts_prev);
        if (rci) return rci;
        D = make_dev(c);
    }
    if (clear_status(c)) return GB2_ERR_CUDA;
    k_pbc<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D, c->P.boxlo[0], c->P.boxlo[1], c->P.boxlo[2], c->P.boxhi[0],
                                                  c->P.boxhi[1], c->P.boxhi[2], c->P.periodic[0], c->P.periodic[1],
                                                  c->P.periodic[2]);
    CKL();
    int st;
    if (read_status(c, &st)) return GB2_ERR_CUDA;
    if (st & ST_LOST_ATOM) return set_err(c, GB2_ERR_LOST, "atom left the non-periodic box (lost atoms unsupported)");
    if (sort_now)
        if (do_atom_sort(c)) return GB2_ERR_CUDA;
    if (do_borders(c)) return GB2_ERR_CUDA;
    if (do_build(c)) return c->err.empty() ? GB2_ERR_CUDA : GB2_ERR_CAPACITY;
    {
        const int rc = do_pre_force(c);
        if (rc) return (rc == GB2_ERR_UNSUPPORTED || rc == GB2_ERR_STATE) ? rc : GB2_ERR_CUDA;
    }
    if (c->split) {   // FP32 kinematics of owned atoms and the new ghosts
        const int nall = c->nlocal + c->nghost;
        Dev D2 = make_dev(c);
        if (nall > 0) k_make_kin<<<nblk(nall), kBlock, 0, c->st>>>(D2, nall);
        CKL();
    }
    // atoms finished by the tail kernel until the next build
    CK(cudaMemsetAsync(c->dtailcnt.p, 0, sizeof(int), c->st));
    if (c->nlocal > 0) {
        Dev D3 = make_dev(c);
        k_tail_list<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D3);
        CKL();
    }
    return 0;
}

// Dynamic shared memory of the pair step: each of its 4 warps lists up to
// item_cap touching entries on each side (8 bytes each).
size_t pair_list_smem(const gb2_ctx *c) { return (size_t)4 * 2 * c->item_cap * sizeof(int2); }

// The pair step counts warps whose touching entries outgrew their lists
// (they take the slower mask enumeration); at setup and at each rebuild the
// lists grow by half, up to kItemCap, while any warp did.  Short lists keep
// shared memory, and with it L1 for the neighbour gathers, on beds with few
// contacts per atom.
int adapt_item_cap(gb2_ctx *c)
{
    if (c->item_cap_fixed || c->item_cap >= kItemCap) return 0;
    CK(cudaMemcpyAsync(&c->h_pinned[6], c->dneed.p + 4, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (c->h_pinned[6] > 0) {
        c->item_cap = std::min(kItemCap, (c->item_cap * 3 / 2 + 31) / 32 * 32);
        c->item_cap_grown++;
    }
    CK(cudaMemsetAsync(c->dneed.p + 4, 0, sizeof(int), c->st));
    return 0;
}

template <bool R, int MINB>
void launch_pair_kernel(gb2_ctx *c, const Dev &D, int shearupdate, int integrate, int fuse_next, int store_f)
{
    k_pair_step<R, MINB, false><<<nblk(c->nlocal), kBlock, pair_list_smem(c), c->st>>>(D, shearupdate, integrate,
                                                                                     fuse_next, store_f);
}

// The pair step kernel of one time step (every atom's pair sums; the
// whole step for atoms without wall work).
void launch_pair(gb2_ctx *c, const Dev &D, int shearupdate, int integrate, int fuse_next, int store_f)
{
    if (c->split) {
        launch_pair_split(D, nblk(c->nlocal), c->st, c->minb, shearupdate, integrate, fuse_next, store_f,
                          pair_list_smem(c));
        return;
    }
    // MINB: minimum resident 128-thread blocks per SM asked of the register
    // allocator; 5 (96 registers, a small spill) measured fastest on the
    // packed 1M hopper, ahead of 4 (128) and 6 (80)
    const int mb = c->minb ? c->minb : 5;
    if (c->P.rolling_cdt) {
        if (mb == 4) launch_pair_kernel<true, 4>(c, D, shearupdate, integrate, fuse_next, store_f);
        else if (mb == 5) launch_pair_kernel<true, 5>(c, D, shearupdate, integrate, fuse_next, store_f);
        else launch_pair_kernel<true, 6>(c, D, shearupdate, integrate, fuse_next, store_f);
    } else {
        if (mb == 4) launch_pair_kernel<false, 4>(c, D, shearupdate, integrate, fuse_next, store_f);
        else if (mb == 5) launch_pair_kernel<false, 5>(c, D, shearupdate, integrate, fuse_next, store_f);
        else launch_pair_kernel<false, 6>(c, D, shearupdate, integrate, fuse_next, store_f);
    }
}

// The tail kernel: the atoms with wall work or more than 64 entries on a side.
void launch_tail(gb2_ctx *c, const Dev &D, int shearupdate, int integrate, int fuse_next, int store_f)
{
    const int tblocks = c->tail_per_sm * c->nsm;
    if (c->split) launch_tail_split(D, tblocks, c->st, shearupdate, integrate, fuse_next, store_f);
    else if (c->P.rolling_cdt)
        launch_pair_tail<true, false>(D, tblocks, c->st, shearupdate, integrate, fuse_next, store_f);
    else
        launch_pair_tail<false, false>(D, tblocks, c->st, shearupdate, integrate, fuse_next, store_f);
}

int do_force(gb2_ctx *c, int shearupdate, int integrate, int fuse_next, int store_f)
{
    if (fuse_next && !c->queue_active) CK(cudaMemsetAsync(c->ddflag.p, 0, sizeof(int), c->st));
    // mesh/surface/stress: FixMesh::pre_force clears the per-element force,
    // MeshModuleStress::pre_force the totals (before the pair step, so the
    // tail kernel stays the pair step's dependent launch)
    for (int k = 0; k < c->nfix; k++) {
        MeshFix *M = c->fix[k].mesh;
        if (!M || !M->stress) continue;
        CK(cudaMemsetAsync(M->trif.p, 0, sizeof(double) * 3 * M->topo.tri.size(), c->st));
        CK(cudaMemsetAsync(M->ftot.p, 0, sizeof(double) * 6, c->st));
    }
    Dev D = make_dev(c);
    gb2_ctx::EvPair e;
    if (prof_begin(c, PROF_PAIR_MAIN, &e)) return GB2_ERR_CUDA;
    launch_pair(c, D, shearupdate, integrate, fuse_next, store_f);
    CKL();
    if (prof_end(c, &e)) return GB2_ERR_CUDA;
    if (prof_begin(c, PROF_PAIR_TAIL, &e)) return GB2_ERR_CUDA;
    launch_tail(c, D, shearupdate, integrate, fuse_next, store_f);
    CKL();
    if (prof_end(c, &e)) return GB2_ERR_CUDA;
    if (c->stream && integrate && !fuse_next && c->nlocal > 0) {
        k_stream_positions<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D);
        CKL();
    }
    if (shearupdate) c->hist.swap(c->hist2);
    if (integrate) {
        c->vel.swap(c->vel2);
        c->omg.swap(c->omg2);
        if (c->split) c->kin.swap(c->kin2);
        if (fuse_next) c->pos.swap(c->pos2);
    }
    c->fused_pending = integrate && fuse_next;
    c->ghost_v_prev = integrate != 0;
    return 0;
}

}  // namespace

// ---------------------------------------------------------------- census without allocation
// Scratch for gb2_census_noalloc: one row of 8 counters per 128-atom block plus
// a final row for the totals.  Shared by every call in the process.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[(GB2_NOALLOC_MAX_BLOCKS + 1) * 8];

// same per-atom census as k_census; each block reduces its atoms in shared
// memory and writes its own row, so no counter needs clearing beforehand
__global__ void __launch_bounds__(128) k_census_rows(Dev D, unsigned long long *rows)
{
    __shared__ unsigned long long red[7][128];
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
    for (int k = 0; k < 7; k++) red[k][threadIdx.x] = c[k];
    __syncthreads();
    for (int w = 64; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 7; k++) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 8) rows[(size_t)blockIdx.x * 8 + threadIdx.x] = threadIdx.x < 7 ? red[threadIdx.x][0] : 0ull;
}

// sums the block rows into the totals row (one block, fixed order)
__global__ void k_census_total(unsigned long long *rows, int nrows)
{
    __shared__ unsigned long long red[8][256];
    unsigned long long c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int r = threadIdx.x; r < nrows; r += blockDim.x)
        for (int k = 0; k < 8; k++) c[k] += rows[(size_t)r * 8 + k];
    for (int k = 0; k < 8; k++) red[k][threadIdx.x] = c[k];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 8; k++) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 8) rows[(size_t)GB2_NOALLOC_MAX_BLOCKS * 8 + threadIdx.x] = red[threadIdx.x][0];
}

// device address of g_noalloc_scratch per device, looked up on first use
static unsigned long long *g_noalloc_ptr[64];

// ====================================================================== C ABI

extern "C" {

const char *gb2_version(void) { return "granb200 0.1 sm_100a"; }

int gb2_create(const gb2_params *p, gb2_ctx **out)
{
    if (!p || !out) return GB2_ERR_ARG;
    *out = nullptr;
    if (p->ntypes < 1 || p->ntypes > kMaxTypes) return GB2_ERR_ARG;
    if (p->dt <= 0 || p->skin < 0) return GB2_ERR_ARG;
    if (p->precision != GB2_PREC_FP64 && p->precision != GB2_PREC_SPLIT) return GB2_ERR_UNSUPPORTED;
    gb2_ctx *c = new gb2_ctx();
    c->P = *p;
    c->split = p->precision == GB2_PREC_SPLIT;
    if (c->P.neigh_every <= 0) c->P.neigh_every = 1;
    if (const char *mb = std::getenv("GB2_PAIR_MINB")) c->minb = std::atoi(mb);
    if (const char *tb = std::getenv("GB2_TAIL_BLOCKS")) c->tail_per_sm = std::max(1, std::atoi(tb));
    if (const char *ic = std::getenv("GB2_ITEM_CAP")) {
        c->item_cap = std::min(std::max(std::atoi(ic), 0), kItemCap);
        c->item_cap_fixed = true;
    }
    if (const char *qd = std::getenv("GB2_QUEUE_DEPTH")) {
        c->queue_depth = std::min(std::max(std::atoi(qd), 0), 15);
        c->queue_ok = c->queue_depth > 0;
    }
    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) {
        delete c;
        return GB2_ERR_CUDA;
    }
    {   // the device pool keeps freed memory for this process's later contexts
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, p->device) == cudaSuccess) {
            uint64_t keep_all = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep_all);
        }
    }
    // one arena slot holds h_pinned (ints 0..31) and the stop-word ring h_stop (ints 32..47)
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
        pinned_slot_get(&c->h_pinned) != 0 || c->dstatus.alloc(1) != cudaSuccess ||
        c->ddflag.alloc(2) != cudaSuccess || c->dneed.alloc(5) != cudaSuccess || c->dstop.alloc(1) != cudaSuccess ||
        c->dtailcnt.alloc(1) != cudaSuccess ||
        cudaMemsetAsync(c->dneed.p, 0, 5 * sizeof(int), c->st) != cudaSuccess ||
        cudaMemsetAsync(c->dtailcnt.p, 0, sizeof(int), c->st) != cudaSuccess ||
        cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, p->device) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess ||
        cudaEventCreate(&c->ev1) != cudaSuccess) {
        pinned_slot_put(c->h_pinned);
        if (c->st) cudaStreamDestroy(c->st);
        delete c;
        return GB2_ERR_CUDA;
    }
    c->h_stop = c->h_pinned + 32;
    *out = c;
    return 0;
}

int gb2_destroy(gb2_ctx *c)
{
    if (!c) return 0;
    cudaStreamSynchronize(c->st);
    for (int k = 0; k < c->nfix; k++) delete c->fix[k].mesh;
    for (auto &e : c->ev_free) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    for (auto &e : c->ev_pending) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    pinned_slot_put(c->h_pinned);   // h_stop lies in the same slot
    for (auto &e : c->qev)
        if (e) cudaEventDestroy(e);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    cudaStream_t st = c->st;
    delete c;
    if (st) cudaStreamDestroy(st);
    return 0;
}

int gb2_set_materials(gb2_ctx *c, const double *youngs, const double *poisson, const double *restitution,
                      const double *friction, const double *rollfriction)
{
    if (!c || !youngs || !poisson || !restitution || !friction) return GB2_ERR_ARG;
    const int nt = c->P.ntypes;
    std::memset(c->hmat, 0, sizeof c->hmat);
    for (int i = 1; i <= nt; i++)
        for (int j = 1; j <= nt; j++) {
            const double Yi = youngs[i - 1], Yj = youngs[j - 1];
            const double vi = poisson[i - 1], vj = poisson[j - 1];
            if (vi < 0. || vi > 0.5 || vj < 0. || vj > 0.5)
                return set_err(c, GB2_ERR_ARG, "0 <= poissonsRatio <= 0.5 required");
            const double cor = restitution[(i - 1) * nt + (j - 1)];
            if (cor <= 0.05 || cor > 1) return set_err(c, GB2_ERR_ARG, "0.05 < coefficientRestitution <= 1 required");
            MatPair &m = c->hmat[i * (kMaxTypes + 1) + j];
            // src/global_properties.cpp:432, :461, :508, :540
            m.Yeff = 1. / ((1. - std::pow(vi, 2.)) / Yi + (1. - std::pow(vj, 2.)) / Yj);
            m.Geff = 1. / (2. * (2. - vi) * (1. + vi) / Yi + 2. * (2. - vj) * (1. + vj) / Yj);
            const double lg = std::log(cor);
            m.betaeff = lg / std::sqrt(std::pow(lg, 2.) + std::pow(M_PI, 2.));
            m.mu = friction[(i - 1) * nt + (j - 1)];
            m.mur = rollfriction ? rollfriction[(i - 1) * nt + (j - 1)] : 0.0;
        }
    if (c->dmat.alloc((kMaxTypes + 1) * (kMaxTypes + 1))) return set_err(c, GB2_ERR_CUDA, "alloc");
    CK(cudaMemcpyAsync(c->dmat.p, c->hmat, sizeof c->hmat, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->have_mat = true;
    return 0;
}

int gb2_upload_atoms(gb2_ctx *c, int n, const double *x, const double *v, const double *omega, const double *radius,
                     const double *rmass, const int *type, const int *tag)
{
    if (!c || n <= 0 || !x || !v || !omega || !radius || !rmass || !type || !tag) return GB2_ERR_ARG;
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "atoms must be uploaded before setup");
    c->have_atoms = false;   // until this upload has passed every check
    c->nlocal = n;
    c->cap = (n + 31) / 32 * 32;
    c->nmax = 0;
    c->nghost = 0;
    if (ensure_nmax(c, n + n / 4 + 1024)) return GB2_ERR_CUDA;
    // x | v | omega | radius | rmass staged as 11 n doubles, one host-to-device
    // copy per array (straight from the caller's memory when it is pinned),
    // packed into the 32-byte records and checked on the device
    const size_t N = (size_t)n;
    CK(c->iostage.alloc(15 * N));   // also the download's five [n][3] planes
    CK(c->iocheck.alloc(2));
    const double *src[5] = {x, v, omega, radius, rmass};
    const size_t off[5] = {0, 3 * N, 6 * N, 9 * N, 10 * N}, len[5] = {3 * N, 3 * N, 3 * N, N, N};
    bool pageable = false;
    for (int k = 0; k < 5; k++) pageable = pageable || !host_pinned(src[k]);
    if (pageable && host_stage(c, 11 * N * sizeof(double))) return GB2_ERR_CUDA;
    for (int k = 0; k < 5; k++) {
        const size_t bytes = len[k] * sizeof(double);
        if (host_pinned(src[k])) {
            CK(cudaMemcpyAsync(c->iostage.p + off[k], src[k], bytes, cudaMemcpyHostToDevice, c->st));
        } else {
            double *h = (double *)c->hstage + off[k];
            host_copy(h, src[k], bytes);
            CK(cudaMemcpyAsync(c->iostage.p + off[k], h, bytes, cudaMemcpyHostToDevice, c->st));
        }
    }
    CK(cudaMemsetAsync(c->iocheck.p, 0x7f, sizeof(int), c->st));   // first bad atom: none (> any index)
    CK(cudaMemsetAsync(c->iocheck.p + 1, 0, sizeof(int), c->st));
    k_pack_atoms<<<nblk(n), kBlock, 0, c->st>>>(c->iostage.p, n, c->pos.p, c->vel.p, c->omg.p, c->iocheck.p);
    CKL();
    CK(cudaMemcpyAsync(c->type.p, type, sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->tag.p, tag, sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
    // the device check's verdict lands in pinned memory, so this readback
    // stays asynchronous and the host work below overlaps the copies
    CK(cudaMemcpyAsync(&c->h_pinned[8], c->iocheck.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
    const size_t cap = c->cap;
    CK(c->f.alloc(cap));
    CK(c->tq.alloc(cap));
    CK(c->tailf.alloc(cap));
    CK(c->tailt.alloc(cap));
    CK(c->tail.alloc(cap));
    CK(c->xhold.alloc(cap));
    CK(c->nnum.alloc(cap));
    CK(c->rnum.alloc(cap));
    CK(c->pnum.alloc(cap));
    CK(c->nbr.alloc((size_t)c->maxn * cap));
    CK(c->flag.alloc((size_t)c->maxn * cap));
    CK(c->hist.alloc((size_t)3 * c->maxn * cap));
    CK(c->hist2.alloc((size_t)3 * c->maxn * cap));
    CK(c->prevmask.alloc(cap));
    CK(c->rev.alloc((size_t)c->maxr * cap));
    CK(c->revs.alloc((size_t)c->maxr * cap));
    CK(c->ptag.alloc((size_t)c->maxp * cap));
    CK(c->phist.alloc((size_t)3 * c->maxp * cap));
    CK(cudaMemsetAsync(c->f.p, 0, sizeof(dbl4) * cap, c->st));
    CK(cudaMemsetAsync(c->tq.p, 0, sizeof(dbl4) * cap, c->st));
    CK(cudaMemsetAsync(c->nnum.p, 0, sizeof(int) * cap, c->st));
    CK(cudaMemsetAsync(c->rnum.p, 0, sizeof(int) * cap, c->st));
    CK(cudaMemsetAsync(c->pnum.p, 0, sizeof(int) * cap, c->st));
    // host checks while the copies are in flight, in one pass over the
    // caller's arrays: type range, per type the largest radius (the
    // neighbour cutoff at setup), the largest tag (Atom::tag_extend)
    const int nt = c->P.ntypes;
    int bad_type = -1;
    double maxrad[kMaxTypes + 1] = {};
    long maxtag = 0;
    for (int i = 0; i < n; i++) {
        const int t = type[i];
        if (t < 1 || t > nt) {
            bad_type = i;
            break;
        }
        if (radius[i] > maxrad[t]) maxrad[t] = radius[i];
        if (tag[i] > maxtag) maxtag = tag[i];
    }
    CK(cudaStreamSynchronize(c->st));
    const int bad0 = c->h_pinned[8], bad1 = c->h_pinned[9];
    if (bad_type >= 0) return set_err(c, GB2_ERR_ARG, "atom type out of range");
    if (bad1 == 2) return set_err(c, GB2_ERR_ARG, "Fix nve/sphere requires extended particles");
    if (bad1 == 3) return set_err(c, GB2_ERR_ARG, "atom mass must be positive");
    if (bad1 == 1) return set_err(c, GB2_ERR_ARG, "non-finite atom state (atom %d)", bad0);
    std::memcpy(c->h_maxrad, maxrad, sizeof maxrad);
    c->maxtag = maxtag;
    c->have_atoms = true;
    return 0;
}

static int add_fix_common(gb2_ctx *c)
{
    if (!c) return GB2_ERR_ARG;
    if (c->nfix >= kMaxFix) return set_err(c, GB2_ERR_CAPACITY, "too many fixes");
    if (!c->have_atoms) return set_err(c, GB2_ERR_STATE, "upload atoms before adding fixes");
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "fixes must be added before setup");
    return 0;
}

int gb2_add_gravity(gb2_ctx *c, double magnitude, const double dir[3])
{
    int rc = add_fix_common(c);
    if (rc) return rc;
    // FixGravity::set_acceleration, style vector (src/fix_gravity.cpp:376-397)
    const double length = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    if (length == 0.) return set_err(c, GB2_ERR_ARG, "Gravity direction vector = 0");
    HostFix &H = c->fix[c->nfix];
    H.kind = FIX_GRAVITY;
    H.acc[0] = magnitude * (dir[0] / length);
    H.acc[1] = magnitude * (dir[1] / length);
    H.acc[2] = magnitude * (dir[2] / length);
    return c->nfix++;
}

int gb2_add_wall_plane(gb2_ctx *c, int dim, double pos, int wall_type, int rolling_cdt)
{
    int rc = add_fix_common(c);
    if (rc) return rc;
    if (dim < 0 || dim > 2) return set_err(c, GB2_ERR_ARG, "plane dimension must be 0, 1 or 2");
    if (wall_type < 1 || wall_type > c->P.ntypes) return set_err(c, GB2_ERR_ARG, "wall type out of range");
    HostFix &H = c->fix[c->nfix];
    H.kind = FIX_WALL_PLANE;
    H.dim = dim;
    H.pos = pos;
    H.wtype = wall_type;
    H.rolling = rolling_cdt;
    CK(H.inlist.alloc(c->cap));
    CK(H.whist.alloc((size_t)3 * c->cap));
    CK(cudaMemsetAsync(H.inlist.p, 0, c->cap, c->st));
    CK(cudaMemsetAsync(H.whist.p, 0, sizeof(double) * 3 * c->cap, c->st));
    return c->nfix++;
}

int gb2_add_wall_cylinder(gb2_ctx *c, int dim, double radius, double c1, double c2, int wall_type, int rolling_cdt)
{
    if (!c) return GB2_ERR_ARG;
    if (!(radius > 0) || !std::isfinite(c1) || !std::isfinite(c2))
        return set_err(c, GB2_ERR_ARG, "cylinder radius must be positive and its axis finite");
    const int k = gb2_add_wall_plane(c, dim, 0.0, wall_type, rolling_cdt);
    if (k < 0) return k;
    HostFix &H = c->fix[k];
    H.cyl = 1;
    H.cr = radius;
    H.cc1 = c1;
    H.cc2 = c2;
    return k;
}

int gb2_add_wall_mesh(gb2_ctx *c, int ntri, const double *nodes, int wall_type, double curvature, int rolling_cdt)
{
    int rc = add_fix_common(c);
    if (rc) return rc;
    if (ntri <= 0 || !nodes) return set_err(c, GB2_ERR_ARG, "empty mesh");
    if (wall_type < 1 || wall_type > c->P.ntypes) return set_err(c, GB2_ERR_ARG, "wall type out of range");
    for (long q = 0; q < 9l * ntri; q++)
        if (!std::isfinite(nodes[q])) return set_err(c, GB2_ERR_ARG, "non-finite mesh node");
    MeshFix *M = new MeshFix();
    const double curv = curvature > 0 ? curvature : 1. - 0.00001;
    if (!build_mesh_topology(nodes, ntri, curv, 1e-8, M->topo, c->err)) {
        delete M;
        return GB2_ERR_ARG;
    }
    const int n = (int)M->topo.tri.size();
    for (int t = 0; t < n; t++)
        for (int k = 0; k < 3; k++)
            for (int d = 0; d < 3; d++)
                if (M->topo.tri[t].node[k][d] < c->P.boxlo[d] || M->topo.tri[t].node[k][d] >= c->P.boxhi[d]) {
                    delete M;
                    return set_err(c, GB2_ERR_UNSUPPORTED, "mesh nodes must lie inside the simulation box");
                }
    if (M->tri.alloc(n) || M->cnn_start.alloc(n + 1) || M->cnn_list.alloc(std::max<size_t>(M->topo.cnn_list.size(), 1))) {
        delete M;
        return set_err(c, GB2_ERR_CUDA, "mesh alloc");
    }
    cudaMemcpyAsync(M->tri.p, M->topo.tri.data(), sizeof(TriGeom) * n, cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(M->cnn_start.p, M->topo.cnn_start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, c->st);
    if (!M->topo.cnn_list.empty())
        cudaMemcpyAsync(M->cnn_list.p, M->topo.cnn_list.data(), sizeof(int) * M->topo.cnn_list.size(),
                        cudaMemcpyHostToDevice, c->st);
    const size_t cap = c->cap;
    if (M->tcnt.alloc(cap) || M->snp.alloc(cap) || M->spartner.alloc((size_t)M->maxt * cap) ||
        M->shist.alloc((size_t)3 * M->maxt * cap) || M->tlist.alloc((size_t)M->maxt * cap)) {
        delete M;
        return set_err(c, GB2_ERR_CUDA, "mesh alloc");
    }
    cudaMemsetAsync(M->tcnt.p, 0, sizeof(int) * cap, c->st);
    cudaMemsetAsync(M->snp.p, 0, sizeof(int) * cap, c->st);
    cudaMemsetAsync(M->spartner.p, 0xff, sizeof(int) * M->maxt * cap, c->st);
    cudaMemsetAsync(M->shist.p, 0, sizeof(double) * 3 * M->maxt * cap, c->st);
    CK(cudaStreamSynchronize(c->st));
    HostFix &H = c->fix[c->nfix];
    H.kind = FIX_WALL_MESH;
    H.wtype = wall_type;
    H.rolling = rolling_cdt;
    H.mesh = M;
    return c->nfix++;
}

int gb2_add_move_mesh_rotate(gb2_ctx *c, int ifix_mesh, const double origin[3], const double axis[3], double period)
{
    if (!c || !origin || !axis) return GB2_ERR_ARG;
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "fix move/mesh must be defined before setup");
    if (ifix_mesh < 0 || ifix_mesh >= c->nfix || !c->fix[ifix_mesh].mesh)
        return set_err(c, GB2_ERR_ARG, "fix move/mesh: mesh fix index does not name a mesh wall");
    MeshFix &M = *c->fix[ifix_mesh].mesh;
    if (M.moving) return set_err(c, GB2_ERR_UNSUPPORTED, "one fix move/mesh per mesh is supported");
    if (!(period != 0.0) || !std::isfinite(period)) return set_err(c, GB2_ERR_ARG, "fix move/mesh: period must be non-zero");
    for (int d = 0; d < 3; d++) {
        M.mv_point[d] = origin[d];
        M.mv_axis[d] = axis[d];
    }
    // vectorNormalize3D (src/vector_liggghts.h:62) as in the MeshMoverRotate constructor
    const double norm = std::sqrt(M.mv_axis[0] * M.mv_axis[0] + M.mv_axis[1] * M.mv_axis[1] + M.mv_axis[2] * M.mv_axis[2]);
    if (norm == 0.) return set_err(c, GB2_ERR_ARG, "fix move/mesh: zero rotation axis");
    const double invnorm = 1. / norm;
    for (int d = 0; d < 3; d++) M.mv_axis[d] *= invnorm;
    M.mv_omega = 2. * M_PI / period;
    M.mover = 1;
    const size_t nt = M.topo.tri.size();
    CK(M.vnode.alloc(9 * nt));
    CK(M.node_last.alloc(9 * nt));
    CK(cudaMemsetAsync(M.vnode.p, 0, sizeof(double) * 9 * nt, c->st));   // FixMoveMesh::setup: v = 0
    CK(cudaStreamSynchronize(c->st));
    M.moving = true;
    return 0;
}

int gb2_add_move_mesh_linear(gb2_ctx *c, int ifix_mesh, const double vel[3])
{
    if (!c || !vel) return GB2_ERR_ARG;
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "fix move/mesh must be defined before setup");
    if (ifix_mesh < 0 || ifix_mesh >= c->nfix || !c->fix[ifix_mesh].mesh)
        return set_err(c, GB2_ERR_ARG, "fix move/mesh: mesh fix index does not name a mesh wall");
    MeshFix &M = *c->fix[ifix_mesh].mesh;
    if (M.moving) return set_err(c, GB2_ERR_UNSUPPORTED, "one fix move/mesh per mesh is supported");
    for (int d = 0; d < 3; d++) {
        if (!std::isfinite(vel[d])) return set_err(c, GB2_ERR_ARG, "fix move/mesh: non-finite velocity");
        M.mv_vel[d] = vel[d];
    }
    const size_t nt = M.topo.tri.size();
    CK(M.vnode.alloc(9 * nt));
    CK(M.node_last.alloc(9 * nt));
    CK(cudaMemsetAsync(M.vnode.p, 0, sizeof(double) * 9 * nt, c->st));   // FixMoveMesh::setup: v = 0
    CK(cudaStreamSynchronize(c->st));
    M.moving = true;
    M.mover = 2;
    return 0;
}

// room for `want` owned atoms in every capacity-strided array (before setup,
// when those arrays hold their initial zeros)
static int reserve_cap(gb2_ctx *c, int want)
{
    const size_t cap = ((size_t)want + 31) / 32 * 32;
    if (cap <= (size_t)c->cap) return 0;
    c->cap = (int)cap;
    if (ensure_nmax(c, (int)(cap + cap / 4 + 1024))) return GB2_ERR_CUDA;
    CK(c->f.alloc(cap));
    CK(c->tq.alloc(cap));
    CK(c->tailf.alloc(cap));
    CK(c->tailt.alloc(cap));
    CK(c->tail.alloc(cap));
    CK(c->xhold.alloc(cap));
    CK(c->nnum.alloc(cap));
    CK(c->rnum.alloc(cap));
    CK(c->pnum.alloc(cap));
    CK(c->nbr.alloc((size_t)c->maxn * cap));
    CK(c->flag.alloc((size_t)c->maxn * cap));
    CK(c->hist.alloc((size_t)3 * c->maxn * cap));
    CK(c->hist2.alloc((size_t)3 * c->maxn * cap));
    CK(c->prevmask.alloc(cap));
    CK(c->rev.alloc((size_t)c->maxr * cap));
    CK(c->revs.alloc((size_t)c->maxr * cap));
    CK(c->ptag.alloc((size_t)c->maxp * cap));
    CK(c->phist.alloc((size_t)3 * c->maxp * cap));
    CK(cudaMemsetAsync(c->f.p, 0, sizeof(dbl4) * cap, c->st));
    CK(cudaMemsetAsync(c->tq.p, 0, sizeof(dbl4) * cap, c->st));
    CK(cudaMemsetAsync(c->nnum.p, 0, sizeof(int) * cap, c->st));
    CK(cudaMemsetAsync(c->rnum.p, 0, sizeof(int) * cap, c->st));
    CK(cudaMemsetAsync(c->pnum.p, 0, sizeof(int) * cap, c->st));
    for (int k = 0; k < c->nfix; k++) {
        HostFix &H = c->fix[k];
        if (H.kind == FIX_WALL_PLANE) {
            CK(H.inlist.alloc(cap));
            CK(H.whist.alloc(3 * cap));
            CK(cudaMemsetAsync(H.inlist.p, 0, cap, c->st));
            CK(cudaMemsetAsync(H.whist.p, 0, sizeof(double) * 3 * cap, c->st));
        }
        if (H.mesh) {
            MeshFix &M = *H.mesh;
            CK(M.tcnt.alloc(cap));
            CK(M.snp.alloc(cap));
            CK(M.spartner.alloc((size_t)M.maxt * cap));
            CK(M.shist.alloc((size_t)3 * M.maxt * cap));
            CK(M.tlist.alloc((size_t)M.maxt * cap));
            CK(cudaMemsetAsync(M.tcnt.p, 0, sizeof(int) * cap, c->st));
            CK(cudaMemsetAsync(M.snp.p, 0, sizeof(int) * cap, c->st));
            CK(cudaMemsetAsync(M.spartner.p, 0xff, sizeof(int) * M.maxt * cap, c->st));
            CK(cudaMemsetAsync(M.shist.p, 0, sizeof(double) * 3 * M.maxt * cap, c->st));
        }
    }
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

int gb2_add_insert_pack(gb2_ctx *c, const gb2_insert_pack *p)
{
    if (!c || !p) return GB2_ERR_ARG;
    if (!c->have_atoms) return set_err(c, GB2_ERR_STATE, "upload atoms before adding fixes");
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "fixes must be added before setup");
    if (c->ins || c->stream) return set_err(c, GB2_ERR_UNSUPPORTED, "one insertion fix per context");
    InsertPack *I = new InsertPack();
    const std::string e = I->init(*p, c->P.boxlo, c->P.boxhi, c->P.ntypes, c->ntimestep);
    if (!e.empty()) {
        delete I;
        return set_err(c, GB2_ERR_ARG, "fix insert/pack: %s", e.c_str());
    }
    if (p->max_atoms < c->nlocal) {
        delete I;
        return set_err(c, GB2_ERR_ARG, "fix insert/pack: max_atoms below the current atom count");
    }
    const int rc = reserve_cap(c, p->max_atoms);
    if (rc) {
        delete I;
        return rc;
    }
    c->ins = I;
    return 0;
}

int gb2_add_insert_stream(gb2_ctx *c, const gb2_insert_stream *p)
{
    if (!c || !p || p->nface <= 0 || !p->face_nodes) return GB2_ERR_ARG;
    if (!c->have_atoms) return set_err(c, GB2_ERR_STATE, "upload atoms before adding fixes");
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "fixes must be added before setup");
    if (c->ins || c->stream) return set_err(c, GB2_ERR_UNSUPPORTED, "one insertion fix per context");
    // the insertion face as fix mesh/surface reads it (element geometry only)
    MeshTopo topo;
    std::string err;
    if (!build_mesh_topology(p->face_nodes, p->nface, 0.0, 1e-8, topo, err))
        return set_err(c, GB2_ERR_ARG, "fix insert/stream face: %s", err.c_str());
    InsertStream *I = new InsertStream();
    const std::string e = I->init(*p, topo.tri, c->P.boxlo, c->P.boxhi, c->P.ntypes, c->ntimestep, c->P.dt);
    if (!e.empty()) {
        delete I;
        return set_err(c, GB2_ERR_ARG, "fix insert/stream: %s", e.c_str());
    }
    if (p->max_atoms < c->nlocal) {
        delete I;
        return set_err(c, GB2_ERR_ARG, "fix insert/stream: max_atoms below the current atom count");
    }
    int rc = reserve_cap(c, p->max_atoms);
    if (!rc && (c->rel.alloc((size_t)4 * c->cap) != cudaSuccess || c->sface.alloc(I->face.size()) != cudaSuccess))
        rc = GB2_ERR_CUDA;
    if (rc) {
        delete I;
        return rc;
    }
    CK(cudaMemsetAsync(c->rel.p, 0, sizeof(dbl4) * 4 * c->cap, c->st));
    CK(cudaMemcpyAsync(c->sface.p, I->face.data(), sizeof(TriGeom) * I->face.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->stream = I;
    return 0;
}

int gb2_insert_stats(gb2_ctx *c, int ifix, long *ninserted, double *massinserted, long *next_step)
{
    if (!c || ifix != 0 || (!c->ins && !c->stream)) return GB2_ERR_ARG;
    if (c->stream) {
        if (ninserted) *ninserted = c->stream->ninserted;
        if (massinserted) *massinserted = c->stream->massinserted;
        if (next_step) *next_step = c->stream->next_reneighbor;
        return 0;
    }
    if (ninserted) *ninserted = c->ins->ninserted;
    if (massinserted) *massinserted = c->ins->massinserted;
    if (next_step) *next_step = c->ins->next_reneighbor;
    return 0;
}

int gb2_download_mesh_nodes(gb2_ctx *c, int ifix, int cap, int *ntri, double *nodes, double *vnode)
{
    if (!c || !ntri) return GB2_ERR_ARG;
    if (ifix < 0 || ifix >= c->nfix || !c->fix[ifix].mesh) return set_err(c, GB2_ERR_ARG, "not a mesh fix");
    MeshFix &M = *c->fix[ifix].mesh;
    const int n = (int)M.topo.tri.size();
    *ntri = n;
    if (cap < n) return 0;
    if (nodes) {
        std::vector<TriGeom> h(n);
        CK(cudaMemcpyAsync(h.data(), M.tri.p, sizeof(TriGeom) * n, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        for (int t = 0; t < n; t++)
            for (int j = 0; j < 3; j++)
                for (int d = 0; d < 3; d++) nodes[9 * t + 3 * j + d] = h[t].node[j][d];
    }
    if (vnode) {
        if (M.moving) {
            CK(cudaMemcpyAsync(vnode, M.vnode.p, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost, c->st));
            CK(cudaStreamSynchronize(c->st));
        } else {
            std::memset(vnode, 0, sizeof(double) * 9 * n);
        }
    }
    return 0;
}

int gb2_set_timestep(gb2_ctx *c, long ntimestep)
{
    if (!c || ntimestep < 0) return GB2_ERR_ARG;
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "the start step is set before setup");
    c->ntimestep = ntimestep;
    return 0;
}

int gb2_setup(gb2_ctx *c)
{
    if (!c) return GB2_ERR_ARG;
    if (!c->have_mat || !c->have_atoms) return set_err(c, GB2_ERR_STATE, "materials and atoms are required before setup");
    c->err.clear();
    neighbor_init(c);
    if (c->P.sort_freq > 0) {
        // Atom::setup_sort_bins (src/atom.cpp:1405)
        const double binsize = c->P.sort_binsize > 0.0 ? c->P.sort_binsize : 0.5 * c->cutneighmax;
        const double bininv = 1.0 / binsize;
        for (int d = 0; d < 3; d++) {
            c->slo[d] = c->P.boxlo[d];
            c->snb[d] = static_cast<int>((c->P.boxhi[d] - c->P.boxlo[d]) * bininv);
            if (c->snb[d] == 0) c->snb[d] = 1;
            c->sinv[d] = c->snb[d] / (c->P.boxhi[d] - c->P.boxlo[d]);
        }
    }
    if (setup_bins(c)) return GB2_ERR_ARG;
    // Verlet::setup: setup_pre_exchange, pbc, exchange, sort (always), borders,
    // neighbor build, setup_pre_force, pair (shearupdate 0), fix setup
    int rc = do_rebuild(c, c->computeflag, c->P.sort_freq > 0, false, false);
    if (rc) return rc;
    if (do_force(c, 0, 0, 0, 1)) return GB2_ERR_CUDA;
    CK(cudaStreamSynchronize(c->st));
    if (adapt_item_cap(c)) return GB2_ERR_CUDA;
    if (c->ins) {   // FixInsert::setup: region volume by Monte Carlo
        const std::string e = c->ins->setup();
        if (!e.empty()) return set_err(c, GB2_ERR_ARG, "fix insert/pack: %s", e.c_str());
    }
    if (c->stream) {   // FixInsert::setup: FixInsertStream::calc_insertion_properties
        const std::string e = c->stream->setup();
        if (!e.empty()) return set_err(c, GB2_ERR_ARG, "fix insert/stream: %s", e.c_str());
    }
    c->setup_done = true;
    c->computeflag = true;
    return 0;
}

// fix insert/pack on an insertion step, after the rebuild's history packing
// (the contact-history fixes run first in Modify::pre_exchange): the device
// selects the owned particles in the region and the particles near it, the
// host places new particles, and they are appended after the owned ones, in
// the first ghost slots.  ghosts_prev: the previous step's ghost positions
// are in pos2 (the step's integration was fused into the previous pair step
// and swapped the buffers).
static int append_inserted(gb2_ctx *c, const std::vector<InsertedParticle> &out, const char *who);

static int do_insert(gb2_ctx *c, bool ghosts_prev)
{
    InsertPack &I = *c->ins;
    const int nl = c->nlocal, nall = c->nlocal + c->nghost;
    const dbl4 *gpos = ghosts_prev ? c->pos2.p : c->pos.p;
    std::vector<double> rr, rm;
    std::vector<NearParticle> nearp;
    if (nall > 0) {
        CK(c->insflag.alloc(2 * (size_t)nall));
        CK(c->insidx.alloc(2 * (size_t)nall + 2));
        k_ins_flags<<<nblk(nall), kBlock, 0, c->st>>>(c->pos.p, gpos, nl, nall, I.R, c->insflag.p,
                                                      c->insflag.p + nall);
        CKL();
        thrust::counting_iterator<int> it(0);
        size_t bytes = 0;
        cub::DeviceSelect::Flagged(nullptr, bytes, it, c->insflag.p, c->insidx.p, c->insidx.p + 2 * nall, nall, c->st);
        if (cub_tmp(c, bytes)) return GB2_ERR_CUDA;
        for (int w = 0; w < 2; w++) {
            bytes = c->cubtmp.n;
            CK(cub::DeviceSelect::Flagged(c->cubtmp.p, bytes, it, c->insflag.p + (size_t)w * nall,
                                          c->insidx.p + (size_t)w * nall, c->insidx.p + 2 * nall + w, nall, c->st));
        }
        int cnt[2] = {0, 0};
        CK(cudaMemcpyAsync(cnt, c->insidx.p + 2 * nall, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        const int ntot = cnt[0] + cnt[1];
        if (ntot > 0) {
            CK(c->insrec.alloc(ntot));
            k_ins_gather<<<nblk(ntot), kBlock, 0, c->st>>>(c->pos.p, c->vel.p, gpos, nl, c->insidx.p, cnt[0],
                                                           c->insidx.p + nall, cnt[1], c->insrec.p);
            CKL();
            std::vector<dbl4> rec(ntot);
            CK(cudaMemcpyAsync(rec.data(), c->insrec.p, sizeof(dbl4) * ntot, cudaMemcpyDeviceToHost, c->st));
            CK(cudaStreamSynchronize(c->st));
            rr.resize(cnt[0]);
            rm.resize(cnt[0]);
            for (int k = 0; k < cnt[0]; k++) {
                rr[k] = rec[k].x;
                rm[k] = rec[k].y;
            }
            nearp.resize(cnt[1]);
            for (int k = 0; k < cnt[1]; k++) {
                const dbl4 &q = rec[cnt[0] + k];
                nearp[k] = NearParticle{{q.x, q.y, q.z}, q.w};
            }
        }
    }
    std::vector<InsertedParticle> out;
    const std::string e = I.insert(c->ntimestep, rr, rm, std::move(nearp), out);
    if (!e.empty()) return set_err(c, GB2_ERR_STATE, "fix insert/pack: %s", e.c_str());
    return append_inserted(c, out, "fix insert/pack");
}

// The accepted particles appended after the owned ones (tags after the
// largest, Atom::tag_extend), over the first ghost slots as create_atom does;
// lists, partners and wall histories of the new atoms start empty.
static int append_inserted(gb2_ctx *c, const std::vector<InsertedParticle> &out, const char *who)
{
    const int nl = c->nlocal, nall = c->nlocal + c->nghost;
    const int k = (int)out.size();
    if (k == 0) return 0;
    if (nl + k > c->cap)
        return set_err(c, GB2_ERR_CAPACITY, "%s: %d atoms exceed the %d reserved (max_atoms)", who, nl + k, c->cap);
    if ((long)c->maxtag + k > 0x7fffffffL) return set_err(c, GB2_ERR_CAPACITY, "atom tags beyond INT_MAX");
    // Atom::tag_extend: tags beyond the largest one, in insertion order
    std::vector<dbl4> hp(k), hv(k), hw(k);
    std::vector<int> ht(k), hg(k);
    for (int q = 0; q < k; q++) {
        const InsertedParticle &a = out[q];
        hp[q] = {a.x[0], a.x[1], a.x[2], a.radius};
        hv[q] = {a.v[0], a.v[1], a.v[2], a.mass};
        hw[q] = {a.omega[0], a.omega[1], a.omega[2], 0.0};
        ht[q] = a.type;
        hg[q] = (int)(c->maxtag + 1 + q);
    }
    // device capacity and copies first; the host mirrors change only once the
    // device holds the new atoms
    if (ensure_nmax(c, nall > nl + k ? nall : nl + k)) return GB2_ERR_CUDA;
    CK(cudaMemcpyAsync(c->pos.p + nl, hp.data(), sizeof(dbl4) * k, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->vel.p + nl, hv.data(), sizeof(dbl4) * k, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->omg.p + nl, hw.data(), sizeof(dbl4) * k, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->type.p + nl, ht.data(), sizeof(int) * k, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->tag.p + nl, hg.data(), sizeof(int) * k, cudaMemcpyHostToDevice, c->st));
    // new atoms start with no list entries, partners or wall history
    CK(cudaMemsetAsync(c->nnum.p + nl, 0, sizeof(int) * k, c->st));
    CK(cudaMemsetAsync(c->rnum.p + nl, 0, sizeof(int) * k, c->st));
    CK(cudaMemsetAsync(c->pnum.p + nl, 0, sizeof(int) * k, c->st));
    CK(cudaMemsetAsync(c->f.p + nl, 0, sizeof(dbl4) * k, c->st));
    CK(cudaMemsetAsync(c->tq.p + nl, 0, sizeof(dbl4) * k, c->st));
    for (int q = 0; q < c->nfix; q++) {
        HostFix &H = c->fix[q];
        if (H.kind == FIX_WALL_PLANE) {
            CK(cudaMemsetAsync(H.inlist.p + nl, 0, k, c->st));
            for (int d = 0; d < 3; d++)
                CK(cudaMemsetAsync(H.whist.p + (size_t)d * c->cap + nl, 0, sizeof(double) * k, c->st));
        }
        if (H.mesh) {
            CK(cudaMemsetAsync(H.mesh->tcnt.p + nl, 0, sizeof(int) * k, c->st));
            CK(cudaMemsetAsync(H.mesh->snp.p + nl, 0, sizeof(int) * k, c->st));
        }
    }
    CK(cudaStreamSynchronize(c->st));
    for (int q = 0; q < k; q++) c->h_maxrad[out[q].type] = std::max(c->h_maxrad[out[q].type], out[q].radius);
    c->maxtag += k;
    c->nlocal = nl + k;
    return 0;
}

// fix insert/stream on an insertion step, at the same place as insert/pack:
// the near list (FixInsertStream::is_nearby) selected on the device, the
// placement on the host, the new atoms appended with their release data
static int do_insert_stream(gb2_ctx *c, bool ghosts_prev)
{
    InsertStream &I = *c->stream;
    const int nl = c->nlocal, nall = c->nlocal + c->nghost;
    const dbl4 *gpos = ghosts_prev ? c->pos2.p : c->pos.p;
    std::vector<NearParticle> nearp;
    if (nall > 0 && I.S.overlapcheck) {
        CK(c->insflag.alloc((size_t)nall));
        CK(c->insidx.alloc((size_t)nall + 1));
        StreamNear SN;
        for (int d = 0; d < 3; d++) {
            SN.p_ref[d] = I.p_ref[d];
            SN.n[d] = I.normalvec[d];
            SN.bblo[d] = I.bblo[d];
            SN.bbhi[d] = I.bbhi[d];
        }
        SN.maxrad = I.maxrad;
        SN.extrude_length = I.extrude_length;
        SN.nface = (int)I.face.size();
        k_ins_near_stream<<<nblk(nall), kBlock, 0, c->st>>>(c->pos.p, gpos, nl, nall, SN, c->sface.p, c->insflag.p);
        CKL();
        thrust::counting_iterator<int> it(0);
        size_t bytes = 0;
        cub::DeviceSelect::Flagged(nullptr, bytes, it, c->insflag.p, c->insidx.p, c->insidx.p + nall, nall, c->st);
        if (cub_tmp(c, bytes)) return GB2_ERR_CUDA;
        bytes = c->cubtmp.n;
        CK(cub::DeviceSelect::Flagged(c->cubtmp.p, bytes, it, c->insflag.p, c->insidx.p, c->insidx.p + nall, nall,
                                      c->st));
        int cnt = 0;
        CK(cudaMemcpyAsync(&cnt, c->insidx.p + nall, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        if (cnt > 0) {
            CK(c->insrec.alloc(cnt));
            k_ins_gather<<<nblk(cnt), kBlock, 0, c->st>>>(c->pos.p, c->vel.p, gpos, nl, nullptr, 0, c->insidx.p, cnt,
                                                          c->insrec.p);
            CKL();
            std::vector<dbl4> rec(cnt);
            CK(cudaMemcpyAsync(rec.data(), c->insrec.p, sizeof(dbl4) * cnt, cudaMemcpyDeviceToHost, c->st));
            CK(cudaStreamSynchronize(c->st));
            nearp.resize(cnt);
            for (int k = 0; k < cnt; k++) nearp[k] = NearParticle{{rec[k].x, rec[k].y, rec[k].z}, rec[k].w};
        }
    }
    std::vector<InsertedParticle> out;
    std::vector<StreamRelease> rel;
    const std::string e = I.insert(c->ntimestep, std::move(nearp), out, rel);
    if (!e.empty()) return set_err(c, GB2_ERR_STATE, "fix insert/stream: %s", e.c_str());
    const int rc = append_inserted(c, out, "fix insert/stream");
    if (rc) return rc;
    const int k = (int)rel.size();
    if (k > 0) {   // release data of the new atoms (release_fix_insert_stream)
        std::vector<dbl4> h((size_t)4 * k);
        for (int q = 0; q < k; q++) {
            const StreamRelease &r = rel[q];
            h[q] = dbl4{r.x[0], r.x[1], r.x[2], r.istep};
            h[k + q] = dbl4{r.vint[0], r.vint[1], r.vint[2], r.rstep};
            h[2 * k + q] = dbl4{r.vrel[0], r.vrel[1], r.vrel[2], 0.0};
            h[3 * k + q] = dbl4{r.wrel[0], r.wrel[1], r.wrel[2], 0.0};
        }
        for (int sl = 0; sl < 4; sl++)
            CK(cudaMemcpyAsync(c->rel.p + (size_t)sl * c->cap + nl, h.data() + (size_t)sl * k, sizeof(dbl4) * k,
                               cudaMemcpyHostToDevice, c->st));
        CK(cudaStreamSynchronize(c->st));
    }
    return 0;
}

// an insertion fix inserts on this step
static bool ins_due(const gb2_ctx *c, long step)
{
    return (c->ins && c->ins->due(step)) || (c->stream && c->stream->due(step));
}

// One Verlet step.  mode 0: the rebuild decision from the device flags
// (one host synchronisation); mode 1: a rebuild requested by a queued step;
// mode 2: queued ahead of the decision (no rebuild, no synchronisation).
static int one_step(gb2_ctx *c, bool last, int mode)
{
    const bool ghosts_prev = c->fused_pending;
    c->ntimestep++;
    c->ago++;
    const bool decide = c->ago >= c->P.neigh_delay && c->ago % c->P.neigh_every == 0;
    const bool check = decide && c->P.neigh_check && mode == 0;
    gb2_ctx::EvPair e;
    if (!c->fused_pending) {
        // first step of this run: initial_integrate as its own kernel (later
        // steps get it fused into the previous step's pair step)
        if (check) CK(cudaMemsetAsync(c->ddflag.p, 0, sizeof(int), c->st));
        Dev D = make_dev(c);
        if (prof_begin(c, PROF_INTEGRATE, &e)) return GB2_ERR_CUDA;
        k_initial_integrate<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D, check ? 1 : 0);
        CKL();
        if (prof_end(c, &e)) return GB2_ERR_CUDA;
    }
    // fix move/mesh: rotate moving meshes (initial_integrate) and test
    // their displacement since the last rebuild
    bool moving = false, forced = mode == 1;
    for (int k = 0; k < c->nfix; k++) {
        MeshFix *M = c->fix[k].mesh;
        if (!M || !M->moving) continue;
        if (!moving) CK(cudaMemsetAsync(c->ddflag.p + 1, 0, sizeof(int), c->st));
        moving = true;
        if (M->next_reneighbor == c->ntimestep) forced = true;   // Neighbor::decide must_check
        const int nt = (int)M->topo.tri.size();
        if (M->mover == 2) {
            const double dt = c->P.dt;
            k_mesh_translate<<<nblk(nt), kBlock, 0, c->st>>>(M->tri.p, nt, M->vnode.p, M->node_last.p,
                                                             M->mv_vel[0] * dt, M->mv_vel[1] * dt, M->mv_vel[2] * dt,
                                                             M->mv_vel[0], M->mv_vel[1], M->mv_vel[2],
                                                             0.25 * c->P.skin * c->P.skin, c->ddflag.p + 1);
        } else {
            MeshRotate mv;
            mesh_rotation(c, *M, mv);
            k_mesh_rotate<<<nblk(nt), kBlock, 0, c->st>>>(M->tri.p, nt, M->vnode.p, M->node_last.p, mv,
                                                          c->ddflag.p + 1);
        }
        CKL();
    }
    // fix insert/pack: its next_reneighbor forces the rebuild (Neighbor::decide must_check)
    const bool insert_now = ins_due(c, c->ntimestep);
    if (insert_now) forced = true;
    bool rebuild = decide && !c->P.neigh_check && mode != 2;
    bool mesh_far = false;
    if (check || (moving && mode != 2)) {
        CK(cudaMemcpyAsync(&c->h_pinned[4], c->ddflag.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        if (check) rebuild = c->h_pinned[4] != 0;
        mesh_far = moving && c->h_pinned[5] != 0;
        if (c->prof) prof_resolve(c);
    }
    if (forced) rebuild = true;
    if (!rebuild && mesh_far)   // FixMesh::pre_force on a regular step (src/fix_mesh.cpp:577-583)
        for (int k = 0; k < c->nfix; k++)
            if (c->fix[k].mesh && c->fix[k].mesh->moving) c->fix[k].mesh->next_reneighbor = c->ntimestep + 1;
    if (rebuild) {
        const bool sort_now = c->P.sort_freq > 0 && c->ntimestep >= c->nextsort;
        if (prof_begin(c, PROF_REBUILD, &e)) return GB2_ERR_CUDA;
        int rc = do_rebuild(c, true, sort_now, insert_now, ghosts_prev);
        if (rc) return rc;
        if (adapt_item_cap(c)) return GB2_ERR_CUDA;
        if (prof_end(c, &e)) return GB2_ERR_CUDA;
        c->nsteps_rebuild++;
    } else if (c->nghost > 0) {
        Dev D = make_dev(c);
        if (prof_begin(c, PROF_FORWARD, &e)) return GB2_ERR_CUDA;
        k_forward_comm<<<nblk(c->nghost), kBlock, 0, c->st>>>(D);
        CKL();
        if (prof_end(c, &e)) return GB2_ERR_CUDA;
    }
    return do_force(c, 1, 1, last ? 0 : 1, last ? 1 : 0);
}

// Undo the host side of a queued step whose kernels returned at once (an
// earlier step asked for a rebuild): the step counters, the buffer swaps of
// do_force and its profiling events.
static void unqueue_step(gb2_ctx *c, bool last, size_t nev)
{
    c->ntimestep--;
    c->ago--;
    c->hist.swap(c->hist2);
    c->vel.swap(c->vel2);
    c->omg.swap(c->omg2);
    if (c->split) c->kin.swap(c->kin2);
    if (!last) c->pos.swap(c->pos2);
    c->fused_pending = true;
    while (c->ev_pending.size() > nev) {
        c->ev_free.push_back(c->ev_pending.back());
        c->ev_pending.pop_back();
    }
}

int gb2_run(gb2_ctx *c, int nsteps)
{
    if (!c) return GB2_ERR_ARG;
    if (!c->setup_done) return set_err(c, GB2_ERR_STATE, "gb2_setup must precede gb2_run");
    // Steps are queued up to queue_depth ahead of the rebuild decision when
    // it can only come from the displacement test (neigh_modify every 1
    // delay 0 check yes, no moving mesh): each queued step's kernels return
    // at once if an earlier step's tail found a displacement beyond skin/2
    // (device word dstop = lowest such step).  The host confirms steps in
    // order from per-step copies of dstop; at the first step that asked, it
    // undoes the queued successors, rebuilds and continues.  Device results
    // are those of the one-step-at-a-time loop; the GPU no longer idles
    // while the host reads the flag every step.
    bool queueable = c->queue_ok && c->P.neigh_check && c->P.neigh_every == 1 && c->P.neigh_delay == 0;
    for (int k = 0; k < c->nfix; k++)
        if (c->fix[k].mesh && c->fix[k].mesh->moving) queueable = false;
    int s = 0;
    while (s < nsteps) {
        if (!queueable || !c->fused_pending || ins_due(c, c->ntimestep + 1)) {
            int rc = one_step(c, s == nsteps - 1, 0);
            if (rc) return rc;
            s++;
            continue;
        }
        // the step just run (not queued) may have asked for a rebuild of the next
        k_queue_start<<<1, 1, 0, c->st>>>(c->dstop.p, c->ddflag.p, (int)c->ntimestep);
        CKL();
        c->queue_active = true;
        struct Queued {
            long ntimestep;
            bool last;
            size_t nev;
        };
        Queued q[16];
        int head = s, launched = s;
        bool stop = false;
        for (;;) {
            // an insertion step is never queued (it rebuilds unconditionally)
            while (launched < nsteps && launched - head < c->queue_depth &&
                   !ins_due(c, c->ntimestep + 1)) {
                Queued &Q = q[launched % 16];
                Q.last = launched == nsteps - 1;
                Q.nev = c->ev_pending.size();
                int rc = one_step(c, Q.last, 2);
                if (rc) {
                    c->queue_active = false;
                    return rc;
                }
                Q.ntimestep = c->ntimestep;
                cudaEvent_t &ev = c->qev[launched % 16];
                if (!ev) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
                CK(cudaMemcpyAsync(&c->h_stop[launched % 16], c->dstop.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
                CK(cudaEventRecord(ev, c->st));
                launched++;
            }
            if (head == launched) break;
            CK(cudaEventSynchronize(c->qev[head % 16]));
            const int v = c->h_stop[head % 16];
            if (v == 0x7f7f7f7f || (long)v > q[head % 16].ntimestep) {
                head++;
                continue;
            }
            // step v asked for a rebuild of step v + 1: v is `head`, or the step
            // run just before the queue (then `head` itself did nothing); the
            // queued steps after v did nothing
            const int first = (long)v < q[head % 16].ntimestep ? head : head + 1;
            for (int r = launched - 1; r >= first; r--) unqueue_step(c, q[r % 16].last, q[r % 16].nev);
            launched = first;
            stop = true;
            break;
        }
        c->queue_active = false;
        s = launched;
        if (stop && s < nsteps) {
            int rc = one_step(c, s == nsteps - 1, 1);
            if (rc) return rc;
            s++;
        }
    }
    int st;
    if (read_status(c, &st)) return GB2_ERR_CUDA;
    if (c->prof) prof_resolve(c);
    if (st & ST_MESH_INTERNAL) return set_err(c, GB2_ERR_STATE, "mesh contact history inconsistent");
    return 0;
}

int gb2_set_profiling(gb2_ctx *c, int on)
{
    if (!c) return GB2_ERR_ARG;
    CK(cudaStreamSynchronize(c->st));
    prof_resolve(c);
    c->prof = on > 0;
    c->prof_every = on > 1 ? on : 1;
    return 0;
}

int gb2_timer_start(gb2_ctx *c)
{
    if (!c) return GB2_ERR_ARG;
    CK(cudaEventRecord(c->ev0, c->st));
    return 0;
}

int gb2_timer_stop(gb2_ctx *c, double *ms)
{
    if (!c || !ms) return GB2_ERR_ARG;
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaEventSynchronize(c->ev1));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, c->ev0, c->ev1));
    *ms = f;
    return 0;
}

int gb2_census(gb2_ctx *c, gb2_contact_census *out)
{
    if (!c || !out) return GB2_ERR_ARG;
    if (!c->setup_done) return set_err(c, GB2_ERR_STATE, "census needs a neighbor list (call gb2_setup)");
    if (c->nlocal == 0) {   // no atoms: nothing to launch
        *out = gb2_contact_census{};
        return 0;
    }
    DBuf<unsigned long long> cnt;
    CK(cnt.alloc(8));
    CK(cudaMemsetAsync(cnt.p, 0, 8 * sizeof(unsigned long long), c->st));
    Dev D = make_dev(c);
    k_census<<<nblk(c->nlocal), kBlock, 0, c->st>>>(D, cnt.p);
    CKL();
    unsigned long long h[8];
    CK(cudaMemcpyAsync(h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    out->nlist = (long)h[0];
    out->ntouch = (long)h[1];
    out->nrev = (long)h[2];
    out->nwall_list = (long)h[3];
    out->nwall_touch = (long)h[4];
    out->nmesh_cand = (long)h[5];
    out->nmesh_touch = (long)h[6];
    return 0;
}

int gb2_census_noalloc(gb2_ctx *c, gb2_contact_census *out)
{
    if (!c || !out) return GB2_ERR_ARG;
    if (!c->setup_done) return set_err(c, GB2_ERR_STATE, "census needs a neighbor list (call gb2_setup)");
    if (c->nlocal == 0) {   // no atoms: nothing to launch
        *out = gb2_contact_census{};
        return 0;
    }
    const int nblocks = nblk(c->nlocal, 128);
    if (nblocks > GB2_NOALLOC_MAX_BLOCKS)
        return set_err(c, GB2_ERR_CAPACITY,
                       "gb2_census_noalloc serves at most %d owned atoms (static scratch); this context has %d",
                       GB2_NOALLOC_MAX_ATOMS, c->nlocal);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_err(c, GB2_ERR_ARG, "device ordinal %d out of range", dev);
    if (!g_noalloc_ptr[dev]) {
        // first call on this device (the device is current): resolve the
        // host-side stand-in symbol to its device address
        unsigned long long *p = nullptr;
        CK(cudaGetSymbolAddress((void **)&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = p;
    }
    unsigned long long *rows = g_noalloc_ptr[dev];
    Dev D = make_dev(c);
    k_census_rows<<<nblocks, 128, 0, c->st>>>(D, rows);
    CKL();
    k_census_total<<<1, 256, 0, c->st>>>(rows, nblocks);
    CKL();
    unsigned long long h[8];
    CK(cudaMemcpyAsync(h, rows + (size_t)GB2_NOALLOC_MAX_BLOCKS * 8, sizeof h, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    out->nlist = (long)h[0];
    out->ntouch = (long)h[1];
    out->nrev = (long)h[2];
    out->nwall_list = (long)h[3];
    out->nwall_touch = (long)h[4];
    out->nmesh_cand = (long)h[5];
    out->nmesh_touch = (long)h[6];
    return 0;
}

int gb2_sync(gb2_ctx *c)
{
    if (!c) return GB2_ERR_ARG;
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

int gb2_download_atoms(gb2_ctx *c, int cap, int *n, double *x, double *v, double *omega, double *f, double *torque,
                       int *tag)
{
    if (!c) return GB2_ERR_ARG;
    if (n) *n = c->nlocal;
    const int m = std::min(cap, c->nlocal);
    if (m <= 0) return 0;
    // the five [m][3] planes unpacked on the device into one block, one
    // device-to-host copy per requested array (straight into the caller's
    // memory when it is pinned, else through the pinned staging buffer)
    const size_t M = (size_t)m;
    CK(c->iostage.alloc(15 * M));
    k_unpack_atoms<<<nblk(m), kBlock, 0, c->st>>>(c->pos.p, c->vel.p, c->omg.p, c->f.p, c->tq.p, m, c->iostage.p);
    CKL();
    double *dst[5] = {x, v, omega, f, torque};
    bool pageable = false;
    for (int k = 0; k < 5; k++) pageable = pageable || (dst[k] && !host_pinned(dst[k]));
    if (pageable && host_stage(c, 15 * M * sizeof(double))) return GB2_ERR_CUDA;
    bool staged[5] = {false, false, false, false, false};
    for (int k = 0; k < 5; k++) {
        if (!dst[k]) continue;
        const size_t bytes = 3 * M * sizeof(double);
        if (host_pinned(dst[k])) {
            CK(cudaMemcpyAsync(dst[k], c->iostage.p + 3 * M * k, bytes, cudaMemcpyDeviceToHost, c->st));
        } else {
            CK(cudaMemcpyAsync((double *)c->hstage + 3 * M * k, c->iostage.p + 3 * M * k, bytes,
                               cudaMemcpyDeviceToHost, c->st));
            staged[k] = true;
        }
    }
    if (tag) CK(cudaMemcpyAsync(tag, c->tag.p, sizeof(int) * m, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int k = 0; k < 5; k++)
        if (staged[k]) host_copy(dst[k], (double *)c->hstage + 3 * M * k, 3 * M * sizeof(double));
    return 0;
}

int gb2_host_alloc(size_t bytes, void **ptr)
{
    if (!ptr) return GB2_ERR_ARG;
    *ptr = nullptr;
    if (cudaHostAlloc(ptr, std::max<size_t>(bytes, 1), cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        return GB2_ERR_CUDA;
    }
    return 0;
}

int gb2_host_free(void *ptr)
{
    if (ptr && cudaFreeHost(ptr) != cudaSuccess) {
        cudaGetLastError();
        return GB2_ERR_CUDA;
    }
    return 0;
}

int gb2_download_pairs(gb2_ctx *c, int cap, int *n, int *tag_i, int *tag_j, int *flag, double *hist)
{
    if (!c) return GB2_ERR_ARG;
    if (!c->setup_done) return set_err(c, GB2_ERR_STATE, "no neighbor list before setup");
    const size_t cp = c->cap;
    const int nl = c->nlocal;
    std::vector<int> nnum(nl), nbr((size_t)c->maxn * cp), fl((size_t)c->maxn * cp), tg(c->nlocal + c->nghost);
    std::vector<double> h((size_t)3 * c->maxn * cp);
    CK(cudaMemcpyAsync(nnum.data(), c->nnum.p, sizeof(int) * nl, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(nbr.data(), c->nbr.p, sizeof(int) * nbr.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(fl.data(), c->flag.p, sizeof(int) * fl.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(h.data(), c->hist.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(tg.data(), c->tag.p, sizeof(int) * tg.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int k = 0;
    for (int i = 0; i < nl; i++)
        for (int s = 0; s < nnum[i]; s++) {
            const size_t e = (size_t)s * cp + i;
            if (k < cap) {
                if (tag_i) tag_i[k] = tg[i];
                if (tag_j) tag_j[k] = tg[nbr[e]];
                if (flag) flag[k] = fl[e];
                if (hist)
                    for (int q = 0; q < 3; q++) hist[3 * k + q] = h[(size_t)(3 * s + q) * cp + i];
            }
            k++;
        }
    if (n) *n = k;
    c->npairs_last = k;
    return 0;
}

int gb2_contact_atom(gb2_ctx *c, int cap, int *n, int *tag, double *contact)
{
    if (!c) return GB2_ERR_ARG;
    if (!c->setup_done) return set_err(c, GB2_ERR_STATE, "no neighbor list before setup");
    const int nl = c->nlocal;
    if (n) *n = nl;
    if (!contact || cap < nl) return 0;
    DBuf<double> d;
    CK(d.alloc(nl > 0 ? nl : 1));
    if (nl > 0) {
        Dev D = make_dev(c);
        k_contact_atom<<<nblk(nl), kBlock, 0, c->st>>>(D, d.p);
        CKL();
        CK(cudaMemcpyAsync(contact, d.p, sizeof(double) * nl, cudaMemcpyDeviceToHost, c->st));
        if (tag) CK(cudaMemcpyAsync(tag, c->tag.p, sizeof(int) * nl, cudaMemcpyDeviceToHost, c->st));
    }
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

// columns of a pair/gran/local row for a keyword mask
static int pgl_ncols(unsigned keys)
{
    static const int width[13] = {6, 6, 3, 3, 3, 3, 3, 3, 3, 3, 1, 1, 3};
    int n = 0;
    for (int b = 0; b < 13; b++)
        if (keys & (1u << b)) n += width[b];
    return n;
}

// compute pair/gran/local on the device: one row per touching pair in list
// order with the columns keys selects
int gb2_pair_gran_local_keys(gb2_ctx *c, unsigned keys, int cap, int *nrows, int *ncols, double *rows)
{
    if (!c || !nrows || keys == 0 || (keys & ~GB2_PGL_ALL)) return GB2_ERR_ARG;
    if (!c->setup_done) return set_err(c, GB2_ERR_STATE, "no neighbor list before setup");
    const int nc = pgl_ncols(keys);
    if (ncols) *ncols = nc;
    const int nl = c->nlocal;
    DBuf<int> cnt, off;
    CK(cnt.alloc(nl + 1));
    CK(off.alloc(nl + 1));
    CK(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (nl + 1), c->st));
    if (c->ghost_v_prev && c->nghost > 0) {
        // ghosts carry the velocities forwarded at the last step's start, as
        // in the reference between steps
        const size_t g0 = (size_t)c->nlocal, ng = (size_t)c->nghost;
        CK(cudaMemcpyAsync(c->vel.p + g0, c->vel2.p + g0, sizeof(dbl4) * ng, cudaMemcpyDeviceToDevice, c->st));
        CK(cudaMemcpyAsync(c->omg.p + g0, c->omg2.p + g0, sizeof(dbl4) * ng, cudaMemcpyDeviceToDevice, c->st));
        c->ghost_v_prev = false;
    }
    Dev D = make_dev(c);
    if (nl > 0) {
        k_pgl_count<<<nblk(nl), kBlock, 0, c->st>>>(D, cnt.p);
        CKL();
    }
    size_t tmp = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt.p, off.p, nl + 1, c->st));
    if (cub_tmp(c, tmp)) return GB2_ERR_CUDA;
    CK(cub::DeviceScan::ExclusiveSum(c->cubtmp.p, tmp, cnt.p, off.p, nl + 1, c->st));
    int total = 0;
    CK(cudaMemcpyAsync(&total, off.p + nl, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    *nrows = total;
    if (!rows || cap < total || total == 0) return 0;
    PglBox B;
    for (int d = 0; d < 3; d++) {
        B.lo[d] = c->P.boxlo[d];
        B.hi[d] = c->P.boxhi[d];
        B.periodic[d] = c->P.periodic[d];
    }
    DBuf<double> d;
    CK(d.alloc((size_t)nc * total));
    k_pgl_rows<<<nblk(nl), kBlock, 0, c->st>>>(D, off.p, d.p, B, keys, nc);
    CKL();
    CK(cudaMemcpyAsync(rows, d.p, sizeof(double) * nc * total, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

// compute pair/gran/local id force torque history: rows of 12 doubles
// (tag_i, tag_j, periodic, f_i[3], torque_i[3], history[3])
int gb2_pair_gran_local(gb2_ctx *c, int cap, int *nrows, double *rows)
{
    return gb2_pair_gran_local_keys(c, GB2_PGL_ID | GB2_PGL_FORCE | GB2_PGL_TORQUE | GB2_PGL_HISTORY, cap, nrows,
                                    nullptr, rows);
}

// fix mesh/surface/stress on mesh wall fix ifix (before setup): per-element
// force and the totals about p_ref accumulated from the wall contacts of each
// step (MeshModuleStress::add_particle_contribution, src/mesh_module_stress.cpp:276)
int gb2_add_mesh_stress(gb2_ctx *c, int ifix, const double p_ref[3])
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_MESH || !p_ref) return GB2_ERR_ARG;
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "mesh/surface/stress is added before setup");
    MeshFix &M = *c->fix[ifix].mesh;
    const int nt = (int)M.topo.tri.size();
    std::vector<double> area(std::max(nt, 1));
    for (int t = 0; t < nt; t++) {   // TriMesh::calcArea of the element as created
        const TriGeom &T0 = M.topo.tri[t];
        const double cx = T0.edgevec[0][1] * T0.edgevec[1][2] - T0.edgevec[0][2] * T0.edgevec[1][1];
        const double cy = T0.edgevec[0][2] * T0.edgevec[1][0] - T0.edgevec[0][0] * T0.edgevec[1][2];
        const double cz = T0.edgevec[0][0] * T0.edgevec[1][1] - T0.edgevec[0][1] * T0.edgevec[1][0];
        area[t] = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz) * T0.edgelen[0] * T0.edgelen[1];
    }
    CK(M.trif.alloc((size_t)3 * std::max<size_t>(M.topo.tri.size(), 1)));
    CK(M.ftot.alloc(6));
    CK(M.tarea.alloc(std::max(nt, 1)));
    CK(cudaMemsetAsync(M.trif.p, 0, sizeof(double) * 3 * M.topo.tri.size(), c->st));
    CK(cudaMemsetAsync(M.ftot.p, 0, sizeof(double) * 6, c->st));
    CK(cudaMemcpyAsync(M.tarea.p, area.data(), sizeof(double) * area.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    M.stress = true;
    for (int d = 0; d < 3; d++) M.pref[d] = p_ref[d];
    return 0;
}

// mesh/surface/stress ... wear finnie on mesh wall fix ifix (after
// gb2_add_mesh_stress, before setup): k_finnie is the ntypes x ntypes
// peratomtypepair property (row-major); the wall's atom type picks the row
int gb2_add_mesh_wear(gb2_ctx *c, int ifix, const double *k_finnie)
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_MESH || !k_finnie) return GB2_ERR_ARG;
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "mesh wear is added before setup");
    MeshFix &M = *c->fix[ifix].mesh;
    if (!M.stress) return set_err(c, GB2_ERR_STATE, "wear needs mesh/surface/stress on this mesh");
    const int nt = (int)M.topo.tri.size(), ntypes = c->P.ntypes;
    const int wt = c->fix[ifix].wtype;
    if (wt < 1 || wt > ntypes) return set_err(c, GB2_ERR_ARG, "wall atom type out of range");
    std::vector<double> kf(kMaxTypes + 1, 0.0);
    for (int j = 1; j <= ntypes; j++) kf[j] = k_finnie[(wt - 1) * ntypes + (j - 1)];
    CK(M.wear.alloc(std::max(nt, 1)));
    CK(M.kfin.alloc(kMaxTypes + 1));
    CK(cudaMemsetAsync(M.wear.p, 0, sizeof(double) * std::max(nt, 1), c->st));
    CK(cudaMemcpyAsync(M.kfin.p, kf.data(), sizeof(double) * kf.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

// cumulative Finnie wear per element (MeshModuleStress "wear")
int gb2_download_mesh_wear(gb2_ctx *c, int ifix, int cap, double *wear)
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_MESH || !wear) return GB2_ERR_ARG;
    MeshFix &M = *c->fix[ifix].mesh;
    if (!M.wear.p) return set_err(c, GB2_ERR_STATE, "wear not enabled on this mesh");
    const int nt = (int)M.topo.tri.size();
    if (cap < nt) return set_err(c, GB2_ERR_ARG, "wear needs %d entries", nt);
    CK(cudaMemcpyAsync(wear, M.wear.p, sizeof(double) * nt, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

// restart of the cumulative wear (MeshModuleStress registers "wear" as a
// restart property, src/mesh_module_stress.cpp:197): after gb2_add_mesh_wear,
// before setup
int gb2_upload_mesh_wear(gb2_ctx *c, int ifix, int n, const double *wear)
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_MESH || !wear) return GB2_ERR_ARG;
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "mesh wear is uploaded before setup");
    MeshFix &M = *c->fix[ifix].mesh;
    if (!M.wear.p) return set_err(c, GB2_ERR_STATE, "wear not enabled on this mesh");
    const int nt = (int)M.topo.tri.size();
    if (n != nt) return set_err(c, GB2_ERR_ARG, "wear needs %d entries, got %d", nt, n);
    CK(cudaMemcpyAsync(M.wear.p, wear, sizeof(double) * nt, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

// per-element force of the last step (3 per triangle), the element normal and
// shear stresses of MeshModuleStress::calc_total_force
// (src/mesh_module_stress.cpp:335-375: |f.n| / area and |f - (f.n) n| / area
// with the current normal and TriMesh::calcArea's area of the element,
// src/tri_mesh_I.h:305, as created and, for a moving mesh, as recomputed at
// its last rebuild), and f_total, torque_total
int gb2_download_mesh_stress(gb2_ctx *c, int ifix, int cap, double *tri_f, double *sigma_n, double *sigma_t,
                             double *tot6)
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_MESH) return GB2_ERR_ARG;
    MeshFix &M = *c->fix[ifix].mesh;
    if (!M.stress) return set_err(c, GB2_ERR_STATE, "mesh/surface/stress not enabled on this mesh");
    const int nt = (int)M.topo.tri.size();
    std::vector<double> f((size_t)3 * nt), area(std::max(nt, 1));
    std::vector<TriGeom> geo(nt);
    CK(cudaMemcpyAsync(f.data(), M.trif.p, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(geo.data(), M.tri.p, sizeof(TriGeom) * nt, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(area.data(), M.tarea.p, sizeof(double) * nt, cudaMemcpyDeviceToHost, c->st));
    if (tot6) CK(cudaMemcpyAsync(tot6, M.ftot.p, sizeof(double) * 6, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (cap < nt) return 0;
    for (int t = 0; t < nt; t++) {
        const double *fi = &f[3 * (size_t)t];
        if (tri_f)
            for (int k = 0; k < 3; k++) tri_f[3 * t + k] = fi[k];
        const double invSurfArea = 1. / area[t];
        const double *sn = geo[t].surfnorm;
        double sn_ = fi[0] * sn[0] + fi[1] * sn[1] + fi[2] * sn[2];
        const double tmp[3] = {fi[0] - sn[0] * sn_, fi[1] - sn[1] * sn_, fi[2] - sn[2] * sn_};
        double st_ = std::sqrt(tmp[0] * tmp[0] + tmp[1] * tmp[1] + tmp[2] * tmp[2]);
        sn_ = std::fabs(sn_);
        st_ = std::fabs(st_);
        if (sigma_n) sigma_n[t] = sn_ * invSurfArea;
        if (sigma_t) sigma_t[t] = st_ * invSurfArea;
    }
    return 0;
}

// Restart: the contact history in FixContactHistory's per-atom partner layout
// (src/fix_contact_history.cpp:588-640, pack_restart / unpack_restart): per
// atom its partner count, then each partner's tag and 3 shear values as seen
// from the atom.  The upload fills the partner arrays before setup, so the
// setup's neighbour build restores the history of pairs touching there,
// as after read_restart (setup_pre_exchange skips the rebuild of the
// partner arrays).
int gb2_upload_history(gb2_ctx *c, int n, const int *npartner, const int *partner_tag, const double *hist)
{
    if (!c || !npartner || (n > 0 && (!partner_tag || !hist))) return GB2_ERR_ARG;
    if (!c->have_atoms || c->setup_done) return set_err(c, GB2_ERR_STATE, "history is uploaded after the atoms, before setup");
    if (n != c->nlocal) return set_err(c, GB2_ERR_ARG, "history for %d atoms, %d uploaded", n, c->nlocal);
    int mx = 0;
    for (int i = 0; i < n; i++) {
        if (npartner[i] < 0) return set_err(c, GB2_ERR_ARG, "negative partner count");
        mx = std::max(mx, npartner[i]);
    }
    if (mx > c->maxp) {
        c->maxp = grown_capacity(c, 1, mx, 1 << 20);
        CK(c->ptag.alloc((size_t)c->maxp * c->cap));
        CK(c->phist.alloc((size_t)3 * c->maxp * c->cap));
    }
    const size_t cp = c->cap;
    std::vector<int> pn(cp, 0), pt((size_t)c->maxp * cp, 0);
    std::vector<double> ph((size_t)3 * c->maxp * cp, 0.0);
    size_t off = 0;
    for (int i = 0; i < n; i++) {
        pn[i] = npartner[i];
        for (int m = 0; m < npartner[i]; m++, off++) {
            pt[(size_t)m * cp + i] = partner_tag[off];
            for (int q = 0; q < 3; q++) ph[(size_t)(3 * m + q) * cp + i] = hist[3 * off + q];
        }
    }
    CK(cudaMemcpyAsync(c->pnum.p, pn.data(), sizeof(int) * cp, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->ptag.p, pt.data(), sizeof(int) * pt.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->phist.p, ph.data(), sizeof(double) * ph.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->computeflag = false;
    return 0;
}

// The current contact history in the same layout (FixContactHistory::
// pre_exchange run on the device from the current list), per owned atom in
// the current atom order with its tag.  *n = atoms, *ntotal = partners; with
// caps too small only the counts are reported.
int gb2_download_history(gb2_ctx *c, int cap_atoms, int cap_partners, int *n, int *ntotal, int *tag, int *npartner,
                         int *partner_tag, double *hist)
{
    if (!c) return GB2_ERR_ARG;
    if (!c->setup_done) return set_err(c, GB2_ERR_STATE, "no neighbor list before setup");
    if (do_partners(c)) return c->err.empty() ? GB2_ERR_CUDA : GB2_ERR_CAPACITY;
    const size_t cp = c->cap;
    const int nl = c->nlocal;
    std::vector<int> pn(nl > 0 ? nl : 1), pt((size_t)c->maxp * cp), tg(nl > 0 ? nl : 1);
    std::vector<double> ph((size_t)3 * c->maxp * cp);
    CK(cudaMemcpyAsync(pn.data(), c->pnum.p, sizeof(int) * nl, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(pt.data(), c->ptag.p, sizeof(int) * pt.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(ph.data(), c->phist.p, sizeof(double) * ph.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(tg.data(), c->tag.p, sizeof(int) * nl, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    long tot = 0;
    for (int i = 0; i < nl; i++) tot += pn[i];
    if (n) *n = nl;
    if (ntotal) *ntotal = (int)tot;
    if (cap_atoms < nl || cap_partners < tot || !tag || !npartner || !partner_tag || !hist) return 0;
    size_t off = 0;
    for (int i = 0; i < nl; i++) {
        tag[i] = tg[i];
        npartner[i] = pn[i];
        for (int m = 0; m < pn[i]; m++, off++) {
            partner_tag[off] = pt[(size_t)m * cp + i];
            for (int q = 0; q < 3; q++) hist[3 * off + q] = ph[(size_t)(3 * m + q) * cp + i];
        }
    }
    return 0;
}

// Primitive-wall shear history (FixWallGran's per-atom history, part of its
// restart data) for the uploaded atoms, before setup.
int gb2_upload_wall_history(gb2_ctx *c, int ifix, int n, const double *hist)
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_PLANE || !hist) return GB2_ERR_ARG;
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "wall history is uploaded before setup");
    if (n != c->nlocal) return set_err(c, GB2_ERR_ARG, "wall history for %d atoms, %d uploaded", n, c->nlocal);
    std::vector<double> h((size_t)3 * c->cap, 0.0);
    for (int i = 0; i < n; i++)
        for (int q = 0; q < 3; q++) h[(size_t)q * c->cap + i] = hist[3 * i + q];
    CK(cudaMemcpyAsync(c->fix[ifix].whist.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

int gb2_download_wall_history(gb2_ctx *c, int ifix, int cap, double *hist)
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_PLANE) return GB2_ERR_ARG;
    const int m = std::min(cap, c->nlocal);
    std::vector<double> h((size_t)3 * c->cap);
    CK(cudaMemcpyAsync(h.data(), c->fix[ifix].whist.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int i = 0; i < m; i++)
        for (int q = 0; q < 3; q++) hist[3 * i + q] = h[(size_t)q * c->cap + i];
    return 0;
}

int gb2_download_mesh_contacts(gb2_ctx *c, int ifix, int cap, int *n, int *tag, int *tri, double *hist)
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_MESH) return GB2_ERR_ARG;
    MeshFix &M = *c->fix[ifix].mesh;
    const size_t cp = c->cap;
    const int nl = c->nlocal;
    std::vector<int> tc(nl), sp((size_t)M.maxt * cp), tg(nl);
    std::vector<double> h((size_t)3 * M.maxt * cp);
    CK(cudaMemcpyAsync(tc.data(), M.tcnt.p, sizeof(int) * nl, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(sp.data(), M.spartner.p, sizeof(int) * sp.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(h.data(), M.shist.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(tg.data(), c->tag.p, sizeof(int) * nl, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int k = 0;
    for (int i = 0; i < nl; i++)
        for (int s = 0; s < tc[i]; s++) {
            const int t = sp[(size_t)s * cp + i];
            if (t < 0) continue;
            if (k < cap) {
                if (tag) tag[k] = tg[i];
                if (tri) tri[k] = t;
                if (hist)
                    for (int q = 0; q < 3; q++) hist[3 * k + q] = h[(size_t)(3 * s + q) * cp + i];
            }
            k++;
        }
    if (n) *n = k;
    return 0;
}

// restart layout of the mesh contact history (FixContactHistoryMesh::
// write_restart sorts the slots first, then FixContactHistory::pack_restart):
// per owned atom its partner count, then per partner the triangle id and 3
// shear values.  The sort runs in place, as in the reference.
int gb2_download_mesh_history(gb2_ctx *c, int ifix, int cap_atoms, int cap_entries, int *n, int *ntotal, int *tag,
                              int *npartner, int *tri, double *hist)
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_MESH) return GB2_ERR_ARG;
    if (!c->setup_done) return set_err(c, GB2_ERR_STATE, "no mesh contact history before setup");
    MeshFix &M = *c->fix[ifix].mesh;
    const size_t cp = c->cap;
    const int nl = c->nlocal;
    if (nl > 0) {
        Dev D = make_dev(c);
        k_mesh_sort_contacts<<<nblk(nl), kBlock, 0, c->st>>>(D, ifix);
        CKL();
    }
    std::vector<int> np(nl), tg(nl);
    CK(cudaMemcpyAsync(np.data(), M.snp.p, sizeof(int) * nl, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(tg.data(), c->tag.p, sizeof(int) * nl, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    long total = 0;
    for (int i = 0; i < nl; i++) total += np[i];
    if (n) *n = nl;
    if (ntotal) *ntotal = (int)total;
    if (tag && npartner && cap_atoms >= nl)
        for (int i = 0; i < nl; i++) {
            tag[i] = tg[i];
            npartner[i] = np[i];
        }
    if (!tri || !hist || cap_entries < total || total == 0) return 0;
    std::vector<int> sp((size_t)M.maxt * cp);
    std::vector<double> h((size_t)3 * M.maxt * cp);
    CK(cudaMemcpyAsync(sp.data(), M.spartner.p, sizeof(int) * sp.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(h.data(), M.shist.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    long k = 0;
    for (int i = 0; i < nl; i++)
        for (int s2 = 0; s2 < np[i]; s2++, k++) {
            tri[k] = sp[(size_t)s2 * cp + i];
            for (int q = 0; q < 3; q++) hist[3 * k + q] = h[(size_t)(3 * s2 + q) * cp + i];
        }
    return 0;
}

// FixContactHistoryMesh::unpack_restart (src/fix_contact_history_mesh.cpp:
// 613-650): the partner triangles and shear of each uploaded atom, in the
// uploaded order (before setup; the setup's mesh list keeps the partners
// that are still candidates, as setup_pre_force does after read_restart)
int gb2_upload_mesh_history(gb2_ctx *c, int ifix, int n, const int *npartner, const int *tri, const double *hist)
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_MESH || !npartner) return GB2_ERR_ARG;
    if (c->setup_done) return set_err(c, GB2_ERR_STATE, "mesh contact history is uploaded before setup");
    if (n != c->nlocal) return set_err(c, GB2_ERR_ARG, "mesh history for %d atoms, %d uploaded", n, c->nlocal);
    MeshFix &M = *c->fix[ifix].mesh;
    const int ntri = (int)M.topo.tri.size();
    int maxnp = 0;
    long total = 0;
    for (int i = 0; i < n; i++) {
        if (npartner[i] < 0 || npartner[i] > 64)
            return set_err(c, GB2_ERR_ARG, "atom %d: %d mesh partners (0..64)", i, npartner[i]);
        maxnp = std::max(maxnp, npartner[i]);
        total += npartner[i];
    }
    if (total > 0 && (!tri || !hist)) return GB2_ERR_ARG;
    for (long k = 0; k < total; k++)
        if (tri[k] < 0 || tri[k] >= ntri) return set_err(c, GB2_ERR_ARG, "mesh partner %d out of range", tri[k]);
    const size_t cp = c->cap;
    if (maxnp > M.maxt) {
        M.maxt = maxnp;
        CK(M.spartner.alloc((size_t)M.maxt * cp));
        CK(M.shist.alloc((size_t)3 * M.maxt * cp));
        CK(M.tlist.alloc((size_t)M.maxt * cp));
    }
    std::vector<int> sp((size_t)M.maxt * cp, -1), np(cp, 0);
    std::vector<double> h((size_t)3 * M.maxt * cp, 0.0);
    long k = 0;
    for (int i = 0; i < n; i++) {
        np[i] = npartner[i];
        for (int s2 = 0; s2 < npartner[i]; s2++, k++) {
            sp[(size_t)s2 * cp + i] = tri[k];
            for (int q = 0; q < 3; q++) h[(size_t)(3 * s2 + q) * cp + i] = hist[3 * k + q];
        }
    }
    CK(cudaMemcpyAsync(M.spartner.p, sp.data(), sizeof(int) * sp.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(M.shist.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(M.snp.p, np.data(), sizeof(int) * cp, cudaMemcpyHostToDevice, c->st));
    // the slot count the setup's sort walks: the unpacked partners
    CK(cudaMemcpyAsync(M.tcnt.p, np.data(), sizeof(int) * cp, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

int gb2_mesh_topology(gb2_ctx *c, int ifix, int cap, int *ntri, unsigned char *edge_active,
                      unsigned char *corner_active, int *obtuse)
{
    if (!c || ifix < 0 || ifix >= c->nfix || c->fix[ifix].kind != FIX_WALL_MESH) return GB2_ERR_ARG;
    const MeshTopo &T = c->fix[ifix].mesh->topo;
    const int n = (int)T.tri.size();
    if (ntri) *ntri = n;
    for (int t = 0; t < std::min(n, cap); t++) {
        for (int k = 0; k < 3; k++) {
            if (edge_active) edge_active[3 * t + k] = (T.tri[t].active >> k) & 1;
            if (corner_active) corner_active[3 * t + k] = (T.tri[t].active >> (3 + k)) & 1;
        }
        if (obtuse) obtuse[t] = T.tri[t].obtuse;
    }
    return 0;
}

int gb2_get_stats(gb2_ctx *c, gb2_stats *s)
{
    if (!c || !s) return GB2_ERR_ARG;
    std::memset(s, 0, sizeof *s);
    s->ntimestep = c->ntimestep;
    s->nlocal = c->nlocal;
    s->nghost = c->nghost;
    s->nbuilds = c->nbuilds;
    s->npairs = c->npairs_last;
    s->maxneigh = c->maxn;
    s->maxpartner = c->maxp;
    s->kernel_launches = c->launches;
    s->t_integrate = c->prof_ms[PROF_INTEGRATE];
    s->t_pair_tail = c->prof_ms[PROF_PAIR_TAIL];
    s->t_pair_main = c->prof_ms[PROF_PAIR_MAIN];
    s->t_forward = c->prof_ms[PROF_FORWARD];
    s->t_rebuild = c->prof_ms[PROF_REBUILD];
    s->time_pair = s->t_pair_tail + s->t_pair_main;
    s->time_neigh = s->t_rebuild;
    s->time_other = s->t_integrate + s->t_forward;
    s->n_pair_main = c->n_pair_main;
    s->n_rebuild_timed = c->n_rebuild_timed;
    s->nsteps_rebuild = c->nsteps_rebuild;
    s->maxrev = c->maxr;
    for (int k = 0; k < c->nfix; k++)
        if (c->fix[k].mesh) s->maxmesh = std::max(s->maxmesh, c->fix[k].mesh->maxt);
    s->ngrow = c->ngrow;
    return 0;
}

int gb2_last_error(gb2_ctx *c, char *buf, int len)
{
    if (!c || !buf || len <= 0) return GB2_ERR_ARG;
    std::snprintf(buf, len, "%s", c->err.c_str());
    return 0;
}

}  // extern "C"
