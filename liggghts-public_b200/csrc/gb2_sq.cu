// gb2_sq.cu -- superquadric time step (pair gran hertz/history on
// superquadric surfaces + fix nve/asphere) and its C ABI (gb2_sq_* in
// include/granb200.h).
//
// Step sequence as Verlet::run with these styles: initial_integrate,
// displacement check, neighbour rebuild with contact-history transfer when
// any particle moved more than skin/2, pair pass (screening of every
// half-list slot, then the contact-point solves in work lists by kind),
// deterministic per-particle sums (reverse slots in ascending owner order,
// then own slots), final_integrate.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <random>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/granb200.h"
#include "gb2_mlp.cuh"

using namespace gb2;
using namespace gb2::sq;

namespace {

constexpr int kB = 128;
inline int nb(long n) { return (int)((n + kB - 1) / kB); }

template <typename T>
struct Buf {
    T *p = nullptr;
    size_t n = 0;
    ~Buf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    // grows with 50% headroom: the neighbour lists are rebuilt every few
    // steps with slightly different sizes and swap roles with the previous
    // list, and a cudaFree/cudaMalloc pair at each of those would stall the
    // device for longer than the rebuild's kernels take
    cudaError_t alloc(size_t m)
    {
        if (m <= n && p) return cudaSuccess;
        release();
        const size_t want = std::max<size_t>(m + m / 2, 1);
        cudaError_t e = cudaMalloc(&p, want * sizeof(T));
        if (e == cudaSuccess) n = want;
        return e;
    }
    void swap(Buf &o)
    {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
};

// ------------------------------------------------------------------ neighbour build kernels

struct Grid {
    double lo[3];
    double inv;
    int nc[3];
};

__global__ void k_sq_cellkey(SqDev D, Grid G, unsigned *keys, int *vals, int *counts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n) return;
    const dbl4 x = D.x[i];
    const double c[3] = {x.x, x.y, x.z};
    int ix[3];
    for (int d = 0; d < 3; d++) ix[d] = min(max((int)((c[d] - G.lo[d]) * G.inv), 0), G.nc[d] - 1);
    const int key = (ix[2] * G.nc[1] + ix[1]) * G.nc[0] + ix[0];
    keys[i] = (unsigned)key;
    vals[i] = i;
    atomicAdd(&counts[key], 1);
}

// count (fill == false) or write (fill == true) the half-list neighbours
// j > i within rb_i + rb_j + skin, then sort the row ascending
__global__ void k_sq_neigh(SqDev D, Grid G, const int *cell_start, const int *cell_atoms, int *cnt, int *nbr,
                           int *own, int fill)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n) return;
    const dbl4 xi = D.x[i];
    const double c[3] = {xi.x, xi.y, xi.z};
    int ix[3];
    for (int d = 0; d < 3; d++) ix[d] = min(max((int)((c[d] - G.lo[d]) * G.inv), 0), G.nc[d] - 1);
    int m = 0;
    const int base = fill ? D.start[i] : 0;
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                const int cx = ix[0] + dx, cy = ix[1] + dy, cz = ix[2] + dz;
                if (cx < 0 || cy < 0 || cz < 0 || cx >= G.nc[0] || cy >= G.nc[1] || cz >= G.nc[2]) continue;
                const int cell = (cz * G.nc[1] + cy) * G.nc[0] + cx;
                for (int a = cell_start[cell]; a < cell_start[cell + 1]; a++) {
                    const int j = cell_atoms[a];
                    if (j <= i) continue;
                    const dbl4 xj = D.x[j];
                    const double ddx = xi.x - xj.x, ddy = xi.y - xj.y, ddz = xi.z - xj.z;
                    const double cut = xi.w + xj.w + D.skin;
                    if (ddx * ddx + ddy * ddy + ddz * ddz > cut * cut) continue;
                    if (fill) {
                        nbr[base + m] = j;
                        own[base + m] = i;
                    }
                    m++;
                }
            }
    if (!fill) {
        cnt[i] = m;
        return;
    }
    for (int a = 1; a < m; a++) {   // ascending j within the row
        const int v = nbr[base + a];
        int b = a - 1;
        while (b >= 0 && nbr[base + b] > v) {
            nbr[base + b + 1] = nbr[base + b];
            b--;
        }
        nbr[base + b + 1] = v;
    }
}

// FixContactHistory transfer at a rebuild: a new slot (i, j) takes the old
// slot's history when the old pair was flagged (touching), else zeros
__global__ void k_sq_transfer(SqDev D, int nslots, const int *own, const int *ostart, const int *onbr,
                              const int *oflag, const int *ostate, const dbl4 *ocp, const double2 *oalpha,
                              const dbl4 *oshear)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int i = own[s], j = D.nbr[s];
    int lo = ostart[i], hi = ostart[i + 1] - 1, hit = -1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int v = onbr[mid];
        if (v == j) {
            hit = mid;
            break;
        }
        if (v < j) lo = mid + 1;
        else hi = mid - 1;
    }
    if (hit >= 0 && oflag[hit]) {
        D.flag[s] = oflag[hit];
        D.state[s] = ostate[hit];
        D.cp[s] = ocp[hit];
        D.alpha[s] = oalpha[hit];
        D.shear[s] = oshear[hit];
    } else {
        D.flag[s] = 0;
        D.state[s] = FAR;
        D.cp[s] = dbl4{0, 0, 0, 0};
        D.alpha[s] = double2{0, 0};
        D.shear[s] = dbl4{0, 0, 0, 0};
    }
}

__global__ void k_sq_rcount(SqDev D, int nslots, int *rcnt)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    atomicAdd(&rcnt[D.nbr[s]], 1);
}
__global__ void k_sq_rfill(SqDev D, int nslots, int *rfill)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int j = D.nbr[s];
    D.rslot[D.rstart[j] + atomicAdd(&rfill[j], 1)] = s;
}
__global__ void k_sq_rsort(SqDev D)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.n) return;
    const int b0 = D.rstart[k], m = D.rstart[k + 1] - b0;
    for (int a = 1; a < m; a++) {
        const int v = D.rslot[b0 + a];
        int b = a - 1;
        while (b >= 0 && D.rslot[b0 + b] > v) {
            D.rslot[b0 + b + 1] = D.rslot[b0 + b];
            b--;
        }
        D.rslot[b0 + b + 1] = v;
    }
}

__global__ void k_sq_hold(SqDev D)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n) return;
    D.xhold[i] = D.x[i];
}

__global__ void k_sq_coords(SqDev D, double *xs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n) return;
    const dbl4 x = D.x[i];
    xs[i] = x.x;
    xs[D.n + i] = x.y;
    xs[2 * D.n + i] = x.z;
}

}  // namespace

struct gb2_sq_ctx {
    gb2_sq_params P{};
    std::string err;
    cudaStream_t st = nullptr;
    int n = 0;
    bool setup_done = false;
    double rbmax = 0;
    Buf<dbl4> x, v, q, L, w, f, t, shape, inert, xhold;
    // list (current and previous for the history transfer)
    long nslots = 0;
    Buf<int> start, nbr, own, flag, state, ostart, onbr, oown, oflag, ostate;
    Buf<dbl4> cp, shear, ocp, oshear, pfi, pti, ptj;
    Buf<double2> alpha, oalpha;
    Buf<int> rstart, rslot, rcnt, cnt;
    // grid
    Buf<unsigned> keys, keys2;
    Buf<int> vals, cell_atoms, cell_start, counts;
    Buf<double> xs, red;
    Buf<char> tmp;
    Buf<unsigned long long> counters;
    Buf<int> dflag;
    int *h_pin = nullptr;
    double Yeff = 0, Geff = 0, betaeff = 0, mu = 0;
    long nbuilds = 0;
    Buf<float> mlp;
    bool mlp_on = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    // work lists of the pair pass: 2 lists of nslots items, then the item
    // counts and the taken counter
    Buf<int> work;
    Buf<signed char> kind;   // per slot: the work list the screen puts it on
    int nsm = 148;
};

namespace {

int sq_err(gb2_sq_ctx *c, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
    return code;
}

#define SQCK(call)                                                                                                \
    do {                                                                                                          \
        cudaError_t e_ = (call);                                                                                  \
        if (e_ != cudaSuccess) return sq_err(c, GB2_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));          \
    } while (0)
#define SQCKL() SQCK(cudaGetLastError())

SqDev sq_dev(gb2_sq_ctx *c)
{
    SqDev D;
    std::memset(&D, 0, sizeof D);
    D.n = c->n;
    D.x = c->x.p;
    D.v = c->v.p;
    D.q = c->q.p;
    D.L = c->L.p;
    D.w = c->w.p;
    D.f = c->f.p;
    D.t = c->t.p;
    D.shape = c->shape.p;
    D.inert = c->inert.p;
    D.xhold = c->xhold.p;
    D.start = c->start.p;
    D.nbr = c->nbr.p;
    D.flag = c->flag.p;
    D.state = c->state.p;
    D.cp = c->cp.p;
    D.shear = c->shear.p;
    D.alpha = c->alpha.p;
    D.pfi = c->pfi.p;
    D.pti = c->pti.p;
    D.ptj = c->ptj.p;
    D.rstart = c->rstart.p;
    D.rslot = c->rslot.p;
    D.dt = c->P.dt;
    D.skin = c->P.skin;
    D.triggersq = 0.25 * c->P.skin * c->P.skin;
    D.Yeff = c->Yeff;
    D.Geff = c->Geff;
    D.betaeff = c->betaeff;
    D.mu = c->mu;
    D.cnt = c->counters.p;
    D.dflag = c->dflag.p;
    D.mlp = c->mlp_on ? c->mlp.p : nullptr;
    return D;
}

int scan(gb2_sq_ctx *c, const int *in, int *out, int n)
{
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, c->st);
    SQCK(c->tmp.alloc(bytes));
    bytes = c->tmp.n;
    SQCK(cub::DeviceScan::ExclusiveSum(c->tmp.p, bytes, in, out, n, c->st));
    return 0;
}

// neighbour list (half, bounding spheres + skin) with history transfer
int sq_build(gb2_sq_ctx *c, bool transfer)
{
    const int n = c->n;
    SqDev D = sq_dev(c);
    // grid over the current particle extent
    SQCK(c->xs.alloc((size_t)3 * n));
    SQCK(c->red.alloc(6));
    k_sq_coords<<<nb(n), kB, 0, c->st>>>(D, c->xs.p);
    SQCKL();
    size_t bytes = 0;
    cub::DeviceReduce::Min(nullptr, bytes, c->xs.p, c->red.p, n, c->st);
    SQCK(c->tmp.alloc(bytes));
    for (int d = 0; d < 3; d++) {
        bytes = c->tmp.n;
        SQCK(cub::DeviceReduce::Min(c->tmp.p, bytes, c->xs.p + (size_t)d * n, c->red.p + d, n, c->st));
        bytes = c->tmp.n;
        SQCK(cub::DeviceReduce::Max(c->tmp.p, bytes, c->xs.p + (size_t)d * n, c->red.p + 3 + d, n, c->st));
    }
    double ext[6];
    SQCK(cudaMemcpyAsync(ext, c->red.p, sizeof ext, cudaMemcpyDeviceToHost, c->st));
    SQCK(cudaStreamSynchronize(c->st));
    Grid G;
    const double cell = 2.0 * c->rbmax + c->P.skin;
    G.inv = 1.0 / cell;
    long ncell = 1;
    for (int d = 0; d < 3; d++) {
        G.lo[d] = ext[d];
        G.nc[d] = std::max(1, (int)((ext[3 + d] - ext[d]) * G.inv) + 1);
        ncell *= G.nc[d];
    }
    if (ncell > (1l << 28)) return sq_err(c, GB2_ERR_UNSUPPORTED, "particle extent too large for the cell grid");
    SQCK(c->keys.alloc(n));
    SQCK(c->keys2.alloc(n));
    SQCK(c->vals.alloc(n));
    SQCK(c->cell_atoms.alloc(n));
    SQCK(c->counts.alloc((size_t)ncell + 1));
    SQCK(c->cell_start.alloc((size_t)ncell + 1));
    SQCK(cudaMemsetAsync(c->counts.p, 0, sizeof(int) * (ncell + 1), c->st));
    k_sq_cellkey<<<nb(n), kB, 0, c->st>>>(D, G, c->keys.p, c->vals.p, c->counts.p);
    SQCKL();
    int endbit = 1;
    while ((1l << endbit) < ncell + 1) endbit++;
    bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, c->keys.p, c->keys2.p, c->vals.p, c->cell_atoms.p, n, 0, endbit,
                                    c->st);
    SQCK(c->tmp.alloc(bytes));
    bytes = c->tmp.n;
    SQCK(cub::DeviceRadixSort::SortPairs(c->tmp.p, bytes, c->keys.p, c->keys2.p, c->vals.p, c->cell_atoms.p, n, 0,
                                         endbit, c->st));
    if (scan(c, c->counts.p, c->cell_start.p, (int)ncell + 1)) return GB2_ERR_CUDA;
    // keep the old list for the transfer
    if (transfer) {
        c->start.swap(c->ostart);
        c->nbr.swap(c->onbr);
        c->own.swap(c->oown);
        c->flag.swap(c->oflag);
        c->state.swap(c->ostate);
        c->cp.swap(c->ocp);
        c->alpha.swap(c->oalpha);
        c->shear.swap(c->oshear);
    }
    SQCK(c->cnt.alloc((size_t)n + 1));
    SQCK(c->start.alloc((size_t)n + 1));
    SQCK(cudaMemsetAsync(c->cnt.p, 0, sizeof(int) * (n + 1), c->st));
    D = sq_dev(c);
    k_sq_neigh<<<nb(n), kB, 0, c->st>>>(D, G, c->cell_start.p, c->cell_atoms.p, c->cnt.p, nullptr, nullptr, 0);
    SQCKL();
    if (scan(c, c->cnt.p, c->start.p, n + 1)) return GB2_ERR_CUDA;
    int tot = 0;
    SQCK(cudaMemcpyAsync(&c->h_pin[0], c->start.p + n, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    SQCK(cudaStreamSynchronize(c->st));
    tot = c->h_pin[0];
    c->nslots = tot;
    const size_t ns = std::max(tot, 1);
    SQCK(c->nbr.alloc(ns));
    SQCK(c->own.alloc(ns));
    SQCK(c->flag.alloc(ns));
    SQCK(c->state.alloc(ns));
    SQCK(c->cp.alloc(ns));
    SQCK(c->alpha.alloc(ns));
    SQCK(c->shear.alloc(ns));
    SQCK(c->pfi.alloc(ns));
    SQCK(c->pti.alloc(ns));
    SQCK(c->ptj.alloc(ns));
    SQCK(c->work.alloc(2 * ns + 4));
    SQCK(c->kind.alloc(ns));
    SQCK(c->rslot.alloc(ns));
    D = sq_dev(c);
    k_sq_neigh<<<nb(n), kB, 0, c->st>>>(D, G, c->cell_start.p, c->cell_atoms.p, nullptr, c->nbr.p, c->own.p, 1);
    SQCKL();
    if (tot > 0) {
        if (transfer && c->ostart.p) {
            k_sq_transfer<<<nb(tot), kB, 0, c->st>>>(D, tot, c->own.p, c->ostart.p, c->onbr.p, c->oflag.p,
                                                      c->ostate.p, c->ocp.p, c->oalpha.p, c->oshear.p);
            SQCKL();
        } else {
            SQCK(cudaMemsetAsync(c->flag.p, 0, sizeof(int) * tot, c->st));
            SQCK(cudaMemsetAsync(c->state.p, 0, sizeof(int) * tot, c->st));
            SQCK(cudaMemsetAsync(c->cp.p, 0, sizeof(dbl4) * tot, c->st));
            SQCK(cudaMemsetAsync(c->alpha.p, 0, sizeof(double2) * tot, c->st));
            SQCK(cudaMemsetAsync(c->shear.p, 0, sizeof(dbl4) * tot, c->st));
        }
    }
    // reverse CSR
    SQCK(c->rcnt.alloc((size_t)n + 1));
    SQCK(c->rstart.alloc((size_t)n + 1));
    SQCK(cudaMemsetAsync(c->rcnt.p, 0, sizeof(int) * (n + 1), c->st));
    if (tot > 0) k_sq_rcount<<<nb(tot), kB, 0, c->st>>>(D, tot, c->rcnt.p);
    SQCKL();
    if (scan(c, c->rcnt.p, c->rstart.p, n + 1)) return GB2_ERR_CUDA;
    SQCK(cudaMemsetAsync(c->rcnt.p, 0, sizeof(int) * (n + 1), c->st));
    D = sq_dev(c);
    if (tot > 0) k_sq_rfill<<<nb(tot), kB, 0, c->st>>>(D, tot, c->rcnt.p);
    SQCKL();
    k_sq_rsort<<<nb(n), kB, 0, c->st>>>(D);
    SQCKL();
    k_sq_hold<<<nb(n), kB, 0, c->st>>>(D);
    SQCKL();
    c->nbuilds++;
    return 0;
}

// the pair pass in work lists (screen, then the solves of the first contacts
// and the warm starts), then the per-particle sums
int sq_force(gb2_sq_ctx *c, int shearupdate)
{
    SqDev D = sq_dev(c);
    if (c->nslots > 0) {
        const size_t ns = (size_t)c->nslots;
        SqWork W;
        for (int l = 0; l < 2; l++) W.list[l] = c->work.p + l * ns;
        W.n = c->work.p + 2 * ns;
        W.next = W.n + 2;
        SQCK(cudaMemsetAsync(W.n, 0, 4 * sizeof(int), c->st));
        k_sq_screen<<<nb(c->nslots), kB, 0, c->st>>>(D, c->own.p, (int)c->nslots, c->kind.p);
        SQCKL();
        // the two work lists in slot order (stable selections; the counts
        // stay on the device for the solve kernel)
        thrust::counting_iterator<int> slots(0);
        size_t bytes = 0;
        cub::DeviceSelect::If(nullptr, bytes, slots, W.list[0], W.n, (int)ns, SlotKindIs{c->kind.p, 0}, c->st);
        SQCK(c->tmp.alloc(bytes));
        for (int l = 0; l < 2; l++) {
            bytes = c->tmp.n;
            SQCK(cub::DeviceSelect::If(c->tmp.p, bytes, slots, W.list[l], W.n + l, (int)ns,
                                       SlotKindIs{c->kind.p, (signed char)l}, c->st));
        }
        // the solves: enough resident warps to fill the GPU; each warp takes
        // the next 32 items (first contacts, then warm starts) until none
        // are left
        k_sq_solve<<<2 * c->nsm, kB, 0, c->st>>>(D, W, c->own.p, shearupdate);
        SQCKL();
    }
    k_sq_sum<<<nb(c->n), kB, 0, c->st>>>(D);
    SQCKL();
    return 0;
}

}  // namespace

extern "C" {

int gb2_sq_create(const gb2_sq_params *p, gb2_sq_ctx **out)
{
    if (!p || !out) return GB2_ERR_ARG;
    *out = nullptr;
    if (!(p->dt > 0) || p->skin < 0) return GB2_ERR_ARG;
    if (p->poisson < 0. || p->poisson > 0.5 || p->restitution <= 0.05 || p->restitution > 1) return GB2_ERR_ARG;
    if (cudaSetDevice(p->device) != cudaSuccess) return GB2_ERR_CUDA;
    gb2_sq_ctx *c = new gb2_sq_ctx();
    c->P = *p;
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, p->device);
    if (c->nsm <= 0) c->nsm = 1;
    // material constants (src/global_properties.cpp:432-540), one atom type
    const double E = p->youngs, nu = p->poisson;
    c->Yeff = 1. / ((1. - std::pow(nu, 2.)) / E + (1. - std::pow(nu, 2.)) / E);
    c->Geff = 1. / (2. * (2. - nu) * (1. + nu) / E + 2. * (2. - nu) * (1. + nu) / E);
    const double lg = std::log(p->restitution);
    c->betaeff = lg / std::sqrt(std::pow(lg, 2.) + std::pow(M_PI, 2.));
    c->mu = p->friction;
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
        pinned_slot_get(&c->h_pin) != 0 || c->counters.alloc(8) != cudaSuccess ||
        c->dflag.alloc(1) != cudaSuccess ||
        cudaMemsetAsync(c->counters.p, 0, 8 * sizeof(unsigned long long), c->st) != cudaSuccess ||
        cudaEventCreate(&c->e0) != cudaSuccess || cudaEventCreate(&c->e1) != cudaSuccess) {
        pinned_slot_put(c->h_pin);
        if (c->st) cudaStreamDestroy(c->st);
        delete c;
        return GB2_ERR_CUDA;
    }
    *out = c;
    return 0;
}

int gb2_sq_destroy(gb2_sq_ctx *c)
{
    if (!c) return 0;
    cudaStreamSynchronize(c->st);
    pinned_slot_put(c->h_pin);
    if (c->e0) cudaEventDestroy(c->e0);
    if (c->e1) cudaEventDestroy(c->e1);
    cudaStream_t st = c->st;
    delete c;
    if (st) cudaStreamDestroy(st);
    return 0;
}

// bounding_sphere_radius_superquadric with n1 = n2 = n, times scale_koef 1.0001
// (src/math_extra_liggghts_superquadric.cpp:206-233)
static double host_pow_abs(double base, double e)
{
    base = std::fabs(base);
    const double tol = 1e-12;
    if (std::fabs(e) < tol || std::fabs(base - 1.0) < tol) return 1.0;
    if (std::fabs(base) < tol) return 0.0;
    const double nn = std::floor(std::fabs(e));
    double r = 1.0;
    for (int i = 0; i < (int)nn; i++) r *= base;
    const double nd = std::fabs(e) - nn;
    if (nd > 0.0) r *= (std::fabs(2.0 * nd - 1.0) < 2.0 * tol) ? std::sqrt(base) : std::pow(base, nd);
    return e > 0.0 ? r : 1.0 / r;
}
static double bounding_radius(const double *shape, double n)
{
    if (n == 2.0 || std::fabs(n - 2.0) < 1e-13) return std::max(std::max(shape[0], shape[1]), shape[2]) * 1.0001;
    const double a = std::max(shape[0], shape[1]), b = std::min(shape[0], shape[1]), c = shape[2];
    const double n1 = std::max(2.1, n), n2 = std::max(2.1, n);
    const double alpha = host_pow_abs(b / a, 2.0 / (n2 - 2.0));
    const double gamma = host_pow_abs(1.0 + host_pow_abs(alpha, n2), n1 / n2 - 1.0);
    const double beta = host_pow_abs(c * c / (a * a) * gamma, 1.0 / (n1 - 2.0));
    const double x0 = 1.0 / host_pow_abs(host_pow_abs(1.0 + host_pow_abs(alpha, n2), n1 / n2) + host_pow_abs(beta, n1), 1.0 / n1);
    const double xt = x0 * a, yt = alpha * x0 * b, zt = beta * x0 * c;
    return std::sqrt(xt * xt + yt * yt + zt * zt) * 1.0001;
}

int gb2_sq_upload(gb2_sq_ctx *c, int n, const double *x, const double *v, const double *quat, const double *angmom,
                  const double *shape, const double *blockiness, const double *rmass, const double *inertia,
                  const double *volume)
{
    if (!c || n <= 0 || !x || !v || !quat || !angmom || !shape || !blockiness || !rmass || !inertia || !volume)
        return GB2_ERR_ARG;
    std::vector<dbl4> hx(n), hv(n), hq(n), hL(n), hs(n), hi(n);
    double rbmax = 0;
    for (int i = 0; i < n; i++) {
        if (!(blockiness[i] >= 2.0) || !(shape[3 * i] > 0) || !(shape[3 * i + 1] > 0) || !(shape[3 * i + 2] > 0) ||
            !(rmass[i] > 0) || !(volume[i] > 0))
            return sq_err(c, GB2_ERR_ARG, "superquadric %d: shape, blockiness (>= 2), mass and volume must be positive", i);
        const double rb = bounding_radius(&shape[3 * i], blockiness[i]);
        rbmax = std::max(rbmax, rb);
        hx[i] = dbl4{x[3 * i], x[3 * i + 1], x[3 * i + 2], rb};
        hv[i] = dbl4{v[3 * i], v[3 * i + 1], v[3 * i + 2], rmass[i]};
        hq[i] = dbl4{quat[4 * i], quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3]};
        hL[i] = dbl4{angmom[3 * i], angmom[3 * i + 1], angmom[3 * i + 2], 0.0};
        hs[i] = dbl4{shape[3 * i], shape[3 * i + 1], shape[3 * i + 2], blockiness[i]};
        // volume-equivalent radius used for the Hertz reff (src/pair_gran_base.h:266-270)
        hi[i] = dbl4{inertia[3 * i], inertia[3 * i + 1], inertia[3 * i + 2], std::cbrt(0.75 * volume[i] / M_PI)};
    }
    c->n = n;
    c->rbmax = rbmax;
    SQCK(c->x.alloc(n));
    SQCK(c->v.alloc(n));
    SQCK(c->q.alloc(n));
    SQCK(c->L.alloc(n));
    SQCK(c->w.alloc(n));
    SQCK(c->f.alloc(n));
    SQCK(c->t.alloc(n));
    SQCK(c->shape.alloc(n));
    SQCK(c->inert.alloc(n));
    SQCK(c->xhold.alloc(n));
    SQCK(cudaMemcpyAsync(c->x.p, hx.data(), sizeof(dbl4) * n, cudaMemcpyHostToDevice, c->st));
    SQCK(cudaMemcpyAsync(c->v.p, hv.data(), sizeof(dbl4) * n, cudaMemcpyHostToDevice, c->st));
    SQCK(cudaMemcpyAsync(c->q.p, hq.data(), sizeof(dbl4) * n, cudaMemcpyHostToDevice, c->st));
    SQCK(cudaMemcpyAsync(c->L.p, hL.data(), sizeof(dbl4) * n, cudaMemcpyHostToDevice, c->st));
    SQCK(cudaMemcpyAsync(c->shape.p, hs.data(), sizeof(dbl4) * n, cudaMemcpyHostToDevice, c->st));
    SQCK(cudaMemcpyAsync(c->inert.p, hi.data(), sizeof(dbl4) * n, cudaMemcpyHostToDevice, c->st));
    SQCK(cudaMemsetAsync(c->f.p, 0, sizeof(dbl4) * n, c->st));
    SQCK(cudaMemsetAsync(c->t.p, 0, sizeof(dbl4) * n, c->st));
    SQCK(cudaStreamSynchronize(c->st));
    c->setup_done = false;
    return 0;
}

int gb2_sq_set_learned_guess(gb2_sq_ctx *c, const float *params, int nparams)
{
    if (!c) return GB2_ERR_ARG;
    if (!params) {
        c->mlp_on = false;
        return 0;
    }
    if (nparams != kMlpSize) return sq_err(c, GB2_ERR_ARG, "learned guess: expected %d parameters, got %d", kMlpSize, nparams);
    SQCK(c->mlp.alloc(kMlpSize));
    SQCK(cudaMemcpyAsync(c->mlp.p, params, sizeof(float) * kMlpSize, cudaMemcpyHostToDevice, c->st));
    SQCK(cudaStreamSynchronize(c->st));
    c->mlp_on = true;
    return 0;
}

int gb2_sq_setup(gb2_sq_ctx *c)
{
    if (!c || c->n <= 0) return GB2_ERR_ARG;
    c->err.clear();
    SqDev D = sq_dev(c);
    k_sq_omega<<<nb(c->n), kB, 0, c->st>>>(D);
    SQCKL();
    int rc = sq_build(c, false);
    if (rc) return rc;
    rc = sq_force(c, 0);
    if (rc) return rc;
    SQCK(cudaStreamSynchronize(c->st));
    c->setup_done = true;
    return 0;
}

int gb2_sq_run(gb2_sq_ctx *c, int nsteps)
{
    if (!c) return GB2_ERR_ARG;
    if (!c->setup_done) return sq_err(c, GB2_ERR_STATE, "gb2_sq_setup must precede gb2_sq_run");
    for (int s = 0; s < nsteps; s++) {
        SQCK(cudaMemsetAsync(c->dflag.p, 0, sizeof(int), c->st));
        SqDev D = sq_dev(c);
        k_sq_initial<<<nb(c->n), kB, 0, c->st>>>(D, 1);
        SQCKL();
        SQCK(cudaMemcpyAsync(&c->h_pin[1], c->dflag.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        SQCK(cudaStreamSynchronize(c->st));
        if (c->h_pin[1]) {
            const int rc = sq_build(c, true);
            if (rc) return rc;
        }
        int rc = sq_force(c, 1);
        if (rc) return rc;
        D = sq_dev(c);
        k_sq_final<<<nb(c->n), kB, 0, c->st>>>(D);
        SQCKL();
    }
    SQCK(cudaStreamSynchronize(c->st));
    return 0;
}

int gb2_sq_run_timed(gb2_sq_ctx *c, int nsteps, double *ms)
{
    if (!c || !ms) return GB2_ERR_ARG;
    SQCK(cudaStreamSynchronize(c->st));
    SQCK(cudaEventRecord(c->e0, c->st));
    const int rc = gb2_sq_run(c, nsteps);
    if (rc) return rc;
    SQCK(cudaEventRecord(c->e1, c->st));
    SQCK(cudaEventSynchronize(c->e1));
    float f = 0;
    SQCK(cudaEventElapsedTime(&f, c->e0, c->e1));
    *ms = f;
    return 0;
}

int gb2_sq_download(gb2_sq_ctx *c, int cap, double *x, double *v, double *quat, double *angmom, double *omega,
                    double *f, double *torque)
{
    if (!c || cap < c->n) return GB2_ERR_ARG;
    const int n = c->n;
    std::vector<dbl4> h(n);
    struct Item {
        Buf<dbl4> *b;
        double *out;
        int k;
    } items[] = {{&c->x, x, 3}, {&c->v, v, 3}, {&c->q, quat, 4}, {&c->L, angmom, 3},
                 {&c->w, omega, 3}, {&c->f, f, 3}, {&c->t, torque, 3}};
    for (auto &it : items) {
        if (!it.out) continue;
        SQCK(cudaMemcpyAsync(h.data(), it.b->p, sizeof(dbl4) * n, cudaMemcpyDeviceToHost, c->st));
        SQCK(cudaStreamSynchronize(c->st));
        for (int i = 0; i < n; i++) {
            const double r[4] = {h[i].x, h[i].y, h[i].z, h[i].w};
            for (int k = 0; k < it.k; k++) it.out[it.k * i + k] = r[k];
        }
    }
    return 0;
}

int gb2_sq_download_pairs(gb2_sq_ctx *c, int cap, int *n, int *tag_i, int *tag_j, int *state, double *cp,
                          double *shear)
{
    if (!c || !n) return GB2_ERR_ARG;
    const long ns = c->nslots;
    *n = (int)ns;
    if (cap < ns || ns == 0) return 0;
    std::vector<int> own(ns), nbr(ns), st(ns);
    std::vector<dbl4> hcp(ns), hsh(ns);
    SQCK(cudaMemcpyAsync(own.data(), c->own.p, sizeof(int) * ns, cudaMemcpyDeviceToHost, c->st));
    SQCK(cudaMemcpyAsync(nbr.data(), c->nbr.p, sizeof(int) * ns, cudaMemcpyDeviceToHost, c->st));
    SQCK(cudaMemcpyAsync(st.data(), c->state.p, sizeof(int) * ns, cudaMemcpyDeviceToHost, c->st));
    SQCK(cudaMemcpyAsync(hcp.data(), c->cp.p, sizeof(dbl4) * ns, cudaMemcpyDeviceToHost, c->st));
    SQCK(cudaMemcpyAsync(hsh.data(), c->shear.p, sizeof(dbl4) * ns, cudaMemcpyDeviceToHost, c->st));
    SQCK(cudaStreamSynchronize(c->st));
    for (long s = 0; s < ns; s++) {
        if (tag_i) tag_i[s] = own[s] + 1;
        if (tag_j) tag_j[s] = nbr[s] + 1;
        if (state) state[s] = st[s];
        if (cp) {
            cp[3 * s] = hcp[s].x;
            cp[3 * s + 1] = hcp[s].y;
            cp[3 * s + 2] = hcp[s].z;
        }
        if (shear) {
            shear[3 * s] = hsh[s].x;
            shear[3 * s + 1] = hsh[s].y;
            shear[3 * s + 2] = hsh[s].z;
        }
    }
    return 0;
}

int gb2_sq_counters(gb2_sq_ctx *c, long long *out)
{
    if (!c || !out) return GB2_ERR_ARG;
    unsigned long long h[8];
    SQCK(cudaMemcpyAsync(h, c->counters.p, sizeof h, cudaMemcpyDeviceToHost, c->st));
    SQCK(cudaStreamSynchronize(c->st));
    for (int k = 0; k < 5; k++) out[k] = (long long)h[k];
    out[5] = c->nbuilds;
    out[6] = c->nslots;
    return 0;
}

int gb2_sq_last_error(gb2_sq_ctx *c, char *buf, int len)
{
    if (!c || !buf || len <= 0) return GB2_ERR_ARG;
    snprintf(buf, len, "%s", c->err.c_str());
    return 0;
}

}  // extern "C"

// ==================================================================== learned initial guess: training

namespace {

__global__ void k_mlp_stats(const float *data, const int *idx, long n, double *acc)
{
    __shared__ double s[2 * 18];
    for (int e = threadIdx.x; e < 36; e += blockDim.x) s[e] = 0.0;
    __syncthreads();
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        const float *o = data + (long)idx[k] * kMlpSample;
        for (int c = 0; c < 18; c++) {
            const double v = o[c];
            atomicAdd(&s[c], v);
            atomicAdd(&s[18 + c], v * v);
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 36; e += blockDim.x) atomicAdd(&acc[e], s[e]);
}

}  // namespace

struct gb2_mlp_ctx {
    std::string err;
    cudaStream_t st = nullptr;
    Buf<float> data, P, G, m, v, loss;
    Buf<int> idx;
    Buf<double> acc, maxd;
    Buf<long long> stats;
    std::vector<int> hidx;
    long nsamples = 0, nvalid = 0;
    long adam_t = 0;
    std::mt19937_64 rng{12345};
};

namespace {
int mlp_err(gb2_mlp_ctx *c, int code, const char *msg)
{
    c->err = msg;
    return code;
}
#define MLCK(call)                                                                                                \
    do {                                                                                                          \
        cudaError_t e_ = (call);                                                                                  \
        if (e_ != cudaSuccess) return mlp_err(c, GB2_ERR_CUDA, cudaGetErrorString(e_));                          \
    } while (0)
}  // namespace

extern "C" {

int gb2_mlp_create(int device, gb2_mlp_ctx **out)
{
    if (!out) return GB2_ERR_ARG;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return GB2_ERR_CUDA;
    gb2_mlp_ctx *c = new gb2_mlp_ctx();
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess || c->P.alloc(kMlpSize) ||
        c->G.alloc(kMlpSize) || c->m.alloc(kMlpSize) || c->v.alloc(kMlpSize) || c->loss.alloc(1) ||
        c->acc.alloc(36) || c->maxd.alloc(1) || c->stats.alloc(16) ||
        cudaFuncSetAttribute(k_mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem)) !=
            cudaSuccess) {
        delete c;
        return GB2_ERR_CUDA;
    }
    *out = c;
    return 0;
}

int gb2_mlp_destroy(gb2_mlp_ctx *c)
{
    if (!c) return 0;
    cudaStreamSynchronize(c->st);
    cudaStream_t st = c->st;
    delete c;
    if (st) cudaStreamDestroy(st);
    return 0;
}

// n random near-contact pairs labelled by the plain solver; out[0] valid
// samples, out[1] mean Newton iterations, out[2] mean solves per sample
int gb2_mlp_make_data(gb2_mlp_ctx *c, long n, unsigned long long seed, double *out)
{
    if (!c || n <= 0 || !out) return GB2_ERR_ARG;
    MLCK(c->data.alloc((size_t)n * kMlpSample));
    k_mlp_make<<<nb(n), kB, 0, c->st>>>(seed, n, c->data.p);
    MLCK(cudaGetLastError());
    std::vector<float> h((size_t)n * kMlpSample);
    MLCK(cudaMemcpyAsync(h.data(), c->data.p, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, c->st));
    MLCK(cudaStreamSynchronize(c->st));
    c->hidx.clear();
    double it = 0, sv = 0;
    for (long k = 0; k < n; k++) {
        const float *o = &h[(size_t)k * kMlpSample];
        if (o[21] != 1.f) continue;
        c->hidx.push_back((int)k);
        it += o[18];
        sv += o[19];
    }
    c->nsamples = n;
    c->nvalid = (long)c->hidx.size();
    if (c->nvalid == 0) return mlp_err(c, GB2_ERR_STATE, "no valid samples");
    MLCK(c->idx.alloc(c->nvalid));
    MLCK(cudaMemcpyAsync(c->idx.p, c->hidx.data(), sizeof(int) * c->nvalid, cudaMemcpyHostToDevice, c->st));
    MLCK(cudaStreamSynchronize(c->st));
    out[0] = (double)c->nvalid;
    out[1] = it / c->nvalid;
    out[2] = sv / c->nvalid;
    return 0;
}

// normalisation statistics from the data, He-uniform weights, zero biases
int gb2_mlp_init(gb2_mlp_ctx *c, unsigned long long seed)
{
    if (!c || c->nvalid == 0) return GB2_ERR_STATE;
    MLCK(cudaMemsetAsync(c->acc.p, 0, sizeof(double) * 36, c->st));
    k_mlp_stats<<<nb(c->nvalid), kB, 0, c->st>>>(c->data.p, c->idx.p, c->nvalid, c->acc.p);
    MLCK(cudaGetLastError());
    double acc[36];
    MLCK(cudaMemcpyAsync(acc, c->acc.p, sizeof acc, cudaMemcpyDeviceToHost, c->st));
    MLCK(cudaStreamSynchronize(c->st));
    std::vector<float> P(kMlpSize, 0.f);
    for (int k = 0; k < 18; k++) {
        const double mean = acc[k] / c->nvalid;
        const double var = std::max(acc[18 + k] / c->nvalid - mean * mean, 0.0);
        const double sd = std::sqrt(var) > 1e-6 ? std::sqrt(var) : 1.0;
        if (k < kMlpIn) {
            P[k] = (float)mean;
            P[kMlpIn + k] = (float)sd;
        } else {
            P[2 * kMlpIn + (k - kMlpIn)] = (float)mean;
            P[2 * kMlpIn + kMlpOut + (k - kMlpIn)] = (float)sd;
        }
    }
    std::mt19937_64 g(seed);
    auto fill = [&](int off, int nout, int nin) {
        const float lim = std::sqrt(6.0f / nin);
        std::uniform_real_distribution<float> U(-lim, lim);
        for (int e = 0; e < nout * nin; e++) P[off + e] = U(g);
    };
    fill(kMlpOffW1, kMlpH, kMlpIn);
    fill(kMlpOffW2, kMlpH, kMlpH);
    fill(kMlpOffW3, kMlpH, kMlpH);
    fill(kMlpOffW4, kMlpOut, kMlpH);
    MLCK(cudaMemcpyAsync(c->P.p, P.data(), sizeof(float) * kMlpSize, cudaMemcpyHostToDevice, c->st));
    MLCK(cudaMemsetAsync(c->m.p, 0, sizeof(float) * kMlpSize, c->st));
    MLCK(cudaMemsetAsync(c->v.p, 0, sizeof(float) * kMlpSize, c->st));
    MLCK(cudaStreamSynchronize(c->st));
    c->adam_t = 0;
    c->rng.seed(seed ^ 0x5DEECE66Dull);
    return 0;
}

// epochs of shuffled mini-batches with Adam; loss[0] = first batch, loss[1] =
// mean over the last epoch
int gb2_mlp_train(gb2_mlp_ctx *c, int epochs, int batch, float lr, float *loss)
{
    if (!c || epochs <= 0 || batch <= 0 || !loss || c->nvalid == 0) return GB2_ERR_ARG;
    const int rows_per_cta = kWarps * kTile;
    double last = 0;
    long nlast = 0;
    loss[0] = -1.f;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(c->hidx.begin(), c->hidx.end(), c->rng);
        MLCK(cudaMemcpyAsync(c->idx.p, c->hidx.data(), sizeof(int) * c->nvalid, cudaMemcpyHostToDevice, c->st));
        std::vector<float> losses;
        for (long b0 = 0; b0 + batch <= c->nvalid; b0 += batch) {
            MLCK(cudaMemsetAsync(c->G.p, 0, sizeof(float) * kMlpSize, c->st));
            MLCK(cudaMemsetAsync(c->loss.p, 0, sizeof(float), c->st));
            const int ncta = (batch + rows_per_cta - 1) / rows_per_cta;
            k_mlp_fwd_bwd<<<ncta, 128, sizeof(MlpSmem), c->st>>>(c->P.p, c->data.p, c->idx.p + b0, batch, c->G.p,
                                                                   c->loss.p);
            MLCK(cudaGetLastError());
            c->adam_t++;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.f - std::pow(b1, (float)c->adam_t), c2 = 1.f - std::pow(b2, (float)c->adam_t);
            k_mlp_adam<<<nb(kMlpSize - kMlpOffW1), kB, 0, c->st>>>(c->P.p, c->G.p, c->m.p, c->v.p, kMlpSize, lr, b1,
                                                                  b2, 1e-8f, c1, c2);
            MLCK(cudaGetLastError());
            if (ep == epochs - 1 || loss[0] < 0) {
                float l;
                MLCK(cudaMemcpyAsync(&l, c->loss.p, sizeof(float), cudaMemcpyDeviceToHost, c->st));
                MLCK(cudaStreamSynchronize(c->st));
                if (loss[0] < 0) loss[0] = l;
                if (ep == epochs - 1) {
                    last += l;
                    nlast++;
                }
            }
        }
    }
    MLCK(cudaStreamSynchronize(c->st));
    loss[1] = nlast ? (float)(last / nlast) : loss[0];
    return 0;
}

int gb2_mlp_get_params(gb2_mlp_ctx *c, float *out, int n)
{
    if (!c || !out || n != kMlpSize) return GB2_ERR_ARG;
    MLCK(cudaMemcpyAsync(out, c->P.p, sizeof(float) * kMlpSize, cudaMemcpyDeviceToHost, c->st));
    MLCK(cudaStreamSynchronize(c->st));
    return 0;
}

int gb2_mlp_set_params(gb2_mlp_ctx *c, const float *in, int n)
{
    if (!c || !in || n != kMlpSize) return GB2_ERR_ARG;
    MLCK(cudaMemcpyAsync(c->P.p, in, sizeof(float) * kMlpSize, cudaMemcpyHostToDevice, c->st));
    MLCK(cudaStreamSynchronize(c->st));
    return 0;
}

// one forward + backward pass over caller-given samples (kMlpSample floats
// each: features 0..13, targets 14..17): loss and the full gradient
int gb2_mlp_grad(gb2_mlp_ctx *c, int nrows, const float *samples, float *loss, float *grad)
{
    if (!c || nrows <= 0 || !samples || !loss || !grad) return GB2_ERR_ARG;
    Buf<float> d;
    Buf<int> ix;
    MLCK(d.alloc((size_t)nrows * kMlpSample));
    MLCK(ix.alloc(nrows));
    std::vector<int> h(nrows);
    for (int k = 0; k < nrows; k++) h[k] = k;
    MLCK(cudaMemcpyAsync(d.p, samples, sizeof(float) * nrows * kMlpSample, cudaMemcpyHostToDevice, c->st));
    MLCK(cudaMemcpyAsync(ix.p, h.data(), sizeof(int) * nrows, cudaMemcpyHostToDevice, c->st));
    MLCK(cudaMemsetAsync(c->G.p, 0, sizeof(float) * kMlpSize, c->st));
    MLCK(cudaMemsetAsync(c->loss.p, 0, sizeof(float), c->st));
    const int ncta = (nrows + kWarps * kTile - 1) / (kWarps * kTile);
    k_mlp_fwd_bwd<<<ncta, 128, sizeof(MlpSmem), c->st>>>(c->P.p, d.p, ix.p, nrows, c->G.p, c->loss.p);
    MLCK(cudaGetLastError());
    MLCK(cudaMemcpyAsync(grad, c->G.p, sizeof(float) * kMlpSize, cudaMemcpyDeviceToHost, c->st));
    MLCK(cudaMemcpyAsync(loss, c->loss.p, sizeof(float), cudaMemcpyDeviceToHost, c->st));
    MLCK(cudaStreamSynchronize(c->st));
    return 0;
}

// learned guess against the plain method on n fresh pairs; stats[9]:
// pairs, plain iterations, plain solves, learned iterations, learned solves,
// learned guesses accepted, plain failures, learned failures, converged more
// than 1e-4 of the size apart; maxdiff = largest point difference / smallest half-axis
int gb2_mlp_evaluate(gb2_mlp_ctx *c, long n, unsigned long long seed, long long *stats, double *maxdiff)
{
    if (!c || n <= 0 || !stats || !maxdiff) return GB2_ERR_ARG;
    MLCK(cudaMemsetAsync(c->stats.p, 0, sizeof(long long) * 16, c->st));
    MLCK(cudaMemsetAsync(c->maxd.p, 0, sizeof(double), c->st));
    k_mlp_eval<<<nb(n), kB, 0, c->st>>>(seed, n, c->P.p, c->stats.p, c->maxd.p);
    MLCK(cudaGetLastError());
    MLCK(cudaMemcpyAsync(stats, c->stats.p, sizeof(long long) * 9, cudaMemcpyDeviceToHost, c->st));
    MLCK(cudaMemcpyAsync(maxdiff, c->maxd.p, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    MLCK(cudaStreamSynchronize(c->st));
    return 0;
}

int gb2_mlp_time_solves(gb2_mlp_ctx *c, long n, unsigned long long seed, double *ms_plain, double *ms_learned,
                        long long *counts)
{
    if (!c || n <= 0 || n > (1L << 24) || !ms_plain || !ms_learned || !counts) return GB2_ERR_ARG;
    Buf<PairSample> pairs;
    Buf<double> pt;
    Buf<int> nv, rej;
    Buf<long long> it;
    MLCK(pairs.alloc(n));
    MLCK(pt.alloc(3 * n));
    MLCK(nv.alloc(2));
    MLCK(rej.alloc(n));
    MLCK(it.alloc(2));
    MLCK(cudaMemsetAsync(nv.p, 0, 2 * sizeof(int), c->st));
    MLCK(cudaMemsetAsync(it.p, 0, 2 * sizeof(long long), c->st));
    k_mlp_store_pairs<<<nb(n), kB, 0, c->st>>>(seed, n, pairs.p, nv.p);
    MLCK(cudaGetLastError());
    cudaEvent_t e[3];
    for (auto &x : e) MLCK(cudaEventCreate(&x));
    // one untimed round of each method (code and data warm), then the timed one
    for (int round = 0; round < 2; round++) {
        MLCK(cudaMemsetAsync(it.p, 0, 2 * sizeof(long long), c->st));
        MLCK(cudaEventRecord(e[0], c->st));
        k_mlp_solve<false><<<nb(n), kB, 0, c->st>>>(pairs.p, nv.p, c->P.p, pt.p, it.p, nullptr, nullptr);
        MLCK(cudaEventRecord(e[1], c->st));
        MLCK(cudaMemsetAsync(nv.p + 1, 0, sizeof(int), c->st));
        k_mlp_solve<true><<<nb(n), kB, 0, c->st>>>(pairs.p, nv.p, c->P.p, pt.p, it.p + 1, rej.p, nv.p + 1);
        k_mlp_solve_rejected<<<nb(n), kB, 0, c->st>>>(pairs.p, rej.p, nv.p + 1, pt.p, it.p + 1);
        MLCK(cudaEventRecord(e[2], c->st));
    }
    MLCK(cudaGetLastError());
    int hv[2] = {0, 0};
    MLCK(cudaMemcpyAsync(hv, nv.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
    MLCK(cudaMemcpyAsync(counts + 1, it.p, 2 * sizeof(long long), cudaMemcpyDeviceToHost, c->st));
    MLCK(cudaStreamSynchronize(c->st));
    float a = 0.f, b = 0.f;
    MLCK(cudaEventElapsedTime(&a, e[0], e[1]));
    MLCK(cudaEventElapsedTime(&b, e[1], e[2]));
    for (auto &x : e) cudaEventDestroy(x);
    counts[0] = hv[0];
    *ms_plain = a;
    *ms_learned = b;
    return 0;
}

int gb2_mlp_last_error(gb2_mlp_ctx *c, char *buf, int len)
{
    if (!c || !buf || len <= 0) return GB2_ERR_ARG;
    snprintf(buf, len, "%s", c->err.c_str());
    return 0;
}

}  // extern "C"
