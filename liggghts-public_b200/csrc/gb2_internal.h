// gb2_internal.h -- device data layout and kernel interfaces of libgranb200.
//
// Layout in HBM (capacities in parentheses):
//   per atom (nmax = owned + ghost images), 32-byte records so one sector
//   serves a neighbour gather:
//     pos  {x, y, z, radius}      vel {vx, vy, vz, rmass}
//     omg  {wx, wy, wz, -}        type, tag (int32)
//   per owned atom:
//     f, tq {., ., ., -}          force / torque of the last step
//     tail[w]                     atoms finished by the tail kernel (wall candidates or
//                                 more than 64 entries on a side), listed at each build
//     tailf, tailt                their pair sums, left by the pair step kernel
//     xhold {x, y, z, -}          positions at the last neighbour build
//   half neighbour list, slot-major so a warp reads consecutive atoms
//   (capacity maxn slots per owned atom, stride `cap`):
//     nnum[i], nbr[s*cap+i] (j index), flag[s*cap+i] (contact flag bits),
//     hist[(3s+c)*cap+i] (shear history, FP64)
//   reverse list (entries where the atom is the j side, ascending owner):
//     rnum[k], rev[r*cap+k] = owner i', revs[r*cap+k] = its slot s'
//   contact-history partners (FixContactHistory::partner_, keyed by tag):
//     pnum[i], ptag[s*cap+i], phist[(3s+c)*cap+i]
//   ghosts: gsrc[g] (owned source atom), gshift[g] {dx, dy, dz, -}
//   split precision: kin {vx, vy, vz, m, wx, wy, wz, -} as FP32 (32 bytes),
//     the neighbour-side operands of the FP32 contact math
#pragma once

#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "gb2_contact.cuh"

namespace gb2 {

struct __align__(32) dbl4 {
    double x, y, z, w;
};

// split-precision kinematics record of one atom (one 32-byte sector):
// velocity, mass and angular velocity rounded to FP32 for the contact math
struct __align__(32) flt8 {
    float vx, vy, vz, m;
    float wx, wy, wz, pad;
};

constexpr int kMaxTypes = 8;      // material table is [kMaxTypes+1]^2
constexpr int kMaxFix = 16;
constexpr int kNeighMax = 5;      // TriMesh = SurfaceMesh<3,5>

// status bits written by device code
enum : int {
    ST_NEIGH_OVERFLOW = 1 << 0,
    ST_PARTNER_OVERFLOW = 1 << 1,
    ST_MESHSLOT_OVERFLOW = 1 << 2,
    ST_LOST_ATOM = 1 << 3,
    ST_REV_OVERFLOW = 1 << 4,
    ST_MESH_INTERNAL = 1 << 5,
    ST_MESH_OUTSIDE_GRID = 1 << 6,
};

enum FixKind : int { FIX_NONE = 0, FIX_GRAVITY = 1, FIX_WALL_PLANE = 2, FIX_WALL_MESH = 3 };

// one triangle, as the narrow phase reads it (all FP64)
struct TriGeom {
    double node[3][3];
    double edgevec[3][3];
    double edgelen[3];
    double edgenorm[3][3];
    double surfnorm[3];
    double center[3];
    double rbound;
    int obtuse;            // obtuse-angle node or -1
    int active;            // bits 0-2 edge active, bits 3-5 corner active
};

struct MeshDev {
    int ntri;
    const TriGeom *tri;
    // coplanar node-neighbour relation (areCoplanarNodeNeighs), CSR sorted
    const int *cnn_start;
    const int *cnn_list;
    // bin -> triangles whose precomputed bin list contains the bin (ascending)
    const int *bin_tri_start;
    const int *bin_tri_list;
    double nl_skin;        // FixNeighlistMesh skin (0.5 * neighbor skin, static mesh)
    int wtype;
    int rolling;
    // per owned atom: candidate triangles (ascending) and contact slots
    int maxt;              // slot capacity per atom
    int *tcnt;             // fix_nneighs
    int *tlist;            // [s*cap + i]
    int *snp;              // npartner
    int *spartner;         // [s*cap + i] triangle id or -1
    double *shist;         // [(3s+c)*cap + i]
    const double *vnode;   // moving mesh: node velocities [9*t + 3*node + c]; null when static
    // mesh/surface/stress: per-element force [3t+c] and f_total, torque_total
    // about pref of the current step; null when not tracked
    double *trif, *ftot;
    double pref[3];
    // Finnie wear (null when not tracked): cumulative per element, element
    // area as created, k_finnie of the wall type against each atom type
    double *wear;
    const double *tarea, *kfin;
};

struct FixDev {
    int kind;
    double acc[3];         // gravity
    int dim;               // plane: axis; cylinder: axis direction
    double pos;
    int cyl;               // 1: {x,y,z}cylinder
    double cr, cc1, cc2;   // cylinder radius and axis position (the other two coordinates, cyclic order)
    int wtype;
    int rolling;
    uint8_t *inlist;       // primitive-wall neighbour flag per owned atom
    double *whist;         // [c*cap + i]
    MeshDev mesh;
};

// everything a step kernel needs, passed by value
struct Dev {
    int nlocal, nghost, nmax, cap;   // cap: stride of slot-major arrays (>= nlocal)
    dbl4 *pos, *vel, *omg;
    dbl4 *pos_out, *vel_out, *omg_out;   // integrate targets (double buffer: pass B reads neighbours' state)
    flt8 *kin, *kin_out;                 // split precision only (null in the FP64 path)
    int *type, *tag;
    dbl4 *f, *tq, *tailf, *tailt, *xhold;
    int *tail, *tailcnt;   // tail-kernel atom list and its length
    // half list
    int maxn;
    int item_cap;          // per-warp list capacity of the pair step's listed rounds (<= kItemCap)
    int *nnum, *nbr, *flag;
    double *hist;          // shear read buffer (current values)
    double *hist_out;      // shear write buffer of the pair step
    unsigned long long *prevmask;   // own slots touching in the previous step
    // reverse list
    int maxr;
    int *rnum, *rev;       // rev[r*cap+k] = owner index i of the pair
    uint8_t *revs;         // revs[r*cap+k] = slot s of the pair in i's list
    // partners
    int maxp;
    int *pnum, *ptag;
    double *phist;
    // ghosts
    int *gsrc;
    dbl4 *gshift;
    // bins
    double bboxlo[3], bboxhi[3], bininv[3], binsize[3];
    int nbin[3], mbinlo[3], mbin[3], mbins;
    int nstencil;
    const int *stencil;
    int nsrow;               // the stencil as runs of consecutive bins {first offset, bins}
    const int2 *srow;
    const int *bin_start;    // [mbins+1]
    const int *bin_atoms;    // atoms sorted by bin, ascending index within a bin
    // materials [(kMaxTypes+1)^2]
    const MatPair *mat;
    int ntypes;
    // physics
    double dt, skin, cutneighmax, triggersq;
    int rolling, tdamp;
    // fixes
    int nfix;
    FixDev fix[kMaxFix];
    int *status;
    int *dflag;              // displacement trigger
    int *dstop;              // queued-ahead steps: lowest step whose tail asked for a rebuild (null when not queuing)
    int step;                // step number of this launch (compared with *dstop)
    const dbl4 *rel;         // fix insert/stream release data [4*cap] (null without a stream):
                             // {x_ins, i_step} {v_int, r_step} {v_release, -} {omega_release, -}
    int *need;               // [5] capacity demand seen by the last overflowing kernel:
                             // neighbour slots, partners, reverse entries, mesh slots;
                             // [4] pair-step warps whose item lists were too short
};

// host-side mesh topology (gb2_mesh.cpp)
struct MeshTopo {
    std::vector<TriGeom> tri;
    std::vector<int> cnn_start, cnn_list;       // coplanar node neighbours, CSR
    std::vector<std::vector<int>> edge_neigh;   // elements sharing an edge
};
bool build_mesh_topology(const double *nodes, int ntri_in, double curvature, double precision, MeshTopo &out,
                         std::string &err);
// split-precision pair step (gb2_split.cu)
void launch_pair_split(const Dev &D, int nblocks, cudaStream_t st, int minb, int shearupdate, int integrate,
                       int fuse_next, int store_f, size_t smem);
void launch_tail_split(const Dev &D, int nblocks, cudaStream_t st, int shearupdate, int integrate, int fuse_next,
                       int store_f);
bool tri_neighbuild_host(const TriGeom &T, double rSphere, const double *c, double treshold);
// Small page-locked host words (flags and counts read back from the device)
// in 256-byte slots of a process-wide arena: locking host pages costs
// milliseconds per allocation, so contexts take a slot instead of locking
// their own pages.  The arena's pages stay locked until the process exits.
constexpr size_t kPinnedSlot = 256;
int pinned_slot_get(int **slot);
void pinned_slot_put(int *slot);

}  // namespace gb2
