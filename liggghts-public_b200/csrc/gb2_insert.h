// fix insert/pack over a region block with a particledistribution/discrete
// of constant-radius particletemplate/sphere templates: the host side of
// particle insertion.  The engine gathers, on the device, the particles in
// the region and the ones near it (InsertRegion below is shared with those
// kernels); this file draws the reference's random numbers in the reference's
// order and places the particles one by one.
//
// Behaviour followed:
//   RanPark::uniform / gaussian          src/random_park.cpp:56-91
//   Random::Random seed checks            src/random.cpp:55-95
//   RegBlock inside / surface_interior / surface_exterior
//                                         src/region_block.cpp:147-259
//   Region::generate_random(_shrinkby_cut), match_cut, match_expandby_cut,
//   volume_mc                             src/region.cpp:531-703
//   FixTemplateSphere volume / mass expectancy, randomize_ptilist
//                                         src/fix_template_sphere.cpp:244-245, 333-361
//   FixParticledistributionDiscrete weights, order, randomize_list
//                                         src/fix_particledistribution_discrete.cpp:130-240, 398-480
//   FixInsert::pre_exchange, distribute_ninsert_this, load_xnear,
//   generate_random_velocity              src/fix_insert.cpp:652-972
//   FixInsertPack::calc_insertion_properties, calc_ninsert_this,
//   is_nearby, getBoundingBox, calc_maxtry, x_v_omega
//                                         src/fix_insert_pack.cpp:199-514
//   RegionNeighborList::hasOverlap (rsq <= radsum^2)
//                                         src/region_neighbor_list_I.h:72-97
#pragma once

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/granb200.h"
#include "gb2_internal.h"

#ifdef __CUDACC__
#define GB2_HD __host__ __device__
#else
#define GB2_HD
#endif

namespace gb2 {

// insertion region (interior side: a block, or a cylinder whose extents are
// lo/hi) and the bounding box of the near-particle list
struct InsertRegion {
    double lo[3], hi[3];     // block, or the cylinder's extents
    double blo[3], bhi[3];   // FixInsertPack::getBoundingBox: region within the box, widened by 2 maxrad
    double maxrad;
    int all_in;
    int cyl;                 // 0 block, 1 cylinder
    int ax, a1, a2;          // cylinder axis and the other two coordinates in x, y, z order
    double c1, c2, rad, clo, chi;

    GB2_HD bool inside(const double *x) const
    {
        if (cyl) {   // RegCylinder::inside
            const double del1 = x[a1] - c1, del2 = x[a2] - c2;
            const double dist = sqrt(del1 * del1 + del2 * del2);
            return dist <= rad && x[ax] >= clo && x[ax] <= chi;
        }
        return x[0] >= lo[0] && x[0] <= hi[0] && x[1] >= lo[1] && x[1] <= hi[1] && x[2] >= lo[2] && x[2] <= hi[2];
    }
    // RegBlock / RegCylinder::surface_interior != 0: inside and closer than cut to a face
    GB2_HD bool surface_interior(const double *x, double cut) const
    {
        if (cyl) {
            const double del1 = x[a1] - c1, del2 = x[a2] - c2;
            const double r = sqrt(del1 * del1 + del2 * del2);
            if (r > rad || x[ax] < clo || x[ax] > chi) return false;
            return (rad - r < cut && r > 0.0) || x[ax] - clo < cut || chi - x[ax] < cut;
        }
        if (x[0] < lo[0] || x[0] > hi[0] || x[1] < lo[1] || x[1] > hi[1] || x[2] < lo[2] || x[2] > hi[2])
            return false;
        for (int d = 0; d < 3; d++)
            if (x[d] - lo[d] < cut || hi[d] - x[d] < cut) return true;
        return false;
    }
    // RegBlock / RegCylinder::surface_exterior != 0: outside (or on the surface) and closer than cut
    GB2_HD bool surface_exterior(const double *x, double cut) const
    {
        if (cyl) {
            const double del1 = x[a1] - c1, del2 = x[a2] - c2;
            const double r = sqrt(del1 * del1 + del2 * del2);
            if (r >= rad + cut || x[ax] <= clo - cut || x[ax] >= chi + cut) return false;
            if (r < rad && x[ax] > clo && x[ax] < chi) return false;
            double p[3];
            if (r > rad) {
                p[a1] = c1 + del1 * rad / r;
                p[a2] = c2 + del2 * rad / r;
            } else {
                p[a1] = x[a1];
                p[a2] = x[a2];
            }
            p[ax] = x[ax] < clo ? clo : (x[ax] > chi ? chi : x[ax]);
            const double dx = x[0] - p[0], dy = x[1] - p[1], dz = x[2] - p[2];
            return sqrt(dx * dx + dy * dy + dz * dz) < cut;
        }
        if (x[0] <= lo[0] - cut || x[0] >= hi[0] + cut || x[1] <= lo[1] - cut || x[1] >= hi[1] + cut ||
            x[2] <= lo[2] - cut || x[2] >= hi[2] + cut)
            return false;
        if (x[0] > lo[0] && x[0] < hi[0] && x[1] > lo[1] && x[1] < hi[1] && x[2] > lo[2] && x[2] < hi[2])
            return false;
        double p[3];
        for (int d = 0; d < 3; d++) p[d] = x[d] < lo[d] ? lo[d] : (x[d] > hi[d] ? hi[d] : x[d]);
        const double dx = x[0] - p[0], dy = x[1] - p[1], dz = x[2] - p[2];
        return sqrt(dx * dx + dy * dy + dz * dz) < cut;
    }
    // FixInsertPack::is_nearby and RegionNeighborList::isInBoundingBox
    GB2_HD bool near(const double *x, double rad) const
    {
        const double cut = all_in ? maxrad : rad + maxrad;
        if (!(inside(x) || surface_exterior(x, cut))) return false;
        return x[0] >= blo[0] && x[0] <= bhi[0] && x[1] >= blo[1] && x[1] <= bhi[1] && x[2] >= blo[2] &&
               x[2] <= bhi[2];
    }
};

// Park-Miller minimal standard generator with Schrage's factorisation
struct ParkRandom {
    int seed = 1;
    int save = 0;
    double second = 0.0;
    void reset(int s)
    {
        seed = s;
        save = 0;
    }
    double uniform()
    {
        const int k = seed / 127773;
        seed = 16807 * (seed - k * 127773) - 2836 * k;
        if (seed < 0) seed += 2147483647;
        return (1.0 / 2147483647) * seed;
    }
    // polar Box-Muller, one pair per two calls
    double gaussian()
    {
        double first;
        if (!save) {
            double v1, v2, rsq;
            for (;;) {
                v1 = 2.0 * uniform() - 1.0;
                v2 = 2.0 * uniform() - 1.0;
                rsq = v1 * v1 + v2 * v2;
                if (rsq < 1.0 && rsq != 0.0) break;
            }
            const double fac = std::sqrt(-2.0 * std::log(rsq) / rsq);
            second = v1 * fac;
            first = v2 * fac;
            save = 1;
        } else {
            first = second;
            save = 0;
        }
        return first;
    }
};

inline bool insert_seed_ok(int seed)
{
    if (seed < 10000) return false;
    for (long d = 2; d * d <= seed; d++)
        if (seed % d == 0) return false;
    return true;
}

struct InsertedParticle {
    double x[3], v[3], omega[3];
    double radius, density, mass;
    int type;
};

// a particle the overlap test sees (existing or accepted this step)
struct NearParticle {
    double x[3], r;
};

class InsertPack {
public:
    gb2_insert_pack P{};
    InsertRegion R{};
    double boxlo[3] = {0, 0, 0}, boxhi[3] = {0, 0, 0};
    double distweight[GB2_INSERT_MAX_TEMPLATES] = {};
    // radius distributions: bounds, uniform's h1/h2, cubic expectancy
    double rmin[GB2_INSERT_MAX_TEMPLATES] = {}, rmax[GB2_INSERT_MAX_TEMPLATES] = {};
    double h1[GB2_INSERT_MAX_TEMPLATES] = {}, h2[GB2_INSERT_MAX_TEMPLATES] = {};
    ParkRandom rtmpl[GB2_INSERT_MAX_TEMPLATES];   // each template's random_insertion
    double tvol[GB2_INSERT_MAX_TEMPLATES] = {}, tmass[GB2_INSERT_MAX_TEMPLATES] = {};
    int distorder[GB2_INSERT_MAX_TEMPLATES] = {};
    double volexpect = 0, massexpect = 0, maxrad = 0, maxrbound = 0;
    double region_volume = 0, region_volume_local = 0, insertion_ratio = 0;
    long next_reneighbor = 0, most_recent = -1;
    long ninserted = 0;
    double massinserted = 0;
    bool props_done = false;
    ParkRandom rnd, rreg, rdist;   // fix insert, its region, the distribution

    // constructor checks of the three commands; returns an error message or ""
    std::string init(const gb2_insert_pack &p, const double lo[3], const double hi[3], int ntypes, long ntimestep)
    {
        P = p;
        for (int d = 0; d < 3; d++) {
            boxlo[d] = lo[d];
            boxhi[d] = hi[d];
        }
        if (!insert_seed_ok(P.seed) || !insert_seed_ok(P.dist_seed))
            return "random seeds must be prime numbers > 10000";
        if (P.ntemplates < 1 || P.ntemplates > GB2_INSERT_MAX_TEMPLATES) return "illegal number of templates";
        if (P.maxattempt <= 0 || P.ntry_mc <= 0) return "maxattempt and ntry_mc must be positive";
        if (P.insert_every < 0) return "insert_every must be >= 0";
        if (P.vel_style < 0 || P.vel_style > 2) return "vel style must be constant, uniform or gaussian";
        int n_defined = (P.volumefraction_region > 0.) + (P.particles_in_region > 0) + (P.mass_in_region > 0.);
        if (n_defined != 1)
            return "must define exactly one keyword out of 'volumefraction_region', 'particles_in_region', and "
                   "'mass_in_region'";
        if (P.volumefraction_region < 0. || P.volumefraction_region > 1.) return "illegal volumefraction_region";
        if (P.region_style == 1) {   // cylinder: extents as RegCylinder's bounding box
            if (P.cyl_axis < 0 || P.cyl_axis > 2 || !(P.cyl_radius > 0.) || !(P.cyl_lo < P.cyl_hi))
                return "illegal region cylinder";
            const int ax = P.cyl_axis, a1 = ax == 0 ? 1 : 0, a2 = ax == 2 ? 1 : 2;
            P.region_lo[ax] = P.cyl_lo;
            P.region_hi[ax] = P.cyl_hi;
            P.region_lo[a1] = P.cyl_c1 - P.cyl_radius;
            P.region_hi[a1] = P.cyl_c1 + P.cyl_radius;
            P.region_lo[a2] = P.cyl_c2 - P.cyl_radius;
            P.region_hi[a2] = P.cyl_c2 + P.cyl_radius;
            R.cyl = 1;
            R.ax = ax;
            R.a1 = a1;
            R.a2 = a2;
            R.c1 = P.cyl_c1;
            R.c2 = P.cyl_c2;
            R.rad = P.cyl_radius;
            R.clo = P.cyl_lo;
            R.chi = P.cyl_hi;
        } else if (P.region_style != 0) {
            return "region style must be block or cylinder";
        }
        for (int d = 0; d < 3; d++)
            if (!(P.region_lo[d] < P.region_hi[d])) return "empty region";
        const int nt = P.ntemplates;
        for (int i = 0; i < nt; i++) {
            if (P.tmpl_type[i] < 1 || P.tmpl_type[i] > ntypes) return "template atom type out of range";
            if (!(P.tmpl_radius[i] > 0.) || !(P.tmpl_density[i] > 0.)) return "template radius and density > 0";
            if (P.tmpl_weight[i] < 0) return "invalid weight";
            if (!insert_seed_ok(P.tmpl_seed[i])) return "template seeds must be prime numbers > 10000";
            rtmpl[i].reset(P.tmpl_seed[i]);
            // ProbabilityDistribution set_params / cubic_expectancy
            const double r = P.tmpl_radius[i], r2 = P.tmpl_radius2[i];
            double cube;
            if (P.tmpl_radius_style[i] == 0) {
                rmin[i] = rmax[i] = r;
                cube = r * r * r;
            } else if (P.tmpl_radius_style[i] == 1) {
                if (!(r2 > r)) return "uniform radius distribution needs max > min";
                rmin[i] = r;
                rmax[i] = r2;
                h1[i] = 2. / (1. / (r * r) - 1. / (r2 * r2));
                h2[i] = h1[i] / (2. * r * r);
                cube = 0.25 * (r2 * r2 * r2 + r2 * r2 * r + r2 * r * r + r * r * r);
            } else if (P.tmpl_radius_style[i] == 2) {
                if (!(r2 > 0.)) return "gaussian radius distribution needs sigma > 0";
                rmin[i] = r - 3. * r2;
                rmax[i] = r + 3. * r2;
                if (rmin[i] < 0.) return "Probablity distribution: mu-3*sigma < 0, please increase mu or decrease sigma";
                cube = r * (r * r + 3 * r2 * r2);
            } else {
                return "radius distribution must be constant, uniform or gaussian";
            }
            // FixTemplateSphere: volume_expect = cubic expectancy * 4 pi / 3, mass_expect = density * volume
            tvol[i] = cube * 4. * M_PI / 3.;
            tmass[i] = P.tmpl_density[i] * tvol[i];
            if (tvol[i] < 1e-12) return "Volume expectancy too small";
            distweight[i] = P.tmpl_weight[i];
        }
        double weightsum = 0;
        for (int i = 0; i < nt; i++) weightsum += distweight[i];
        for (int i = 0; i < nt; i++) distweight[i] /= weightsum;
        if (P.dist_mass_based) {
            for (int i = 0; i < nt; i++) distweight[i] = distweight[i] / tmass[i];
            weightsum = 0;
            for (int i = 0; i < nt; i++) weightsum += distweight[i];
            for (int i = 0; i < nt; i++) distweight[i] /= weightsum;
        }
        volexpect = massexpect = 0.;
        for (int i = 0; i < nt; i++) {
            volexpect += tvol[i] * distweight[i];
            massexpect += tmass[i] * distweight[i];
        }
        // templates by volume, descending (the reference's bubble sort)
        for (int i = 0; i < nt; i++) distorder[i] = i;
        bool swapped;
        int n = nt;
        do {
            swapped = false;
            for (int i = 0; i < nt - 1; i++)
                if (tvol[distorder[i]] < tvol[distorder[i + 1]]) {
                    std::swap(distorder[i], distorder[i + 1]);
                    swapped = true;
                }
            n--;
        } while (swapped && n > 0);
        maxrbound = 0.;
        for (int i = 0; i < nt; i++) maxrbound = std::max(maxrbound, rmax[i]);
        maxrad = 0.;
        for (int t = 1; t <= ntypes; t++) maxrad = std::max(maxrad, max_rad(t));
        rnd.reset(P.seed);
        rdist.reset(P.dist_seed);
        long first = P.start > 0 ? P.start : ntimestep + 1;
        if (first < ntimestep + 1) return "'start' step can not be before current step";
        next_reneighbor = first;
        for (int d = 0; d < 3; d++) {
            R.lo[d] = P.region_lo[d];
            R.hi[d] = P.region_hi[d];
        }
        R.all_in = P.all_in;
        R.maxrad = maxrad;
        // FixInsertPack::getBoundingBox: the block shrunk to the (single) subdomain, widened by 2 maxrad
        for (int d = 0; d < 3; d++) {
            double a = R.lo[d], b = R.hi[d];
            if (a < boxlo[d]) a = boxlo[d];
            if (b > boxhi[d]) b = boxhi[d];
            R.blo[d] = a - 2 * maxrad;
            R.bhi[d] = b + 2 * maxrad;
        }
        return "";
    }

    // FixParticledistributionDiscrete::max_rad(type): largest template radius of that type
    double max_rad(int type) const
    {
        double m = 0.;
        for (int i = 0; i < P.ntemplates; i++)
            if (P.tmpl_type[i] == type && rmax[i] > m) m = rmax[i];
        return m;
    }

    // FixInsertPack::calc_insertion_properties (FixInsert::setup, once)
    std::string setup()
    {
        if (props_done) return "";
        props_done = true;
        rreg.reset(P.seed + 12);   // reset_random(seed + SEED_OFFSET)
        // Region::volume_mc(ntry_mc, all_in, max_r_bound)
        const double *lo = P.region_lo, *hi = P.region_hi;
        long n_in_global = 0, n_in_local = 0;
        for (int i = 0; i < P.ntry_mc; i++) {
            double pos[3];
            pos[0] = lo[0] + rreg.uniform() * (hi[0] - lo[0]);
            pos[1] = lo[1] + rreg.uniform() * (hi[1] - lo[1]);
            pos[2] = lo[2] + rreg.uniform() * (hi[2] - lo[2]);
            if (!(pos[0] >= boxlo[0] && pos[0] <= boxhi[0] && pos[1] >= boxlo[1] && pos[1] <= boxhi[1] &&
                  pos[2] >= boxlo[2] && pos[2] <= boxhi[2]))
                continue;
            if (R.inside(pos)) {
                n_in_global++;
                if (!P.all_in || !R.surface_interior(pos, maxrbound)) n_in_local++;
            }
        }
        if (n_in_global == 0) return "Unable to calculate region volume";
        const double vol_bbox = (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
        const double vol_global = static_cast<double>(n_in_global) / static_cast<double>(P.ntry_mc) * vol_bbox;
        double vol_local = static_cast<double>(n_in_local) / static_cast<double>(P.ntry_mc) * vol_bbox;
        const double vol_local_all = vol_local;
        if (vol_local_all < 1.e-10) return "Unable to calculate region volume (too small for all_in)";
        vol_local *= (vol_global / vol_local_all);
        region_volume = vol_global;
        region_volume_local = vol_local;
        if (region_volume <= 0. || region_volume_local < 0. ||
            (region_volume_local - region_volume) / region_volume > 1e-3)
            return "Fix insert: Region volume calculation with MC failed";
        return "";
    }

    bool due(long step) const { return next_reneighbor == step && most_recent != step; }

    // FixParticledistributionDiscrete::randomize_list (particles per
    // template, exact or uncorrelated) and FixTemplateSphere::randomize_ptilist
    // (each particle's radius from its template's generator); the list runs
    // from large to small templates
    void randomize(int nlocal_ins, bool exact, std::vector<int> &plist, std::vector<double> &prad)
    {
        const int nt = P.ntemplates;
        int parttogen[GB2_INSERT_MAX_TEMPLATES];
        if (!exact) {
            for (int i = 0; i < nt; i++)
                parttogen[i] = static_cast<int>(static_cast<double>(nlocal_ins) * distweight[i] + rdist.uniform());
        } else {
            int ntrunc = 0;
            double remainder[GB2_INSERT_MAX_TEMPLATES];
            for (int i = 0; i < nt; i++) {
                parttogen[i] = static_cast<int>(static_cast<double>(nlocal_ins) * distweight[i]);
                ntrunc += parttogen[i];
                remainder[i] = static_cast<double>(nlocal_ins) * distweight[i] - static_cast<double>(parttogen[i]);
            }
            const int gap = nlocal_ins - ntrunc;
            for (int i = 0; i < gap; i++) {
                const double r = rdist.uniform() * static_cast<double>(gap);
                int j = 0;
                double rsum = remainder[0];
                while (rsum < r && j < nt - 1) {
                    j++;
                    rsum += remainder[j];
                }
                parttogen[j]++;
            }
        }
        std::vector<double> rad[GB2_INSERT_MAX_TEMPLATES];
        for (int i = 0; i < nt; i++)
            for (int j = 0; j < parttogen[i]; j++) rad[i].push_back(draw_radius(i));
        plist.clear();
        prad.clear();
        for (int i = 0; i < nt; i++) {
            const int t = distorder[i];
            for (int j = 0; j < parttogen[t]; j++) {
                plist.push_back(t);
                prad.push_back(rad[t][j]);
            }
        }
    }

    // one insertion (FixInsert::pre_exchange on step `step`): rreg_r / rreg_m
    // are radius and mass of the owned particles inside the region in index
    // order, nearp the particles near it; the accepted particles are appended
    // to out.  Returns an error message or "".
    std::string insert(long step, const std::vector<double> &rreg_r, const std::vector<double> &rreg_m,
                       std::vector<NearParticle> nearp, std::vector<InsertedParticle> &out)
    {
        out.clear();
        most_recent = step;
        // FixInsertPack::calc_ninsert_this
        int np_region = (int)rreg_r.size();
        double vol_region = 0., mass_region = 0.;
        const double _4Pi3 = 4. * M_PI / 3.;
        for (int i = 0; i < np_region; i++) {
            vol_region += _4Pi3 * rreg_r[i] * rreg_r[i] * rreg_r[i];
            mass_region += rreg_m[i];
        }
        int ninsert_this = 0;
        if (P.volumefraction_region > 0.) {
            ninsert_this = static_cast<int>((P.volumefraction_region * region_volume - vol_region) / volexpect +
                                            rnd.uniform());
            insertion_ratio = vol_region / (P.volumefraction_region * region_volume);
        } else if (P.particles_in_region > 0) {
            ninsert_this = P.particles_in_region - np_region;
            insertion_ratio = static_cast<double>(np_region) / static_cast<double>(P.particles_in_region);
        } else {
            ninsert_this = static_cast<int>((P.mass_in_region - mass_region) / massexpect + rnd.uniform());
            insertion_ratio = mass_region / P.mass_in_region;
        }
        if (ninsert_this < -200000) return "overflow in particle number calculation";
        if (ninsert_this < 0) ninsert_this = 0;
        if (insertion_ratio < 0.) insertion_ratio = 0.;
        if (insertion_ratio > 1.) insertion_ratio = 1.;
        // distribute_ninsert_this on one process
        const double fraction_local = region_volume_local / region_volume;
        int nlocal_ins;
        if (!P.exact_number) {
            nlocal_ins = static_cast<int>(fraction_local * static_cast<double>(ninsert_this) + rnd.uniform());
        } else {
            double f = fraction_local;
            if (f < 0.02) f = 0.;
            if (f == 0.) return "Internal error distributing particles to processes";
            f /= f;
            nlocal_ins = static_cast<int>(f * static_cast<double>(ninsert_this));
            // the remainder f * n - n is zero: no gap draws
        }
        // FixParticledistributionDiscrete::randomize_list
        std::vector<int> plist;
        std::vector<double> prad;
        randomize(nlocal_ins, P.exact_number != 0, plist, prad);
        const int ntot = (int)plist.size();
        if (ntot == 0) {
            if (P.insert_every) next_reneighbor += P.insert_every;
            else next_reneighbor = -1;
            return "";
        }
        // the near list grows by each accepted particle
        NearGrid grid(R, maxrad);
        if (P.overlapcheck)
            for (const NearParticle &q : nearp) grid.add(q);
        // FixInsertPack::x_v_omega
        const int maxtry = insertion_ratio >= 1.
                               ? ntot * P.maxattempt
                               : static_cast<int>(static_cast<double>(ntot * P.maxattempt) / (1. - insertion_ratio));
        int ntry = 0;
        int done = 0;
        double mass_this = 0.;
        if (!P.overlapcheck) {
            for (int it = 0; it < ntot; it++) {
                const int t = plist[done];
                double pos[3], v[3];
                if (!random_position(pos, prad[done])) return "region too small for all_in";
                random_velocity(v);
                if (pos[0] == 0. && pos[1] == 0. && pos[2] == 0.) return "FixInsertPack::x_v_omega() illegal position";
                out.push_back(make(t, prad[done], pos, v));
                mass_this += out.back().mass;
                done++;
            }
        } else {
            while (ntry < maxtry && done < ntot) {
                const int t = plist[done];
                const double rbound = prad[done];
                int nins = 0;
                while (nins == 0 && ntry < maxtry) {
                    double pos[3];
                    do {
                        if (!random_position(pos, rbound)) return "region too small for all_in";
                        ntry++;
                    } while (P.check_dist_from_subdomain_border && ntry < maxtry && dist_box_borders(pos) < rbound);
                    if (ntry == maxtry) break;
                    double v[3];
                    random_velocity(v);
                    if (!grid.overlaps(pos, rbound)) {
                        grid.add(NearParticle{{pos[0], pos[1], pos[2]}, rbound});
                        out.push_back(make(t, rbound, pos, v));
                        nins = 1;
                    }
                }
                if (nins > 0) {
                    mass_this += out.back().mass;
                    done++;
                }
            }
        }
        ninserted += done;
        massinserted += mass_this;
        if (P.insert_every) next_reneighbor += P.insert_every;
        else next_reneighbor = 0;
        return "";
    }

    // dense cell list over the near-list bounding box (every near particle and
    // every candidate lies in it): a test sees every particle whose sphere
    // reaches the candidate's (exact, unlike a fixed stencil); cell indices
    // are clamped, which keeps the lookup exact because it is monotone
    struct NearGrid {
        double lo[3], h, inv;
        int n[3];
        double rmax = 0.;
        std::vector<int> head, next;
        std::vector<NearParticle> parts;
        NearGrid(const InsertRegion &R, double maxrad_)
        {
            h = 4 * maxrad_ > 0 ? 4 * maxrad_ : 1.0;
            for (;;) {
                inv = 1.0 / h;
                long cells = 1;
                for (int d = 0; d < 3; d++) {
                    lo[d] = R.blo[d];
                    n[d] = std::max(1, (int)std::ceil((R.bhi[d] - R.blo[d]) * inv) + 1);
                    cells *= n[d];
                }
                if (cells <= (1L << 24)) break;   // at most 16M cells (64 MB of heads)
                h *= 2;
            }
            head.assign((size_t)n[0] * n[1] * n[2], -1);
        }
        int cell(double x, int d) const
        {
            const double f = std::floor((x - lo[d]) * inv);
            return f < 0 ? 0 : (f >= n[d] ? n[d] - 1 : (int)f);
        }
        void add(const NearParticle &q)
        {
            rmax = std::max(rmax, q.r);
            const size_t c = ((size_t)cell(q.x[2], 2) * n[1] + cell(q.x[1], 1)) * n[0] + cell(q.x[0], 0);
            parts.push_back(q);
            next.push_back(head[c]);
            head[c] = (int)parts.size() - 1;
        }
        bool overlaps(const double *x, double r) const
        {
            const double reach = r + rmax;
            int clo[3], chi[3];
            for (int d = 0; d < 3; d++) {
                clo[d] = cell(x[d] - reach, d);
                chi[d] = cell(x[d] + reach, d);
            }
            for (int cz = clo[2]; cz <= chi[2]; cz++)
                for (int cy = clo[1]; cy <= chi[1]; cy++)
                    for (int cx = clo[0]; cx <= chi[0]; cx++)
                        for (int k = head[((size_t)cz * n[1] + cy) * n[0] + cx]; k >= 0; k = next[k]) {
                            const NearParticle &p = parts[k];
                            double del[3] = {x[0] - p.x[0], x[1] - p.x[1], x[2] - p.x[2]};
                            const double rsq = del[0] * del[0] + del[1] * del[1] + del[2] * del[2];
                            const double radsum = r + p.r;
                            if (rsq <= radsum * radsum) return true;
                        }
            return false;
        }
    };

    // ProbabilityDistribution rand_value (src/probability_distribution.h:143-226)
    double draw_radius(int t)
    {
        const double r = P.tmpl_radius[t], r2 = P.tmpl_radius2[t];
        if (P.tmpl_radius_style[t] == 1) {
            const double rn = rtmpl[t].uniform();
            return std::sqrt(h1[t] / (2. * (h2[t] - rn)));
        }
        if (P.tmpl_radius_style[t] == 2) {
            double value;
            do {
                value = r + rtmpl[t].gaussian() * r2;
            } while (value < rmin[t] || value > rmax[t]);
            return value;
        }
        return r;
    }

    InsertedParticle make(int t, double radius, const double *pos, const double *v) const
    {
        InsertedParticle q;
        for (int d = 0; d < 3; d++) {
            q.x[d] = pos[d];
            q.v[d] = v[d];
            q.omega[d] = P.omega[d];
        }
        q.radius = radius;
        q.density = P.tmpl_density[t];
        q.mass = q.density * (q.radius * q.radius * q.radius * 4. * M_PI / 3.);
        q.type = P.tmpl_type[t];
        return q;
    }

private:
    // Region::generate_random / generate_random_shrinkby_cut on the block
    // within the single subdomain (the box)
    bool random_position(double *pos, double rbound)
    {
        double lo[3], hi[3], diff[3];
        for (int d = 0; d < 3; d++) {
            lo[d] = std::max(P.region_lo[d], boxlo[d]);
            hi[d] = std::min(P.region_hi[d], boxhi[d]);
            diff[d] = hi[d] - lo[d];
        }
        if (P.all_in)
            for (int d = 0; d < 3; d++)
                if (P.region_hi[d] - P.region_lo[d] < 2. * rbound) return false;
        for (;;) {
            pos[0] = lo[0] + rreg.uniform() * diff[0];
            pos[1] = lo[1] + rreg.uniform() * diff[1];
            pos[2] = lo[2] + rreg.uniform() * diff[2];
            if (!R.inside(pos)) continue;
            if (P.all_in && R.surface_interior(pos, rbound)) continue;
            return true;
        }
    }

    // FixInsert::generate_random_velocity
    void random_velocity(double *v)
    {
        for (int d = 0; d < 3; d++) v[d] = P.vel[d];
        if (P.vel_style == 1) {
            v[0] = P.vel[0] + P.vel_fluct[0] * 2.0 * (rnd.uniform() - 0.50);
            v[1] = P.vel[1] + P.vel_fluct[1] * 2.0 * (rnd.uniform() - 0.50);
            v[2] = P.vel[2] + P.vel_fluct[2] * 2.0 * (rnd.uniform() - 0.50);
        } else if (P.vel_style == 2) {
            v[0] = P.vel[0] + P.vel_fluct[0] * rnd.gaussian();
            v[1] = P.vel[1] + P.vel_fluct[1] * rnd.gaussian();
            v[2] = P.vel[2] + P.vel_fluct[2] * rnd.gaussian();
        }
    }

    // Domain::dist_subbox_borders with the box as the subdomain
    double dist_box_borders(const double *pos) const
    {
        double dlo = std::fabs(boxlo[0] - pos[0]), dhi = std::fabs(boxhi[0] - pos[0]);
        for (int d = 1; d < 3; d++) {
            dlo = std::min(dlo, std::fabs(boxlo[d] - pos[d]));
            dhi = std::min(dhi, std::fabs(boxhi[d] - pos[d]));
        }
        return dlo < dhi ? dlo : dhi;
    }
};



// Release data of a particle inserted by fix insert/stream (the reference's
// per-atom property release_fix_insert_stream): position at insertion and
// insertion step, integration velocity v_n and release step, velocity and
// angular velocity given at release.
struct StreamRelease {
    double x[3], istep;
    double vint[3], rstep;
    double vrel[3], wrel[3];
};

// fix insert/stream over a planar face (src/fix_insert_stream.cpp with
// src/fix_insert.cpp), host side: the same particle distribution and
// templates as insert/pack (an embedded InsertPack holds them), the face's
// area-weighted random points (its own generator, MultiNodeMesh's fixed seed)
// extruded against the normal velocity, the Monte-Carlo insertion fraction,
// and the release data of each inserted particle.
//   FixInsertStream::calc_insertion_properties   src/fix_insert_stream.cpp:254-373
//   calc_ins_fraction, is_nearby, getBoundingBox,
//   generate_random(_global), x_v_omega,
//   finalize_insertion                          src/fix_insert_stream.cpp:469-836
//   FixInsert::calc_ninsert_this, pre_exchange,
//   distribute_ninsert_this                     src/fix_insert.cpp:637-914
//   SurfaceMesh::randomOwnedGhostElement, searchElementByAreaAcc,
//   TriMesh::generateRandomOwnedGhost, isInElement, calcArea
//                                               src/surface_mesh_I.h:167-274, src/tri_mesh_I.h:305-401
//   Domain::is_in_subdomain, dist_subbox_borders src/domain_I.h:65-143
class InsertStream {
public:
    gb2_insert_stream S{};
    InsertPack dist;
    std::vector<TriGeom> face;
    std::vector<double> area, areaAcc;
    double area_owned = 0.;
    double boxlo[3] = {0, 0, 0}, boxhi[3] = {0, 0, 0};
    double v_insert[3] = {0, 0, 0}, normalvec[3] = {0, 0, 0}, v_normal[3] = {0, 0, 0}, p_ref[3] = {0, 0, 0};
    double vn_mag = 0.;
    double extrude_length = 0., extrude_length_min = 0., extrude_length_max = 0.;
    int insert_every = -1, duration = 0;
    long ninsert = 0;
    bool ninsert_exists = true;
    double massinsert = 0., nflowrate = 0., massflowrate = 0., ninsert_per = 0.;
    long next_reneighbor = 0, most_recent = -1;
    long ninserted = 0;
    double massinserted = 0.;
    bool exact_number = true;
    double ins_fraction = 0.;
    bool frac_done = false, props_done = false;
    double maxrad = 0., maxrbound = 0.;
    double bblo[3] = {0, 0, 0}, bbhi[3] = {0, 0, 0};   // getBoundingBox of the near list
    double dt = 0.;
    ParkRandom rnd, rmesh;

    // the three commands' constructor checks; face = the element geometry of
    // the insertion mesh in its element order
    std::string init(const gb2_insert_stream &p, std::vector<TriGeom> faces, const double lo[3], const double hi[3],
                     int ntypes, long ntimestep, double dt_)
    {
        S = p;
        dt = dt_;
        for (int d = 0; d < 3; d++) {
            boxlo[d] = lo[d];
            boxhi[d] = hi[d];
        }
        if (!insert_seed_ok(S.seed)) return "random seeds must be prime numbers > 10000";
        // the distribution and templates through insert/pack's checks (its
        // region and target are placeholders here and never used)
        gb2_insert_pack q{};
        q.seed = S.seed;
        for (int d = 0; d < 3; d++) {
            q.region_lo[d] = lo[d];
            q.region_hi[d] = hi[d];
        }
        q.particles_in_region = 1;
        q.maxattempt = S.maxattempt;
        q.ntry_mc = S.ntry_mc;
        q.vel_style = 0;
        q.dist_seed = S.dist_seed;
        q.dist_mass_based = S.dist_mass_based;
        q.ntemplates = S.ntemplates;
        for (int i = 0; i < GB2_INSERT_MAX_TEMPLATES; i++) {
            q.tmpl_type[i] = S.tmpl_type[i];
            q.tmpl_radius[i] = S.tmpl_radius[i];
            q.tmpl_density[i] = S.tmpl_density[i];
            q.tmpl_weight[i] = S.tmpl_weight[i];
            q.tmpl_radius_style[i] = S.tmpl_radius_style[i];
            q.tmpl_radius2[i] = S.tmpl_radius2[i];
            q.tmpl_seed[i] = S.tmpl_seed[i];
        }
        q.max_atoms = S.max_atoms;
        const std::string e = dist.init(q, lo, hi, ntypes, ntimestep);
        if (!e.empty()) return e;
        if (S.maxattempt <= 0 || S.ntry_mc < 1000) return "maxattempt must be > 0 and ntry_mc >= 1000";
        if (S.vel_style < 0 || S.vel_style > 2) return "vel style must be constant, uniform or gaussian";
        if (S.insert_every == 0) return "insert_every 0 (once) is not supported with insert/stream";
        if (S.nparticles > 0. && S.mass > 0.) return "must not define both 'nparticles' and 'mass'";
        if (S.particlerate > 0. && S.massrate > 0.) return "must not define both 'particlerate' and 'massrate'";
        if (S.extrude_length < 0.) return "invalid extrude_length";
        if (S.duration < 0) return "'duration' can not be < 1";
        if (faces.empty()) return "must define an insertion face";
        // TriMesh::isPlanar: every element's normal parallel to the first
        for (const TriGeom &t : faces)
            if (std::fabs(t.surfnorm[0] * faces[0].surfnorm[0] + t.surfnorm[1] * faces[0].surfnorm[1] +
                          t.surfnorm[2] * faces[0].surfnorm[2]) < 1. - 1e-10)
                return "command requires a planar face for insertion";
        face = std::move(faces);
        // SurfaceMesh::recalcLocalSurfProperties: area, accumulated area, owned area
        const int n = (int)face.size();
        area.resize(n);
        areaAcc.resize(n);
        area_owned = 0.;
        for (int i = 0; i < n; i++) {
            const TriGeom &t = face[i];
            const double c[3] = {t.edgevec[0][1] * t.edgevec[1][2] - t.edgevec[0][2] * t.edgevec[1][1],
                                 t.edgevec[0][2] * t.edgevec[1][0] - t.edgevec[0][0] * t.edgevec[1][2],
                                 t.edgevec[0][0] * t.edgevec[1][1] - t.edgevec[0][1] * t.edgevec[1][0]};
            area[i] = 0.5 * std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) * t.edgelen[0] * t.edgelen[1];
            areaAcc[i] = area[i];
            if (i > 0) areaAcc[i] += areaAcc[i - 1];
            area_owned += area[i];
        }
        rnd.reset(S.seed);
        rmesh.reset(179424799);   // MultiNodeMesh's generator
        for (int d = 0; d < 3; d++) v_insert[d] = S.vel[d];
        ninsert_exists = !S.ninsert_inf;
        ninsert = ninsert_exists ? static_cast<long>(S.nparticles) : 0;
        massinsert = S.mass;
        nflowrate = S.particlerate;
        massflowrate = S.massrate;
        insert_every = S.insert_every;
        duration = S.duration;
        extrude_length = S.extrude_length;
        exact_number = S.exact_number != 0;
        maxrad = dist.maxrad;
        maxrbound = dist.maxrbound;
        const long first = S.start > 0 ? S.start : ntimestep + 1;
        if (first < ntimestep + 1) return "'start' step can not be before current step";
        next_reneighbor = first;
        return "";
    }

    double max_rad(int type) const { return dist.max_rad(type); }

    // FixInsertStream::calc_insertion_properties (FixInsert::setup, once)
    std::string setup()
    {
        if (props_done) return "";
        props_done = true;
        for (int d = 0; d < 3; d++) normalvec[d] = face[0].surfnorm[d];
        double dot = v_insert[0] * normalvec[0] + v_insert[1] * normalvec[1] + v_insert[2] * normalvec[2];
        if (dot < 0)
            for (int d = 0; d < 3; d++) normalvec[d] = normalvec[d] * -1.;
        dot = v_insert[0] * normalvec[0] + v_insert[1] * normalvec[1] + v_insert[2] * normalvec[2];
        for (int d = 0; d < 3; d++) v_normal[d] = normalvec[d] * dot;
        vn_mag = std::sqrt(v_normal[0] * v_normal[0] + v_normal[1] * v_normal[1] + v_normal[2] * v_normal[2]);
        if (vn_mag < 1.e-3) return "insertion velocity projected on face normal is < 1e-3";
        for (int d = 0; d < 3; d++) p_ref[d] = face[0].node[0][d];
        if (std::sqrt(v_insert[0] * v_insert[0] + v_insert[1] * v_insert[1] + v_insert[2] * v_insert[2]) < 1e-5)
            return "insertion velocity too low";
        if (insert_every == -1 && extrude_length == 0.) return "must define either 'insert_every' or 'extrude_length'";
        if (insert_every > -1 && extrude_length > 0.) return "must not provide both 'insert_every' and 'extrude_length'";
        if (extrude_length > 0. && duration > 0) return "must not provide both 'extrude_length' and 'duration'";
        if (insert_every == -1) {
            if (extrude_length < 3. * maxrbound && S.overlapcheck) return "'extrude_length' is too small";
            insert_every = static_cast<int>((extrude_length + 1e-14) / (dt * vn_mag));
            if (insert_every == 0) return "insertion velocity too high or extrude_length too low";
        } else {
            if (insert_every < 1) return "'insert_every' must be > 0";
            if (duration == 0) duration = insert_every;
            else if (duration > insert_every) return "'duration' > 'insert_every' not allowed";
            extrude_length = static_cast<double>(duration) * dt * vn_mag;
            if (extrude_length < 2. * maxrbound)
                return "'insert_every' or 'vel' is too small, or (bounding) radius of inserted particles too large";
        }
        const double mass_expect = dist.massexpect;
        if (ninsert == 0 && ninsert_exists) {
            if (massinsert / mass_expect > 2.e9) return "attempting to insert more than 2e9 particles";
            if (massinsert > 0.) ninsert = static_cast<int>((massinsert + 1e-14) / mass_expect);
            else return "must define either 'nparticles' or 'mass'";
        }
        if (nflowrate == 0.) {
            if (massflowrate == 0.) return "must define either 'massrate' or 'particlerate'";
            nflowrate = massflowrate / mass_expect;
        } else {
            massflowrate = nflowrate * mass_expect;
        }
        ninsert_per = nflowrate * (static_cast<double>(insert_every) * dt);
        if (ninsert_exists) massinsert = static_cast<double>(ninsert) * mass_expect;
        extrude_length_min = 0.;
        extrude_length_max = extrude_length;
        // getBoundingBox: face box extruded by -(extrude_length + 2 cut), shrunk
        // to the (single) subdomain, widened by 3 maxrad + 2 max bounding radius
        double lo[3], hi[3];
        for (int d = 0; d < 3; d++) {
            lo[d] = face[0].node[0][d];
            hi[d] = face[0].node[0][d];
        }
        for (const TriGeom &t : face)
            for (int k = 0; k < 3; k++)
                for (int d = 0; d < 3; d++) {
                    lo[d] = std::min(lo[d], t.node[k][d]);
                    hi[d] = std::max(hi[d], t.node[k][d]);
                }
        const double cut = 3 * maxrad;
        const double delta = -(extrude_length + 2 * cut);
        for (int d = 0; d < 3; d++) {
            double a = std::min(lo[d], lo[d] + delta * normalvec[d]);
            double b = std::max(hi[d], hi[d] + delta * normalvec[d]);
            if (a < boxlo[d]) a = boxlo[d];
            if (b > boxhi[d]) b = boxhi[d];
            const double extend = 3 * maxrad + 2. * maxrbound;
            bblo[d] = a - extend;
            bbhi[d] = b + extend;
        }
        return "";
    }

    bool due(long step) const { return next_reneighbor == step && most_recent != step; }

    // one insertion (FixInsert::pre_exchange with FixInsertStream's parts);
    // nearp = the owned and ghost particles FixInsertStream::is_nearby keeps
    // inside getBoundingBox; accepted particles and their release data are
    // appended to out / rel
    std::string insert(long step, std::vector<NearParticle> nearp, std::vector<InsertedParticle> &out,
                       std::vector<StreamRelease> &rel)
    {
        out.clear();
        rel.clear();
        most_recent = step;
        // FixInsert::calc_ninsert_this
        if (ninsert_per == 0.) return "ninsert_per == 0.";
        int ninsert_this = static_cast<int>(ninsert_per + rnd.uniform());
        if (ninsert_exists && ninserted + ninsert_this > ninsert) ninsert_this = static_cast<int>(ninsert - ninserted);
        if (ninsert_exists && ninserted + ninsert_this >= ninsert) {
            ninsert_this = static_cast<int>(ninsert - ninserted);
            if (ninsert_this < 0) ninsert_this = 0;
            exact_number = true;
        }
        // distribute_ninsert_this on one process
        if (!frac_done) {
            const std::string e = calc_ins_fraction();
            if (!e.empty()) return e;
        }
        int nlocal_ins;
        if (!exact_number) {
            nlocal_ins = static_cast<int>(ins_fraction * static_cast<double>(ninsert_this) + rnd.uniform());
        } else {
            double f = ins_fraction;
            if (f < 0.02) f = 0.;
            if (f == 0.) return "Internal error distributing particles to processes";
            f /= f;
            nlocal_ins = static_cast<int>(f * static_cast<double>(ninsert_this));
        }
        std::vector<int> plist;
        std::vector<double> prad;
        dist.randomize(nlocal_ins, exact_number, plist, prad);
        const int ntot = (int)plist.size();
        if (ntot == 0) {
            if (insert_every && (!ninsert_exists || ninserted < ninsert)) next_reneighbor += insert_every;
            else if (0 == insert_every) next_reneighbor = -1;
            return "";
        }
        // x_v_omega: positions in the extruded face, velocity v_n, no omega
        const int maxtry = ntot * S.maxattempt;
        int ntry = 0, done = 0;
        double mass_this = 0.;
        const double zero3[3] = {0., 0., 0.};
        if (!S.overlapcheck) {
            for (int it = 0; it < ntot; it++) {
                const double rad = prad[done];
                double pos[3];
                do {
                    generate_random(pos, rad);
                    ntry++;
                } while (ntry < maxtry && !in_subdomain(pos));
                if (ntry < maxtry) {
                    out.push_back(dist.make(plist[done], rad, pos, v_normal));
                    for (int d = 0; d < 3; d++) out.back().omega[d] = zero3[d];
                    mass_this += out.back().mass;
                    done++;
                }
            }
        } else {
            NearGrid grid(bblo, bbhi, maxrad);
            for (const NearParticle &q : nearp) grid.add(q);
            while (ntry < maxtry && done < ntot) {
                const double rad = prad[done];
                int nins = 0;
                while (nins == 0 && ntry < maxtry) {
                    double pos[3];
                    do {
                        generate_random(pos, rad);
                        ntry++;
                    } while (ntry < maxtry && (!in_subdomain(pos) || dist_box_borders(pos) < rad));
                    if (ntry < maxtry && !grid.overlaps(pos, rad)) {
                        grid.add(NearParticle{{pos[0], pos[1], pos[2]}, rad});
                        out.push_back(dist.make(plist[done], rad, pos, v_normal));
                        for (int d = 0; d < 3; d++) out.back().omega[d] = zero3[d];
                        nins = 1;
                    }
                }
                if (nins > 0) {
                    mass_this += out.back().mass;
                    done++;
                }
            }
        }
        // finalize_insertion: release data, in insertion order
        for (const InsertedParticle &a : out) {
            StreamRelease r;
            const double pos_rel[3] = {p_ref[0] - a.x[0], p_ref[1] - a.x[1], p_ref[2] - a.x[2]};
            const double dist_normal = pos_rel[0] * normalvec[0] + pos_rel[1] * normalvec[1] + pos_rel[2] * normalvec[2];
            const int n_steps = static_cast<int>((dist_normal + 1e-14) / (vn_mag * dt));
            for (int d = 0; d < 3; d++) r.x[d] = a.x[d];
            r.istep = static_cast<double>(step);
            r.rstep = static_cast<double>(step + n_steps);
            for (int d = 0; d < 3; d++) r.vint[d] = v_normal[d];
            double v[3] = {v_insert[0], v_insert[1], v_insert[2]};
            random_velocity(v);
            for (int d = 0; d < 3; d++) {
                r.vrel[d] = v[d];
                r.wrel[d] = S.omega[d];
            }
            rel.push_back(r);
        }
        ninserted += done;
        massinserted += mass_this;
        if (insert_every && (!ninsert_exists || ninserted < ninsert)) next_reneighbor += insert_every;
        else next_reneighbor = 0;
        return "";
    }

    // FixInsertStream::is_nearby for a particle at x (the face test of the
    // near list, SMALL_TRIMESH = 1e-10), with the list's bounding box
    bool nearby(const double *x) const
    {
        if (!(x[0] >= bblo[0] && x[0] <= bbhi[0] && x[1] >= bblo[1] && x[1] <= bbhi[1] && x[2] >= bblo[2] &&
              x[2] <= bbhi[2]))
            return false;
        const double pos_rel[3] = {x[0] - p_ref[0], x[1] - p_ref[1], x[2] - p_ref[2]};
        const double dist_normal = pos_rel[0] * normalvec[0] + pos_rel[1] * normalvec[1] + pos_rel[2] * normalvec[2];
        if (dist_normal > maxrad) return false;
        if (dist_normal < -(extrude_length + 3. * maxrad)) return false;
        double pp[3];
        for (int d = 0; d < 3; d++) pp[d] = x[d] + normalvec[d] * dist_normal;
        for (const TriGeom &t : face)
            if (in_element(t, pp)) return true;
        return false;
    }

private:
    struct NearGrid : InsertPack::NearGrid {
        NearGrid(const double *blo, const double *bhi, double maxrad_) : InsertPack::NearGrid(box(blo, bhi), maxrad_) {}
        static InsertRegion box(const double *blo, const double *bhi)
        {
            InsertRegion R{};
            for (int d = 0; d < 3; d++) {
                R.blo[d] = blo[d];
                R.bhi[d] = bhi[d];
            }
            return R;
        }
    };

    static bool in_element(const TriGeom &t, const double *pos)
    {
        double v0[3], v1[3], v2[3];
        for (int d = 0; d < 3; d++) {
            v0[d] = t.node[2][d] - t.node[0][d];
            v1[d] = t.node[1][d] - t.node[0][d];
            v2[d] = pos[d] - t.node[0][d];
        }
        const double dot00 = v0[0] * v0[0] + v0[1] * v0[1] + v0[2] * v0[2];
        const double dot01 = v0[0] * v1[0] + v0[1] * v1[1] + v0[2] * v1[2];
        const double dot02 = v0[0] * v2[0] + v0[1] * v2[1] + v0[2] * v2[2];
        const double dot11 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
        const double dot12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
        const double invDenom = 1. / (dot00 * dot11 - dot01 * dot01);
        const double u = (dot11 * dot02 - dot01 * dot12) * invDenom;
        const double v = (dot00 * dot12 - dot01 * dot02) * invDenom;
        return (u > -1e-10) && (v > -1e-10) && (u + v < 1. + 1e-10);
    }

    // SurfaceMesh::searchElementByAreaAcc (recursive in the reference)
    int element_by_area(double a, int lo, int hi) const
    {
        for (;;) {
            if ((lo < 1 || a > areaAcc[lo - 1]) && (a <= areaAcc[lo])) return lo;
            if ((hi < 1 || a > areaAcc[hi - 1]) && (a <= areaAcc[hi])) return hi;
            const int mid = static_cast<int>((lo + hi) / 2);
            if (a > areaAcc[mid]) lo = mid;
            else hi = mid;
        }
    }

    // TriMesh::generateRandomOwnedGhost on the face
    void face_point(double *pos)
    {
        const double a = area_owned + 0.;   // areaMeshOwned + areaMeshGhost (no ghosts)
        const double r = rmesh.uniform() * a;
        const int chosen = element_by_area(r, 0, (int)face.size() - 1);
        double u, v;
        do {
            u = rmesh.uniform();
            v = rmesh.uniform();
        } while (u + v > 1);
        const double b0 = 1. - u - v, b1 = v, b2 = u;
        const TriGeom &t = face[chosen];
        for (int d = 0; d < 3; d++) pos[d] = b0 * t.node[0][d] + b1 * t.node[1][d] + b2 * t.node[2][d];
    }

    // FixInsertStream::generate_random (all_in no)
    void generate_random(double *pos, double rad)
    {
        face_point(pos);
        double r;
        if (S.overlapcheck) r = -1. * (rnd.uniform() * (extrude_length_max) + rad + extrude_length_min);
        else r = -1. * (rnd.uniform() * (extrude_length_max - 2. * rad) + rad + extrude_length_min);
        for (int d = 0; d < 3; d++) pos[d] = pos[d] + normalvec[d] * r;
    }

    // FixInsertStream::calc_ins_fraction (parallel no)
    std::string calc_ins_fraction()
    {
        frac_done = true;
        int n_in_local = 0;
        const int n_test = S.ntry_mc;
        for (int i = 0; i < n_test; i++) {
            double pos[3];
            face_point(pos);
            const double r = -1. * (rnd.uniform() * extrude_length);
            for (int d = 0; d < 3; d++) pos[d] = pos[d] + normalvec[d] * r;
            if (in_subdomain(pos)) n_in_local++;
        }
        ins_fraction = static_cast<double>(n_in_local) / static_cast<double>(n_test);
        if (ins_fraction < 0.9 || ins_fraction > 1.1)
            return "insertion volume could not be distributed properly in parallel. Bad decomposition or insertion "
                   "face extrusion is too small or outside domain";
        return "";
    }

    // Domain::is_in_subdomain on the single subdomain (the box, padded by
    // SMALL_DMBRDR at the box boundary)
    bool in_subdomain(const double *pos) const
    {
        for (int d = 0; d < 3; d++)
            if (!(pos[d] >= boxlo[d] - 1.0e-8 && pos[d] < boxhi[d] + 1.0e-8)) return false;
        return true;
    }

    double dist_box_borders(const double *pos) const
    {
        double dlo = std::fabs(boxlo[0] - pos[0]), dhi = std::fabs(boxhi[0] - pos[0]);
        for (int d = 1; d < 3; d++) {
            dlo = std::min(dlo, std::fabs(boxlo[d] - pos[d]));
            dhi = std::min(dhi, std::fabs(boxhi[d] - pos[d]));
        }
        return dlo < dhi ? dlo : dhi;
    }

    // FixInsert::generate_random_velocity
    void random_velocity(double *v)
    {
        if (S.vel_style == 1) {
            v[0] = v_insert[0] + S.vel_fluct[0] * 2.0 * (rnd.uniform() - 0.50);
            v[1] = v_insert[1] + S.vel_fluct[1] * 2.0 * (rnd.uniform() - 0.50);
            v[2] = v_insert[2] + S.vel_fluct[2] * 2.0 * (rnd.uniform() - 0.50);
        } else if (S.vel_style == 2) {
            v[0] = v_insert[0] + S.vel_fluct[0] * rnd.gaussian();
            v[1] = v_insert[1] + S.vel_fluct[1] * rnd.gaussian();
            v[2] = v_insert[2] + S.vel_fluct[2] * rnd.gaussian();
        }
    }
};

}  // namespace gb2
