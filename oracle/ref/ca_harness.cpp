/*
 * ca_harness.cpp -- the reference's own cellular-automaton processors, compiled
 * from the reference tree (oracle/Makefile), run on one block to pin the
 * oracle's serial CA order (oracle.c, orc_ca_redistribute with serial = 1).
 * Test infrastructure only.
 *
 *   ref_ca_block   one CA block of src/complab.cpp:1453-1715 and the age pass
 *                  of :1736-1739, with the reference's processors doing all the
 *                  per-voxel work: updateLocalMaskNtotalLattices3D,
 *                  pushExcessBiomass3D / halfPushExcessBiomass3D and
 *                  updateAgeDistance3D.  The loop around them (the maximum,
 *                  the stall and sweep limits, the age relaxation every 50
 *                  sweeps) is complab.cpp's, restated here because it lives
 *                  inside main().  pullExcessBiomass3D is not run: on one block
 *                  no push crosses a block boundary, so it has nothing to pull.
 *   ref_ca_update_mask  updateLocalMaskNtotalLattices3D alone (complab.cpp:1068-1076).
 *
 * std::random_shuffle and std::rand (seeded from the clock in the reference,
 * complab.cpp:189) are replaced, by macro, with draws from a counter-based
 * generator whose stream the oracle's serial order also draws from; the state
 * is the draw counter passed in and out.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <random>
#include <string>
#include <vector>
#include "plb_ca_stub.h"

// declarations that other processors of the same headers name (never instantiated here)
namespace plb {
template<typename T1, template<typename U> class D1, typename T2, template<typename U> class D2>
class BoxProcessingFunctional3D_LL { public: virtual ~BoxProcessingFunctional3D_LL() {} };
template<typename T1, template<typename U> class D1> class BounceBack { public: BounceBack() {} };
template<typename T1, template<typename U> class D1> class IncBGKdynamics { public: explicit IncBGKdynamics(T1) {} };
}
#define COMPLAB_THRD 1e-14            /* src/complab_functions.hh:64 */

namespace capin {
uint64_t seed = 0, draws = 0;
inline uint64_t hash(uint64_t s, uint64_t stream, uint64_t site) {
    uint64_t z = s ^ (stream * 0x9E3779B97F4A7C15ull) ^ (site * 0xD1B54A32D192ED03ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline uint64_t next() { return hash(seed, ~0ull, draws++); }
}  // namespace capin

namespace std {
template<class It> void capin_random_shuffle(It first, It last) {
    const long n = (long)(last - first);
    const uint64_t r = ::capin::next();
    for (long i = n - 1; i > 0; --i) {
        const long j = (long)((r >> (8 * i)) & 0xff) % (i + 1);
        std::swap(first[i], first[j]);
    }
}
inline int capin_rand() { return (int)(::capin::next() & 0x7fffffff); }
}  // namespace std
#define random_shuffle capin_random_shuffle
#define rand capin_rand

#include "src/complab3d_processors_part1.hh"
#include "src/complab3d_processors_part2.hh"

typedef plb::BlockLattice3D<double, CaStubD3Q7> Lat;

namespace {

struct Block {
    plint nx, ny, nz, M;
    std::vector<Lat*> bio, copy;
    Lat *total, *mask, *age, *dist;
    Block(plint nx_, plint ny_, plint nz_, plint M_) : nx(nx_), ny(ny_), nz(nz_), M(M_) {
        for (plint m = 0; m < M; ++m) { bio.push_back(new Lat(nx, ny, nz)); copy.push_back(new Lat(nx, ny, nz)); }
        total = new Lat(nx, ny, nz); mask = new Lat(nx, ny, nz); age = new Lat(nx, ny, nz); dist = new Lat(nx, ny, nz);
    }
    ~Block() {
        for (auto* p : bio) delete p;
        for (auto* p : copy) delete p;
        delete total; delete mask; delete age; delete dist;
    }
    // [B.., copies.., total, mask, age]: ptr_ca_lattices (complab.cpp:1010-1022)
    std::vector<Lat*> ca() const {
        std::vector<Lat*> v(bio);
        v.insert(v.end(), copy.begin(), copy.end());
        v.push_back(total); v.push_back(mask); v.push_back(age);
        return v;
    }
    // [age, dist, total]: ageNdistance_lattices (complab.cpp:1063-1066)
    std::vector<Lat*> agedist() const { return {age, dist, total}; }
    Box3D box() const { return Box3D{0, nx - 1, 0, ny - 1, 0, nz - 1}; }
    size_t idx(plint x, plint y, plint z) const { return ((size_t)x * ny + (size_t)y) * nz + (size_t)z; }
    template<class F> void each(F f) const {
        for (plint x = 0; x < nx; ++x) for (plint y = 0; y < ny; ++y) for (plint z = 0; z < nz; ++z) f(x, y, z, idx(x, y, z));
    }
    double max_total() {
        double mx = -std::numeric_limits<double>::infinity();
        each([&](plint x, plint y, plint z, size_t) { mx = std::max(mx, total->get(x, y, z).computeDensity()); });
        return mx;
    }
    long long sum_of(Lat* l) {
        double s = 0;
        each([&](plint x, plint y, plint z, size_t) { s += l->get(x, y, z).computeDensity(); });
        return (long long)util::roundToInt(s);
    }
};

struct Args {
    int nx, ny, nz, M, half;
    double bmax, frac;
    int solid, bb, n_pore;
    const int* pore;
    const int* codes;
};

std::vector<plint> pores(const Args& a) { return std::vector<plint>(a.pore, a.pore + a.n_pore); }
std::vector<std::vector<plint>> bio_dyn(const Args& a) {
    std::vector<std::vector<plint>> v;
    for (int m = 0; m < a.M; ++m) v.push_back({(plint)a.codes[m]});
    return v;
}

void load(Block& b, const Args& a, const uint8_t* mask, const double* bio, const double* total,
          const int32_t* age, const uint8_t* distpos) {
    const size_t N = (size_t)a.nx * a.ny * a.nz;
    b.each([&](plint x, plint y, plint z, size_t n) {
        b.mask->setScalar(x, y, z, mask[n]);
        for (int m = 0; m < a.M; ++m) b.bio[m]->setScalar(x, y, z, bio[m * N + n]);
        b.total->setScalar(x, y, z, total[n]);
        b.age->setScalar(x, y, z, age[n]);
        b.dist->setScalar(x, y, z, distpos[n] ? 1.0 : 0.0);
    });
}

void store(Block& b, const Args& a, uint8_t* mask, double* bio, double* total, int32_t* age) {
    const size_t N = (size_t)a.nx * a.ny * a.nz;
    b.each([&](plint x, plint y, plint z, size_t n) {
        mask[n] = (uint8_t)util::roundToInt(b.mask->get(x, y, z).computeDensity());
        for (int m = 0; m < a.M; ++m) bio[m * N + n] = b.bio[m]->get(x, y, z).computeDensity();
        total[n] = b.total->get(x, y, z).computeDensity();
        age[n] = (int32_t)util::roundToInt(b.age->get(x, y, z).computeDensity());
    });
}

void update_mask(Block& b, const Args& a) {
    const plint len = 2 * a.M + 3;
    updateLocalMaskNtotalLattices3D<double, CaStubD3Q7> p(a.nx, a.ny, a.nz, len, a.bb, a.solid, bio_dyn(a), pores(a),
                                                          a.frac, a.bmax);
    p.process(b.box(), b.ca());
}

void age_pass(Block& b, const Args& a) {
    updateAgeDistance3D<double, CaStubD3Q7> p(a.bmax, a.nx, a.ny, a.nz);
    p.process(b.box(), b.agedist());
}

}  // namespace

extern "C" {

long long ref_ca_update_mask(int nx, int ny, int nz, int M, int half, double bmax, double frac, int solid, int bb,
                             const int* pore, int n_pore, const int* codes, uint8_t* mask, double* bio,
                             double* total, int32_t* age, const uint8_t* distpos, long long* mask_sum) {
    Args a{nx, ny, nz, M, half, bmax, frac, solid, bb, n_pore, pore, codes};
    Block b(nx, ny, nz, M);
    load(b, a, mask, bio, total, age, distpos);
    const long long before = b.sum_of(b.mask);
    update_mask(b, a);
    *mask_sum = b.sum_of(b.mask);
    std::vector<uint8_t> old(mask, mask + (size_t)nx * ny * nz);
    store(b, a, mask, bio, total, age);
    long long changed = 0;
    for (size_t n = 0; n < old.size(); ++n) changed += old[n] != mask[n];
    (void)before;
    return changed;
}

/* returns 0, or 1 where the reference ends the run (stall, age relaxation or
 * sweep limit); *mask_sum is complab.cpp's old_totMask in and out */
int ref_ca_block(int nx, int ny, int nz, int M, int half, double bmax, double frac, int solid, int bb,
                 const int* pore, int n_pore, const int* codes, uint64_t seed, uint64_t* draws,
                 uint8_t* mask, double* bio, double* total, int32_t* age, const uint8_t* distpos,
                 long long* mask_sum, int32_t* sweeps_out, long long* changes_out, double* gmax_out) {
    Args a{nx, ny, nz, M, half, bmax, frac, solid, bb, n_pore, pore, codes};
    capin::seed = seed;
    capin::draws = *draws;
    Block b(nx, ny, nz, M);
    load(b, a, mask, bio, total, age, distpos);
    std::vector<uint8_t> before(mask, mask + (size_t)nx * ny * nz);
    const plint len = 2 * M + 3;
    update_mask(b, a);                                   // complab.cpp:1454
    double gmax = b.max_total();                         // :1455
    int status = 0, sweeps = 0;
    plint whilecount = 0;                                // :1680-1712
    double prev = gmax;
    plint stall = 0;
    if (gmax - bmax > thrd) {
        while (gmax - bmax > thrd) {
            if (half == 0) {
                pushExcessBiomass3D<double, CaStubD3Q7> p(bmax, nx, ny, nz, 1, len, solid, bb, pores(a));
                p.process(b.box(), b.ca());
            } else {
                halfPushExcessBiomass3D<double, CaStubD3Q7> p(bmax, nx, ny, nz, 1, len, solid, bb, pores(a));
                p.process(b.box(), b.ca());
            }
            ++sweeps;
            update_mask(b, a);
            gmax = b.max_total();
            if (gmax > prev - thrd) { if (++stall >= 100) { status = 1; break; } }
            else stall = 0;
            prev = gmax;
            if (whilecount % 50 == 0) {
                long long diff = 1;
                plint whilecount1 = 0;
                bool settled = true;
                while (diff != 0) {
                    const long long old_tot = b.sum_of(b.age);
                    age_pass(b, a);
                    diff = b.sum_of(b.age) - old_tot;
                    ++whilecount1;
                    if (whilecount1 > 1000) { settled = false; break; }
                }
                if (!settled) { status = 1; break; }
            }
            if (whilecount > 1000) { status = 1; break; }
            ++whilecount;
        }
    }
    const long long new_tot = b.sum_of(b.mask);          // :1736-1739
    if (new_tot != *mask_sum) {
        *mask_sum = new_tot;
        age_pass(b, a);
    }
    store(b, a, mask, bio, total, age);
    long long changed = 0;
    for (size_t n = 0; n < before.size(); ++n) changed += before[n] != mask[n];
    *draws = capin::draws;
    *sweeps_out = sweeps;
    *changes_out = changed;
    *gmax_out = gmax;
    return status;
}

/* fdDiffusion3D (complab3d_processors_part2.hh:258-420) on one block: the
 * copies taken from the biomass, [B.., copies.., mask], bdryGap 1, nu */
void ref_fd_diffuse(int nx, int ny, int nz, int M, double nu, const uint8_t* mask, double* bio) {
    Block b(nx, ny, nz, M);
    const size_t N = (size_t)nx * ny * nz;
    b.each([&](plint x, plint y, plint z, size_t n) {
        b.mask->setScalar(x, y, z, mask[n]);
        for (int m = 0; m < M; ++m) { b.bio[m]->setScalar(x, y, z, bio[m * N + n]); b.copy[m]->setScalar(x, y, z, bio[m * N + n]); }
    });
    std::vector<Lat*> v(b.bio);
    v.insert(v.end(), b.copy.begin(), b.copy.end());
    v.push_back(b.mask);
    fdDiffusion3D<double, CaStubD3Q7> p(nx, ny, nz, (plint)v.size(), 1, nu);
    p.process(b.box(), v);
    b.each([&](plint x, plint y, plint z, size_t n) {
        for (int m = 0; m < M; ++m) bio[m * N + n] = b.bio[m]->get(x, y, z).computeDensity();
    });
}

}  // extern "C"
