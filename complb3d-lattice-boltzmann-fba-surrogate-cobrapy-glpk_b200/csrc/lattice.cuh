// lattice.cuh -- lattice constants and AA-pattern addressing shared by the
// flow (D3Q19) and transport (D3Q7) kernels.
//
// Storage is structure-of-arrays: population i of site n lives at
// pop[i*N + n], n = (x*ny + y)*nz + z.  Streaming is the in-place AA pattern:
//   even step: site n reads pop[i][n], collides, writes pop[opp(i)][n];
//   odd step:  site n reads pop[opp(i)][n - c_i], collides, writes pop[i][n + c_i].
// After an even number of steps the array holds the natural post-stream state.
// Each memory slot belongs to exactly one site's read/write set, so a launch
// over any subset of sites is race-free and no second buffer is needed.
// y and z are periodic.  A population whose upstream/downstream site lies
// outside 0..nx-1 is reflected into its own site's opposite slot; that is what
// a swap-based streaming step leaves in a slot with no neighbour.
#pragma once
#include <cstdint>

namespace cl {

// D3Q19 in Palabos order (opp(i) = i +/- 9)
__host__ __device__ constexpr int c19x(int i) {
    return i == 1 ? -1 : i == 4 ? -1 : i == 5 ? -1 : i == 6 ? -1 : i == 7 ? -1 :
           i == 10 ? 1 : i == 13 ? 1 : i == 14 ? 1 : i == 15 ? 1 : i == 16 ? 1 : 0;
}
__host__ __device__ constexpr int c19y(int i) {
    return i == 2 ? -1 : i == 4 ? -1 : i == 8 ? -1 : i == 9 ? -1 : i == 14 ? -1 :
           i == 5 ? 1 : i == 11 ? 1 : i == 13 ? 1 : i == 17 ? 1 : i == 18 ? 1 : 0;
}
__host__ __device__ constexpr int c19z(int i) {
    return i == 3 ? -1 : i == 6 ? -1 : i == 8 ? -1 : i == 16 ? -1 : i == 18 ? -1 :
           i == 7 ? 1 : i == 9 ? 1 : i == 12 ? 1 : i == 15 ? 1 : i == 17 ? 1 : 0;
}
__host__ __device__ constexpr int opp19(int i) { return i == 0 ? 0 : (i <= 9 ? i + 9 : i - 9); }
__host__ __device__ constexpr float t19(int i) {
    return i == 0 ? 1.0f / 3.0f : ((i == 1 || i == 2 || i == 3 || i == 10 || i == 11 || i == 12) ? 1.0f / 18.0f : 1.0f / 36.0f);
}

// D3Q7 (t0 = 1/4, ti = 1/8, cs2 = 1/4), opp(i) = i +/- 3
__host__ __device__ constexpr int c7x(int i) { return i == 1 ? -1 : i == 4 ? 1 : 0; }
__host__ __device__ constexpr int c7y(int i) { return i == 2 ? -1 : i == 5 ? 1 : 0; }
__host__ __device__ constexpr int c7z(int i) { return i == 3 ? -1 : i == 6 ? 1 : 0; }
__host__ __device__ constexpr int opp7(int i) { return i == 0 ? 0 : (i <= 3 ? i + 3 : i - 3); }
__host__ __device__ constexpr float t7(int i) { return i == 0 ? 0.25f : 0.125f; }

// node classes (low two bits of a class byte)
enum : uint8_t { NODYN = 0, BB = 1, FLUID = 2, BIO = 3 };
// class-byte flags: reactive (interior x, not solid / bounce-back), surface (a
// face neighbour is solid / bounce-back), phase-neighbour (a face neighbour in
// x = 1..nx-2 carries a dissolvable phase), phase-self (carries one itself)
enum : uint8_t { F_REACTIVE = 4, F_SURFACE = 8, F_PHASE_NBR = 16, F_PHASE_SELF = 32 };

// Unsigned 32-bit division by a divisor fixed at set-up (Granlund and
// Montgomery, "Division by invariant integers using multiplication", 1994,
// the round-down variant with the extra add): q = (t + ((n - t) >> s1)) >> s2,
// t = umulhi(m, n), exact for every 32-bit n.  Site decoding uses it instead
// of a hardware-less 32/64-bit division on every site of every launch.
struct FastDiv {
    uint32_t d, m, s1, s2;
    __host__ void init(uint32_t div) {
        d = div;
        uint32_t l = 0;
        while (l < 32 && (1ull << l) < (unsigned long long)div) ++l;     // ceil(log2 d)
        m = (uint32_t)((((1ull << 32) * ((1ull << l) - div)) / div) + 1);
        s1 = l > 0 ? 1u : 0u;
        s2 = l > 0 ? l - 1 : 0u;
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const {
#ifdef __CUDA_ARCH__
        const uint32_t t = __umulhi(m, n);
#else
        const uint32_t t = (uint32_t)(((unsigned long long)m * n) >> 32);
#endif
        return (t + ((n - t) >> s1)) >> s2;
    }
};

struct Geo {
    int nx, ny, nz;
    int64_t N, plane;   // N = nx*ny*nz, plane = ny*nz
    FastDiv by_nz, by_ny;
};

// site index -> (x, y, z); the context keeps N below 2^32
__device__ __forceinline__ void decode(const Geo& g, int64_t n, int& x, int& y, int& z) {
    const uint32_t n32 = (uint32_t)n;
    const uint32_t q = g.by_nz.div(n32);
    z = (int)(n32 - q * (uint32_t)g.nz);
    x = (int)g.by_ny.div(q);
    y = (int)(q - (uint32_t)x * (uint32_t)g.ny);
}

// Site index of (x+dx, y+dy, z+dz) with y,z periodic; returns -1 when x+dx
// leaves 0..nx-1.
__device__ __forceinline__ int64_t nbr(const Geo& g, int64_t n, int x, int y, int z,
                                       int dx, int dy, int dz) {
    int xd = x + dx;
    if (xd < 0 || xd >= g.nx) return -1;
    int64_t m = n + (int64_t)dx * g.plane;
    if (dy) {
        int yd = y + dy;
        m += (int64_t)dy * g.nz;
        if (yd < 0) m += g.plane; else if (yd >= g.ny) m -= g.plane;
    }
    if (dz) {
        int zd = z + dz;
        m += dz;
        if (zd < 0) m += g.nz; else if (zd >= g.nz) m -= g.nz;
    }
    return m;
}

// Row-blocked traversal: a block walks whole z-rows (x, y fixed), so x and y
// come from one 32-bit division per row and the neighbour offsets are row
// constants.  Offsets inside one population array are 32-bit (the context
// refuses lattices with 19*N >= 2^32).
struct Site {
    uint32_t n;
    int32_t oxm, oxp, oym, oyp, ozm, ozp;
    bool hxm, hxp;     // x-1 / x+1 inside 0..nx-1
    __device__ __forceinline__ uint32_t at(int dx, int dy, int dz) const {
        int32_t o = 0;
        if (dx < 0) o += oxm; else if (dx > 0) o += oxp;
        if (dy < 0) o += oym; else if (dy > 0) o += oyp;
        if (dz < 0) o += ozm; else if (dz > 0) o += ozp;
        return (uint32_t)((int32_t)n + o);
    }
    __device__ __forceinline__ bool inx(int dx) const { return dx < 0 ? hxm : (dx > 0 ? hxp : true); }
};

__device__ __forceinline__ Site make_site(const Geo& g, int x, int y, int z, uint32_t n) {
    Site s;
    s.n = n;
    const int32_t plane = (int32_t)g.plane, nz = g.nz;
    s.oxm = -plane; s.oxp = plane;
    s.oym = (y == 0) ? (g.ny - 1) * nz : -nz;
    s.oyp = (y == g.ny - 1) ? -(g.ny - 1) * nz : nz;
    s.ozm = (z == 0) ? nz - 1 : -1;
    s.ozp = (z == nz - 1) ? -(nz - 1) : 1;
    s.hxm = x > 0;
    s.hxp = x < g.nx - 1;
    return s;
}

// Threads of a block cover `rows_per_block` consecutive z-rows when nz is
// smaller than the block, or loop over z in block-sized chunks otherwise.
struct RowMap {
    int rpb;      // rows per block iteration
    int lrow;     // this thread's row within the block's rows
    int z0;       // this thread's first z
    int zstep;    // z stride
    bool active;  // thread maps to a z
};

__device__ __forceinline__ RowMap make_rowmap(int nz) {
    RowMap r;
    const int bd = blockDim.x, t = threadIdx.x;
    if (nz >= bd) { r.rpb = 1; r.lrow = 0; r.z0 = t; r.zstep = bd; r.active = true; }
    else {
        r.rpb = bd / nz;
        r.lrow = t / nz;
        r.z0 = t - r.lrow * nz;
        r.zstep = nz;
        r.active = r.lrow < r.rpb;
    }
    return r;
}

}  // namespace cl
