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
// class-byte flags
enum : uint8_t { F_REACTIVE = 4, F_SURFACE = 8 };

struct Geo {
    int nx, ny, nz;
    int64_t N, plane;   // N = nx*ny*nz, plane = ny*nz
};

__device__ __forceinline__ void decode(const Geo& g, int64_t n, int& x, int& y, int& z) {
    int64_t q = n / g.nz;
    z = (int)(n - q * g.nz);
    x = (int)(q / g.ny);
    y = (int)(q - (int64_t)x * g.ny);
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

}  // namespace cl
