// biofilm.cu -- cellular-automaton biofilm: the reference's CA block
// (src/complab.cpp:1453-1715) as whole-lattice sweeps.
//
//   updateLocalMaskNtotalLattices3D (complab3d_processors_part2.hh:71-235):
//     total biomass per voxel and the pore <-> biofilm reclassification at
//     thrd_biofilm_fraction * Bmax;
//   pushExcessBiomass3D / halfPushExcessBiomass3D (part1.hh:432-894): an
//     over-full voxel hands its excess to its non-wall face neighbours in a
//     random order, up to each one's room below Bmax, and whatever is left to
//     one neighbour chosen by the age wavefront (or at random);
//   updateAgeDistance3D (part2.hh:717-842): the age wavefront, every 50 sweeps.
//
// The reference runs each sweep serially over the lattice, writing the
// neighbours' biomass in place, but it reads the capacities from its total
// lattice, which only the update between sweeps refreshes.  Here every
// over-full voxel plans its outflows at once from the sweep's starting totals
// and biomass (its per-face, per-microbe outflows go to ca_out), and every
// voxel then gathers: its biomass minus its own outflows plus what its face
// neighbours sent it, in a fixed order, so a sweep is deterministic.  A
// counter-based hash of (seed, sweep, site) replaces std::random_shuffle and
// std::rand.  The age sweeps read the previous ages (Jacobi) and run to the
// fixed point.
#include <cmath>
#include <cstring>
#include "internal.h"

namespace cl {

constexpr double kCaThrd = 1e-12;        // thrd (src/complab3d_processors.hh:60): push and loop
constexpr double kCaEps = 1e-14;         // COMPLAB_THRD (src/complab_functions.hh:64): mask, total, age

// splitmix64 finaliser over (seed, stream, site)
__host__ __device__ __forceinline__ uint64_t ca_hash(uint64_t seed, uint64_t stream, uint64_t site) {
    uint64_t z = seed ^ (stream * 0x9E3779B97F4A7C15ull) ^ (site * 0xD1B54A32D192ED03ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct CaK {
    Geo g;
    uint8_t* mask;
    uint8_t* mask_new;
    double* bio;                 // M*N
    double* total;               // N
    const int32_t* age_in;
    int32_t* age_out;
    const uint8_t* distpos;
    double* out;                 // 6*M*N
    int M, half;
    double bmax, thrd_mass;
    int solid, bb, n_pore;
    int pore[CL_MAX_CODES];
    int code[CL_MAX_MICROBES];
    uint64_t seed, sweep;
    unsigned long long* counter;
};

__device__ __forceinline__ bool ca_pore(const CaK& k, int m) {
    for (int i = 0; i < k.n_pore; ++i) if (k.pore[i] == m) return true;
    return false;
}
__device__ __forceinline__ bool ca_wall(const CaK& k, int m) { return m == k.solid || m == k.bb; }

// face directions in the reference's order +x -x +y -y +z -z
__device__ __constant__ int kD6[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};

// one sweep, phase 1: outflows of every over-full voxel
__global__ void ca_plan_kernel(CaK k) {
    const int64_t N = k.g.N;
    const int M = k.M;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) {
        for (int d = 0; d < 6; ++d)
            for (int m = 0; m < M; ++m) k.out[((int64_t)d * M + m) * N + n] = 0.0;
        int x, y, z;
        decode(k.g, n, x, y, z);
        if (x < 1 || x > k.g.nx - 2) continue;
        const int mk = k.mask[n];
        if (ca_wall(k, mk) || (k.half && ca_pore(k, mk))) continue;
        double bMt = k.total[n];
        if (!(bMt > k.bmax)) continue;
        double bMd = k.half ? bMt * 0.5 : bMt - k.bmax;
        if (!k.half && !(bMd > kCaThrd)) continue;
        int cand[6], nc = 0;
        int64_t qn[6];
        for (int d = 0; d < 6; ++d) {
            const int ax = x + kD6[d][0], ay = y + kD6[d][1], az = z + kD6[d][2];
            if (ax < 1 || ax > k.g.nx - 2 || ay < 0 || ay >= k.g.ny || az < 0 || az >= k.g.nz) continue;
            const int64_t q = ((int64_t)ax * k.g.ny + ay) * k.g.nz + az;
            if (ca_wall(k, k.mask[q])) continue;
            qn[nc] = q;
            cand[nc++] = d;
        }
        if (nc == 0) continue;          // boxed in: the excess stays
        double Bc[CL_MAX_MICROBES];
        for (int m = 0; m < M; ++m) Bc[m] = k.bio[(int64_t)m * N + n];
        int order[6];
        for (int t = 0; t < nc; ++t) order[t] = t;
        if (nc > 1) {
            const uint64_t r = ca_hash(k.seed, 2 * k.sweep, (uint64_t)n);
            for (int i = nc - 1; i > 0; --i) {
                const int j = (int)((r >> (8 * i)) & 0xff) % (i + 1);
                const int tmp = order[i]; order[i] = order[j]; order[j] = tmp;
            }
        }
        bool chk = false;
        for (int t = 0; t < nc; ++t) {
            const int d = cand[order[t]];
            const int64_t q = qn[order[t]];
            const double nbrbMt = ca_pore(k, k.mask[q]) ? 0.0 : k.total[q];
            if (nbrbMt < k.bmax) {
                const double cap = k.bmax - nbrbMt;
                double partial = bMd;
                if (bMd > cap) { partial = cap; bMd -= cap; }
                else { bMd = 0.0; chk = true; }
                for (int m = 0; m < M; ++m) {
                    const double shove = __dmul_rn(Bc[m] / bMt, partial);
                    if (shove > kCaThrd) { Bc[m] -= shove; k.out[((int64_t)d * M + m) * N + n] += shove; }
                }
                bMt -= partial;
            }
            if (chk) break;
        }
        if (chk) continue;
        // the rest to one neighbour: older-age side first (age directed), else any
        int tl[6], nt = 0;
        const int a0 = k.age_in[n];
        for (int t = 0; t < nc; ++t) {
            const int a1 = k.age_in[qn[t]];
            if (k.half ? a0 >= a1 : a0 > a1) tl[nt++] = cand[t];
        }
        const uint64_t r = ca_hash(k.seed, 2 * k.sweep + 1, (uint64_t)n);
        int pick;
        if (nt > 1) pick = tl[r % (uint64_t)nt];
        else if (nt == 1) pick = tl[0];
        else pick = cand[nc > 1 ? (int)(r % (uint64_t)nc) : 0];
        for (int m = 0; m < M; ++m) {
            const double shove = __dmul_rn(Bc[m] / bMt, bMd);
            Bc[m] -= shove;
            k.out[((int64_t)pick * M + m) * N + n] += shove;
        }
    }
}

// one sweep, phase 2: every voxel gathers (own outflows out, neighbours' in)
__global__ void ca_apply_kernel(CaK k) {
    const int64_t N = k.g.N;
    const int M = k.M;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) {
        int x, y, z;
        decode(k.g, n, x, y, z);
        for (int m = 0; m < M; ++m) {
            double b = k.bio[(int64_t)m * N + n];
            for (int d = 0; d < 6; ++d) b -= k.out[((int64_t)d * M + m) * N + n];
            for (int d = 0; d < 6; ++d) {
                const int wx = x - kD6[d][0], wy = y - kD6[d][1], wz = z - kD6[d][2];
                if (wx < 1 || wx > k.g.nx - 2 || wy < 0 || wy >= k.g.ny || wz < 0 || wz >= k.g.nz) continue;
                const int64_t w = ((int64_t)wx * k.g.ny + wy) * k.g.nz + wz;
                b += k.out[((int64_t)d * M + m) * N + w];
            }
            k.bio[(int64_t)m * N + n] = b;
        }
    }
}

// updateLocalMaskNtotalLattices3D: total and reclassification, new masks into
// mask_new (the pore relabel reads the neighbours' previous masks).  Counters:
// [0] masks changed, [1] sum of the new masks, [2] the largest total as the
// bits of a non-negative double (their integer order is the numeric order).
__global__ void ca_mask_total_kernel(CaK k) {
    const int64_t N = k.g.N;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long changed = 0, masksum = 0, maxbits = 0;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) {
        const int mk = k.mask[n];
        int newmask_out = mk;
        if (!ca_wall(k, mk)) {
            double bmass = 0.0;
            int newmask = 0;
            for (int m = 0; m < k.M; ++m) {
                const double bm = k.bio[(int64_t)m * N + n];
                if (bm > kCaEps) { bmass += bm; newmask += k.code[m]; }
            }
            if (fabs(bmass - k.total[n]) > kCaEps) k.total[n] = bmass;
            const bool poreflag = ca_pore(k, mk);
            if (!poreflag && bmass < k.thrd_mass) {
                newmask = k.pore[0];
                if (k.n_pore > 1) {
                    int x, y, z;
                    decode(k.g, n, x, y, z);
                    for (int d = 0; d < 6; ++d) {
                        const int ax = x + kD6[d][0], ay = y + kD6[d][1], az = z + kD6[d][2];
                        if (ax < 0 || ax >= k.g.nx || ay < 0 || ay >= k.g.ny || az < 0 || az >= k.g.nz) continue;
                        const int nm = k.mask[((int64_t)ax * k.g.ny + ay) * k.g.nz + az];
                        if (!ca_wall(k, nm) && ca_pore(k, nm)) { newmask = nm; break; }
                    }
                }
                newmask_out = newmask;
            } else if (poreflag && bmass >= k.thrd_mass && newmask > 0) {
                newmask_out = newmask;
            }
        }
        // the maximum covers every voxel, walls included (a sealed voxel keeps
        // its last total, as the reference's total lattice does)
        const double t = k.total[n];
        const unsigned long long tb = (unsigned long long)__double_as_longlong(t);
        if (t > 0.0 && tb > maxbits) maxbits = tb;
        k.mask_new[n] = (uint8_t)newmask_out;
        if (newmask_out != mk) ++changed;
        masksum += (unsigned long long)newmask_out;
    }
    for (int o = 16; o > 0; o >>= 1) {
        changed += __shfl_down_sync(0xffffffffu, changed, o);
        masksum += __shfl_down_sync(0xffffffffu, masksum, o);
        const unsigned long long mb = __shfl_down_sync(0xffffffffu, maxbits, o);
        if (mb > maxbits) maxbits = mb;
    }
    if ((threadIdx.x & 31) == 0) {
        if (changed) atomicAdd(k.counter, changed);
        if (masksum) atomicAdd(k.counter + 1, masksum);
        if (maxbits) atomicMax(k.counter + 2, maxbits);
    }
}

// updateAgeDistance3D, one Jacobi sweep
__global__ void ca_age_kernel(CaK k) {
    const int64_t N = k.g.N;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long changed = 0;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) {
        const int age = k.age_in[n];
        int out_age = age;
        const double B = k.total[n];
        if (B > kCaEps) {
            int x, y, z;
            decode(k.g, n, x, y, z);
            int64_t qs[6];
            int nq = 0;
            for (int d = 0; d < 6; ++d) {
                const int ax = x + kD6[d][0], ay = y + kD6[d][1], az = z + kD6[d][2];
                if (ax < 0 || ax >= k.g.nx || ay < 0 || ay >= k.g.ny || az < 0 || az >= k.g.nz) continue;
                const int64_t q = ((int64_t)ax * k.g.ny + ay) * k.g.nz + az;
                if (k.distpos[q]) qs[nq++] = q;
            }
            if (age == 0) out_age = 1;
            else if (age == 1 && (B - k.bmax) > -kCaEps) {
                bool upd = true;
                for (int t = 0; t < nq; ++t) if (k.age_in[qs[t]] == 0) { upd = false; break; }
                if (upd) out_age = 2;
            } else {
                int count = 0;
                for (int t = 0; t < nq; ++t)
                    if (k.age_in[qs[t]] >= age && (k.total[qs[t]] - k.bmax) > -kCaEps) ++count;
                if (count == nq) out_age = age + 1;
            }
        }
        k.age_out[n] = out_age;
        if (out_age != age) ++changed;
    }
    for (int o = 16; o > 0; o >>= 1) changed += __shfl_down_sync(0xffffffffu, changed, o);
    if ((threadIdx.x & 31) == 0 && changed) atomicAdd(k.counter, changed);
}

// ages from the mask (createAgeDomain3D, complab3d_processors_part3.hh:350-370:
// -1 wall, 0 pore, 1 biofilm) and the sign of the reference's distance field
// (calculateDistanceFromSolid, complab.cpp:581: positive on non-wall voxels
// except on the last index of each axis, which it does not visit)
// (and the mask sum into counter[1])
__global__ void ca_init_kernel(CaK k) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long masksum = 0;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < k.g.N; n += stride) {
        int x, y, z;
        decode(k.g, n, x, y, z);
        const int m = k.mask[n];
        const bool wall = ca_wall(k, m);
        k.age_out[n] = wall ? -1 : (ca_pore(k, m) ? 0 : 1);
        const_cast<uint8_t*>(k.distpos)[n] = (uint8_t)(!wall && x < k.g.nx - 1 && y < k.g.ny - 1 && z < k.g.nz - 1);
        masksum += (unsigned long long)m;
    }
    for (int o = 16; o > 0; o >>= 1) masksum += __shfl_down_sync(0xffffffffu, masksum, o);
    if ((threadIdx.x & 31) == 0 && masksum) atomicAdd(k.counter + 1, masksum);
}

__global__ void ca_age_to_double(const int32_t* age, double* out, int64_t N) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) out[n] = (double)age[n];
}

static CaK make_cak(Ctx* c) {
    CaK k{};
    const int src = c->ca_age_src;
    k.g = c->geo;
    k.mask = c->d_mask;
    k.mask_new = reinterpret_cast<uint8_t*>(c->d_scratch);       // N bytes at the start of scratch
    k.bio = c->d_bio;
    k.total = c->d_ca_total;
    k.age_in = c->d_ca_age + (int64_t)src * c->geo.N;
    k.age_out = c->d_ca_age + (int64_t)(1 - src) * c->geo.N;
    k.distpos = c->d_ca_distpos;
    k.out = c->d_ca_out;
    k.M = c->cfg.n_microbes;
    k.half = c->cfg.ca_half;
    k.bmax = c->cfg.ca_bmax;
    k.thrd_mass = c->cfg.ca_thrd_frac * c->cfg.ca_bmax;
    k.solid = c->cfg.solid_code;
    k.bb = c->cfg.bb_code;
    k.n_pore = c->cfg.n_pore_codes;
    for (int i = 0; i < CL_MAX_CODES; ++i) k.pore[i] = c->cfg.pore_codes[i];
    for (int m = 0; m < CL_MAX_MICROBES; ++m) k.code[m] = c->cfg.microbe_code[m];
    k.seed = c->cfg.ca_seed;
    k.sweep = c->ca_sweeps;
    // three counters in the last doubles of scratch (N + 65536 doubles), clear of mask_new
    k.counter = reinterpret_cast<unsigned long long*>(c->d_scratch + c->scratch_bytes / sizeof(double) - 3);
    return k;
}

static int ca_blocks(const Ctx* c) { return grid_for(c->geo.N, 256, 148 * 16); }



// launch one counting kernel and read its three counters back
template <class F>
static int counted(Ctx* c, const CaK& k, F launch, unsigned long long out[3]) {
    CL_CUDA(cudaMemsetAsync(k.counter, 0, 3 * sizeof(unsigned long long), c->stream));
    launch();
    CL_LAUNCH_CHECK("ca kernel");
    c->launches += 1;
    CL_CUDA(cudaMemcpyAsync(out, k.counter, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return CL_OK;
}

// the ages, the distance sign and the mask-sum baseline (complab.cpp:1070)
int ca_init(Ctx* c) {
    if (!c->d_ca_age) return CL_OK;
    c->ca_age_src = 1;                 // make_cak writes age_out = plane 0
    CaK k = make_cak(c);
    unsigned long long h[3] = {0, 0, 0};
    int r = counted(c, k, [&] { ca_init_kernel<<<ca_blocks(c), 256, 0, c->stream>>>(k); }, h);
    if (r) return r;
    c->ca_age_src = 0;
    CL_CUDA(cudaMemsetAsync(c->d_ca_total, 0, sizeof(double) * c->geo.N, c->stream));
    CL_CUDA(cudaMemsetAsync(c->d_ca_out, 0, sizeof(double) * 6 * c->cfg.n_microbes * c->geo.N, c->stream));
    c->ca_sweeps = 0;
    c->ca_mask_sum = (int64_t)h[1];
    return CL_OK;
}

// updateLocalMaskNtotalLattices3D over the lattice; *masksum = sum of the new
// masks, *tmax = the largest total (computeMax of the total lattice)
static int mask_total(Ctx* c, int64_t* changes, int64_t* masksum, double* tmax = nullptr) {
    CaK k = make_cak(c);
    unsigned long long h[3] = {0, 0, 0};
    int r = counted(c, k, [&] { ca_mask_total_kernel<<<ca_blocks(c), 256, 0, c->stream>>>(k); }, h);
    if (r) return r;
    if (h[0]) CL_CUDA(cudaMemcpyAsync(c->d_mask, k.mask_new, c->geo.N, cudaMemcpyDeviceToDevice, c->stream));
    *changes += (int64_t)h[0];
    if (masksum) *masksum = (int64_t)h[1];
    if (tmax) { double t; std::memcpy(&t, &h[2], sizeof t); *tmax = t; }
    return CL_OK;
}

// one updateAgeDistance3D pass; *changed = voxels whose age changed
static int age_sweep(Ctx* c, int64_t* changed) {
    CaK k = make_cak(c);
    unsigned long long h[3] = {0, 0, 0};
    int r = counted(c, k, [&] { ca_age_kernel<<<ca_blocks(c), 256, 0, c->stream>>>(k); }, h);
    if (r) return r;
    c->ca_age_src ^= 1;
    *changed = (int64_t)h[0];
    return CL_OK;
}

int ca_update_mask(Ctx* c, int64_t* changes_out) {
    if (!c->d_ca_age) { set_error("the cellular automaton is not enabled in this context"); return CL_ERR_STATE; }
    int64_t changes = 0, sum = 0;
    int r = mask_total(c, &changes, &sum);
    if (r) return r;
    c->ca_mask_sum = sum;
    if (changes && (r = refresh_flags(c))) return r;
    if (changes_out) *changes_out = changes;
    return CL_OK;
}

int ca_redistribute(Ctx* c, int32_t* sweeps_out, int64_t* changes_out, double* bmax_after) {
    if (!c->d_ca_age) { set_error("the cellular automaton is not enabled in this context"); return CL_ERR_STATE; }
    int64_t changes = 0, sum = 0;
    double gmax = 0.0;
    int r = mask_total(c, &changes, &sum, &gmax);
    if (r) return r;
    if (!std::isfinite(gmax)) { set_error("cellular automaton: non-finite biomass"); return CL_ERR_DIVERGED; }
    int status = CL_OK, sweeps = 0;
    const double bmax = c->cfg.ca_bmax;
    if (gmax - bmax > kCaThrd) {
        double prev = gmax;
        int stall = 0;
        for (int64_t whilecount = 0; gmax - bmax > kCaThrd; ++whilecount) {
            CaK k = make_cak(c);
            ca_plan_kernel<<<ca_blocks(c), 256, 0, c->stream>>>(k);
            CL_LAUNCH_CHECK("ca_plan_kernel");
            ca_apply_kernel<<<ca_blocks(c), 256, 0, c->stream>>>(k);
            CL_LAUNCH_CHECK("ca_apply_kernel");
            c->launches += 2;
            c->ca_sweeps += 1;
            ++sweeps;
            if ((r = mask_total(c, &changes, &sum, &gmax))) return r;
            // complab.cpp:1696-1710: the reference ends the run when 100 sweeps
            // bring no decrease of the maximum, when the age relaxation takes
            // more than 1000 passes, or after 1001 sweeps
            if (gmax > prev - kCaThrd) { if (++stall >= 100) { status = CL_WARN_NOT_CONVERGED; break; } }
            else stall = 0;
            prev = gmax;
            if (whilecount % 50 == 0) {
                int64_t changed = 1;
                int passes = 0;
                while (changed != 0) {
                    if ((r = age_sweep(c, &changed))) return r;
                    if (++passes > 1000) break;
                }
                if (changed != 0) { status = CL_WARN_NOT_CONVERGED; break; }
            }
            if (whilecount > 1000) { status = CL_WARN_NOT_CONVERGED; break; }
        }
    }
    // complab.cpp:1736-1739: one age pass when the mask sum moved since the
    // last check (this call's CA changes and any conversions before it)
    if (sum != c->ca_mask_sum) {
        int64_t changed = 0;
        if ((r = age_sweep(c, &changed))) return r;
        c->ca_mask_sum = sum;
    }
    if (changes && (r = refresh_flags(c))) return r;
    if (sweeps_out) *sweeps_out = sweeps;
    if (changes_out) *changes_out = changes;
    if (bmax_after) *bmax_after = gmax;
    return status;
}

// field reads: the age plane in use and the totals
int ca_field(Ctx* c, int which, double* d_out) {
    if (!c->d_ca_age) { set_error("the cellular automaton is not enabled in this context"); return CL_ERR_STATE; }
    if (which == CL_FIELD_CA_TOTAL) {
        CL_CUDA(cudaMemcpyAsync(d_out, c->d_ca_total, sizeof(double) * c->geo.N, cudaMemcpyDeviceToDevice, c->stream));
        return CL_OK;
    }
    ca_age_to_double<<<ca_blocks(c), 256, 0, c->stream>>>(c->d_ca_age + (int64_t)c->ca_age_src * c->geo.N, d_out, c->geo.N);
    CL_LAUNCH_CHECK("ca_age_to_double");
    return CL_OK;
}

// ---- finite-difference sessile biomass (solver_type FD) ---------------------
// fdDiffusion3D (src/complab3d_processors_part2.hh:258-420): one explicit
// step B += nu * (d2B/dx2 + d2B/dy2 + d2B/dz2) of the biomass of the microbes
// in `sel`, on the sites of x = 1 .. nx-2 whose material number exceeds 1,
// reading the copy taken before the step.  Per direction, the upstream side
// at the lattice's first plane or next to a site with a material number
// below 2 takes the centre value (no flux); otherwise the downstream side
// does so at the last plane or next to such a site; otherwise both
// neighbours are read (the reference's order of tests, so a site walled on
// both sides still reads its downstream neighbour).  Values below thrd count
// as zero; a result not above thrd leaves the biomass as it was.  A
// neighbour outside the lattice reads zero.  The sums follow the reference's
// order with no fused multiply-adds, so the oracle's FP64 result is matched
// bit for bit.
__global__ void fd_diffuse_kernel(Geo g, const uint8_t* __restrict__ mask, const double* __restrict__ copy,
                                  double* __restrict__ bio, int M, uint32_t sel, double nu) {
    const int64_t N = g.N, plane = g.plane, nz = g.nz;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) {
        int x, y, z;
        decode(g, n, x, y, z);
        if (x < 1 || x > g.nx - 2 || mask[n] <= 1) continue;
        int mxp = 0, mxn = 0, myp = 0, myn = 0, mzp = 0, mzn = 0;
        if (x == 1) mxp = mask[n + plane];
        else if (x == g.nx - 2) mxn = mask[n - plane];
        else { mxp = mask[n + plane]; mxn = mask[n - plane]; }
        if (y == 0) { if (y + 1 < g.ny) myp = mask[n + nz]; }
        else if (y == g.ny - 1) myn = mask[n - nz];
        else { myp = mask[n + nz]; myn = mask[n - nz]; }
        if (z == 0) { if (z + 1 < g.nz) mzp = mask[n + 1]; }
        else if (z == g.nz - 1) mzn = mask[n - 1];
        else { mzp = mask[n + 1]; mzn = mask[n - 1]; }
        for (int m = 0; m < M; ++m) {
            if (!((sel >> m) & 1u)) continue;
            const double* cp = copy + (int64_t)m * N;
            auto at = [&](int64_t q, bool inside) { return inside ? cp[q] : 0.0; };
            double b0 = cp[n], bxp, bxn, byp, byn, bzp, bzn;
            if (x == 1 || mxn < 2) { bxp = at(n + plane, x + 1 < g.nx); bxn = b0; }
            else if (x == g.nx - 2 || mxp < 2) { bxp = b0; bxn = cp[n - plane]; }
            else { bxp = cp[n + plane]; bxn = cp[n - plane]; }
            if (y == 0 || myn < 2) { byp = at(n + nz, y + 1 < g.ny); byn = b0; }
            else if (y == g.ny - 1 || myp < 2) { byp = b0; byn = cp[n - nz]; }
            else { byp = cp[n + nz]; byn = cp[n - nz]; }
            if (z == 0 || mzn < 2) { bzp = at(n + 1, z + 1 < g.nz); bzn = b0; }
            else if (z == g.nz - 1 || mzp < 2) { bzp = b0; bzn = cp[n - 1]; }
            else { bzp = cp[n + 1]; bzn = cp[n - 1]; }
            if (b0 < kCaEps) b0 = 0.0;
            if (bxp < kCaEps) bxp = 0.0;
            if (bxn < kCaEps) bxn = 0.0;
            if (byp < kCaEps) byp = 0.0;
            if (byn < kCaEps) byn = 0.0;
            if (bzp < kCaEps) bzp = 0.0;
            if (bzn < kCaEps) bzn = 0.0;
            const double b2 = 2.0 * b0;
            const double lx = __dadd_rn(__dadd_rn(bxp, -b2), bxn);
            const double ly = __dadd_rn(__dadd_rn(byp, -b2), byn);
            const double lz = __dadd_rn(__dadd_rn(bzp, -b2), bzn);
            const double nb = __dadd_rn(b0, __dmul_rn(nu, __dadd_rn(__dadd_rn(lx, ly), lz)));
            if (nb > kCaEps) bio[(int64_t)m * N + n] = nb;
        }
    }
}

int fd_diffuse(Ctx* c, double nu, uint32_t sel) {
    const int M = c->cfg.n_microbes;
    const int64_t N = c->geo.N;
    if (M <= 0 || !c->d_bio) { set_error("cl_fd_diffuse: no sessile biomass"); return CL_ERR_STATE; }
    if (!c->d_fd_copy) { int r = dalloc(c, &c->d_fd_copy, (size_t)M * N); if (r) return r; }
    CL_CUDA(cudaMemcpyAsync(c->d_fd_copy, c->d_bio, sizeof(double) * M * N, cudaMemcpyDeviceToDevice, c->stream));
    fd_diffuse_kernel<<<grid_for(N, 256, 148 * 16), 256, 0, c->stream>>>(c->geo, c->d_mask, c->d_fd_copy, c->d_bio, M,
                                                                        sel, nu);
    CL_LAUNCH_CHECK("fd_diffuse_kernel");
    c->launches += 1;
    return CL_OK;
}

}  // namespace cl
