// storage.cu -- compact storage of the transport populations (and the
// index assignment the flow's compact storage shares).
//
// A step reads and writes the slots of the live sites (the AA read and write
// sets of a site are its own slots and, in the odd parity, the slots its face
// neighbours own), so only the live sites and their face neighbours need
// storage; solid interiors behind the bounce-back shell never do.  Stored
// sites get storage indices in site order, so the slots of a run of pore
// sites along z are contiguous in every population array and a warp's loads
// fill whole sectors, where the full-lattice layout fetched the solid sites'
// slots at the ends of every run with them.
//
// The set only grows: a site whose slots were never read or written still
// holds the values the initialisation gave every site (t_i * c0), so a site
// entering the set starts from those, and a site leaving the need keeps its
// slots.  Reads of sites without storage (field output) fall back to the same
// initial values.
#include <vector>
#include "internal.h"

namespace cl {

constexpr int kStoreBlocks = 148 * 8;

struct InitPop { float c0[CL_MAX_SOLUTES]; };   // per mobile slot

__device__ __forceinline__ bool ade_live(uint8_t cls, int nodyn_coupled) {
    const uint8_t dyn = cls & 3;
    return !((dyn == BB && !(cls & F_REACTIVE)) || (dyn == NODYN && !nodyn_coupled));
}

// need[n] = 1 when site n has no storage yet and is live, next to a live site, or all is set
__global__ void store_need_kernel(Geo g, const uint8_t* cls, int nodyn_coupled, int all, const int32_t* sidx,
                                  const uint8_t* extra, uint8_t* need) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        bool nd = false;
        if (sidx[n] < 0) {
            if (all || ade_live(cls[n], nodyn_coupled) || (extra && extra[n])) nd = true;
            else {
                int x, y, z;
                decode(g, n, x, y, z);
                const int d6[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};
                for (int d = 0; d < 6 && !nd; ++d) {
                    const int64_t q = nbr(g, n, x, y, z, d6[d][0], d6[d][1], d6[d][2]);
                    if (q >= 0 && ade_live(cls[q], nodyn_coupled)) nd = true;
                }
            }
        }
        need[n] = nd ? 1 : 0;
    }
}

__global__ void store_count_kernel(const uint8_t* need, int64_t N, int64_t chunk, int64_t* counts) {
    __shared__ int64_t s_part[8];
    const int64_t b0 = (int64_t)blockIdx.x * chunk, b1 = min(N, b0 + chunk);
    int64_t cnt = 0;
    for (int64_t n = b0 + threadIdx.x; n < b1; n += blockDim.x) cnt += need[n];
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_part[w];
        counts[blockIdx.x] = t;
    }
}

// blockDim.x == 256; writes the new sites in site order from base + offsets[block]
__global__ void store_write_kernel(const uint8_t* need, int64_t N, int64_t chunk, const int64_t* offsets,
                                   int64_t base, uint32_t* site_of, int32_t* sidx) {
    __shared__ int s_warp[8];
    __shared__ int64_t s_base;
    const int64_t b0 = (int64_t)blockIdx.x * chunk, b1 = min(N, b0 + chunk);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_base = base + offsets[blockIdx.x];
    __syncthreads();
    for (int64_t r0 = b0; r0 < b1; r0 += blockDim.x) {
        const int64_t n = r0 + threadIdx.x;
        const bool hit = n < b1 && need[n];
        const unsigned ball = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) s_warp[w] = __popc(ball);
        __syncthreads();
        int before = 0, total = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { if (q < w) before += s_warp[q]; total += s_warp[q]; }
        if (hit) {
            const int64_t idx = s_base + before + __popc(ball & ((1u << lane) - 1u));
            if (site_of) site_of[idx] = (uint32_t)n;
            sidx[n] = (int32_t)idx;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_base += total;
        __syncthreads();
    }
}

// the initial populations (t_i * c0) into the slots of storage indices [lo, hi)
__global__ void store_init_kernel(float* pop, int64_t N, int n_mob, InitPop ip, int64_t lo, int64_t hi) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < hi; s += stride)
        for (int m = 0; m < n_mob; ++m) {
            const float c = ip.c0[m];
#pragma unroll
            for (int i = 0; i < 7; ++i) pop[((int64_t)m * 7 + i) * N + s] = t7(i) * c;
        }
}

// Storage indices for the sites flagged in need (scratch, N bytes), in site
// order after the *n_stored already assigned; *first and *added give the new
// range.  site_of (may be null) records the site of each new index.
int assign_storage(Ctx* c, const uint8_t* need, int32_t* sidx, uint32_t* site_of, int64_t* n_stored,
                   int64_t* first, int64_t* added) {
    const int64_t N = c->geo.N;
    int64_t* counts = reinterpret_cast<int64_t*>(c->d_scratch + N / 8 + 8);  // after the need bytes
    const int64_t chunk = (N + kStoreBlocks - 1) / kStoreBlocks;
    store_count_kernel<<<kStoreBlocks, 256, 0, c->stream>>>(need, N, chunk, counts);
    CL_LAUNCH_CHECK("store_count_kernel");
    std::vector<int64_t> h(kStoreBlocks);
    CL_CUDA(cudaMemcpyAsync(h.data(), counts, sizeof(int64_t) * kStoreBlocks, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    int64_t total = 0;
    for (int b = 0; b < kStoreBlocks; ++b) { const int64_t v = h[b]; h[b] = total; total += v; }
    *first = *n_stored;
    *added = total;
    if (total == 0) return CL_OK;
    if (*n_stored + total > N) { set_error("storage overflow"); return CL_ERR_STATE; }
    CL_CUDA(cudaMemcpyAsync(counts, h.data(), sizeof(int64_t) * kStoreBlocks, cudaMemcpyHostToDevice, c->stream));
    store_write_kernel<<<kStoreBlocks, 256, 0, c->stream>>>(need, N, chunk, counts, *n_stored, site_of, sidx);
    CL_LAUNCH_CHECK("store_write_kernel");
    CL_CUDA(cudaStreamSynchronize(c->stream));   // h is read by the copy above
    *n_stored += total;
    return CL_OK;
}

int store_update(Ctx* c, int all, const uint8_t* extra) {
    const int64_t N = c->geo.N;
    if (!c->d_sidx) {
        int r = CL_OK;
        if ((r = dalloc(c, &c->d_sidx, (size_t)N)) || (r = dalloc(c, &c->d_site_of, (size_t)N))) return r;
        CL_CUDA(cudaMemsetAsync(c->d_sidx, 0xff, sizeof(int32_t) * N, c->stream));
        c->n_stored = 0;
    }
    if (c->n_stored == N) { c->store_dirty = false; return CL_OK; }
    uint8_t* need = reinterpret_cast<uint8_t*>(c->d_scratch);            // N bytes
    store_need_kernel<<<grid_for(N, 256, 148 * 16), 256, 0, c->stream>>>(
        c->geo, c->d_ade_cls, c->ade_nodyn_coupled ? 1 : 0, all, c->d_sidx, extra, need);
    CL_LAUNCH_CHECK("store_need_kernel");
    int64_t first = 0, total = 0;
    int r = assign_storage(c, need, c->d_sidx, c->d_site_of, &c->n_stored, &first, &total);
    if (r) return r;
    if (total > 0) {
        InitPop ip{};
        for (int m = 0; m < c->ap.n_mob; ++m) ip.c0[m] = (float)c->cfg.c0[c->ap.mob_index[m]];
        store_init_kernel<<<grid_for(total, 256, 148 * 16), 256, 0, c->stream>>>(
            c->d_g, N, c->ap.n_mob, ip, first, first + total);
        CL_LAUNCH_CHECK("store_init_kernel");
    }
    c->store_dirty = false;
    return CL_OK;
}

}  // namespace cl
