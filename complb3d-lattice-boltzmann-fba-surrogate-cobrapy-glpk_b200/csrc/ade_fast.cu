// ade_fast.cu -- the transport step of a compiled chemistry in one launch.
//
// For a configuration that matches a chemistry of chem.cuh every size is a
// compile-time constant, so the reaction chain of a voxel (run_kinetics +
// update_rxnLattices, abiotic + dissolution + update_abiotic_rxnLattices,
// run_equilibrium_biotic with Newton; src/complab.cpp:1252-1374) keeps its
// concentrations, increments and Newton state in registers, and the chain and
// the collide-stream of the voxel's populations run in the same thread:
//
//   per live site (one thread):
//     gather the populations of this step, sum each mobile solute's density
//     (the BGK collision keeps it, so it is the post-collision density the
//     processors read), run the chain, apply the immobile and biomass
//     increments;
//     gather again (the same slots, still in L1 / L2), collide, add t_i*dC,
//     scatter (AA pattern, in place).
//
// DRAM sees each population read once and written once.  The AA read and
// write sets of a site coincide and belong to no other site, so one thread
// owns its slots from the first gather to the scatter.
//
// The arithmetic is that of the run-time-table launches (ade_kernels.cuh)
// operation for operation, so both give the same fields.
#include "ade_kernels.cuh"
#include "chem.cuh"
#include "learned.cuh"

namespace cl {

// dissolution increments reaching voxel n (dissol_gather with the solute loop
// unrolled): the products of each phase-carrying face neighbour, and the
// voxel's own decrement at its phase substrate, in the reference's order
template <int S>
__device__ __forceinline__ void fast_dissol_gather(const AdeK& k, int64_t n, int x, int y, int z, uint8_t cls,
                                                   double (&D)[S]) {
    const AdeParams& p = k.p;
    const int64_t N = k.g.N, plane = k.g.plane, nz = k.g.nz;
    const int64_t q[7] = {n - plane, n - nz, n - 1, n, n + 1, n + nz, n + plane};
    const bool ok[7] = {x - 1 >= 1, y > 0, z > 0, (cls & F_PHASE_SELF) != 0,
                        z < k.g.nz - 1, y < k.g.ny - 1, x + 1 <= k.g.nx - 2};
#pragma unroll
    for (int j = 0; j < 7; ++j) {
        if (!ok[j]) continue;
        const int pid = k.phase[q[j]];
        if (pid == 0) continue;
        const int sM = p.phase[pid - 1].substrate;
        if (j == 3) {
            const double v = k.rel[(int64_t)sM * N + n];
#pragma unroll
            for (int s = 0; s < S; ++s) if (s == sM) D[s] += v;
            continue;
        }
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (s != sM) D[s] += k.rel[(int64_t)s * N + q[j]];
    }
}

// The reaction chain of one voxel on register arrays (reaction_chain with
// the Newton solver).  C: densities, updated as each processor applies its
// increments; A: the total increment per solute.  Returns 1 if the
// equilibrium solve did not converge.
template <class Chem>
__device__ __forceinline__ int fast_chain(const AdeK& k, const typename Chem::Consts& kc, int64_t n, uint32_t sto,
                                          int x, int y, int z, uint8_t cls, double (&C)[Chem::S],
                                          double (&A)[Chem::S]) {
    constexpr int S = Chem::S, M = Chem::M, MW = Chem::MW, NC = Chem::NC;
    const AdeParams& p = k.p;
    const int64_t N = k.g.N;
    int nonconv = 0;
    double R[S];
    // kinetics and the surrogate networks deposit into the same increments,
    // applied together (kinetics_increments + the update of reaction_chain)
    if (p.do_kin || (Chem::kSrg && p.n_srg > 0)) {
        double B[MW], BR[MW];
#pragma unroll
        for (int m = 0; m < MW; ++m) {
            const double b = m < M ? k.bio[m * N + n] : 0.0;
            B[m] = b < THRD ? 0.0 : b;
        }
        if (p.do_kin) {
            Chem::kinetics(p, C, B, R, BR, k.mask[n]);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const double d = R[s] * p.dt;
                R[s] = (d > THRD || d < -THRD) ? d : 0.0;
            }
#pragma unroll
            for (int m = 0; m < MW; ++m) {
                const double d = BR[m] * p.dt;
                BR[m] = (d > THRD || d < -THRD) ? d : 0.0;
            }
        } else {
#pragma unroll
            for (int s = 0; s < S; ++s) R[s] = 0.0;
#pragma unroll
            for (int m = 0; m < MW; ++m) BR[m] = 0.0;
        }
        if constexpr (Chem::kSrg) {
            if (p.n_srg > 0) Chem::surrogate(p, kc, C, B, R, BR);
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double d = R[s];
            if (d > THRD || d < -THRD) { C[s] += d; A[s] += d; }
        }
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const double d = BR[m];
            if (d > THRD || d < -THRD) {
                k.bio[m * N + n] += d;
            }
        }
    }
    const bool abio = p.do_abio && (!p.surface_only || (cls & F_SURFACE));
    const bool dis = p.do_dissol && (cls & (F_PHASE_NBR | F_PHASE_SELF));
    if (abio || dis) {
        if (abio) {
            Chem::abiotic(p, C, R, k.mask[n]);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const double d = R[s] * p.dt;
                R[s] = (d > THRD || d < -THRD) ? d : 0.0;
            }
        } else {
#pragma unroll
            for (int s = 0; s < S; ++s) R[s] = 0.0;
        }
        if (dis) fast_dissol_gather<S>(k, n, x, y, z, cls, R);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double d = R[s];
            if (d > THRD || d < -THRD) { C[s] += d; A[s] += d; }
        }
    }
    if constexpr (NC > 0) {
        if (!p.do_eq) return 0;
        const EqDev& e = k.e;
        const typename Chem::Tab tb{e};
        double x[NC], T[NC];
#pragma unroll
        for (int j = 0; j < NC; ++j) T[j] = 0.0;
#pragma unroll
        for (int i = 0; i < S; ++i) {
            if (!tb.active(i)) continue;
            const double c = fmin(fmax(C[i], 1e-30), 10.0);
#pragma unroll
            for (int j = 0; j < NC; ++j) {
                if constexpr (Chem::Tab::kFixed) { if (tb.ipow(i, j) == 0) continue; }
                T[j] = fma(tb.s(i, j), c, T[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < NC; ++j) T[j] = fmax(T[j], 1e-30);
        int conv = 0, it = 0;
        bool warm = false;
        double xprev[NC];
        if (k.eq_x) {
            warm = true;
            bool two = true;
#pragma unroll
            for (int j = 0; j < NC; ++j) {
                xprev[j] = (double)k.eq_x[(int64_t)j * N + sto];
                warm = warm && (xprev[j] == xprev[j]);
                const double xq = (double)k.eq_xp[(int64_t)j * N + sto];
                two = two && (xq == xq);
                x[j] = xprev[j];
                if (two) x[j] = fmin(fmax(2.0 * xprev[j] - xq, -30.0), 1.0);
            }
            if (!two) {
#pragma unroll
                for (int j = 0; j < NC; ++j) x[j] = xprev[j];
            }
        }
        // the reference's cold start: log10 of each component's own species
        auto cold = [&](double* xs) {
#pragma unroll
            for (int j = 0; j < NC; ++j) {
                const int idx = e.comp_species[j];
                double c = 1e-7;
#pragma unroll
                for (int s = 0; s < S; ++s) if (s == idx) c = C[s];
                xs[j] = log10(fmin(fmax(c, 1e-30), 10.0));
            }
        };
        // no previous solution of its own: the network's guess, once trained,
        // where it is closer to equilibrium than the cold start by the relative
        // mass-balance residual (the cold start reads the voxel's own species,
        // which transport keeps near equilibrium)
        if (!warm && k.learn_w) {
            LearnVec<NC> tv;
#pragma unroll
            for (int j = 0; j < NC; ++j) tv.v[j] = T[j];
            const LearnVec<NC> xv = learn_start<NC>(k.learn_w, k.learn_norm, tv);
#pragma unroll
            for (int j = 0; j < NC; ++j) x[j] = xv.v[j];
            double xc[NC], F[NC];
            cold(xc);
            warm = eq_residual_t<NC, S>(tb, T, x, F) < eq_residual_t<NC, S>(tb, T, xc, F);
        }
        for (int phase = warm ? 0 : 1; phase < 2; ++phase) {
            if (phase == 1) cold(x);
            it += eq_newton_t<NC, S>(tb, T, x, phase == 0 ? p.eq.warm_iter : p.eq.max_iter, p.eq.tol, &conv, R, 1);
            if (conv) break;
        }
        if (k.eq_x && conv) {
#pragma unroll
            for (int j = 0; j < NC; ++j) {
                k.eq_xp[(int64_t)j * N + sto] = (float)xprev[j];
                k.eq_x[(int64_t)j * N + sto] = (float)x[j];
            }
        }
        if (k.eq_iters) k.eq_iters[n] = it;
        if (conv && k.pair_T && learn_sampled((uint32_t)n, k.pair_salt, k.pair_mask))
            learn_store<NC>(k.pair_T, k.pair_X, k.pair_count, k.pair_cap, T, x);
        if (!conv) nonconv = 1;
        else {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const double conc = fmax(C[s], 1e-30);
                double eqc = !tb.active(s) ? fmin(conc, 10.0) : (NC <= 3 ? R[s] : species_c<NC>(e, s, x));
                eqc = fmin(fmax(eqc, 1e-30), 10.0);
                double d = eqc - conc;
                const double mx = fmax(1e-9, 0.1 * fabs(conc));
                if (fabs(d) > mx) d = d > 0 ? mx : -mx;
                if (conc + d < 1e-20) d = 1e-20 - conc;
                if (fabs(d) > THRD) { C[s] += d; A[s] += d; }
            }
        }
    }
    return nonconv;
}

template <class Chem, int PARITY, int kFastBlock, int kMinBlocks>
__global__ void __launch_bounds__(kFastBlock, kMinBlocks)
ade_fast_kernel(const __grid_constant__ AdeK k, const __grid_constant__ typename Chem::Consts kc,
                const uint32_t* __restrict__ list, int64_t count, int any_rxn) {
    constexpr int S = Chem::S, NMOB = Chem::NMOB;
    const AdeParams& p = k.p;
    const int64_t N = k.g.N, plane = k.g.plane;
    const uint32_t N32 = (uint32_t)N;
    unsigned long long nonconv = 0;
    for (int64_t r = (int64_t)blockIdx.x * kFastBlock + threadIdx.x; r < count; r += (int64_t)gridDim.x * kFastBlock) {
        const uint32_t n = list[r];
        const uint8_t cls = k.cls[n];
        const uint8_t dyn = cls & 3;
        int x, y, z;
        decode(k.g, n, x, y, z);
        SSite st;
        if (!make_ssite<PARITY>(k.g, k.sidx, x, y, z, n, st)) atomicAdd(&k.counters[1], 1ull);
        float dcv[NMOB];
#pragma unroll
        for (int m = 0; m < NMOB; ++m) dcv[m] = 0.f;
        if (any_rxn && (cls & F_REACTIVE)) {
            double C[S], A[S];
#pragma unroll
            for (int s0 = 0; s0 < S; s0 += kGroup) {
                float f[kGroup][7];
#pragma unroll
                for (int g = 0; g < kGroup; ++g)
                    if (s0 + g < S && Chem::mobile(s0 + g))
                        gather7<PARITY>(k.pop + (int64_t)Chem::slot(s0 + g) * 7 * N, N32, st, f[g]);
#pragma unroll
                for (int g = 0; g < kGroup; ++g) {
                    const int s = s0 + g;
                    if (s >= S) continue;
                    if (Chem::mobile(s)) {
                        float rr = 0.f;
#pragma unroll
                        for (int i = 0; i < 7; ++i) rr += f[g][i];
                        C[s] = (double)rr;
                    } else {
                        C[s] = k.imm[(int64_t)s * N + n];
                    }
                    A[s] = 0.0;
                }
            }
            nonconv += fast_chain<Chem>(k, kc, n, st.s, x, y, z, cls, C, A);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                if (Chem::mobile(s)) dcv[Chem::slot(s)] = (float)A[s];
                else if (A[s] != 0.0) k.imm[(int64_t)s * N + n] += A[s];
            }
        }
        const float ux = k.u[n], uy = k.u[N + n], uz = k.u[2 * N + n];
        const bool adj = (x == 1 || x == k.g.nx - 2);
        constexpr int kSG = stream_group<PARITY>();
#pragma unroll
        for (int m0 = 0; m0 < NMOB; m0 += kSG) {
            float f[kSG][7];
#pragma unroll
            for (int g = 0; g < kSG; ++g)
                if (m0 + g < NMOB) gather7<PARITY>(k.pop + (int64_t)(m0 + g) * 7 * N, N32, st, f[g]);
#pragma unroll
            for (int g = 0; g < kSG; ++g) {
                const int m = m0 + g;
                if (m >= NMOB) continue;
                float rho = 0.f;
                if (dyn == BB) {
#pragma unroll
                    for (int i = 1; i < 4; ++i) { const float tmp = f[g][i]; f[g][i] = f[g][i + 3]; f[g][i + 3] = tmp; }
                } else if (dyn != NODYN) {
                    const float om = (dyn == BIO) ? p.omega_bio[m] : p.omega_pore[m];
                    collide7(f[g], om, ux, uy, uz, rho);
                } else if (adj) {
#pragma unroll
                    for (int i = 0; i < 7; ++i) rho += f[g][i];
                }
                const float d = dcv[m];
                if (d != 0.f) {
#pragma unroll
                    for (int i = 0; i < 7; ++i) f[g][i] += t7(i) * d;
                }
                if (adj && dyn != BB) {
                    const int side = (x == 1) ? 0 : 1;
                    k.rho_adj[((int64_t)m * 2 + side) * plane + (n - (int64_t)x * plane)] = rho;
                }
            }
#pragma unroll
            for (int g = 0; g < kSG; ++g)
                if (m0 + g < NMOB) scatter7<PARITY>(k.pop + (int64_t)(m0 + g) * 7 * N, N32, st, f[g]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) nonconv += __shfl_down_sync(0xffffffffu, nonconv, o);
    if ((threadIdx.x & 31) == 0 && nonconv) atomicAdd(&k.counters[0], nonconv);
}

template <class Chem, int B, int MB>
int fast_launch(Ctx* c, const AdeK& k, const typename Chem::Consts& kc, int any_rxn) {
    // one thread per live site: the block scheduler balances the reactive
    // sites' long chains against the cheap streaming-only sites (at
    // 512x256x256: 2.76 ms, against 2.83 ms with a grid of 16 waves of
    // 148 x MB blocks striding over the list and 2.90 ms with one wave)
    const int blocks = grid_for(c->n_live, B, 1 << 30);
    if (c->ade_parity == 0)
        ade_fast_kernel<Chem, 0, B, MB><<<blocks, B, 0, c->stream>>>(k, kc, c->d_live, c->n_live, any_rxn);
    else
        ade_fast_kernel<Chem, 1, B, MB><<<blocks, B, 0, c->stream>>>(k, kc, c->d_live, c->n_live, any_rxn);
    CL_LAUNCH_CHECK("ade_fast_kernel");
    return CL_OK;
}

template <class Chem>
int fast_step(Ctx* c) {
    AdeK k = make_adek(c);
    const bool any_rxn = c->ap.do_kin || c->ap.do_abio || c->ap.do_dissol || (Chem::NC > 0 && c->ap.do_eq) ||
                         (Chem::kSrg && c->ap.n_srg > 0);
    typename Chem::Consts kc{};
    if constexpr (Chem::kSrg) {
        for (int o = 0; o < 2; ++o) {
            if (c->h_srg_params[o].size() != (size_t)Chem::kP) { set_error("surrogate network not set"); return CL_ERR_STATE; }
            for (int i = 0; i < Chem::kP; ++i) kc.w[o][i] = c->h_srg_params[o][i];
        }
    }
    int r = CL_OK;
    if (c->store_dirty && (r = store_update(c, 0))) return r;
    if (c->live_dirty && (r = build_live_list(c))) return r;
    if (any_rxn && c->ap.do_dissol && (r = dissol_release(c, k))) return r;
    if (c->n_live > 0) {
        if ((r = timing_begin(c, CL_KERNEL_ADE_MAIN))) return r;
        const int ar = any_rxn ? 1 : 0;
        // launch shapes (threads per block x blocks per SM, which sets the
        // register cap): 128x4 measured fastest on the coupled workload
        switch (c->fast_variant) {
            case 1: r = fast_launch<Chem, 128, 3>(c, k, kc, ar); break;
            case 2: r = fast_launch<Chem, 64, 6>(c, k, kc, ar); break;
            case 3: r = fast_launch<Chem, 64, 5>(c, k, kc, ar); break;
            default: r = fast_launch<Chem, 128, 4>(c, k, kc, ar); break;
        }
        if (r) return r;
        c->launches += 1;
        if ((r = timing_end(c, CL_KERNEL_ADE_MAIN))) return r;
    }
    const int bblocks = grid_for(2 * c->geo.plane, 256, 148 * 4);
    if (c->ade_parity == 0) ade_boundary_kernel<Chem::NMOB, 0><<<bblocks, 256, 0, c->stream>>>(k);
    else ade_boundary_kernel<Chem::NMOB, 1><<<bblocks, 256, 0, c->stream>>>(k);
    CL_LAUNCH_CHECK("ade_boundary_kernel");
    c->launches += 1;
    c->ade_parity ^= 1;
    return CL_OK;
}

int chem_match(const cl_config& cfg) {
    // microbes solved by LBM run the rate table's launches
    for (int m = 0; m < CL_MAX_MICROBES; ++m) if (cfg.microbe_carrier[m]) return 0;
    if (ChemCoupled::matches(cfg)) return ChemCoupled::kId;
    if (ChemBiotic4::matches(cfg)) return ChemBiotic4::kId;
    if (ChemZhao24::matches(cfg)) return ChemZhao24::kId;
    if (ChemSurrogate2::matches(cfg)) return ChemSurrogate2::kId;
    return 0;
}

const char* chem_name(int id) {
    switch (id) {
        case ChemCoupled::kId: return ChemCoupled::kName;
        case ChemBiotic4::kId: return ChemBiotic4::kName;
        case ChemZhao24::kId: return ChemZhao24::kName;
        case ChemSurrogate2::kId: return ChemSurrogate2::kName;
        default: return "run-time rate table";
    }
}

// whether the context holds what its compiled chemistry's step needs (a
// surrogate chemistry: both networks set, of the compiled shape); otherwise
// the step runs the run-time-table launches
bool chem_ready(const Ctx* c) {
    if (c->chem == ChemSurrogate2::kId) return ChemSurrogate2::ready(c->ap);
    return true;
}

int ade_step_fast(Ctx* c) {
    switch (c->chem) {
        case ChemCoupled::kId: return fast_step<ChemCoupled>(c);
        case ChemBiotic4::kId: return fast_step<ChemBiotic4>(c);
        case ChemZhao24::kId: return fast_step<ChemZhao24>(c);
        case ChemSurrogate2::kId: return fast_step<ChemSurrogate2>(c);
        default: set_error("no compiled chemistry selected"); return CL_ERR_STATE;
    }
}

}  // namespace cl
