// ade_nc0.cu -- instantiations of the fused transport step with 0 equilibrium
// components (0: no equilibrium), one translation unit per count so they build in parallel.
#include "ade_kernels.cuh"
#include "ops.cuh"

namespace cl {

int ade_step_nc0(Ctx* c) {
    AdeK k = make_adek(c);
    switch (c->ap.n_mob) {
        case 1: return launch_step<1, 0>(c, k);
        case 2: return launch_step<2, 0>(c, k);
        case 3: return launch_step<3, 0>(c, k);
        case 4: return launch_step<4, 0>(c, k);
        case 5: return launch_step<5, 0>(c, k);
        case 6: return launch_step<6, 0>(c, k);
        case 7: return launch_step<7, 0>(c, k);
        case 8: return launch_step<8, 0>(c, k);
        default: set_error("the fused transport step supports 1..8 mobile solutes");
                 return CL_ERR_ARG;
    }
}

int ade_ops_nc0(Ctx* c, const AdeK& k, int ops) { return launch_ops<0>(c, k, ops); }

}  // namespace cl
