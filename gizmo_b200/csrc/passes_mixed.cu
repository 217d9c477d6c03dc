// gizmo_b200/csrc/passes_mixed.cu -- mixed form: FP32 pair arithmetic, FP64
// positions / membership / accumulation (see passes.cuh).
#include "passes.cuh"

namespace gz {

void density_sums_mixed(const PassParams &p, const Particles &ps, const DensityWork &w, int tpt, cudaStream_t s)
{
    launch_density_sums<float>(p, ps, w, tpt, s);
}

void gradients_mixed(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                     cudaStream_t s)
{
    launch_gradients<float>(p, ps, targets, n_targets, rows, tpt, s);
}

void force_mixed(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                 DevStatus *st, cudaStream_t s)
{
    launch_force<float>(p, ps, targets, n_targets, rows, tpt, st, s);
}

}  // namespace gz
