// gizmo_b200/csrc/passes_mixed.cu -- mixed form: FP32 pair arithmetic, FP64
// positions / membership / accumulation (see passes.cuh).
#include "passes.cuh"

namespace gz {

// The density sums feed the bracketed kernel-length iteration, whose
// accept/bracket decisions are discontinuous in NumNgb, DrkernNgb, NV_T and
// the face weights: computing them in FP32 moves the converged h of any
// particle whose count sits within ~1e-7 of a band edge by up to the band
// width (~1e-3). The mixed form therefore takes them in FP64 -- the same
// kernel as the FP64 form, so both forms converge to identical h -- and uses
// FP32 for the gradient and force pair arithmetic.
void density_sums_mixed(const PassParams &p, const Particles &ps, const DensityWork &w, int tpt, cudaStream_t s)
{
    density_sums_fp64(p, ps, w, tpt, s);
}

void gradients_mixed(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                     void *rec, const EventPair *ev, cudaStream_t s)
{
    launch_gradients<float>(p, ps, targets, n_targets, rows, tpt, rec, ev, s);
}

void force_mixed(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                 DevStatus *st, void *rec, void *flux, double *sums, const EventPair *ev, cudaStream_t s)
{
    launch_force<float>(p, ps, targets, n_targets, rows, tpt, st, rec, flux, sums, ev, s);
}

}  // namespace gz
