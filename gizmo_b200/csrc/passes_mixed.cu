// gizmo_b200/csrc/passes_mixed.cu -- mixed form: FP32 force pair arithmetic,
// FP64 positions / membership / density and gradient sums / accumulation (see
// passes.cuh). Built with the approximate FP32 division and square root; the
// pairs whose FP32 branch decisions are too close to call are evaluated again
// by force_refine in passes_fp64.cu.
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

void force_mixed(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                 DevStatus *st, void *rec, void *flux, bool all, const RefineQueue &q, double *sums,
                 const EventPair *ev, cudaStream_t s)
{
    launch_force<float>(p, ps, targets, n_targets, rows, tpt, st, rec, flux, all, q, sums, ev, s);
}

}  // namespace gz
