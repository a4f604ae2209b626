// fg_adjoint.cuh -- adjoint kernels (hand-written reverse mode of the forward path stage).
#pragma once
#include "fg_kernels.cuh"

namespace fg {

template <typename R, int EDGE>
fg_status Launch<R, EDGE>::cchi_bwd(const StageView &, const Tables<R> &, int64_t, int, const void *, int,
                                    const int64_t *, const void *, const void *, void *, unsigned char *, int,
                                    cudaStream_t)
{
    return fail(FG_ERR_NOT_IMPLEMENTED, "adjoint not built yet");
}

template <typename R, int EDGE>
fg_status Launch<R, EDGE>::fused_bwd(const StageView &, const Tables<R> &, const fg_paths *, int, const double *,
                                     const double *, const int *, const double *, const void *, const double *,
                                     double *, double *, unsigned char *, int, cudaStream_t)
{
    return fail(FG_ERR_NOT_IMPLEMENTED, "adjoint not built yet");
}

template <typename R>
fg_status LaunchCommon<R>::chi_fine_bwd(const StageView &, int64_t, const void *, const void *, int, const void *,
                                        const void *, const int *, const void *, void *, void *, cudaStream_t)
{
    return fail(FG_ERR_NOT_IMPLEMENTED, "adjoint not built yet");
}

}  // namespace fg
