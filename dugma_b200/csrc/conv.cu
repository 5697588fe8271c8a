// conv.cu -- CONV model (convolved GMM with a per-pair combined covariance).
#include "context.hpp"

namespace dugma {

int conv_launch(Context& c, const double* pose_dev, bool grad, int i0, int i1, double* out_dev, double* dEdx_dev,
                cudaStream_t s, const KernelShape* force)
{
    (void)c; (void)pose_dev; (void)grad; (void)i0; (void)i1; (void)out_dev; (void)dEdx_dev; (void)s; (void)force;
    return set_error(DUGMA_ERR_ARG, "CONV model is not available in this build");
}

}  // namespace dugma
