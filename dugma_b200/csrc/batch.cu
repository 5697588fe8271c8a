// batch.cu -- many registration problems in one persistent launch.
#include "context.hpp"

extern "C" {
int dugma_batch_create(int, int, const int*, const int*, const double* const*, const double* const*,
                       const double* const*, const double* const*, void**)
{
    return dugma::set_error(DUGMA_ERR_ARG, "batched problems are not available in this build");
}
int dugma_batch_energy_grad(void*, int, const double*, int, double*)
{
    return dugma::set_error(DUGMA_ERR_ARG, "batched problems are not available in this build");
}
int dugma_batch_destroy(void*) { return DUGMA_OK; }
}
