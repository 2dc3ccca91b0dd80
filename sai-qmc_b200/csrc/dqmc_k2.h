/* Host-callable entry points of the two-CTAs-per-SM kernel build. */
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include "dqmc_common.h"

namespace dq2x {
size_t smem_bytes(int n, int kb);
cudaError_t set_attrs(size_t smem, size_t msmem);
void launch_sweep(unsigned nc, size_t smem, cudaStream_t st, DqmcChainDev *c,
                  const DqmcModelDev *m, int flags, int nsweeps, const int *order);
void launch_measure(unsigned nc, size_t msmem, cudaStream_t st, DqmcChainDev *c,
                    const DqmcModelDev *m, int bin);
void launch_init(unsigned nc, size_t smem, cudaStream_t st, DqmcChainDev *c,
                 const DqmcModelDev *m);
}  // namespace dq2x
