/* Two-CTAs-per-SM instantiation of the sweep kernels (128 registers per
 * thread, 128-column reflector chunks so two CTAs fit in shared memory):
 * for batches of more chains than SMs, a second chain on each SM fills the
 * latency of the first one's reductions and panel factorizations. */
#define DQMC_NS dq2
#define DQMC_MINB 2
#define DQMC_WCOLS 128
#include <cuda_runtime.h>
#include "dqmc_kernels.cuh"
#include "dqmc_k2.h"

namespace dq2x {
size_t smem_bytes(int n, int kb) { return dq2::smem_bytes(n, kb); }
cudaError_t set_attrs(size_t smem, size_t msmem) { return dq2::set_attrs(smem, msmem); }
void launch_sweep(unsigned nc, size_t smem, cudaStream_t st, DqmcChainDev *c,
                  const DqmcModelDev *m, int flags, int nsweeps, const int *order)
{
    dq2::launch_sweep(nc, smem, st, c, m, flags, nsweeps, order);
}
void launch_measure(unsigned nc, size_t msmem, cudaStream_t st, DqmcChainDev *c,
                    const DqmcModelDev *m, int bin)
{
    dq2::launch_measure(nc, msmem, st, c, m, bin);
}
void launch_init(unsigned nc, size_t smem, cudaStream_t st, DqmcChainDev *c,
                 const DqmcModelDev *m)
{
    dq2::launch_init(nc, smem, st, c, m);
}
}  // namespace dq2x
