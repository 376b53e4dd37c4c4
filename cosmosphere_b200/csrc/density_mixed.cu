/*
 * density_mixed.cu -- the mixed-precision instantiations of the single-set Newton kernels
 * (newton_kernels.cuh).  This file is compiled with contraction into fused multiply-adds:
 * the mixed form's FP32 pair arithmetic and Kahan sums are not bit-compared with anything,
 * so -fmad=false, which the plain form needs for parity with the oracle, would only cost
 * it instructions.
 */
#include "newton_kernels.cuh"

namespace cosmo {

NrKernelFn mixed_density_nr_kernel(bool periodic, bool staged)
{
    if (staged) return periodic ? density_nr_kernel<true, true, true> : density_nr_kernel<false, true, true>;
    return periodic ? density_nr_kernel<true, true, false> : density_nr_kernel<false, true, false>;
}

RowsKernelFn mixed_newton_rows_kernel(bool periodic)
{
    return periodic ? newton_rows_kernel<true, true> : newton_rows_kernel<false, true>;
}

RowKernelFn mixed_density_row_kernel(bool periodic)
{
    return periodic ? density_row_kernel<true, true> : density_row_kernel<false, true>;
}

} // namespace cosmo
