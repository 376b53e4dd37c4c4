// Exposes the reference's own M4/M6 kernel (include/kernel.hpp, compiled where it lies)
// through a C interface, so the oracle's restatement can be checked against it bit for
// bit.  Built twice: cubic, and quintic with -DCOSMO_KERNEL_QUINTIC, as the reference's
// KERNEL switch does (Makefile:39-46).
#include "kernel.hpp"

extern "C" void ref_kernel_eval(int n, const double* q, double* w, double* dw)
{
    for (int i = 0; i < n; ++i) sph::kern(q[i] * q[i], q[i], w[i], dw[i]);
}

extern "C" void ref_kernel_consts(double* out4)
{
    out4[0] = sph::radkernel;
    out4[1] = sph::radk2;
    out4[2] = sph::cnormk;
    out4[3] = sph::hfact_default;
}
