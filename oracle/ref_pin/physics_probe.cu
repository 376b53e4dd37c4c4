// TEST INFRASTRUCTURE -- the parity checker, never part of the product.
//
// The reference's own density, gradient and force kernels, compiled for sm_100a from
// the reference's sources where they lie (src/density_base.cu, src/force.cu,
// src/gpu_state.cu; oracle/Makefile target `ref` passes their directory), and launched
// on arrays a test hands in:
//   sphDensityKernelJList<Periodic>          src/density_base.cu:237-334 (one NR step)
//   sphGradientsKernel<Periodic> + xiLimiter src/density_base.cu:511-714
//   forcePrepKernel                          src/force.cu:92-137
//   sphForceKernelJList<Periodic,Disc,Heat>  src/force.cu:145-383
// The Cornerstone headers those files include are interface stand-ins
// (ref_pin/shim_cuda): types only, no Cornerstone algorithm.  The test supplies the
// Hilbert-ordered particles, the leaf layout and CSR j-leaf lists; the kernels do all the
// physics arithmetic exactly as the reference builds it (nvcc -O3, default contraction).
//
// Every entry point takes HOST arrays, copies them to the device, launches one kernel
// (two for the force pass) with the reference's launch shape (256 threads per block),
// copies the outputs back and returns 0, or -1 on a CUDA error.
#include "gpu_state.cu"
#include "density_base.cu"
#include "force.cu"

#include <cstring>
#include <vector>

// buildTree is defined in the reference's src/tree.cu, which needs Cornerstone's tree
// algorithms and is not compiled here; solveDensH (compiled, never called by the probe)
// references it.  This body does nothing.
void buildTree(GpuState&, const std::vector<thrust::device_vector<double>*>&, TreeTimings&, const double*) {}

namespace {

struct DevArrays
{
    std::vector<void*> ptrs;
    bool ok = true;
    ~DevArrays()
    {
        for (void* p : ptrs) cudaFree(p);
    }
    template<class T>
    T* in(const T* host, size_t count)
    {
        T* d = nullptr;
        const size_t bytes = (count > 0 ? count : 1) * sizeof(T);
        if (cudaMalloc(&d, bytes) != cudaSuccess) { ok = false; return nullptr; }
        ptrs.push_back(d);
        if (host && count > 0 && cudaMemcpy(d, host, count * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
            ok = false;
        return d;
    }
    template<class T>
    T* out(size_t count) { return in<T>(nullptr, count); }
    template<class T>
    void back(T* host, const T* dev, size_t count)
    {
        if (count > 0 && cudaMemcpy(host, dev, count * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess) ok = false;
    }
};

Box<double> make_box(int periodic, const double* b)
{
    if (periodic)
        return Box<double>{b[0], b[1], b[2], b[3], b[4], b[5], BoundaryType::periodic, BoundaryType::periodic,
                           BoundaryType::periodic};
    return Box<double>{0.0, 1.0, BoundaryType::open};
}

int finish(DevArrays& d)
{
    if (cudaGetLastError() != cudaSuccess) return -1;
    if (cudaDeviceSynchronize() != cudaSuccess) return -1;
    return d.ok ? 0 : -1;
}

} // namespace

extern "C" {

// One Newton-Raphson step of the reference's flat kernel over the active particles.
// h (in/out), rho, gradh, converged (in/out) are length n; lists are CSR over nLeaves.
int ref_density_step(int periodic, const double* box6, int n, int nActive, const int* active, const double* x,
                     const double* y, const double* z, double* h, double* rho, double* gradh, int* converged,
                     double pmass, const int* particleLeaf, int nLeaves, const int* jOffset, const int* jcount,
                     const int* jlist, int listLen, const unsigned* layout, double tolh, double hfact)
{
    DevArrays d;
    const double *dx = d.in(x, n), *dy = d.in(y, n), *dz = d.in(z, n);
    double* dh = d.in(h, n);
    double* drho = d.in(rho, n);
    double* dgr = d.in(gradh, n);
    int* dconv = d.in(converged, n);
    const int* dact = d.in(active, nActive);
    const int* dpl = d.in(particleLeaf, n);
    const int* doff = d.in(jOffset, size_t(nLeaves) + 1);
    const int* dcnt = d.in(jcount, nLeaves);
    const int* dlist = d.in(jlist, listLen);
    const unsigned* dlay = d.in(layout, size_t(nLeaves) + 1);
    if (!d.ok) return -1;
    const Box<double> box = make_box(periodic, box6);
    if (nActive > 0)
    {
        if (periodic)
            sphDensityKernelJList<true><<<iceil(nActive, 256), 256>>>(dx, dy, dz, dh, drho, dgr, dconv, nActive, dact,
                                                                     pmass, dpl, doff, dcnt, dlist, dlay, box, tolh,
                                                                     hfact);
        else
            sphDensityKernelJList<false><<<iceil(nActive, 256), 256>>>(dx, dy, dz, dh, drho, dgr, dconv, nActive,
                                                                      dact, pmass, dpl, doff, dcnt, dlist, dlay, box,
                                                                      tolh, hfact);
    }
    if (const int e = finish(d)) return e;
    d.back(h, dh, n);
    d.back(rho, drho, n);
    d.back(gradh, dgr, n);
    d.back(converged, dconv, n);
    return d.ok ? 0 : -1;
}

// The reference's post-convergence sweep over all n particles at the converged h:
// rho, gradh, div v, xi, d(div v)/dt.  vel3/acc3 are component-major (3n).
int ref_gradients(int periodic, const double* box6, int n, const double* x, const double* y, const double* z,
                  const double* vel3, const double* acc3, const double* h, double* rho, double* gradh, double* divv,
                  double* xi, double* ddivvdt, double pmass, const int* particleLeaf, int nLeaves,
                  const int* jOffset, const int* jcount, const int* jlist, int listLen, const unsigned* layout)
{
    DevArrays d;
    const double *dx = d.in(x, n), *dy = d.in(y, n), *dz = d.in(z, n);
    const double* dv = d.in(vel3, 3 * size_t(n));
    const double* da = d.in(acc3, 3 * size_t(n));
    const double* dh = d.in(h, n);
    double *drho = d.out<double>(n), *dgr = d.out<double>(n), *ddiv = d.out<double>(n);
    double *dxi = d.out<double>(n), *ddd = d.out<double>(n);
    const int* dpl = d.in(particleLeaf, n);
    const int* doff = d.in(jOffset, size_t(nLeaves) + 1);
    const int* dcnt = d.in(jcount, nLeaves);
    const int* dlist = d.in(jlist, listLen);
    const unsigned* dlay = d.in(layout, size_t(nLeaves) + 1);
    if (!d.ok) return -1;
    const Box<double> box = make_box(periodic, box6);
    if (periodic)
        sphGradientsKernel<true><<<iceil(n, 256), 256>>>(dx, dy, dz, dv, dv + n, dv + 2 * n, da, da + n, da + 2 * n,
                                                         dh, drho, dgr, ddiv, dxi, ddd, n, pmass, dpl, doff, dcnt,
                                                         dlist, dlay, box);
    else
        sphGradientsKernel<false><<<iceil(n, 256), 256>>>(dx, dy, dz, dv, dv + n, dv + 2 * n, da, da + n, da + 2 * n,
                                                          dh, drho, dgr, ddiv, dxi, ddd, n, pmass, dpl, doff, dcnt,
                                                          dlist, dlay, box);
    if (const int e = finish(d)) return e;
    d.back(rho, drho, n);
    d.back(gradh, dgr, n);
    d.back(divv, ddiv, n);
    d.back(xi, dxi, n);
    d.back(ddivvdt, ddd, n);
    return d.ok ? 0 : -1;
}

// The reference's force pass: forcePrepKernel, then sphForceKernelJList over the
// symmetric lists.  thermo4 = {pro2, cs, alphaAV, u} component-major (4n); force6 out =
// {fx, fy, fz, du/dt, vsigmax, div v} component-major (6n).
int ref_force(int periodic, const double* box6, int n, const double* x, const double* y, const double* z,
              const double* vel3, const double* h, const double* gradh, const double* thermo4, double* force6,
              double pmass, double beta, double alphau, double hfact, int disc, int pdv, int shock,
              const int* particleLeaf, int nLeaves, const int* jOffset, const int* jcount, const int* jlist,
              int listLen, const unsigned* layout)
{
    DevArrays d;
    const double *dx = d.in(x, n), *dy = d.in(y, n), *dz = d.in(z, n);
    const double* dv = d.in(vel3, 3 * size_t(n));
    const double* dh = d.in(h, n);
    const double* dgr = d.in(gradh, n);
    const double* dth = d.in(thermo4, 4 * size_t(n));
    double* prep = d.out<double>(8 * size_t(n));
    double* df = d.out<double>(6 * size_t(n));
    const int* dpl = d.in(particleLeaf, n);
    const int* doff = d.in(jOffset, size_t(nLeaves) + 1);
    const int* dcnt = d.in(jcount, nLeaves);
    const int* dlist = d.in(jlist, listLen);
    const unsigned* dlay = d.in(layout, size_t(nLeaves) + 1);
    if (!d.ok) return -1;
    const Box<double> box = make_box(periodic, box6);
    double *hsqinv = prep, *hinv = prep + n, *rhoh = prep + 2 * n, *rho1 = prep + 3 * n, *grkfac = prep + 4 * n;
    double *pres = prep + 5 * n, *auterm = prep + 6 * n, *divfac = prep + 7 * n;
    forcePrepKernel<<<iceil(n, 256), 256>>>(dh, dgr, dth, hsqinv, hinv, rhoh, rho1, grkfac, pres, auterm, divfac, n,
                                            pmass, alphau, hfact);
    const bool full = pdv && shock;
    auto launch = [&](auto per, auto dsc, auto heat) {
        sphForceKernelJList<decltype(per)::value, decltype(dsc)::value, decltype(heat)::value>
            <<<iceil(n, 256), 256>>>(dx, dy, dz, dv, dv + n, dv + 2 * n, dh, dth, dth + n, dth + 2 * n, dth + 3 * n,
                                     hsqinv, hinv, rhoh, rho1, grkfac, pres, auterm, divfac, df, df + n, df + 2 * n,
                                     df + 3 * n, df + 4 * n, df + 5 * n, n, pmass, beta, pdv != 0, shock != 0, dpl,
                                     doff, dcnt, dlist, dlay, box, hfact);
    };
    auto with_heat = [&](auto per, auto dsc) {
        if (full) launch(per, dsc, std::true_type{});
        else      launch(per, dsc, std::false_type{});
    };
    auto with_disc = [&](auto per) {
        if (disc) with_heat(per, std::true_type{});
        else      with_heat(per, std::false_type{});
    };
    if (periodic) with_disc(std::true_type{});
    else          with_disc(std::false_type{});
    if (const int e = finish(d)) return e;
    d.back(force6, df, 6 * size_t(n));
    return d.ok ? 0 : -1;
}

} // extern "C"
