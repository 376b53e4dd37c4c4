/*
 * cosmo_density.hpp -- the reference's C++ density interface (include/density.hpp:85-91),
 * exported by libcosmoSPHere with the same names and layout so the reference's own
 * standalone driver (src/main.cu) links against this library unchanged.
 *
 * The enum and struct must stay layout-identical to the reference's: a caller compiled
 * against its header passes and receives them by value.
 */
#pragma once

enum class KernelMode { FLAT_PARTICLE, WARP_PER_LEAF };

struct DensTimings
{
    double     upload;          // host-to-device transfer (accumulated by cosmo_upload)
    double     bboxAndSetup;    // bounding box
    double     keysAndSort;     // Hilbert keys + radix sort + gathers
    double     treeBuild;       // leaf tree + octree prefixes
    double     nodeCenters;     // node geometry and maps
    double     jleafBuild;      // j-leaf lists, all Newton iterations
    double     densKernel;      // Newton density kernel, all iterations
    double     gradJleafBuild;  // list rebuild before the gradient sweep
    double     gradKernel;      // gradient sweep
    double     download;        // device-to-host (accumulated by cosmo_download)
    int        itersRun;
    int        nParticles;
    int        nLeavesOut;
    KernelMode kernelMode;
};

// Solve for h and rho of the particles uploaded with cosmo_upload.  Both kernel modes
// run the same warp-per-leaf Newton kernel; withGradients adds the gradient sweep.
DensTimings solveDensH(int n, double pmass, KernelMode mode = KernelMode::FLAT_PARTICLE,
                       bool withGradients = false, const double* periodicBox = nullptr, double tolh = 1.0e-4,
                       double hfact = -1.0);
