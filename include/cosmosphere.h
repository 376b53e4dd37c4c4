/*
 * cosmosphere.h -- the C-ABI of libcosmoSPHere for B200 (sm_100a).
 *
 * A drop-in for the library Phantom's Fortran links (-lcosmoSPHere): the same symbols,
 * argument meanings and error behaviour as the reference's include/arrays.hpp:15-61,
 * src/dens_c_api.cu:47 and :128, src/force_c_api.cu:26 and src/pin_c_api.cu:22-34.
 *
 * Conventions (unchanged from the reference):
 *   - one process-wide state on the current CUDA device; single host thread;
 *   - every call returns only when its device work is done;
 *   - errors print a "FATAL:" line on stderr and abort(); nothing returns a code;
 *   - a slot moves as one host block of ncomp*n doubles, component-major;
 *   - the device keeps particles in Hilbert order; transfers permute through it.
 * Kernel choice is fixed when the library is built, as in the reference (KERNEL=cubic
 * gives libcosmoSPHere.so, KERNEL=quintic gives libcosmoSPHere_quintic.so).
 */
#ifndef COSMOSPHERE_H
#define COSMOSPHERE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Slot ids, shared with Phantom's gpu_arrays ibun_* (include/arrays.hpp:15-25). */
enum CosmoSlot
{
    COSMO_POS       = 1, /* x, y, z */
    COSMO_HSML      = 2, /* h */
    COSMO_VEL       = 3, /* vx, vy, vz */
    COSMO_ACCEL     = 4, /* ax, ay, az */
    COSMO_DENS_OUT  = 5, /* rho, d(rho)/d(h) */
    COSMO_GRAD_OUT  = 6, /* div v, xi, d(div v)/dt */
    COSMO_THERMO    = 7, /* p/rho^2, c_s, alpha_AV, u */
    COSMO_FORCE_OUT = 8  /* fx, fy, fz, du/dt, vsigmax, div v */
};

/* Size every particle-length device array for n particles; n <= 0 is a no-op and a
 * repeated n is free.  Replaces src/arrays_c_api.cu:31 (cosmo_arrays_init). */
void cosmo_arrays_init(int n);

/* Components of a slot, 0 if unknown.  Replaces src/arrays_c_api.cu:152. */
int cosmo_slot_ncomp(int slot);

/* Send a slot in the caller's particle order, for the next density solve to sort.
 * Aborts if n differs from cosmo_arrays_init's or the slot is unknown.
 * Replaces src/arrays_c_api.cu:158 (cosmo_upload). */
void cosmo_upload(int slot, const double* host, int n);

/* Send a slot and gather it into the device's Hilbert order; needs a density solve for
 * this n to have built the ordering, else aborts.  Replaces src/arrays_c_api.cu:164. */
void cosmo_upload_sorted(int slot, const double* host, int n);

/* Fetch a slot back in the caller's order (scatter through the ordering, then copy).
 * Replaces src/arrays_c_api.cu:178 (cosmo_download). */
void cosmo_download(int slot, double* host, int n);

/* Page-lock / release a caller buffer (cudaHostRegister).  Null or zero size is a
 * no-op; failure is silent.  Replaces src/pin_c_api.cu:22 and :29. */
void cosmo_pin_host(void* ptr, size_t nbytes);
void cosmo_unpin_host(void* ptr);

/* Kernel support radius in units of h: 2 (cubic) or 3 (quintic).
 * Replaces src/dens_c_api.cu:128 (cosmo_kernel_radius). */
double cosmo_kernel_radius(void);

/* Density / smoothing-length solve with the gradient sweep: Hilbert keys, sort, leaf
 * tree, octree, j-leaf lists, Newton-Raphson to |dh/h| < tolh, then div v, xi and
 * d(div v)/dt at the converged h.  box = {xmin,xmax,ymin,ymax,zmin,zmax} is read only
 * when periodic != 0; hfact <= 0 selects the kernel's default.  Results stay on the
 * device (HSML, DENS_OUT, GRAD_OUT).  Aborts on a size mismatch, non-convergence within
 * the iteration cap (100, or COSMO_MAX_ITER) or a kernel support reaching half the
 * periodic box.  Replaces src/dens_c_api.cu:47 (densityiterate_gpu_c). */
void densityiterate_gpu_c(int n, double pmass, int periodic, const double* box, double tolh, double hfact);

/* Force pass on the tree of the last density solve: pressure + artificial-viscosity
 * accelerations, du/dt, vsigmax and div v over the symmetric (gather + scatter) lists.
 * Uses THERMO (and VEL if re-sent) uploaded with cosmo_upload_sorted.  Aborts without a
 * density solve for this n.  Replaces src/force_c_api.cu:26 (force_gpu_c). */
void force_gpu_c(int n, double pmass, double beta, double alphau, int disc_viscosity, int pdv_heating,
                 int shock_heating);

/* Arithmetic of the pair kernels for the following density solves and force passes:
 * COSMO_PRECISION_FP64 (default; the drop-in form, bit-for-bit with the FP64 oracle) or
 * COSMO_PRECISION_MIXED (FP32 pair arithmetic on leaf-relative coordinates with Kahan-
 * compensated sums combined in FP64; FP64 keys, tree, Newton-Raphson update and Omega).
 * The environment variable COSMO_PRECISION=mixed sets the same at start-up.  No
 * counterpart in the reference, which is FP64 only. */
enum CosmoPrecision { COSMO_PRECISION_FP64 = 0, COSMO_PRECISION_MIXED = 1 };
void cosmo_set_precision(int mode);
int cosmo_get_precision(void);

/* ---- batched form: many independent particle sets in one solve (no counterpart in
 * the reference, which solves one set per call) ----
 * The sets are concatenated set-major: set s owns entries [offsets[s], offsets[s+1]).
 * One segmented (set, key) sort, one forest with a tree per set, and one density launch
 * per Newton-Raphson iteration for all sets; per particle the arithmetic is the
 * single-set form's (cosmo_set_precision), so each set's h, rho and d(rho)/dh equal those
 * of solving it alone.  No gradient sweep or force pass in this form.
 * cosmo_batch_init returns 0, or -1 for bad offsets. */
int cosmo_batch_init(int nsets, const int* offsets);
/* Per-set particle mass, periodicity (nonzero: periodic) and box {xmin,xmax,...} (6 per
 * set, read where periodic); periodic/box6 may be NULL for all-open sets. */
void cosmo_batch_set_params(const double* pmass, const int* periodic, const double* box6);
/* Leaf capacity of each set's tree (default 64, the reference's BUCKET_SIZE). */
void cosmo_batch_set_bucket(const int* bucket_per_set);
/* The batched Newton kernel's j-stream feed for every set of the batch: 1 staged into
 * shared memory by bulk copies, 0 (default) loaded directly.  Results do not depend on
 * it; the autotuner picks it for the whole batch. */
void cosmo_batch_set_staging(int on);

/* Per-set launch parameters, as an autotuner picks them (NULL keeps a parameter):
 * bucket = leaf capacity (8..1024); list_margin = widening of the gather radius the lists
 * are walked at, which lets them serve later iterations (1..2, default 1.15);
 * split_stream = gather stream (particles) above which a leaf's active particles are cut
 * into smaller work items, split_work = the particle-pairs of one cut item (>= 32; default
 * 4096 and 131072).  None of them changes a result of the plain form.  Returns 0, or -1
 * (nothing set) when a value is out of range or no batch is initialised. */
int cosmo_batch_set_tuning(const int* bucket, const double* list_margin, const int* split_stream,
                           const int* split_work);
/* Positions and initial h of all sets (host arrays, length offsets[nsets]); a no-op
 * before cosmo_batch_init, as is cosmo_batch_download. */
void cosmo_batch_upload(const double* x, const double* y, const double* z, const double* h);
/* Solve every set; 0 ok, 1 some particle unconverged within max_iter (<= 0: 100; at
 * most 128).  flags: COSMO_BATCH_GRAPH runs the whole Newton loop as one CUDA graph
 * whose body (hmax, lists, density, bookkeeping) repeats under a device-side while
 * condition, with no host round trip per iteration; COSMO_BATCH_FINAL_RHO adds one
 * gather pass that re-evaluates rho and d(rho)/dh at the converged h (without it they
 * are the last iteration's, taken at the h before its update, as the reference's
 * solve without gradients returns them). */
enum { COSMO_BATCH_GRAPH = 1, COSMO_BATCH_FINAL_RHO = 2 };
int cosmo_batch_density(double tolh, double hfact, int max_iter, int flags);
/* Converged h, rho and d(rho)/dh of all sets, in the upload order. */
void cosmo_batch_download(double* h, double* rho, double* gradh);
/* Counters and timings (seconds) of the last batch solve; NaN if unknown. */
double cosmo_batch_scalar(const char* name);

/* ---- served form: a request loop with continuous batching (no counterpart in the
 * reference) ----
 * cosmo_serve_start launches `slots` worker threads on the current device with the
 * current precision; each runs one request at a time on its particle set's own CUDA
 * stream, so requests overlap on the GPU.  A queued request starts as soon as a slot is
 * free and, for a new set, the library's device memory plus admitted estimates fit
 * hbm_budget_gb (idle resident sets are evicted least-recently-used first; a request
 * larger than the whole budget is rejected).  Returns 0, or -1 if already running. */
int cosmo_serve_start(int slots, double hbm_budget_gb);
/* Submit a new set: density solve with gradients, then force.  pos3 (3n), h (n), vel3
 * (3n, may be NULL), thermo4 (4n: p/rho^2, c_s, alpha, u) are copied at submission,
 * component-major, caller order.  keep_resident keeps the set on the device for
 * cosmo_serve_continue.  Returns the request id (also the set id), or -1. */
long cosmo_serve_submit(int n, double pmass, int periodic, const double* box6, double tolh, double hfact,
                        const double* pos3, const double* h, const double* vel3, const double* thermo4, double beta,
                        double alphau, int keep_resident);
/* Continue a set one step: positions advance on the device by v*dt (wrapped into a
 * periodic box), the Newton iteration starts from the previous converged h; thermo4 may
 * be NULL (keep).  The set may be resident or still queued for admission (its first
 * request submitted with keep_resident); continuations of one set run in submission
 * order.  Returns the request id, or -1 if the set is unknown or was dropped. */
long cosmo_serve_continue(long set_id, double dt, const double* thermo4, int keep_resident);
/* Block until a request finishes and copy its results (caller order) into the given,
 * non-NULL outputs: h (n), dens (rho, gradh: 2n), grad (div v, xi, d(div v)/dt: 3n),
 * force (fx, fy, fz, du/dt, vsigmax, div v: 6n).  Returns 1 done, -1 rejected or
 * unknown, -2 unconverged. */
int cosmo_serve_wait(long request_id, double* h, double* dens, double* grad, double* force);
/* Per-request figures in seconds or counts: latency, queue, service, submit, start,
 * done, updates, iters, slot, n, status. */
double cosmo_serve_request_stat(long request_id, const char* name);
/* Drop an idle resident set (0), or -1 if unknown or busy. */
int cosmo_serve_release(long set_id);
/* Server figures: device_bytes, budget, resident_sets, max_inflight, completed,
 * rejected, evicted, queued, slots, and the admission estimate of a new set
 * (bytes_fixed + bytes_per_particle x n). */
double cosmo_serve_stat(const char* name);
/* Stop the workers (after the running requests) and release every resident set. */
int cosmo_serve_stop(void);

/* Hilbert keys and the stable sort order of n particles, computed without allocating
 * any device memory.  No counterpart in the reference: it exists for callers that cannot
 * call cudaMalloc at this point -- a caller that fixes its device-memory budget at start
 * and treats a later allocation as a failure, or one that keeps its own GPU work in
 * flight (cudaMalloc/cudaFree synchronise the device).  Inputs d_x, d_y, d_z, d_h and
 * outputs d_keys (n sorted keys) and d_order (sorted position -> input index) are DEVICE
 * pointers the caller owns; box6 is a host array read only when periodic != 0.  The
 * results equal the keys and ordering a density solve of the same particles builds.
 * Scratch is a fixed 7.06 MiB array inside the library, held by every GPU that loads it
 * until exit; n must be in [1, 524288], else it returns -1 (with a message on stderr)
 * and does nothing; so does periodic != 0 with box6 == NULL.  The first call on a device
 * looks up that array's address; make that first call before any stream capture.  Runs
 * on the calling thread's default stream (cudaStreamPerThread, which neither waits for
 * nor holds up the caller's other streams) and returns when done: 0 ok, -1 input
 * rejected, -2 CUDA error (also when an error from the caller's earlier CUDA calls is
 * pending on entry; that error is left in place), -3 device wait gave up.
 * Every call uses the same array: calls that overlap on the GPU (from several threads
 * or streams) race and corrupt each other's results. */
int cosmo_hilbert_order_noalloc(int n, const double* d_x, const double* d_y, const double* d_z,
                                const double* d_h, int periodic, const double* box6,
                                unsigned long long* d_keys, int* d_order);

/* ---- harness hooks (no counterpart in the reference; used by tests and bench) ---- */

/* Set the Newton iteration cap (default 100, as src/density_base.cu:50). */
void cosmo_x_set_max_iter(int max_iter);

/* Density solve that returns a status instead of aborting: 0 ok, 1 unconverged,
 * 2 periodic support too large, -1 size mismatch. */
int cosmo_x_density(int n, double pmass, int periodic, const double* box, double tolh, double hfact, int max_iter,
                    int with_gradients);

/* Wait for the library's stream. */
void cosmo_x_sync(void);

/* Select a kernel variant of the single-set solve (results do not depend on it):
 * "staging" 1 stages the Newton kernels' j-stream into shared memory with bulk copies
 * (cp.async.bulk completing on an mbarrier), 0 (default) loads it directly;
 * "sym_prefilter" 1 puts the symmetric row builder's tests behind the FP32 prefilter;
 * "split_stream" / "split_work" set the Newton work queue's leaf cut (a leaf whose gather
 * list streams more than split_stream particles is cut into groups of about
 * split_work / stream particles that scan the tree for their own box; 0 restores the
 * built-in 4096 and 131072); "spread_groups" sets how many h-ordered groups, at least, a
 * 64-particle window whose smoothing lengths spread by more than 1.5x is cut into (0 restores
 * the built-in 1; also COSMO_SPREAD_GROUPS); "newton_graph" 1 (default) runs the Newton loop
 * as one graph launch, 0 with a host round trip per iteration (also COSMO_NEWTON_GRAPH);
 * "graph_list_store" sets the graph loop's list storage as a percentage of its first lists'
 * total (0: the built-in; under 100 forces the fallback to the host loop, for tests);
 * "sym_from_rows" 1 (default) runs the gradient and force passes over the Newton rows' j
 * (with the pairs other particles' supports add merged in) when every live particle's row
 * covers its converged h, 0 builds the symmetric lists and rows after every solve (also
 * COSMO_SYM_FROM_ROWS); "sym_extra_cap" k > 0 holds at most k of the pairs other
 * particles' supports add to those rows (0: the built-in, one per live particle), so that
 * a solve that finds more hands the force pass to the list-built rows (a test of that
 * fallback).
 * Returns 0, or -1 for an unknown name or a value out of range. */
int cosmo_x_set_option(const char* name, int value);

/* Open boundaries: the particle extents (xmin, xmax, ymin, ymax, zmin, zmax) the next
 * solves make their bounding box, keys and order from, instead of the uploaded particles'
 * own; NULL returns to the latter.  A rank of a set decomposed over several GPUs gives the
 * whole set's extents, so its particles and halo sort in the whole set's order and its
 * sums run in the order of a solve of the whole set. */
void cosmo_x_set_key_extent(const double* ext6);

/* Particles the next solves of n particles take as neighbours only (mask in caller order,
 * nonzero = fixed): they start converged, so the Newton loop never updates them and the
 * loop ends when the others have converged (a rank's halo particles).  NULL or n <= 0
 * clears it.  Returns 0. */
int cosmo_x_set_frozen(const int* mask, int n);

/* After h (HSML) and rho/gradh (DENS_OUT) were replaced with cosmo_upload_sorted -- a
 * rank of a decomposed set takes its halo particles' converged values from their owners
 * -- refresh what the force pass derives from h: the leaves' hmax, and the symmetric
 * lists and rows, rebuilt by the next force pass.  Returns 0, or -1 with no solved set. */
int cosmo_x_refresh_h(void);

/* Time limit of every bounded device wait (the sort's look-back on its predecessor
 * tiles, the staging barriers of the bulk copies), in nanoseconds; <= 0 restores the
 * default of 1 s.  A wait that runs out raises a bit in the device error word, and the
 * entry point reports it (FATAL, or -3 where a status is returned). */
void cosmo_x_set_wait_limit(long long ns);
long long cosmo_x_get_wait_limit(void);

/* Run a device wait that can never be satisfied, through the library's bounded-wait code:
 * kind 0 polls a flag no block sets, kind 1 waits on a staging mbarrier whose bulk copy is
 * never issued.  Returns the device error bits it raised (8 flag wait, 4 staging wait) and
 * clears them, or -1 for an unknown kind; with fatal_on_error the library reports them as
 * a solve does (a FATAL line and abort). */
int cosmo_x_wait_test(int kind, int fatal_on_error);

/* Format a statistics line (0 COSMO_STATS, 1 COSMO_FORCE, 2 COSMO_MEM) from its values,
 * in the field order the entry points print it; returns the snprintf length or -1.  No
 * device work. */
int cosmo_x_stats_line(int which, const double* values, char* buf, int len);

/* Make device dev current for the library (before its first call on this thread). */
void cosmo_x_set_device(int dev);

/* Record mark id (0..15) on the library's stream; seconds between two marks. */
void cosmo_x_mark(int id);
double cosmo_x_mark_elapsed(int a, int b);

/* Number of the library's kernel launches so far in this process. */
unsigned long long cosmo_x_launches(void);

/* Measured FP64 FMA throughput of the current GPU, TFLOP/s. */
double cosmo_x_fp64_peak(void);

/* Named scalar of the last solve (counts, timings in seconds); NaN if unknown. */
double cosmo_x_scalar(const char* name);

/* Copy a named device array (Hilbert order / tree / lists) to the host; returns its
 * length or -1.  dtype: 0 f64, 1 i32, 2 u32, 3 u64, 4 i64.  out == NULL only queries. */
long cosmo_x_array(const char* name, void* out, int* dtype);

#ifdef __cplusplus
}
#endif

#endif /* COSMOSPHERE_H */
