/*
 * ssmd.h — C ABI of the B200 (sm_100a) two-phase jet lattice-Boltzmann step.
 *
 * One time step of the reference (ssmdLBM) is the CUDA graph
 *   computePhase -> computeForces -> computeMoments -> streamCollide
 * (src/cuda/CUDAGraph.cuh:41-56) followed by five boundary launches
 * (src/main.cu:165-169).  This library replaces that sequence with one fused
 * bulk kernel plus light surface kernels, behind the entry points below.
 *
 * Conventions shared by every entry point
 *   - All pointers inside LBMFields and ssmd_params are DEVICE pointers that
 *     the caller owns (cudaMalloc, a caching allocator, ...).  No entry point
 *     allocates or frees device memory.
 *   - Every call is asynchronous on the given stream unless it says it
 *     synchronises.  Return value: 0 (SSMD_OK) or a positive SSMD_ERR_* code;
 *     ssmd_last_error() returns a message for the calling thread.  The library
 *     never aborts the process (the reference's checkCudaErrors* macros do,
 *     src/cuda/utils.cuh:101-161; that policy stays with the caller).
 *   - Scalar fields are FP32, structure of arrays, index x + nx*(y + ny*z)
 *     (reference src/functions/deviceFunctions.cuh:33-39).  Populations are
 *     [q][cell] arrays with q in the reference's velocity order
 *     (src/velocitySet/D3Q19.cuh:82-131, D3Q27.cuh:91-140, D3Q7.cuh:73-122),
 *     stored in PULL layout: slot q of cell s holds the post-collision value
 *     that cell s + c_q reads next step.  ssmd_populations_to_push() converts
 *     to the reference's post-stream (push) layout.  Cell indices are 32-bit,
 *     population offsets 64-bit, so nx*ny*nz may reach 2^32 - 1 cells.
 *   - One host thread per stream.  Graph capture of ssmd_step is legal on the
 *     caller's stream (no host synchronisation inside a step).
 */
#ifndef SSMD_H
#define SSMD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque CUDA handles, layout-identical to cudaStream_t / cudaGraphExec_t. */
typedef struct CUstream_st *ssmd_stream_t;
typedef struct CUgraphExec_st *ssmd_graph_exec_t;

#define SSMD_ABI_VERSION 1

/* ---------------------------------------------------------------- status */
#define SSMD_OK 0
#define SSMD_ERR_INVALID_ARGUMENT 1 /* bad size, pointer or parameter      */
#define SSMD_ERR_CUDA 2             /* a CUDA runtime call failed          */
#define SSMD_ERR_UNSTABLE 3         /* NaN/Inf or |u| above the limit       */
#define SSMD_ERR_UNSUPPORTED 4      /* combination not built into library  */

/* ------------------------------------------------------ face-pair kinds */
#define SSMD_BC_PERIODIC_COPY 0 /* reference periodicX: ghost layers at 0 and n-1,
                                   slots copied between planes 1 and n-2
                                   (src/BoundaryConditions.cuh:295-349)       */
#define SSMD_BC_PERIODIC 1      /* exact periodic wrap, no ghost layers       */
#define SSMD_BC_JET 2           /* y: water inflow disc at y=0 + outflow at
                                   y=ny-1 (BoundaryConditions.cuh:36-99,170-233);
                                   z: oil inflow disc at z=0 + outflow at
                                   z=nz-1 (:101-168, :235-293)                 */

/* ------------------------------------------------------- storage types */
#define SSMD_STORAGE_F32 0  /* f - w_q and g as float                        */
#define SSMD_STORAGE_F16 1  /* f - w_q and g as IEEE half (round to nearest) */
#define SSMD_STORAGE_BF16 2 /* f - w_q as bfloat16, g as IEEE half (both round
                               to nearest; g carries phi in [0, 1], which
                               needs mantissa bits rather than range)     */
#define SSMD_STORAGE_F16_G32 3 /* f - w_q as IEEE half, g as float: the layout
                                  of the reference's ENABLE_FP16=1 build
                                  (src/cuda/utils.cuh:67-99, pop_t f and
                                  scalar_t g in src/structs/LBMFields.cuh) */

/* ------------------------------------------------- bulk kernel variants */
#define SSMD_PATH_AUTO 0   /* library choice (currently SSMD_PATH_GATHER)        */
#define SSMD_PATH_GATHER 1 /* per-cell loads of populations and of the phi halo */
#define SSMD_PATH_TMA 2    /* TMA boxes of g for the phi halo                    */
#define SSMD_PATH_SLAB 3   /* TMA slabs of the populations, one plane ahead      */
/* (the TMA paths return SSMD_ERR_UNSUPPORTED unless nx * element size is a
 * multiple of 16 bytes) */

/* ------------------------------------------------------------ step flags */
#define SSMD_STEP_STORE_MACROS 1u /* write rho, ux, uy, uz, phi at every cell */
#define SSMD_STEP_AVERAGE 2u      /* update the running means of ssmd_params.derived
                                     in the step itself (no macroscopic store needed) */

/* ssmd_derived_update: what to compute */
#define SSMD_DERIVED_AVERAGES 1u  /* running means, t = number of updates so far + 1 */
#define SSMD_DERIVED_VORTICITY 2u /* curl u and |curl u| from the stored u          */

/* Closure network: 12 features -> 64 -> 64 -> 2, GELU.  A network is one FP32
 * device buffer of SSMD_MLP_NET_FLOATS: the SSMD_MLP_PARAMS trainable values
 * W1 [64][16] (input columns 12..15 zero), b1 [64], W2 [64][64], b2 [64],
 * W3 [2][64], b3 [2], then feature mean [12], feature 1/std [12], output
 * scale [2] and output offset [2]. */
#define SSMD_MLP_IN 12
#define SSMD_MLP_HIDDEN 64
#define SSMD_MLP_OUT 2
#define SSMD_MLP_PARAMS 5378
#define SSMD_MLP_NET_FLOATS 5406

/*
 * Field container.  Member order and meaning are those of the reference's
 * struct LBMFields (src/structs/LBMFields.cuh:26-49) so code that reads
 * fields.phi / fields.rho after a step keeps working.  f and g point at the
 * "A" population buffers; the "B" buffers are ssmd_params.f_alt / g_alt.
 * normx/normy/normz/ind are never used (the reference never allocates them
 * either, src/main.cu:55-70).
 */
typedef struct LBMFields {
    float *rho;
    float *ux;
    float *uy;
    float *uz;
    float *pxx;
    float *pyy;
    float *pzz;
    float *pxy;
    float *pxz;
    float *pyz;
    float *phi;
    float *normx;
    float *normy;
    float *normz;
    float *ind;
    float *fsx;
    float *fsy;
    float *fsz;
    void *f; /* Q * cells populations, element type from ssmd_params.storage */
    void *g; /* 7 * cells phase populations: float for SSMD_STORAGE_F32 and
                SSMD_STORAGE_F16_G32, IEEE half otherwise                */
} LBMFields;

/*
 * Run-time parameters.  The reference fixes all of these at compile time
 * (src/constants.cuh:70-101, src/functions/globalFunctions.cuh:68-104,
 * 232-283); here they are per call so one library serves every grid.
 * Floating-point members are the FP32 values the kernels use, so a caller can
 * reproduce the reference's constexpr arithmetic bit for bit
 * (ssmd_params_reference does exactly that).
 */
typedef struct ssmd_params {
    uint32_t nx, ny, nz;  /* lattice size, ghost layers included              */
    int32_t velocity_set; /* 19 or 27 (hydrodynamics); phase field is D3Q7    */
    int32_t storage;      /* SSMD_STORAGE_*                                   */
    int32_t bc_x;         /* SSMD_BC_PERIODIC_COPY | SSMD_BC_PERIODIC          */
    int32_t bc_y;         /* SSMD_BC_PERIODIC_COPY | SSMD_BC_PERIODIC | SSMD_BC_JET */
    int32_t bc_z;         /* SSMD_BC_JET | SSMD_BC_PERIODIC                    */

    float nu_water;   /* kinematic viscosity of phi = 0 (lattice units)       */
    float nu_oil;     /* kinematic viscosity of phi = 1                       */
    float omco_water; /* 1 - omega(nu_water), water inflow regularisation     */
    float omco_oil;   /* 1 - omega(nu_oil), oil inflow regularisation         */
    float omco_ref;   /* 1 - omega used by the outflows (reference: water)    */
    float sigma;      /* surface tension                                      */
    float gamma;      /* interface sharpening 4 M / (W cs2)                   */
    float omega_g;    /* phase-field BGK rate 1/(1/2 + M/cs2); 1 = reference  */

    float u_oil;     /* oil inlet speed (+z) at z = 0                        */
    float oil_cx;    /* oil disc centre x                                    */
    float oil_cy;    /* oil disc centre y                                    */
    float oil_r2;    /* oil disc radius squared (cells with r^2 <= oil_r2)   */
    float u_water;   /* water inlet speed (+y) at y = 0                      */
    float water_cx;  /* water disc centre x                                  */
    float water_cz;  /* water disc centre z                                  */
    float water_r2;  /* water disc radius squared                            */
    float noise_amp; /* oil inlet speed u_oil * (1 + noise_amp * N(0,1))     */
    float u_limit;   /* |u| above this is reported as SSMD_ERR_UNSTABLE      */
    uint64_t seed;   /* key of the counter-based inlet noise                 */

    void *f_alt;      /* "B" hydrodynamic populations, same size as fields->f */
    void *g_alt;      /* "B" phase populations, same size as fields->g        */
    void *workspace;  /* ssmd_workspace_bytes() bytes of device scratch       */
    size_t workspace_bytes;

    int32_t tile_z;   /* z planes per bulk work item (0: library default)     */
    int32_t bulk_path; /* SSMD_PATH_*: how the bulk kernel feeds the phi halo */
    const struct ssmd_derived *derived; /* derived-field arrays (NULL: none)   */
    const struct ssmd_closure *closure; /* per-cell closure arrays read by the
                                           bulk kernel (NULL: plain method)    */
    int32_t reserved[2];
} ssmd_params;

/*
 * Derived fields (reference src/derivedFields/DerivedFields.cuh:39-58 and
 * LBMFields.cuh:51-84): FP32 arrays of nx*ny*nz cells, each may be NULL.
 * Running means follow timeAverage.cuh:58-61 / reynoldsMoments.cuh:58-61,
 * avg <- avg + (value - avg) / t with t the 1-based index of the step just
 * completed; vorticity follows vorticityFields.cuh:37-96.
 */
typedef struct ssmd_derived {
    float *avg_phi, *avg_ux, *avg_uy, *avg_uz;
    float *avg_uxux, *avg_uyuy, *avg_uzuz, *avg_uxuy, *avg_uxuz, *avg_uyuz;
    float *vort_x, *vort_y, *vort_z, *vort_mag;
} ssmd_derived;

/*
 * Learned closure state of a (coarse) lattice: per-cell eddy viscosity added
 * to nu(phi) and a factor on the surface tension, both FP32 nx*ny*nz arrays
 * written by ssmd_closure_apply and read by the bulk kernel.  No reference
 * counterpart: the reference runs the plain method only.
 */
typedef struct ssmd_closure {
    const float *nut;         /* eddy viscosity (lattice units), > -nu(phi)    */
    const float *sigma_scale; /* factor on sigma at the cell                   */
} ssmd_closure;

/* Global reductions, accumulated in FP64 over the fluid (non-ghost) cells. */
typedef struct ssmd_stats {
    double phi_sum;      /* sum of phi from the macroscopic field             */
    double phi_sum_next; /* sum over cells of sum_q g (next step's phi)        */
    double mass;         /* sum of rho                                        */
    double momentum[3];  /* sum of rho u                                      */
    double kinetic;      /* sum of rho |u|^2 / 2                              */
    double u_max;        /* max |u|                                           */
    double nonfinite;    /* count of cells with non-finite rho, u or phi      */
    double cells;        /* number of fluid cells reduced                     */
} ssmd_stats;

/* One connected component of phi > threshold (ssmd_droplets). */
typedef struct ssmd_droplet {
    uint32_t root;          /* smallest cell index of the component              */
    uint32_t cells;         /* number of cells                                   */
    double volume;          /* FP64 sum of phi over those cells                  */
    uint32_t touches_inlet; /* 1 when it reaches the first fluid plane (z = 1 for
                               inflow faces): the intact jet, not a droplet      */
    uint32_t reserved;
} ssmd_droplet;

/* -------------------------------------------------------------- queries */
int ssmd_abi_version(void);
const char *ssmd_last_error(void);

/* Bytes of one scalar field, of fields->f (== f_alt), of fields->g
 * (== g_alt) and of the workspace, for these parameters. */
size_t ssmd_scalar_bytes(const ssmd_params *p);
size_t ssmd_f_bytes(const ssmd_params *p);
size_t ssmd_g_bytes(const ssmd_params *p);
size_t ssmd_workspace_bytes(const ssmd_params *p);

/* Checks sizes, BC kinds, relaxation ranges (tau > 1/2) and geometry. */
int ssmd_validate(const ssmd_params *p);

/*
 * Fills p the way the reference derives its constants:
 *   nu = u * diam / Re (FP64 then FP32, globalFunctions.cuh:234-242),
 *   omega = 1/(1/2 + 3 nu) in FP64 (:244-247), omco = 1 - omega (:269-282),
 *   sigma = u_oil^2 diam_oil / We (constants.cuh:93),
 *   gamma = 4 cs2 (tau_g - 1/2) / W / cs2 with tau_g = 1 (constants.cuh:97-100),
 *   disc radius = diam / 2 in integers, r^2 = radius^2 (globalFunctions.cuh:70-78),
 *   oil centre ((nx-1)/2, (ny-1)/4), water centre ((nx-1)/2, 0.35 (nz-1)).
 * Boundary kinds default to the reference's two-jet crossflow:
 * bc_x = PERIODIC_COPY, bc_y = JET, bc_z = JET.
 * radius_* may be passed separately from diam_* (radius < 0: diam / 2).
 */
int ssmd_params_reference(ssmd_params *p, uint32_t nx, uint32_t ny, uint32_t nz,
                          int32_t velocity_set, float u_water, float u_oil,
                          int32_t diam_water, int32_t diam_oil, int32_t radius_water,
                          int32_t radius_oil, double reynolds_water, double reynolds_oil,
                          double weber, float interface_width);

/* ------------------------------------------------------------- the path */

/*
 * Initial state of the reference (src/initialConditions.cu:33-140):
 * rho = 1, u = 0, phi = 0; phi = 0, uy = u_water on the water disc (bc_y = JET);
 * phi = 1, uz = u_oil on the oil disc (bc_z = JET); f = f_eq(rho, u) and
 * g = g_eq(phi, u) in both population buffers.  Zeroes pxx..pyz and fsx..fsz.
 * Resets the device step counter to 0.
 */
int ssmd_init(const ssmd_params *p, LBMFields *fields, ssmd_stream_t stream);

/*
 * Same, but takes rho, ux, uy, uz and phi as the caller left them in fields
 * (the reference's setDistros on an arbitrary macroscopic state,
 * initialConditions.cu:99-140).
 */
int ssmd_init_from_macros(const ssmd_params *p, LBMFields *fields, ssmd_stream_t stream);

/*
 * One time step n = step: reads populations from the A buffers (fields->f/g)
 * when step is even, from the B buffers (p->f_alt/g_alt) when odd, writes the
 * other pair.  After the call, rho/u/Pi/phi are valid on the planes the
 * boundaries read, phi/rho/u on the boundary faces, and, with
 * SSMD_STEP_STORE_MACROS, rho/ux/uy/uz/phi on every cell (phi is the
 * step-n field Sum_q g^n, as in the reference).
 */
int ssmd_step(LBMFields *fields, const ssmd_params *p, uint64_t step, uint32_t flags,
              ssmd_stream_t stream);

/*
 * Captures steps [first_step, first_step + steps) into a CUDA graph and
 * instantiates it (graph::captureGraph, src/cuda/CUDAGraph.cuh:34-57, which
 * holds only the four bulk kernels; here the boundaries are inside too).
 * steps must be even so that replays keep the A/B parity.  The inlet-noise
 * step index lives in device memory and advances on every replayed step.
 */
int ssmd_capture_graph(const ssmd_params *p, LBMFields *fields, uint64_t first_step,
                       int32_t steps, uint32_t flags, ssmd_stream_t stream,
                       ssmd_graph_exec_t *out);

/* Replays / frees a graph from ssmd_capture_graph (cudaGraphLaunch /
 * cudaGraphExecDestroy through this library's runtime). */
int ssmd_graph_launch(ssmd_graph_exec_t exec, ssmd_stream_t stream);
int ssmd_graph_destroy(ssmd_graph_exec_t exec);

/*
 * FP64 reductions over the fluid cells (synchronises the stream).  Reads the
 * macroscopic arrays (valid after a step with SSMD_STEP_STORE_MACROS or after
 * init) and the current phase populations of step `steps_done` (number of
 * steps taken since init).  Returns SSMD_ERR_UNSTABLE (with *out filled) when
 * a non-finite value or |u| > p->u_limit is found.
 */
int ssmd_reduce(const ssmd_params *p, const LBMFields *fields, uint64_t steps_done,
                ssmd_stats *out, ssmd_stream_t stream);

/*
 * ssmd_reduce without any device allocation.  No counterpart in the
 * reference.  For callers that cannot allocate device memory (a plugin handed
 * the fields by the host application with no memory of its own, or code that
 * must not call cudaMalloc because it synchronises the whole device):
 * p->workspace is not used; the partial sums live in a fixed 41 KiB array
 * inside the library (512 partials of 10 doubles + result, per GPU, held
 * until exit).  512 blocks striding over the cells cover every lattice that
 * ssmd_validate accepts; larger lattices are refused by ssmd_validate.  The
 * first call in each CUDA context of a device looks the array up
 * (cudaGetSymbolAddress); after a device reset the next call looks it up
 * again.  The call reads its result back and synchronises the stream, so it
 * cannot be captured: a capturing stream is refused with
 * SSMD_ERR_INVALID_ARGUMENT, and it must not be called on the legacy default
 * stream while another stream captures.  All calls share the array:
 * overlapping calls race.  Same results as ssmd_reduce up to FP64 summation
 * order.
 */
int ssmd_reduce_static(const ssmd_params *p, const LBMFields *fields, uint64_t steps_done,
                       ssmd_stats *out, ssmd_stream_t stream);

/*
 * Copies the current populations (after `steps_done` steps) to the
 * reference's push layout: which = 0 -> hydrodynamic f (element type of the
 * storage), which = 1 -> g.  out has ssmd_f_bytes / ssmd_g_bytes bytes.
 * Slots whose pull home lies outside the lattice are written as zero.
 */
int ssmd_populations_to_push(const ssmd_params *p, const LBMFields *fields,
                             uint64_t steps_done, int32_t which, void *out,
                             ssmd_stream_t stream);

/*
 * Kernel timing for benchmarks (host-side state of the calling thread, no
 * device allocation): after ssmd_profile_enable(n), the next n ssmd_step
 * calls record a CUDA event pair around their bulk-kernel launch;
 * ssmd_profile_read synchronises and returns the launch durations in ms
 * (count = recorded launches); ssmd_profile_disable frees the events.
 */
int ssmd_profile_enable(int32_t max_launches);
int ssmd_profile_read(float *ms, int32_t max, int32_t *count);
int ssmd_profile_disable(void);

/* ------------------------------------------------------------ batched sweep
 * Many independent lattices (a parameter sweep: different sizes, inlet
 * speeds, nozzles, sigma, tau, mobility) advanced by ONE persistent bulk
 * launch per step whose blocks pull (lattice, tile, z-chunk) work items from
 * an atomic counter, plus one launch per boundary kind for all lattices.
 * params[i] / fields[i] are complete single-lattice descriptions (own
 * buffers and workspace); all share velocity set and storage.  The device
 * table (ssmd_batch_table_bytes) is filled once by ssmd_batch_prepare
 * (synchronous); the batch's z-chunk comes from params[i].tile_z (0: 16).
 * ssmd_batch_step advances every lattice by one step (parity = step & 1, as
 * ssmd_step); ssmd_batch_capture_graph captures an even number of them.   */
size_t ssmd_batch_table_bytes(const ssmd_params *params, int32_t count);
int ssmd_batch_prepare(const ssmd_params *params, const LBMFields *fields, int32_t count, void *table,
                       size_t table_bytes, ssmd_stream_t stream);
int ssmd_batch_step(const ssmd_params *params, int32_t count, uint64_t step, uint32_t flags, void *table,
                    ssmd_stream_t stream);
int ssmd_batch_capture_graph(const ssmd_params *params, int32_t count, uint64_t first_step, int32_t steps,
                             uint32_t flags, void *table, ssmd_stream_t stream, ssmd_graph_exec_t *out);

/* ------------------------------------------------------------ checkpoints
 * Bit-exact save / resume (the reference's phi / rho dumps cannot restart a
 * run): current populations, the eleven macroscopic arrays and the device
 * step counter.  Loading requires the same lattice, velocity set, storage and
 * face kinds, writes the populations into both buffers and returns the step
 * count to continue from in *steps_done.  Both synchronise the stream.     */
int ssmd_checkpoint_save(const ssmd_params *p, const LBMFields *fields, uint64_t steps_done,
                         const char *path, ssmd_stream_t stream);
int ssmd_checkpoint_load(const ssmd_params *p, LBMFields *fields, const char *path,
                         uint64_t *steps_done, ssmd_stream_t stream);

/* ------------------------------------------------------------- statistics
 * Both read the macroscopic arrays (a step with SSMD_STEP_STORE_MACROS first).
 * ssmd_centreline: for every z, mean u_z and phi over the cells nearest the
 *   oil-nozzle axis (oil_cx, oil_cy); uz_out and phi_out are DEVICE arrays of
 *   nz doubles.  Asynchronous.
 * ssmd_droplets: connected components (6-neighbour, exact-periodic axes wrap)
 *   of fluid cells with phi > threshold; writes up to max_droplets entries to
 *   the HOST array out (unordered) and the number found to *n_out
 *   (SSMD_ERR_INVALID_ARGUMENT when more than max_droplets exist).  Needs
 *   ssmd_droplets_scratch_bytes() bytes of device scratch.  Synchronises.  */
/*
 * Phase-field budget of the step that produced `steps_done`: the FP64 sums of
 * the D3Q7 populations that stream from ghost cells into the fluid region
 * (inflow) and from the fluid region into ghost cells (outflow), so that
 * sum phi after the next gather = sum phi before + inflow - outflow
 * (ssmd_stats.phi_sum_next before and after).  Synchronous; uses the
 * workspace, like ssmd_reduce.  No reference counterpart.
 */
int ssmd_phase_flux(const ssmd_params *p, const LBMFields *fields, uint64_t steps_done, double *inflow,
                    double *outflow, ssmd_stream_t stream);
int ssmd_centreline(const ssmd_params *p, const LBMFields *fields, double *uz_out, double *phi_out,
                    ssmd_stream_t stream);
size_t ssmd_droplets_scratch_bytes(const ssmd_params *p, int32_t max_droplets);
int ssmd_droplets(const ssmd_params *p, const LBMFields *fields, float threshold, void *scratch,
                  size_t scratch_bytes, ssmd_droplet *out, int32_t max_droplets, int32_t *n_out,
                  ssmd_stream_t stream);

/* ------------------------------------------------------------ output files
 * The reference's file formats (host code, no GPU needed):
 *   ssmd_output_bin:  <dir>/<name><step:06>.bin, count raw FP32 values
 *                     (src/postProcess/PostProcess.cuh:44-98)
 *   ssmd_output_vti:  <dir>/step_<step:06>.vti, VTK ImageData whose appended
 *                     raw arrays are the existing <name><step>.bin files, in
 *                     the given order (PostProcess.cuh:100-262)
 *   ssmd_output_info: <dir>/<id>_info.txt run metadata
 *                     (src/functions/hostFunctions.cuh:47-87)              */
int ssmd_output_bin(const char *dir, const char *name, uint64_t step, const float *values,
                    uint64_t count);
int ssmd_output_vti(const char *dir, uint64_t step, uint32_t nx, uint32_t ny, uint32_t nz,
                    const char *const *names, int32_t count);
int ssmd_output_info(const char *dir, const char *id, const char *velocity_set, float u_water,
                     float u_oil, double reynolds_water, double reynolds_oil, double weber,
                     uint32_t nx, uint32_t ny, uint32_t nz, int32_t diam_water, int32_t diam_oil,
                     int64_t nsteps, int64_t macro_save);

/* Reads and clears the device status word (synchronises the stream):
 * bit 0 = a bulk cell produced a non-finite density. */
int ssmd_check_status(const ssmd_params *p, uint32_t *status_out, ssmd_stream_t stream);

/*
 * Derived fields (reference DerivedFields::launch, src/derivedFields/
 * DerivedFields.cuh:184-206, called once per step at src/main.cu:175): the
 * non-null arrays of p->derived, from the macroscopic fields of the last
 * step (run it with SSMD_STEP_STORE_MACROS).  Running means use t = (updates
 * since ssmd_init) + 1, which is the reference's STEP + 1 when every step is
 * averaged; a step with SSMD_STEP_AVERAGE performs the same update inside
 * the step (bulk kernel for fluid cells, a ghost-layer pass after the
 * boundaries) and counts as one update.  Device-side counter: graph-safe.
 */
int ssmd_derived_update(const ssmd_params *p, const LBMFields *fields, uint32_t what, ssmd_stream_t stream);

/*
 * Learned closure (no reference counterpart).  The network runs on the
 * tcgen05 tensor cores, 128 cells per CTA, bf16 operands, FP32 accumulation,
 * GELU in its tanh form z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))).
 *   ssmd_mlp_forward: out[i][0..1] = scale * net(features[i]) + offset
 *     (out 8-byte aligned).
 *   ssmd_mlp_grad: overwrites grad (SSMD_MLP_PARAMS floats) with dL/dparams
 *     and *loss (device double) with L = (1/n) sum_i sum_k w_ik (r_ik -
 *     (t_ik - offset_k)/scale_k)^2, r the raw output; weights may be NULL (1).
 *     The CTAs' sums meet in floating-point atomics, so the last bits vary
 *     from run to run.
 *   ssmd_mlp_grad_ws: the same, reproducible bit for bit: every CTA writes its
 *     sums to a row of `workspace` (ssmd_mlp_grad_workspace_bytes() bytes,
 *     device memory) and a second kernel adds the rows in CTA order.
 *   ssmd_mlp_adam: one Adam step (bias-corrected, step t >= 1) on the params.
 *   ssmd_mlp_average: avg = decay * avg + (1 - decay) * net on the params (an
 *     exponential moving average of the weights along training; the
 *     normalisation part of avg is left as it is).
 *   ssmd_mlp_status: bit 0 set when an MMA wait timed out (the CTA aborted).
 * Features (ssmd_closure_features), per cell, from rho, ux, uy, uz, phi with
 * central differences (periodic axes wrap, others clamp at the faces):
 *   phi, 4 phi (1 - phi), |grad phi|, laplacian phi, |S| = sqrt(2 S:S),
 *   |curl u|, n.S.n (n = grad phi / |grad phi|), |u|, u_z, rho - 1, div u,
 *   nu(phi).
 * ssmd_closure_filter box-filters a fine lattice 2x (even sizes) into coarse
 * rho, ux, uy, uz, phi (5 arrays of the coarse cell count, in that order),
 * the subgrid stress tau_ij = <u_i u_j> - <u_i><u_j> (6 arrays: xx, yy, zz,
 * xy, xz, yz) and the mean fine |grad phi| (1 array).  ssmd_closure_targets
 * turns them into training targets on the coarse lattice: nu_t* =
 * clamp(-tau^d : S / (2 S:S + 1e-12), -nut_max, nut_max) and sigma* = the ratio of
 * the fine interface area density to the coarse one, 2 <|grad phi|> /
 * |grad phi_c|, clamped to [0.25, 4] (1 where |grad phi_c| < 1e-2), with
 * weights 1 and 4 phi (1 - phi) + 0.01.  ssmd_closure_apply evaluates the
 * network on features and writes nut = clamp(out0, max(-nu(phi)/2, -nut_max),
 * nut_max) (nu(phi) is feature 11) and
 * sigma_scale = clamp(out1, 0.25, 4); out is 2 * cells floats of scratch.
 * ssmd_closure_refresh does features, network and apply in one kernel (the
 * features never leave the chip): the same nut and sigma_scale as
 * ssmd_closure_features + ssmd_closure_apply, without their buffers.
 */
int ssmd_mlp_forward(const float *net, const float *features, int64_t n, float *out, ssmd_stream_t stream);
int ssmd_mlp_grad(const float *net, const float *features, const float *targets, const float *weights, int64_t n,
                  float *grad, double *loss, ssmd_stream_t stream);
size_t ssmd_mlp_grad_workspace_bytes(void);
int ssmd_mlp_grad_ws(const float *net, const float *features, const float *targets, const float *weights,
                     int64_t n, float *grad, double *loss, float *workspace, size_t workspace_bytes,
                     ssmd_stream_t stream);
int ssmd_mlp_adam(float *net, const float *grad, float *m, float *v, int64_t t, float lr, float beta1,
                  float beta2, float eps, ssmd_stream_t stream);
int ssmd_mlp_average(float *avg, const float *net, float decay, ssmd_stream_t stream);
int ssmd_mlp_status(uint32_t *status);
int ssmd_closure_features(const ssmd_params *p, const LBMFields *fields, float *features, ssmd_stream_t stream);
int ssmd_closure_filter(const ssmd_params *fine, const LBMFields *fine_fields, float *coarse, float *tau,
                        float *area, ssmd_stream_t stream);
int ssmd_closure_targets(const ssmd_params *coarse, const float *coarse_fields, const float *tau,
                         const float *area, float nut_max, float *targets, float *weights, ssmd_stream_t stream);
int ssmd_closure_apply(const ssmd_params *coarse, const float *net, const float *features, float *out,
                       float *nut, float *sigma_scale, float nut_max, ssmd_stream_t stream);
int ssmd_closure_refresh(const ssmd_params *coarse, const LBMFields *fields, const float *net, float nut_max,
                         float *nut, float *sigma_scale, ssmd_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* SSMD_H */
