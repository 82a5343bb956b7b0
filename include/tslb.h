/*
 * tslb.h -- C-ABI of the B200 thread-safe lattice Boltzmann (TSLB) step.
 *
 * One call advances the two-component, recursive-regularized D3Q27 TSLB
 * step by n time steps on one GPU.  The state lives on the device as 11
 * moment fields per node (rho, u, v, w, pxx, pxy, pxz, pyy, pyz, pzz, phi),
 * where p** is the non-equilibrium second moment Pi^neq.  Host arrays
 * passed to the upload/download calls are Fortran column-major with x
 * fastest: element (i,j,k) of an nx*ny*nz field sits at
 * (i-1) + nx*((j-1) + ny*(k-1)) for 1-based i,j,k, exactly the layout of
 * the reference's vars-module arrays rho(1:nx,1:ny,1:nz) etc.
 *
 * Every entry point returns an int status (TSLB_OK = 0) and never aborts
 * the process; tslb_last_error() gives the message of the last failure.
 * Host pointers are borrowed for the duration of the call only.
 *
 * Which reference interface each entry point replaces (paths relative to
 * the reference repository):
 *   tslb_create          allocate(...) + parameter block of
 *                        recursive_2c_TSLB3D.f90:20-77 and the
 *                        "!$acc data copy" region at :316-317
 *   tslb_upload_pops     the device copy-in of f, g after the initial
 *                        conditions (recursive_2c_TSLB3D.f90:106-287,316)
 *                        followed by the moments pass (:346-542)
 *   tslb_upload_moments  the same copy-in for a moment-space state
 *                        (TSLB_2C-mpi/lb_kernels_module.f90:938-1142 builds
 *                        the state from rho, u, Pi)
 *   tslb_step            one loop iteration of recursive_2c_TSLB3D.f90:344-839:
 *                        moments (:346-542) + normals (:543-577) +
 *                        collision and streaming (:607-836) + boundary
 *                        conditions (:838 -> boundary_cds_3D_module.f90);
 *                        module form lb_kernels_module.f90:213,738; the
 *                        colour-gradient operator of
 *                        turbulent_benchmark/couette/recursive_colorTSLB3D.f90:468-1108
 *   tslb_download_moments "!$acc update host(rho,phi,u,v,w)"
 *                        (recursive_2c_TSLB3D.f90:597) before print_module writers
 *   tslb_download_normals "!$acc update host" of normx/normy/normz
 *   tslb_set_inlet       the inlet-plane refresh of bcs_2c_turbulent_jet
 *                        (boundary_cds_3D_module.f90:866-877)
 *   tslb_reduce          the diagnostics the drivers compute on the host
 *                        (mass, momentum) and the Laplace pressure check
 *   tslb_destroy         "!$acc end data" + deallocate (:841)
 */
#ifndef TSLB_H
#define TSLB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define TSLB_OK               0
#define TSLB_ERR_ARG          1  /* bad argument (null pointer, size, parameter) */
#define TSLB_ERR_CUDA         2  /* a CUDA runtime call failed                   */
#define TSLB_ERR_NAN          3  /* the step produced a non-finite moment        */
#define TSLB_ERR_TIMEOUT      4  /* a bounded device wait ran out                */
#define TSLB_ERR_UNSUPPORTED  5  /* valid request this build does not implement  */
#define TSLB_ERR_STATE        6  /* call out of order (e.g. step before upload)  */

/* ---- two-component operator ---- */
#define TSLB_MODE_PHASEFIELD  0  /* D3Q7 conservative phase field + CSF velocity shift
                                    (recursive_2c_TSLB3D.f90); phi in [0,1]          */
#define TSLB_MODE_COLOUR      1  /* colour gradient: perturbation + recolouring
                                    (recursive_colorTSLB3D.f90); phi in [-1,1]       */
#define TSLB_MODE_SINGLE      2  /* single component (fused_TSLB_1c / fused_TSLB_force_1c,
                                    TSLB_2C-mpi/lb_kernels_module.f90:414-736): the f
                                    step of the phase-field mode with no phase field,
                                    force as the velocity shift u + F of the equilibrium;
                                    phi is held at 1 and not stepped; tau = tau_a    */

/* ---- storage precision of the device moment state ---- */
#define TSLB_PREC_FP32        0
#define TSLB_PREC_BF16        1  /* shifted moments in bf16, collision in fp32       */
#define TSLB_PREC_FP16S       2  /* shifted moments in fp16 with per-field 2^k scale */
/* The step stores 16-bit moments with stochastic rounding (seeded by node,
 * field and step counter, reproducible; ensembles count their steps on the
 * device, so their members round as single lattices do). */

/* ---- face boundary kinds; faces are ordered x-, x+, y-, y+, z-, z+ ---- */
#define TSLB_BC_PERIODIC      0  /* wrap (mpi_module.f90:2083-2118 exchange_pops_intpbc) */
#define TSLB_BC_BOUNCEBACK    1  /* half-way bounce-back (boundary_cds_3D_module.f90:10-76) */
#define TSLB_BC_VELOCITY      2  /* regularized wall of velocity bc_u
                                    (bcs_couette_w_regularized..., :405-629)              */
#define TSLB_BC_INLET         3  /* regularized inlet, per-node velocity and colour plane
                                    (bcs_2c_turbulent_jet inlet, :931-988)                */
#define TSLB_BC_OUTLET        4  /* regularized zero-gradient outlet (:990-1048)          */
#define TSLB_BC_PRESSURE      5  /* regularized pressure outlet: density 1, velocity and
                                    phi of the fluid node (zero gradient).  No reference
                                    counterpart: the reference outlet (kind 4) takes the
                                    density of the fluid node too, which lets density and
                                    velocity drift together at low viscosity (in a jet at
                                    tau 0.5024 the outlet planes grow without bound within
                                    ~2700 steps); fixing the density removes that mode.   */

#define TSLB_NREDUCE         12

/* indices into the tslb_reduce output (all FP64, summed on the device) */
#define TSLB_RED_MASS         0  /* sum rho                                         */
#define TSLB_RED_MASS_A       1  /* colour: sum rho(1+phi)/2; phase field: sum phi  */
#define TSLB_RED_MASS_B       2  /* colour: sum rho(1-phi)/2; phase field: sum 1-phi*/
#define TSLB_RED_MOM_X        3  /* sum rho u                                       */
#define TSLB_RED_MOM_Y        4
#define TSLB_RED_MOM_Z        5
#define TSLB_RED_KINETIC      6  /* sum rho |u|^2 / 2                               */
#define TSLB_RED_UMAX         7  /* max |u|                                         */
#define TSLB_RED_RHO_IN       8  /* mean rho where phi > 0.9                        */
#define TSLB_RED_RHO_OUT      9  /* mean rho where phi < 0.1 (PF) / < -0.9 (colour)  */
#define TSLB_RED_DP          10  /* Laplace jump cs^2 (rho_in - rho_out)            */
#define TSLB_RED_N_IN        11  /* number of nodes with phi > 0.9                  */

typedef struct tslb_params {
    int32_t mode;           /* TSLB_MODE_*                                          */
    int32_t precision;      /* TSLB_PREC_*                                          */
    float   tau_a;          /* relaxation time of component A (phase field: both)   */
    float   tau_b;          /* relaxation time of component B (colour mode)         */
    float   sigma;          /* surface tension                                      */
    float   beta;           /* recolouring parameter (colour mode)                  */
    float   sharp_c;        /* interface sharpening coefficient (phase field)       */
    float   grad_threshold; /* colour mode: |grad phi| below which neither the
                               perturbation nor the recolouring is applied          */
    float   force[3];       /* constant body force                                  */
    int32_t bc[6];          /* TSLB_BC_* per face x-, x+, y-, y+, z-, z+            */
    float   bc_u[6][3];     /* wall / inlet velocity per face (TSLB_BC_VELOCITY);
                               outlet: x,y used, z replaced by the fluid value;
                               phase-field outlet: z is the advection speed of g    */
    float   bc_phi[6];      /* colour carried by incoming populations at velocity
                               faces (<-2: use the fluid node's own phi) and the
                               ghost phi of solid faces when wall_phi_mode == 0     */
    int32_t wall_phi_mode;  /* ghost phi on solid faces: 0 = bc_phi, 1 = mirror     */
    int32_t reserved[7];
} tslb_params;

typedef struct tslb_ctx tslb_ctx;

/* Fill *p with the defaults of the reference's two-component program
 * (recursive_2c_TSLB3D.f90:20-28,45-48): phase field, tau 0.5004,
 * sigma 0.001, sharp_c 0.9, periodic faces, FP32 storage. */
void tslb_default_params(tslb_params* p);

/* Validate *p and the sizes, allocate the device state of nx*ny*nz nodes
 * and a CUDA stream on the current device.  *out is NULL on failure. */
int  tslb_create(const tslb_params* p, int nx, int ny, int nz, tslb_ctx** out);
void tslb_destroy(tslb_ctx* ctx);

/* Upload the 11 moment fields (host, Fortran layout, nx*ny*nz floats each).
 * Pi arguments are the non-equilibrium second moments. */
int  tslb_upload_moments(tslb_ctx* ctx,
                         const float* rho, const float* u, const float* v, const float* w,
                         const float* pxx, const float* pxy, const float* pxz,
                         const float* pyy, const float* pyz, const float* pzz,
                         const float* phi);

/* Upload populations in the reference's halo layout f(0:nx+1,0:ny+1,0:nz+1,0:26)
 * and g(...,0:6) (phase field) or g(...,0:26) (colour: f = component A,
 * g = component B) and run the moments pass on the device. */
int  tslb_upload_pops(tslb_ctx* ctx, const float* f, const float* g);

/* Advance nsteps time steps (asynchronous on the context stream). */
int  tslb_step(tslb_ctx* ctx, int nsteps);

/* Download the moment fields (synchronises).  Any pointer may be NULL. */
int  tslb_download_moments(tslb_ctx* ctx,
                           float* rho, float* u, float* v, float* w,
                           float* pxx, float* pxy, float* pxz,
                           float* pyy, float* pyz, float* pzz,
                           float* phi);

/* Download the interface normals n = grad(phi)/(|grad(phi)|+1e-9) of the
 * current state (recursive_2c_TSLB3D.f90:555-571). */
int  tslb_download_normals(tslb_ctx* ctx, float* nx, float* ny, float* nz);

/* FP64 diagnostics of the current state, see TSLB_RED_* (synchronises). */
int  tslb_reduce(tslb_ctx* ctx, double out[TSLB_NREDUCE]);

/* The same diagnostics without waiting: tslb_reduce_async queues the
 * reduction of the state after the steps queued so far, and its copy into
 * page-locked host memory of the context; tslb_reduce_collect waits for the
 * stream and writes the queued results in queue order to
 * out[i * TSLB_NREDUCE ...] for i < *count = min(max, queued), dropping the
 * rest.  At most TSLB_REDUCE_QUEUE results wait at a time.  This is the
 * reference's pattern of reading diagnostics at the print stamps
 * (recursive_2c_TSLB3D.f90:580-599) with a result per step kept, and no
 * host wait per step. */
#define TSLB_REDUCE_QUEUE 256
int  tslb_reduce_async(tslb_ctx* ctx);
int  tslb_reduce_collect(tslb_ctx* ctx, double* out, int max, int* count);

/* Set the inlet plane of face (TSLB_BC_INLET faces only): uvw_phi holds
 * four planes (u, v, w, phi) of the face's extent, Fortran order. */
int  tslb_set_inlet(tslb_ctx* ctx, int face, const float* uvw_phi);

/* ---- moment-space boundary planes (TSLB_newBCS/boundary_cds_3D_module.f90:1233-1292) ----
 * Before every step the moments of the face plane (z faces: z = 0 or nz-1)
 * are rewritten from the plane next to it, between the moments pass and the
 * collision as bcs_TSLB_only_z_turbojet does:
 *   TSLB_MBC_COPY  all moments copied from the next plane inward (its k = nz side)
 *   TSLB_MBC_JET   rho and Pi copied from the next plane, u = v = 0; w keeps the
 *                  stepped value, except on every 10th step (reference step
 *                  numbering, step = steps done + 1) when the nodes of the disc
 *                  (i - nx/2)^2 + (j - ny/2)^2 <= radius^2 (1-based i, j) get
 *                  w = uwall + amp sqrt(-2 ln r) cos(2 pi r), r = rand_noseeded(i, j, 1, step)
 *                  (its k = 1 side; r is floored at 2^-25 so w stays finite)
 * The populations that enter the plane from outside follow the face's kind
 * as usual (the reference leaves its z halo untouched). */
#define TSLB_MBC_NONE  0
#define TSLB_MBC_COPY  1
#define TSLB_MBC_JET   2
int  tslb_set_moment_bc(tslb_ctx* ctx, int face, int kind, float uwall, float radius, float amp);
/* The reference's counter-based uniform rand_noseeded(i, j, k, l)
 * (TSLB_2C-mpi/vars_single_3D_module.f90:150-215), bit-exact. */
float tslb_rand_noseeded(int i, int j, int k, int l);

/* Interior solid nodes: isfluid holds nx*ny*nz bytes (Fortran order), 1 for
 * a fluid node and 0 for a solid one, as the reference's isfluid array
 * (recursive_2c_TSLB3D.f90:79-85); NULL removes them.  Populations that
 * would leave a fluid node toward a solid one come back to it (half-way
 * bounce-back, boundary_cds_3D_module.f90:10-76 applied at every
 * isfluid == 0 node), solid nodes keep their moments (their phi is the wall
 * value the colour gradient and the phase field see), and phase-field
 * normals at solid nodes are 0.  Face conditions apply as before; a source
 * behind a face follows the face.  FP32 storage; not combined with a tau
 * correction or a closure. */
int  tslb_set_solid_mask(tslb_ctx* ctx, const unsigned char* isfluid);

/* Jet inlet drawn on the device (asynchronous, no host copy): the plane of
 * inlet face `face` becomes a disc of radius `radius` centred at in-plane
 * coordinates (c0, c1) -- (x, y) for z faces, (x, z) for y faces, (y, z)
 * for x faces, node indices from 0 -- with normal velocity
 * speed * (1 + amp * xi) into the lattice and phi = +1; outside the disc the
 * velocity is 0 and phi = -1.  xi is uniform in [-1, 1): the top 24 bits of
 * h = m(m(seed * 0x9E3779B97F4A7C15 + counter) ^ i), m the splitmix64
 * finaliser and i the plane index (first coordinate fastest), times 2^-23,
 * minus 1.  Replaces the host random_number refresh of the jet inlet
 * (boundary_cds_3D_module.f90:866-877); call it with counter = step / 10
 * to refresh every 10 steps. */
int  tslb_set_inlet_disc(tslb_ctx* ctx, int face, float c0, float c1, float radius, float speed, float amp,
                         unsigned long long seed, unsigned long long counter);

/* Static per-node correction dtau of the relaxation time (colour mode,
 * FP32 storage): node x relaxes with tau(phi_x) + dtau[x], i.e. an added
 * local viscosity dtau/3, in the collision and in the regularized faces; the
 * surface-tension coefficient follows the corrected omega.  dtau holds
 * nx*ny*nz values (Fortran order) with tau + dtau > 1/2; NULL switches the
 * correction off.  Typical use: a sponge layer in front of an outlet.  With
 * a learned closure attached (tslb_closure.h) the closure's output is added
 * to this field.  The reference has no counterpart. */
int  tslb_set_tau_correction(tslb_ctx* ctx, const float* dtau);
/* The correction in effect (static field plus closure output; zeros when
 * there is none). */
int  tslb_download_tau_correction(tslb_ctx* ctx, float* dtau);

/* Time averages on the device: tslb_stats_accumulate adds u, v, w, phi,
 * the six products u_a u_b and the six Pi^neq components of the current
 * state to running sums (asynchronous; 16 FP32 fields per node);
 * tslb_stats_download returns the means of u, v, w, phi and w^2 over the
 * accumulated samples, averaged over coarsen^3 blocks (coarsen divides nx,
 * ny, nz; outputs have nc = (nx/coarsen)*(ny/coarsen)*(nz/coarsen) values;
 * any pointer may be NULL) and the sample count;
 * tslb_stats_download_stress the means of the products into uu (6 x nc:
 * uu, uv, uw, vv, vw, ww) and of Pi^neq into pineq (6 x nc: xx, xy, xz, yy,
 * yz, zz), for Reynolds and viscous stresses.  They stand in for the
 * host-side averaging the reference's drivers do on frames written by
 * print_module.f90 (no counterpart in its step). */
int  tslb_stats_reset(tslb_ctx* ctx);
int  tslb_stats_accumulate(tslb_ctx* ctx);
int  tslb_stats_download(tslb_ctx* ctx, int coarsen, float* u, float* v, float* w, float* phi, float* ww,
                         long long* count);
int  tslb_stats_download_stress(tslb_ctx* ctx, int coarsen, float* uu, float* pineq, long long* count);

/* Wait for all work queued on the context stream. */
int  tslb_synchronize(tslb_ctx* ctx);

/* The context's cudaStream_t, for callers that order their own work or
 * CUDA events against the step. */
void* tslb_stream(tslb_ctx* ctx);

/* Device memory of destroyed lattices stays cached for the next lattice (up
 * to 1/8 of each device's memory); this returns all of it to the devices,
 * e.g. before the host allocates large buffers of its own.  No counterpart
 * in the reference, which allocates its arrays once. */
int tslb_release_memory(void);

/* Number of kernel launches the context has issued since creation. */
long long tslb_launch_count(tslb_ctx* ctx);

/* Message of the last failed call on ctx (or, when ctx is NULL, of the
 * calling thread's last failed tslb_create or tslb_step_noalloc: each host
 * thread keeps its own).  Never NULL.  A context is used by one thread at a
 * time; different contexts may be used by different threads concurrently. */
const char* tslb_last_error(tslb_ctx* ctx);

/* ---- z slabs: one lattice over several GPUs ----
 *
 * Replaces the reference's MPI domain decomposition and halo exchange
 * (TSLB_2C-mpi/mpi_module.f90:2120-2258: pack, mpi_isend/mpi_irecv, wait,
 * unpack; periodic wrap :2083-2118).  The lattice of nx*ny*nz nodes is cut
 * along z; a slab context owns planes [z_begin, z_end) and keeps H halo
 * planes on every side that has a neighbouring slab (a periodic z axis, or
 * an inner cut): H = 2 in colour mode, 3 in phase-field mode, 1 in
 * single-component mode.  Its device array holds halo_lo + (z_end -
 * z_begin) + halo_hi planes, bottom up; the upload/download calls take and
 * return that whole local array (host layout, Fortran order), tslb_step
 * updates the own planes only, and tslb_reduce covers the own planes.  The
 * z faces of the lattice apply on the slabs that own them.
 *
 * After every step the halos must be refreshed before the next one:
 *   tslb_halo_pack(ctx, side, d_buf) copies the own edge planes that the
 *   neighbour on `side` (0: z-, 1: z+) needs into the device buffer d_buf of
 *   tslb_halo_bytes(ctx) bytes -- the 10 non-phi moments of the edge plane,
 *   then phi of H edge planes, in the storage type;
 *   the caller moves the buffer to that neighbour (NCCL send/recv, a peer
 *   copy), whose tslb_halo_unpack(ctx, other side, d_buf) writes it into its
 *   halo planes.  Both are queued on the context stream.
 * Inlet faces and moment-space boundary planes must lie on the slab that
 * owns their face. */
int  tslb_create_slab(const tslb_params* p, int nx, int ny, int nz, int z_begin, int z_end, tslb_ctx** out);
/* out = {nz (whole lattice), z_begin, z_end, halo_lo, halo_hi, H} */
int  tslb_slab_geometry(const tslb_ctx* ctx, int out[6]);
long long tslb_halo_bytes(const tslb_ctx* ctx);
int  tslb_halo_pack(tslb_ctx* ctx, int side, void* d_buf);
int  tslb_halo_unpack(tslb_ctx* ctx, int side, const void* d_buf);

/* ---- batched ensemble of independent lattices ----
 *
 * Many independent lattices of different sizes (all of one mode and one
 * storage precision) advanced together: every time step is ONE kernel
 * launch whose blocks walk a work list of (lattice, tile, z chunk) items,
 * and tslb_ensemble_step_graph captures K such steps in a CUDA graph.  This
 * replaces running the reference program once per domain (the reference
 * has no batching).  Member i is addressed by its index. */
typedef struct tslb_ensemble tslb_ensemble;

/* params[i] and dims[3*i .. 3*i+2] = (nx, ny, nz) of member i. */
int  tslb_ensemble_create(const tslb_params* params, const int* dims, int n, tslb_ensemble** out);
void tslb_ensemble_destroy(tslb_ensemble* e);
int  tslb_ensemble_upload_moments(tslb_ensemble* e, int i,
                                  const float* rho, const float* u, const float* v, const float* w,
                                  const float* pxx, const float* pxy, const float* pxz,
                                  const float* pyy, const float* pyz, const float* pzz,
                                  const float* phi);
/* nsteps steps, one launch each, on the ensemble stream (asynchronous). */
int  tslb_ensemble_step(tslb_ensemble* e, int nsteps);
/* The same nsteps steps replayed from a CUDA graph (captured on first use). */
int  tslb_ensemble_step_graph(tslb_ensemble* e, int nsteps);
int  tslb_ensemble_download_moments(tslb_ensemble* e, int i,
                                    float* rho, float* u, float* v, float* w,
                                    float* pxx, float* pxy, float* pxz,
                                    float* pyy, float* pyz, float* pzz, float* phi);
int  tslb_ensemble_reduce(tslb_ensemble* e, int i, double out[TSLB_NREDUCE]);
/* Autotuner of the persistent kernel: time 10 steps of each candidate z
 * chunk with each resident grid (two and one blocks per SM, taking the work
 * items in list order, longest first, as they finish) on the uploaded state
 * (restored afterwards) and keep the fastest; returns the choice.  One block
 * per work item (grid 0) is set only by tslb_ensemble_set_launch. */
int  tslb_ensemble_tune(tslb_ensemble* e, int* zchunk, int* grid);
/* The last tuning's timings, in the order they ran: *count rows (at most
 * max written) of z chunk (1 << 20: whole lattices), grid and milliseconds
 * per step.  No reference counterpart (the reference has no ensembles). */
int  tslb_ensemble_tune_results(tslb_ensemble* e, int max, int* count, int* zchunk, int* grid, float* ms_per_step);
/* Set the z chunk (>= 1) and grid (>= 0, as above) without tuning.  No
 * reference counterpart. */
int  tslb_ensemble_set_launch(tslb_ensemble* e, int zchunk, int grid);
int  tslb_ensemble_synchronize(tslb_ensemble* e);
void* tslb_ensemble_stream(tslb_ensemble* e);
const char* tslb_ensemble_last_error(tslb_ensemble* e);

/* Size of tslb_step_noalloc's device scratch (32-bit words). */
#define TSLB_NOALLOC_SCRATCH_WORDS 64

/* One time step on caller-owned device buffers, allocating nothing.
 *
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc -- a host that owns all device memory itself (an OpenACC data
 * region, a memory pool, a real-time loop that must not allocate).  The
 * only scratch the step needs, its non-finite flag, lives in a fixed device
 * array inside the library (TSLB_NOALLOC_SCRATCH_WORDS words on every GPU
 * that loads the library, held until the process exits); it does not grow
 * with the lattice (the phase-field step forms its interface normals
 * itself), so the call takes any lattice size the context API takes.
 *
 * d_in and d_out hold the 11 fields in the library's device layout: field
 * f at d_x + f * field_stride (floats), x fastest, field 0 = rho - 1, then
 * u, v, w, pxx, pxy, pxz, pyy, pyz, pzz, phi.  Both 16-byte aligned,
 * field_stride >= nx*ny*nz and a multiple of 4; the two ranges of
 * 11 * field_stride floats must not overlap.  Inlet faces are not supported
 * (their planes need storage).  The work is queued on `stream`
 * (cudaStream_t, NULL = default stream) and not waited for.  A step that
 * produces a non-finite moment sets the flag; read it with
 * tslb_noalloc_check.
 *
 * The first call on a device (of this function or tslb_noalloc_check)
 * resolves the scratch address and sets the attributes of every kernel this
 * function launches; make that first call before any stream capture.  All
 * calls share the one scratch array, so calls that overlap on the GPU
 * (other streams, other threads) race: order them on one stream. */
int tslb_step_noalloc(const tslb_params* p, int nx, int ny, int nz,
                      const float* d_in, float* d_out, long long field_stride,
                      void* stream);

/* Wait for `stream` (cudaStream_t, NULL = default stream) and report whether
 * any tslb_step_noalloc step on the current device since the previous check
 * produced a non-finite moment: TSLB_ERR_NAN if so (the flag is then
 * cleared), TSLB_OK if not.  Allocates nothing.  Like tslb_step_noalloc it
 * has no counterpart in the reference. */
int tslb_noalloc_check(void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TSLB_H */
