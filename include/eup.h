/*
 * eup.h -- C ABI of the B200 (sm_100a) D3Q19 BGK lattice-Boltzmann time step.
 *
 * Drop-in for the time-step loop of giacomofalcucci/Euplectella_HPC
 * (CODE/SRC/bgk3d.F90:114-152).  The reference's Fortran driver keeps its
 * input files, its arrays a01..a19(0:l+1,0:m+1,0:n+1) and its output layout;
 * a `bind(c)` interface (fortran/eup_mod.F90) calls these entry points in
 * place of boundaries/propagation/collision.  Plain pointers and sizes only;
 * every entry point returns an eup_status (0 = success) and never aborts,
 * exits or throws.
 *
 * Conventions shared with the reference:
 *  - population q = 1..19 is the reference's aQQ; arrays passed as `pops[19]`
 *    are indexed q-1 and velocity q is the table of CODE/SRC/bgk3d.F90:30-49;
 *  - every population array is haloed, Fortran order (i fastest), extent
 *    (l+2)*(m+2)*(n+2) elements, element type float (4 bytes, the reference's
 *    default mykind) or double (8 bytes, -DDOUBLE_P);
 *  - `obs` is obs(1:l,1:m,1:n), int32, Fortran order, value 1 = solid;
 *  - boundary flags use the reference codes of CODE/SRC/build.bcond.F90:11-17.
 *
 * Threading: one host thread per handle (the reference runs one MPI rank per
 * GPU, MPI_THREAD_SINGLE).  Calls on one handle are serialised.  eup_step is
 * asynchronous on the handle's stream; entry points that return data
 * synchronise.  Host arrays belong to the caller and are never retained.
 */
#ifndef EUP_H
#define EUP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EUP_ABI_VERSION 1

typedef enum eup_status {
    EUP_OK = 0,
    EUP_ERR_INVALID_ARG = 1,    /* bad pointer, size, flag or call order */
    EUP_ERR_CUDA = 2,           /* a CUDA runtime call failed; text in eup_last_error */
    EUP_ERR_OOM = 3,            /* device or pinned-host allocation failed */
    EUP_ERR_DIVERGED = 4,       /* a monitored FP64 sum is not finite */
    EUP_ERR_UNSUPPORTED = 5,    /* valid in the reference but not offered here (text says why) */
    EUP_ERR_IO = 6,             /* file missing, short or malformed */
    EUP_ERR_NO_DEVICE = 7       /* no usable CUDA device */
} eup_status;

/* Boundary flag codes (CODE/SRC/build.bcond.F90:11-17). */
enum {
    EUP_BC_PERIODIC = 0,
    EUP_BC_NOSLIP = 1,
    EUP_BC_LID = 2,       /* up face only */
    EUP_BC_FREESLIP = 3,  /* up/down/left/right */
    EUP_BC_INFLOW = 4,    /* rear face only */
    EUP_BC_OUTFLOW = 5,   /* front face only */
    EUP_BC_EXCHANGE = 6   /* front/rear: an x-slab face whose halo plane the caller fills from the
                             neighbouring slab (eup_set_x_planes); no reference flag, the
                             reference's MPI faces are implied by its process grid */
};

/* Face order of eup_config.bc (reference names front/rear/right/left/up/down). */
enum { EUP_FRONT = 0, EUP_REAR = 1, EUP_RIGHT = 2, EUP_LEFT = 3, EUP_UP = 4, EUP_DOWN = 5 };

/* Population storage in device memory. */
typedef enum eup_precision {
    EUP_FP32 = 0,       /* float storage and arithmetic (the reference's default) */
    EUP_FP64 = 1,       /* double storage and arithmetic (-DDOUBLE_P) */
    EUP_FP16_DEV = 2,   /* half storage of (f_q - w_q)*scale, float arithmetic */
    EUP_BF16_DEV = 3    /* bfloat16 storage of (f_q - w_q)*scale, float arithmetic */
} eup_precision;

typedef struct eup_config {
    int32_t lx, ly, lz;     /* lattice nodes (one GPU: l=lx, m=ly, n=lz) */
    int32_t bc[6];          /* reference flag per face, order EUP_FRONT..EUP_DOWN */
    double svisc;           /* kinematic viscosity; omega = 2/(6 svisc+1) as in CODE/SRC/hencol.F90:30 */
    double u0;              /* body-force scale; fgrad = 4 u0 svisc/(5 lz^2), CODE/SRC/hencol.F90:37 (0 with an inlet) */
    double u_inflow;        /* inlet velocity of EUP_BC_INFLOW, CODE/SRC/bcond.bc.F90:262 */
    double u00;             /* lid velocity scale, force = u00/6, CODE/SRC/bcond.bc.F90:50-56 */
    int32_t precision;      /* eup_precision */
    int32_t device;         /* CUDA device ordinal */
    double dev_scale;       /* scale of the 16-bit deviation storage; 0 selects 4096 */
    /* drag coefficient normalisation C_d = F_x / (0.5 rho0 u_ref^2 length span) */
    double cd_rho0, cd_uref, cd_length, cd_span;
    int64_t series_capacity;  /* force history entries kept on the device; 0 selects 1<<20 */
} eup_config;

typedef struct eup_handle eup_handle;

/* ---- life cycle --------------------------------------------------------- */

/* Library ABI version (EUP_ABI_VERSION). */
int32_t eup_abi_version(void);

/* Number of usable CUDA devices, 0 when none (never fails). */
int32_t eup_device_count(void);

/* Creates a solver on cfg->device and allocates both population lattices, the
 * halo shell and the diagnostic buffers.  Replaces the set-up half of
 * CODE/SRC/initialize.F90:22-158 (build_bcond, alloca, hencol). */
int eup_create(const eup_config* cfg, eup_handle** out);

/* Frees every device resource of the handle; h may be NULL. */
int eup_destroy(eup_handle* h);

/* Text of the last failure on h (h == NULL: last failure of eup_create or of
 * a handle-less call on this thread).  Valid until the next call. */
const char* eup_last_error(const eup_handle* h);

/* ---- state ---------------------------------------------------------------- */

/* Installs the solid mask obs(1:l,1:m,1:n) (1 = solid): builds the bit-packed
 * mask, the list of solid voxels adjacent to fluid or halo (which takes the place
 * of the reference's bounding box) and their neighbour classification.  Replaces
 * CODE/SRC/build.obs.F90:33-194 as consumed by CODE/SRC/bcond.obs.F90:47-77.
 * Solid voxels on the outflow plane i = l are rejected (EUP_ERR_UNSUPPORTED):
 * there the reference's result depends on the iteration order of its
 * bounce-back loop.  A rejected mask, or one whose buffers cannot be
 * allocated, leaves the previous mask installed. */
int eup_set_obstacles(eup_handle* h, const int32_t* obs);

/* ---- obstacles built on the device ------------------------------------------ */

/* Voxel shapes (eup_geometry.kind). */
enum {
    EUP_GEOM_NONE = 0,            /* no solid voxel */
    EUP_GEOM_REF_SPHERE = 1,      /* spherical shell, CODE/SRC/build.obs.F90:207-268 (flag2 = 1) */
    EUP_GEOM_REF_COLUMN = 2,      /* z-column, CODE/SRC/build.obs.F90:271-441 (flag2 = 2 and 3) */
    EUP_GEOM_CYLINDER_Z = 3,      /* solid circular cylinder along z, as eup_geometry_cylinder_z */
    EUP_GEOM_RETICULAR_SHELL = 4, /* as eup_geometry_reticular_shell */
    EUP_GEOM_RIDGED_SHELL = 5     /* eup_geometry_ridged_shell with smooth_w = 0, as a 0/1 mask */
};

/* A voxel shape in global node coordinates (global index = local index + offset). */
typedef struct eup_geometry {
    int32_t kind;
    int32_t offset[3];  /* global index of this lattice's node (1,1,1) minus 1: the reference's
                           mpicoords(d) * (l, m, n) (CODE/SRC/build.obs.F90:233-235), an x-slab's x0 - 1 */
    /* REF_SPHERE: solid where d2 = |center - global index|^2 (integers) satisfies
     * r2_lo < d2 < r2_hi.  REF_COLUMN: the same in x and y with r2_lo <= d2 < r2_hi, for
     * center[2] <= global k < kstop.  eup_geometry_reference fills them as the reference does. */
    int32_t center[3];
    int32_t kstop;
    int64_t r2_lo, r2_hi;
    /* CYLINDER_Z: xc, yc, radius.  Shells: x0, length, yc, zc, outer_d, strut_d, pitch, seed;
     * RIDGED_SHELL also ridge_h, ridge_t, cap_t, pore_d (the eup_geometry_* helpers' arguments). */
    double xc, yc, zc, radius;
    double x0, length, outer_d, strut_d, pitch;
    double ridge_h, ridge_t, cap_t, pore_d;
    uint64_t seed;
} eup_geometry;

/* Variant bits of eup_geometry_reference: compile-time choices of the reference's build_obs. */
enum { EUP_GEOM_VARIANT_CYLINDER_INF = 1, EUP_GEOM_VARIANT_TEST1 = 2 };

/* The obstacle CODE/SRC/build.obs.F90 creates for flag1 = 2 on a global lattice
 * lx x ly x lz: flag2 = 1 sphere (radius 20; min(ly/4, lz/4) with TEST1), 2 column
 * (radius min(20, lx/8) over 1 <= k < lz; radius 100 over every k with CYLINDER_INF),
 * 3 half column (radius min(20, lz/8), 1 <= k < 60), centred at (lx/4, ly/2[, lz/2]),
 * offset 0.  No GPU.  -DCHECK2D leaves the reference's radius unset and is not offered. */
int eup_geometry_reference(int32_t flag2, int32_t lx, int32_t ly, int32_t lz, int32_t variant,
                           eup_geometry* g);

/* Voxelises g on the device straight into the handle's bit-packed mask (one warp
 * per 32 nodes of an x row; no host array, no host-to-device copy of a mask) and
 * installs it with the checks of eup_set_obstacles.  The mask equals
 * eup_voxelise's bit for bit. */
int eup_build_obstacles(eup_handle* h, const eup_geometry* g);

/* The installed mask as obs(1:l,1:m,1:n) (obs may be NULL) and its number of
 * solid voxels (nobs may be NULL).  The bit-packed mask crosses to the host. */
int eup_get_obstacles(eup_handle* h, int32_t* obs, int64_t* nobs);

/* Writes the installed mask as an obstacle file (CODE/SRC/build.obs.F90:506-541:
 * a record with the count, then one (i,j,k) record per solid voxel, i fastest).
 * The list is compacted and laid out as records on the device and crosses to the
 * host in one copy.  The count written is the number of records: the reference
 * writes that count minus 100 for the obstacles it creates (its counter starts
 * at -100, CODE/SRC/build.obs.F90:68), so reading its file back drops 100 voxels. */
int eup_write_obstacles(eup_handle* h, const char* path);

/* Copies the 19 haloed host arrays (elem_bytes 4 or 8) into device storage:
 * interior nodes into the lattice (converted to the storage precision), halo
 * nodes into the persistent halo shell.  Replaces the host-to-device copy of
 * CODE/SRC/bgk3d.F90:113 / CODE/SRC/initialize.F90:164-175; also the
 * restart path (CODE/SRC/restore_raw.F90:43-63).  Sets the step counter.
 * A value that is not finite (NaN, Inf) anywhere in the 19 arrays is
 * EUP_ERR_INVALID_ARG naming the populations; the handle then holds no state
 * (eup_restore_state and eup_init_state check the same way).  The host copy of
 * each population overlaps the device-side conversion of the previous one
 * (two staging buffers, a copy stream of the handle's own): page-locked host
 * arrays move at the host link's full rate. */
int eup_upload(eup_handle* h, const void* const pops[19], int32_t elem_bytes, int64_t itime);

/* The seeded equilibrium state of eup_init_equilibrium generated on the
 * device: the same bits as eup_upload of eup_init_equilibrium's arrays
 * (elem_bytes 8 for an FP64 handle, else 4), without host arrays or a
 * host-to-device copy of the lattice.  No reference counterpart (the
 * reference initialises on the host, CODE/SRC/init.F90). */
int eup_init_state(eup_handle* h, double u_in, double amp, uint64_t seed, int64_t itime);

/* Checkpoint files in the reference's raw format (CODE/SRC/save_raw.F90:41-78,
 * restore_raw.F90:34-63: a record holding itime as int32, then 19 records of
 * the haloed arrays, elem_bytes 4 or 8, gfortran 4-byte record markers)
 * written from and read into the device state directly, one population at a
 * time through a pinned buffer, with no 19-array host copy: 16-bit storage is
 * expanded to float/double on the way out.  A 16-bit state crosses a double file
 * (elem_bytes 8) bit for bit; in a float file f = w + D/scale is rounded to float,
 * which drops low bits of deviations below 2^-6 (the same holds for eup_download and
 * eup_upload with elem_bytes 4 and 8).  Records over 2 GiB (a population
 * beyond 2^29 FP32 nodes) are rejected.  eup_restore_state sets the step
 * counter from the file. */
int eup_save_state(eup_handle* h, const char* path, int32_t elem_bytes);
int eup_restore_state(eup_handle* h, const char* path, int32_t elem_bytes);

/* Copies the current state back into 19 haloed host arrays: the interior from
 * the lattice, the halo from the halo shell, exactly what the reference's
 * arrays hold after a step.  Replaces the device-to-host copies of
 * CODE/SRC/diagnostic.F90:47-58,110-120,163-174 and CODE/SRC/bgk3d.F90:153.
 * Like eup_upload, each population's copy overlaps the gather of the next. */
int eup_download(eup_handle* h, void* const pops[19], int32_t elem_bytes);

/* ---- time step ------------------------------------------------------------ */

/* Advances nsteps time steps of CODE/SRC/bgk3d.F90:128-138: bounce-back on
 * solid voxels (CODE/SRC/bcond.obs.F90), halo planes in the reference's order
 * (CODE/SRC/bcond.bc.F90), then one fused pull stream-collide kernel
 * (CODE/SRC/movef.F90 + CODE/SRC/col.F90).  The momentum-exchange force of
 * every state reached is recorded in FP64.  Asynchronous. */
int eup_step(eup_handle* h, int32_t nsteps);

/* Same work as eup_step, with CUDA events on the handle's stream around each
 * phase; adds to ms[0..2] the device milliseconds spent in bounce-back + drag,
 * halo planes and stream-collide over the nsteps, and sets ms[3] to the
 * elapsed device time of the whole call.  Synchronises.  Replaces the phase
 * timers of CODE/SRC/boundaries.F90, propagation.F90 and collision.F90
 * (time_obs, time_bc, time_move, time_coll of CODE/SRC/finalize.F90:58-124). */
int eup_step_profiled(eup_handle* h, int32_t nsteps, double ms[4]);

/* Waits for all work queued on the handle; reports deferred CUDA errors. */
int eup_synchronize(eup_handle* h);

/* The handle's CUDA stream (a cudaStream_t), so callers can order their own
 * device work, events or copies with the solver's. */
int eup_get_stream(eup_handle* h, void** stream);

/* Number of CUDA kernels the time-step entry points have launched on this
 * handle so far (bounce-back/drag, halo planes, stream-collide, and for an
 * x slab the plane pack/unpack kernels). */
int eup_get_launch_count(eup_handle* h, int64_t* launches);

/* Current step counter (itime of the state held on the device). */
int eup_get_itime(eup_handle* h, int64_t* itime);

/* ---- diagnostics ---------------------------------------------------------- */

/* Momentum-exchange force on the solid for the current state, FP64:
 * F = sum over fluid nodes x and directions q with solid neighbour x + c_q
 * (wrapped across periodic axes) of 2 c_q f_q(x), post-collision.  No
 * reference counterpart (the reference's drag is CODE/SRC/drag.F90:33-79).
 * EUP_ERR_DIVERGED when a component is not finite (the values are still
 * written), the same for eup_get_force_series and eup_get_cd_series. */
int eup_get_forces(eup_handle* h, double fxyz[3]);

/* Force history: entries for steps first_step .. first_step+count-1 (step t =
 * the state after t time steps), 3 doubles each.  Steps older than the ring
 * capacity or not yet reached are EUP_ERR_INVALID_ARG. */
int eup_get_force_series(eup_handle* h, int64_t first_step, int32_t count, double* fxyz);

/* Drag coefficient history C_d(t) = F_x/(0.5 cd_rho0 cd_uref^2 cd_length cd_span). */
int eup_get_cd_series(eup_handle* h, int64_t first_step, int32_t count, double* cd);

/* Global sums of CODE/SRC/diagno.F90:67-120 in FP64 over the interior, solid
 * voxels counted as rho = 1, u = 0: out = {sum rho, sum ux, sum uy, sum uz,
 * sum u^2}.  EUP_ERR_DIVERGED when any sum is not finite. */
int eup_get_monitor(eup_handle* h, double out[5]);

/* Line profile of CODE/SRC/prof_i.F90 (axis 0, nodes (1..l, c1, c2)),
 * prof_j.F90 (axis 1, (c1, 1..m, c2)) and prof_k.F90 (axis 2, (c1, c2, 1..n)):
 * out[4t .. 4t+3] = u, w (y velocity), v (z velocity), den of the t-th node,
 * computed in the arithmetic type in the reference's expression order (so FP32
 * and FP64 runs reproduce the reference's values exactly), widened to double. */
int eup_get_line(eup_handle* h, int32_t axis, int32_t c1, int32_t c2, double* out);

/* Means over every plane normal to `axis` of u, w, v and den, as
 * CODE/SRC/varm.F90:42-98 computes them for axis 2 (u_med files): per-node
 * values in the arithmetic type, sums in FP64 (the reference sums in mykind).
 * out[4p .. 4p+3] for plane p = 0..extent-1.  All nodes count, solid ones too,
 * as in the reference (values at solid voxels are not those of the reference:
 * see eup_set_obstacles). */
int eup_get_plane_means(eup_handle* h, int32_t axis, double* out);

/* Control-volume drag of CODE/SRC/drag.F90:51-67: box = {xstart, xstop,
 * ystart, ystop, zstart, zstop} (1-based, clipped to the lattice with the face
 * weights of CODE/SRC/flux_X.F90:56-156); out[0] = fluxX (sigma_xx over the
 * two x faces), out[1] = fluxY (sigma_xy over the two y faces).  Per-node
 * stresses in the arithmetic type as CODE/SRC/flux_X.F90:162-240 writes them,
 * face sums in FP64. */
int eup_get_cv_drag(eup_handle* h, const int32_t box[6], double out[2]);

/* FP64 sums over the fluid nodes whose byte in region (Fortran order, l*m*n,
 * nonzero = included) is set: out = {count, sum rho, sum ux, sum uy, sum uz,
 * sum u^2}.  Region means (the velocity inside a shell's cavity, a probe box)
 * without downloading the populations.  No reference counterpart: the
 * reference's diagnostics of this kind (CODE/SRC/varm.F90, prof_*.F90) sum
 * whole planes and lines of the host arrays. */
int eup_get_region_sums(eup_handle* h, const uint8_t* region, double out[6]);

/* rho, ux, uy, uz (FP64) at npts interior nodes (1-based i,j,k triples), as
 * CODE/SRC/probe_global.F90:58-77 computes them. */
int eup_get_probes(eup_handle* h, int32_t npts, const int32_t* ijk, double* rho_u);

/* Link classification per interior node (Fortran order): bit q-1 set when the
 * node is fluid and x - c_q is an interior solid voxel (its pull is served by
 * bounce-back); bit 31 marks a solid voxel. */
int eup_get_links(eup_handle* h, uint32_t* links);

/* Interior linear indices (i-1 + l*(j-1 + m*(k-1))) of the solid voxels that
 * touch fluid or halo, ascending.  *count receives the total; at most cap
 * entries are written. */
int eup_get_boundary_solid(eup_handle* h, int64_t* list, int64_t cap, int64_t* count);

/* No counterpart in the reference.  Momentum-exchange force (same definition
 * as eup_get_forces) of a state that lives in the CALLER's device memory, for
 * callers that cannot let a library allocate: e.g. a Fortran driver whose
 * a01..a19 and obs are already device-resident under its own OpenACC data
 * region and whose runtime owns the device memory, or a code with a fixed
 * device-memory budget handed out by its own allocator, where an extra
 * cudaMalloc would fail or stall the device.  Needs no handle and allocates nothing: its
 * scratch is one fixed device array in the library (one FP64 partial per
 * z-plane, at most 4096 planes, about 96 KiB per GPU, held until the process
 * exits); lz > 4096 is rejected with EUP_ERR_UNSUPPORTED.
 *   pops[19]  device pointers to the haloed arrays a01..a19(0:l+1,0:m+1,0:n+1),
 *             float (elem_bytes 4) or double (8);
 *   obs       device pointer to obs(1:l,1:m,1:n), 1 = solid;
 *   bc[6]     reference face flags (axes with both faces periodic wrap);
 *   force     device pointer receiving 3 doubles;
 *   stream    cudaStream_t to run on (NULL: the legacy default stream).
 * Asynchronous on `stream`.  Every call looks up the scratch address on the
 * current device (cudaGetSymbolAddress), so it stays valid across a device
 * reset.  The CUDA runtime loads device code lazily by default, so the
 * scratch comes into being on a device at the first call there: a caller with
 * a fixed device-memory budget makes one call before its allocator takes the
 * budget, and makes that first call before any stream capture.  All calls
 * share the scratch: calls that overlap on the GPU race. */
int eup_mem_force_noalloc(int32_t l, int32_t m, int32_t n, const int32_t bc[6], const void* const pops[19],
                          int32_t elem_bytes, const int32_t* obs, double* force, void* stream);

/* ---- x-slab decomposition (one GPU per slab) ----------------------------- */
/* The time step in two halves for a lattice that is one x-slab of a larger
 * one: eup_step_boundaries enqueues the bounce-back (with the force of the
 * current state) and the halo planes; the caller then moves the x-face planes
 * between neighbouring slabs (eup_get_x_planes / eup_set_x_planes, e.g. NCCL
 * send/recv on the handle's stream); eup_step_stream enqueues stream-collide
 * and advances the step.  Faces flagged EUP_BC_EXCHANGE get no halo kernel.
 * With the planes exchanged after the halo kernels (their y/z halo rows
 * included), an FP32 or FP64 run split into slabs equals the single-lattice
 * run bit for bit (16-bit storage: to FP32 rounding of f, the halo's type),
 * provided no solid voxel lies on a column next to an exchange face
 * (eup_set_obstacles rejects that: its bounce-back would read the
 * neighbour's state of the previous step).  Replaces the x part of
 * CODE/SRC/bcond.comm.packed.F90:203-286, which exchanges before bcond_bc and
 * so lags the halo rows by one step. */
int eup_step_boundaries(eup_handle* h);
int eup_step_stream(eup_handle* h);

/* eup_step_stream in two parts, so that the plane exchange can overlap compute:
 * eup_step_stream_interior streams and collides every column that does not pull
 * from the x halo planes (x = 2..l-1) and may be enqueued right after
 * eup_get_x_planes, before the planes arrive; eup_step_stream_faces, after
 * eup_set_x_planes, does the columns x = 1 and x = l and advances the step.  Same
 * bits as eup_step_stream.  No reference counterpart (the reference exchanges with
 * blocking MPI calls before its step, CODE/SRC/bcond.comm.packed.F90). */
int eup_step_stream_interior(eup_handle* h);
int eup_step_stream_faces(eup_handle* h);

/* The five populations that cross an x face, (m+2)(n+2) values each, index
 * (q', j + (m+2) k) for j = 0..m+1, k = 0..n+1, in the arithmetic type (float,
 * or double for FP64), device pointers.  side 0: column x = 1, populations
 * a10..a14 (heading to -x), for the left neighbour's x = l+1 plane; side 1:
 * column x = l, a01..a05 (heading to +x), for the right neighbour's x = 0
 * plane.  Enqueued on the handle's stream after eup_step_boundaries. */
int eup_get_x_planes(eup_handle* h, int32_t side, void* dst);
/* Writes received planes into the halo: side 0 fills x = 0 with a01..a05 (from
 * the left neighbour's side 1), side 1 fills x = l+1 with a10..a14. */
int eup_set_x_planes(eup_handle* h, int32_t side, const void* src);

/* The same plane message with no pack kernel: *dev receives a device pointer
 * into the handle's own x-face copy, where the stream-collide kernel's
 * epilogue writes the face columns' populations as it produces them (and the
 * bounce-back keeps them in step) and eup_step_boundaries adds the halo rows
 * after its halo kernels.  5 (m+2)(n+2) values in the arithmetic type, in two
 * parts: the blocks, the five populations on rows j = 1..m, k = 1..n
 * ((q', (j-1) + m (k-1))); and the rim, per population the halo rows k = 0 and
 * k = n+1 (j = 0..m+1), then j = 0 and j = m+1 (k = 1..n).  Side 1 (x = l,
 * a01..a05) holds the blocks then the rim, side 0 (x = 1, a10..a14) the rim
 * then the blocks.  Valid, and to be sent, between eup_step_boundaries and the
 * next eup_step_stream / eup_step_stream_faces, which overwrites it; the
 * pointer itself is fixed for the handle's life.  Only for an exchange face.
 * Replaces the pack of CODE/SRC/bcond.comm.packed.F90:60-62 for x. */
int eup_get_x_planes_view(eup_handle* h, int32_t side, const void** dev);
/* Writes a message from the neighbour's opposite side, in that side's order,
 * into the x = 0 (side 0) or x = l+1 (side 1) halo plane, like
 * eup_set_x_planes. */
int eup_set_x_planes_view(eup_handle* h, int32_t side, const void* src);

/* ---- partial bounce-back and its adjoint ----------------------------------- */
/* No counterpart in the reference (its solids are all-or-nothing voxels).  A
 * solid fraction n_s(1:l,1:m,1:n) in [0,1] switches the handle to the
 * partial-bounce-back collision of Walsh, Burwinkle & Saar (2009),
 * f*_i = (1-n_s) BGK_i(f) + n_s f_opp(i), whose drag is sum 2 n_s j_x; the force
 * of every step is recorded like eup_get_forces'.  Any storage (16-bit
 * deviations mix as D*_i = (1-n_s) D_i + n_s D_opp(i), since w_i = w_opp(i)), no
 * obstacles.  NULL switches the field off. */
int eup_set_solid_fraction(eup_handle* h, const double* ns);

typedef struct eup_adjoint_config {
    int32_t nsteps;       /* forward steps T from the current state */
    int32_t avg_steps;    /* objective: mean C_d over the last avg_steps steps (at most the
                             handle's force history, eup_config.series_capacity) */
    int32_t checkpoints;  /* stored states (snapshot slots); 0 selects 64 */
    int32_t reserved;
} eup_adjoint_config;

/* Runs T partial-bounce-back steps from the current state and the discrete
 * adjoint back to it: *objective = mean C_d over the last avg_steps steps,
 * grad_ns[l*m*n] = d objective / d n_s per voxel (FP64, Fortran order).
 * Binomial checkpointing (Griewank 1992; Griewank & Walther 2000): with c =
 * checkpoints stored states the reverse sweep recomputes the fewest forward
 * steps possible, t(T, c) - (T - 1) beyond the forward sweep, where t(n, c) =
 * r n - C(c + r, r - 1) and r is the smallest repetition number with
 * C(c + r, c) >= n; device memory is c + 4 states.  Leaves the handle at step
 * itime + T.  stats (may be NULL): forward ms, reverse ms (recomputation +
 * adjoint), recomputed steps, stored states c, repetition number r, device
 * bytes of the states, T, avg_steps. */
int eup_adjoint_run(eup_handle* h, const eup_adjoint_config* cfg, double* objective, double* grad_ns,
                    double stats[8]);

/* No counterpart in the reference.  The checkpoint schedule eup_adjoint_run
 * would follow for nsteps steps and `checkpoints` stored states (0 selects 64),
 * built on the host without a GPU, to size the budget before a run:
 * *forward_steps = forward steps of the whole schedule, t(nsteps, c) (the
 * forward sweep's first nsteps-1 included), *recomputed = those of the reverse
 * sweep (eup_adjoint_run's stats[2]), *repetitions = r. */
int eup_adjoint_plan(int32_t nsteps, int32_t checkpoints, int64_t* forward_steps, int64_t* recomputed,
                     int32_t* repetitions);

/* ---- host utilities (no GPU) ---------------------------------------------- */

/* Reads obs.RRRR.TTTTTTTT.bin (CODE/SRC/build.obs.F90:147-177): Fortran
 * unformatted sequential, record 1 = nobs, then nobs records of (i,j,k).
 * Fills obs(1:l,1:m,1:n) with 0/1; *nobs receives the count. */
int eup_read_obs_file(const char* path, int32_t l, int32_t m, int32_t n, int32_t* obs,
                      int64_t* nobs);

/* Writes obs in the same format (CODE/SRC/build.obs.F90:506-541). */
int eup_write_obs_file(const char* path, int32_t l, int32_t m, int32_t n, const int32_t* obs);

/* Reads restore.XX.YY.ZZ.bin / save.*.bin (CODE/SRC/restore_raw.F90:43-63,
 * CODE/SRC/save_raw.F90:54-74): record 1 = itime, then 19 records of the
 * haloed arrays. */
int eup_read_raw_state(const char* path, int32_t l, int32_t m, int32_t n, int32_t elem_bytes,
                       void* const pops[19], int64_t* itime);

/* Writes the same format (CODE/SRC/save_raw.F90:54-74). */
int eup_write_raw_state(const char* path, int32_t l, int32_t m, int32_t n, int32_t elem_bytes,
                        const void* const pops[19], int64_t itime);

/* The initial states of CODE/SRC/init.F90:42-236 (init(opt), called with the
 * namelist's init_v): the equilibrium at rho = 1 of 0 rest, 1 Poiseuille
 * u_x = 0.1 (1 - z^2), 2 decaying shear u_x = u0 sin(2 pi z), 3 Kida vortices
 * u = 0.1 (sin 2pi x cos 2pi z, 0, -cos 2pi x sin 2pi z), over the haloed arrays,
 * with the reference's coordinates and constants (single-precision literals,
 * x scaled by lz; periodic != 0 selects the -DPERIODIC coordinates (k - 1/2)/lz).
 * global = (lx, ly, lz) of the whole lattice; start = mpicoords * (l, m, n) places
 * this block in it.  u0 is the one the reference holds after build_bcond (0 with an
 * inlet or a lid).  Options 4 and 5 stop the reference ("still to port") and return
 * EUP_ERR_UNSUPPORTED. */
int eup_init_reference(int32_t opt, int32_t l, int32_t m, int32_t n, const int32_t global[3],
                       const int32_t start[3], int32_t periodic, double u0, int32_t elem_bytes,
                       void* const pops[19]);

/* Equilibrium state of CODE/SRC/init.F90:194-232 with rho = 1 and
 * u = (u_in + amp*xi_x, amp*xi_y, amp*xi_z), xi uniform in [-1,1) from
 * splitmix64(seed + 3 L + c) (L haloed linear index, c the component), halos
 * included.  The synthetic workloads inject it through eup_upload the way the
 * reference restarts from restore.*.bin. */
int eup_init_equilibrium(int32_t l, int32_t m, int32_t n, double u_in, double amp, uint64_t seed,
                         int32_t elem_bytes, void* const pops[19]);

/* ---- synthetic geometries (no GPU) ---------------------------------------- */

/* The host voxeliser: obs(1:l,1:m,1:n) of shape g on this lattice (OpenMP).  The
 * same node tests as eup_build_obstacles, so the two masks are identical. */
int eup_voxelise(const eup_geometry* g, int32_t l, int32_t m, int32_t n, int32_t* obs);

/* Solid circular cylinder with axis along z: node (i,j,k) is solid when
 * (i-xc)^2 + (j-yc)^2 <= r^2 (1-based node coordinates). */
int eup_geometry_cylinder_z(int32_t l, int32_t m, int32_t n, double xc, double yc, double r,
                            int32_t* obs);

/* Reticular cylindrical shell with its axis along x (Euplectella-like
 * lattice): cylindrical struts of diameter strut_d on the shell of outer
 * diameter outer_d, a square grid of pitch `pitch` (longitudinal struts and
 * rings) plus both diagonals in alternate cells; the shell spans x0..x0+length
 * and is centred at (yc, zc).  seed sets the angular phase of the grid. */
int eup_geometry_reticular_shell(int32_t l, int32_t m, int32_t n, double x0, double length,
                                 double yc, double zc, double outer_d, double strut_d,
                                 double pitch, uint64_t seed, int32_t* obs);

/* Ridged lattice shell: the reticular shell above plus two counter-rotating
 * helical ridges at +-45 degrees (height ridge_h, width ridge_t) on its outer
 * surface and a porous cap (thickness cap_t, seeded circular pores of
 * diameter pore_d) closing its downstream end, as a solid fraction ns in
 * [0,1] (double, Fortran order).  With smooth_w > 0 the ridges' radial extent
 * is smoothed over smooth_w and dns_dh (may be NULL) receives d ns / d ridge_h,
 * the chain from a ridge-height parameter to the voxel field; with
 * smooth_w = 0 the field is 0/1 (ns >= 0.5 gives an obstacle mask). */
int eup_geometry_ridged_shell(int32_t l, int32_t m, int32_t n, double x0, double length, double yc, double zc,
                              double outer_d, double strut_d, double pitch, double ridge_h, double ridge_t,
                              double cap_t, double pore_d, double smooth_w, uint64_t seed, double* ns,
                              double* dns_dh);

#ifdef __cplusplus
}
#endif
#endif /* EUP_H */
