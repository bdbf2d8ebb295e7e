/*
 * scaletrack.h -- C ABI of the B200 Lagrangian parcel step (libscaletrack.so).
 *
 * The library replaces the parcel step that SCALE-TRACK's icoFoam coupling calls once per
 * fluid time step: cell-value fluid velocity lookup at each parcel, drag plus time
 * integration, relocation into the owning cell with wall bounce, and the two-way momentum
 * source deposited back to the cells.  Exchange arrays keep the reference layout: cell
 * velocity U in, per-cell momentum source out, both cell-major [nCells][3].
 *
 * Reference files cited below:
 *   A: run/icoJuliaParcelFoam/cavity3D/asyncParallelTracking.jl
 *   F: sol/icoJuliaParcelFoam/  (the C++ side of the coupling)
 *
 * Conventions: every function returns an int status (ST_OK = 0) unless stated otherwise;
 * st_last_error() returns a thread-local message for the last failure on the calling
 * thread.  Host pointers are plain host memory (pageable or pinned); "_device" entry points
 * take device pointers.  No CUDA types appear in the signatures: a stream is passed as
 * void* holding a cudaStream_t.  Cell indices are 0-based (the reference's posI - 1).
 */
#ifndef SCALETRACK_H
#define SCALETRACK_H

#include <stdint.h>

#if defined(__GNUC__)
#define ST_API __attribute__((visibility("default")))
#else
#define ST_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------- */
enum {
    ST_OK = 0,
    ST_ERR_INVALID_ARGUMENT = 1, /* bad size, pointer, name or parameter                    */
    ST_ERR_CUDA = 2,             /* a CUDA runtime call failed (message has the CUDA error) */
    ST_ERR_PARCEL_OUTSIDE = 3,   /* a parcel could not be located inside the mesh           */
    ST_ERR_SOURCE_RANGE = 4,     /* a deposit exceeded the deterministic fixed-point range  */
    ST_ERR_NOT_INITIALISED = 5,  /* shim called before st_setup                             */
    ST_ERR_OUT_OF_MEMORY = 6
};

/* ---- models and modes ---------------------------------------------------------------- */
enum {
    ST_DRAG_STOKES_IMPLICIT = 0, /* f = 18 mu dt/(rho_d d^2); v' = (v + f u)/(1 + f): A:1294-1295 */
    ST_DRAG_SCHILLER_NAUMANN = 1 /* v' = v + f (1 + 0.15 Re^0.687)(u - v), explicit Euler       */
};
enum {
    ST_PREC_FP32 = 0,  /* all single precision: the reference's arithmetic (A:172)   */
    ST_PREC_MIXED = 1, /* FP64 positions and cell location, FP32 drag and velocity   */
    ST_PREC_FP64 = 2   /* all double precision                                        */
};
enum {
    ST_DEPOSIT_DETERMINISTIC = 0, /* warp-aggregated fixed-point sums: bitwise reproducible */
    ST_DEPOSIT_ATOMIC = 1         /* one FP64 atomicAdd per deposit (A:714-725 in FP64)     */
};

/* Uniform cuboid mesh, cells numbered x fastest (A:222-270, A:684-691). */
typedef struct st_mesh_desc {
    int32_t n[3];      /* cells per direction */
    double origin[3];  /* lower corner */
    double ending[3];  /* upper corner */
} st_mesh_desc;

typedef struct st_params {
    double mu_c;              /* carrier dynamic viscosity      (A: μᶜ)   */
    double rho_c;             /* carrier density                (A: ρᶜ)   */
    double rho_d;             /* parcel density                 (A: ρᵈ)   */
    int32_t drag_model;       /* ST_DRAG_*                                 */
    int32_t precision;        /* ST_PREC_*                                 */
    int32_t deposit;          /* ST_DEPOSIT_*                              */
    int32_t n_substeps;       /* substeps per call; 10 in the reference (A:1260) */
    int32_t sort_interval;    /* Morton re-sort of the parcels every k steps; 0 = never */
    int32_t n_clouds;         /* independent parcel clouds, each with its own source field */
    int32_t block_size;       /* threads per block of the step kernel; 0 = default (256) */
    int32_t grid_blocks;      /* blocks of the step kernel; 0 = from occupancy x SM count */
    double drag_multiplier;   /* multiplies the drag factor; 1 reproduces the reference */
    double diameter_scale;    /* multiplies every diameter;  1 reproduces the reference */
} st_params;

typedef struct st_handle st_handle;

/* Library version, e.g. "scaletrack-b200 0.1 sm_100a". */
ST_API const char* st_version(void);
/* Thread-local message describing the last failure on this thread ("" if none). */
ST_API const char* st_last_error(void);

/* Defaults: the reference's physics (setup.jl: mu_c 1e-3, rho_c 1e3, rho_d 1), Stokes
 * implicit drag, FP32, deterministic deposit, 10 substeps, one cloud, no re-sort. */
ST_API void st_params_default(st_params* p);

/* Creates a handle on CUDA device `device`.  Allocates the per-cell arrays (U, source,
 * fixed-point accumulators) and a stream.  Replaces the Julia-side set-up of Mesh,
 * TwoWayEulerian and the device arrays (A:1560-1620, A:934-964). */
ST_API int st_create(const st_params* p, const st_mesh_desc* mesh, int device, st_handle** out);
ST_API int st_destroy(st_handle* h);

/* Parcels of cloud `cloud` (0 <= cloud < n_clouds), SoA host arrays: xyz = [3][n]
 * (x block, y block, z block), uvw = [3][n], d = [n].  Values are converted to the handle's
 * precision.  Every parcel must lie inside the mesh (else ST_ERR_PARCEL_OUTSIDE).  Replaces
 * allocate!/initWithHilbert! (A:474-482, A:559-638) with caller-provided parcels. */
ST_API int st_set_parcels(st_handle* h, int cloud, int64_t n, const double* xyz, const double* uvw,
                   const double* d);
/* n parcels of cloud `cloud` generated on the device, clustered along a Hilbert curve as
 * the reference's initWithHilbert! (A:559-638): the cloud takes its own segment of a 1024^3
 * Hilbert curve, each parcel a random point of the cell its curve point selects, velocity
 * zero, diameter uniform in [d_min, d_max).  Counter-based random numbers: the same seed
 * gives the same parcels on any GPU and in the CPU oracle. */
ST_API int st_init_parcels(st_handle* h, int cloud, int64_t n, uint64_t seed, double d_min,
                           double d_max);
/* Injection: m more parcels (same SoA layout as st_set_parcels) appended to a cloud of a
 * cuboid mesh, in place on the device; they take the order positions n .. n+m-1.  The next
 * step re-derives the fixed-point scale.  The reference injects only at start-up. */
ST_API int st_append_parcels(st_handle* h, int cloud, int64_t m, const double* xyz,
                             const double* uvw, const double* d);
/* Current parcel state in the order given to st_set_parcels (re-sorting is undone). */
ST_API int st_get_parcels(st_handle* h, int cloud, double* xyz, double* uvw, double* d);
/* 0-based owning cell of each parcel (locate, A:680-693), order as st_set_parcels. */
ST_API int st_get_cells(st_handle* h, int cloud, int32_t* cells);
/* A sample of one cloud's parcels by their st_set_parcels index (ids[m], each in [0, n)):
 * positions and velocities as FP64 [3][m] each, and the owning cell [m] (tet meshes: the
 * tracked tet; cuboid meshes: the located cell, -1 outside).  Any output may be NULL.
 * Copies 56 bytes per sampled parcel instead of the whole cloud; synchronises the stream.
 * No counterpart in the reference. */
ST_API int st_get_parcel_sample(st_handle* h, int cloud, int64_t m, const int32_t* ids,
                                double* xyz, double* uvw, int32_t* cells);
/* Device-side order of a cloud: ids[k] = index (in the order given to st_set_parcels) of the
 * parcel stored at position k of the device arrays, which the periodic re-sort groups by
 * owning cell.  Diagnostic; no counterpart in the reference. */
ST_API int st_get_order(st_handle* h, int cloud, int32_t* ids);
ST_API int64_t st_num_parcels(st_handle* h, int cloud);
ST_API int64_t st_num_cells(st_handle* h);

/* Cell velocity U, [nCells][3] with 4- or 8-byte components (host or device memory).
 * Replaces copyto!(deviceEulerian.U, eulerian.U) (A:1079-1083). */
ST_API int st_set_fluid_velocity(st_handle* h, const void* U, int elem_bytes);
ST_API int st_set_fluid_velocity_device(st_handle* h, const void* U, int elem_bytes);

/* One call of the parcel step for every cloud: n_substeps substeps of dt/n_substeps
 * (evolve_on_device!, A:1258-1365), fluid velocity U scaled by fluid_scale, followed by the
 * source reduction.  Asynchronous on the handle's stream.  Errors found on the device
 * (lost parcels, fixed-point range) are reported by the next st_synchronize,
 * st_get_source, st_get_parcels or st_get_cells. */
ST_API int st_step(st_handle* h, double dt, double fluid_scale);

/* Per-cell momentum source of the last step for `cloud`, [nCells][3], 4- or 8-byte
 * components: the sum over deposits of (rho_d/rho_c)(pi d^3/6)(state0 - v) (A:703-725),
 * not divided by the cell volume or dt, exactly as the reference's UTrans.  Synchronous. */
ST_API int st_get_source(st_handle* h, int cloud, void* S, int elem_bytes);
/* Device pointer to the FP64 source [nCells][3] of `cloud`, valid until st_destroy.  The
 * call orders the handle's stream after the computation of the last step's source (see
 * st_set_finalize_overlap): work enqueued on that stream afterwards reads it complete. */
ST_API const double* st_source_device(st_handle* h, int cloud);

/* Waits for the handle's stream and reports device-side errors. */
ST_API int st_synchronize(st_handle* h);
/* The handle's cudaStream_t, and a way to run on a caller-owned stream instead. */
ST_API void* st_get_stream(st_handle* h);
ST_API int st_set_stream(st_handle* h, void* stream);

/* ---- unstructured tetrahedral meshes (no counterpart in the reference) -------------- */
/* A conforming tet mesh filling the box [origin, ending] (planar walls).  Face f of a tet is
 * the face opposite its local vertex f; neighbors[4t + f] is the tet across it, or -1 on the
 * boundary.  Parcels carry their owning tet; after each position update a greedy walk moves
 * across the face with the largest positive signed distance (planes in FP64 from the face's
 * vertices taken in increasing id order, ties to the face opposite the smaller vertex id)
 * until the position is inside.  A position outside the box keeps its old
 * coordinate on that axis and mirrors the old velocity component, as on cuboid meshes
 * (A:1313-1329).  Deposits go to the tet of the last velocity sample.  Mixed and FP64
 * precision only (positions in FP64). */
typedef struct st_tet_mesh_desc {
    int64_t n_vertices;
    const double* vertices;    /* [n_vertices][3] (host) */
    int64_t n_tets;
    const int32_t* tets;       /* [n_tets][4] vertex ids (host) */
    const int32_t* neighbors;  /* [n_tets][4] tet across face f, -1 on the boundary (host) */
    double origin[3];          /* box walls */
    double ending[3];
    int32_t hop_limit;         /* walk hops per substep before a parcel counts as lost; 0 = 64 */
    int32_t pad;
} st_tet_mesh_desc;
/* Like st_create for a tet mesh; cells are tets (st_num_cells = n_tets, U and the source
 * are [n_tets][3]).  The mesh arrays are copied to the device. */
ST_API int st_create_tet(const st_params* p, const st_tet_mesh_desc* mesh, int device,
                         st_handle** out);
/* Like st_set_parcels, with a starting tet per parcel (`hint`, [n], may be NULL for tet 0)
 * from which the walk looks for the owning tet.  st_set_parcels on a tet handle walks from
 * tet 0. */
ST_API int st_set_parcels_tet(st_handle* h, int cloud, int64_t n, const double* xyz,
                              const double* uvw, const double* d, const int32_t* hint);
/* Walk lengths of every substep since the last reset: out[k] = substeps whose walk took k
 * hops (k < 7), out[7] = 7 or more.  Synchronises the stream. */
ST_API int st_tet_hop_histogram(st_handle* h, uint64_t out[8], int reset);

/* ---- output and restart -------------------------------------------------------------- */
/* ParaView dump of one cloud (the reference's write, A:1367-1430): a VTK XML
 * UnstructuredGrid file with one vertex per parcel, point data "U" (velocity) and "d"
 * (diameter), FP64, appended raw binary; parcels in the order of st_set_parcels. */
ST_API int st_write_vtu(st_handle* h, int cloud, const char* path);
/* ParaView collection (.pvd) listing n dumps with their times (A:1414-1430). */
ST_API int st_write_pvd(const char* path, int n, const double* times, const char* const* files);
/* Restart file of the whole handle: every cloud's parcels (and owning tets on tet meshes),
 * the fixed-point scale of the next step and the step bookkeeping.  Loading it into a handle
 * created with the same parameters and mesh continues the run bit for bit (after the same
 * fluid velocity is set).  No counterpart in the reference, which has no restart. */
ST_API int st_save_state(st_handle* h, const char* path);
ST_API int st_load_state(st_handle* h, const char* path);

/* ---- CUDA-graph replay and autotuning ---------------------------------------------- */
/* Captures n_steps calls of st_step (dt, fluid_scale[k] or 1) into a CUDA graph on the
 * handle's stream; st_graph_launch replays them (asynchronously), which removes the host
 * launch cost of a multi-cloud step sequence.  With re-sorting on, capture right after set-up
 * or a re-sort and a multiple of 2 x sort_interval steps, so every replay starts from the same
 * buffers.  st_set_parcels and st_autotune release the graph. */
ST_API int st_graph_capture(st_handle* h, int n_steps, double dt, const double* fluid_scale);
ST_API int st_graph_launch(st_handle* h);
ST_API int st_graph_release(st_handle* h);

typedef struct st_tune_result {
    int32_t block_size;   /* threads per block of the step kernel */
    int32_t grid_blocks;  /* persistent grid: SMs x resident blocks at that size */
    int32_t sort_interval;
    int32_t pad;
    double ms_per_step;   /* measured, including the amortised re-sort */
} st_tune_result;
/* Times trial_steps steps for every block size in {128, 256} and re-sort interval in
 * {never, 10, 20, 40} on a copy of the handle (the caller's parcels do not advance) and keeps
 * the fastest.  The results of a step do not depend on either choice: parcel order never
 * changes positions, velocities or the fixed-point source. */
ST_API int st_autotune(st_handle* h, double dt, int trial_steps, st_tune_result* out);

/* Step kernel of a handle with one cloud (cuboid or tet mesh).  ST_STEP_KERNEL_RING (the
 * default): a persistent block per SM streams block tiles of 1024 parcels through a
 * shared-memory ring with bulk copies.  ST_STEP_KERNEL_WARP: every warp loads and steps its
 * own 32 parcels.  Both give bit-identical positions, velocities, cells, sources and walk
 * lengths; handles with several clouds, and the first (probe) pass of a run, always use the
 * warp kernel.  No counterpart in the
 * reference (one kernel, A:1258-1269). */
enum { ST_STEP_KERNEL_RING = 0, ST_STEP_KERNEL_WARP = 1 };
ST_API int st_set_step_kernel(st_handle* h, int kind);
/* With one cloud and the deterministic deposit, a step's conversion of the fixed-point sums
 * to the FP64 source (and the clearing of its accumulator) runs on a second stream of the
 * library, concurrent with the next step on the handle's stream; the two steps use two
 * accumulators in turn.  st_get_source, st_synchronize and st_source_device order the
 * handle's stream after it, so work the caller enqueues on that stream afterwards sees the
 * source.  on = 0 runs the conversion in the handle's stream after each step instead (as
 * graph capture, several clouds, tet meshes, the sharded phases and the coupling shims always
 * do).  Results do not depend on the choice.  Default: on. */
ST_API int st_set_finalize_overlap(st_handle* h, int on);
/* Failure detection of the ring step kernels: every wait of their shared-memory pipeline
 * (on a copy into a stage, or on the consumers releasing it) gives up after `cycles` SM clock
 * cycles, records the fault in the cloud's control block and lets the kernel drain and exit;
 * the next st_synchronize (or other synchronous call) then returns ST_ERR_CUDA, and that
 * step's parcels and source are incomplete (set the parcels again).  cycles = 0: the default
 * of about one second, far above any wait of a correct run.  stall != 0 (with cycles > 0)
 * tests this path: the consumer warps of every ring block first wait on a barrier that
 * nothing completes, give up after `cycles`, and the block drains (its own copies in flight
 * are always waited for, with the default limit, before it exits).  stall = 0 ends the test.
 * No counterpart in the reference (its kernels have no such waits). */
ST_API int st_set_wait_limit(st_handle* h, int64_t cycles, int stall);

/* ---- instrumentation --------------------------------------------------------------- */
enum { ST_KERNEL_STEP = 0, ST_KERNEL_FINALIZE = 1, ST_KERNEL_SORT = 2, ST_KERNEL_PROBE = 3,
       ST_KERNEL_OTHER = 4, ST_KERNEL_ADJ_FORWARD = 5, ST_KERNEL_ADJ_REVERSE = 6,
       ST_KERNEL_KINDS = 7 };
/* Record CUDA events around every kernel the library launches (on the launching stream). */
ST_API int st_profile_enable(st_handle* h, int on);
/* Launch count and summed device time (ms) of one kernel kind since the last reset;
 * synchronises the stream.  reset != 0 clears the counters afterwards. */
ST_API int st_profile_read(st_handle* h, int kind, int64_t* launches, double* ms, int reset);
/* Total number of kernels the library launched on this handle. */
ST_API int64_t st_launch_count(st_handle* h);

/* ---- adjoint of the time-averaged source (no counterpart in the reference) ---------- */
/* The differentiable map is Sbar = (1/T) sum_{n<T} S_n over T steps of one cloud starting
 * from its current state (which is not modified), Schiller-Naumann drag, one substep,
 * mixed or FP64 precision.  Cell ownership and wall-bounce decisions are frozen at the
 * forward pass.  This is the backend of a Julia ChainRules rrule: the forward call is the
 * primal, the pull-back call the backward closure. */
typedef struct st_adjoint_desc {
    int32_t n_steps;             /* T >= 1 */
    int32_t checkpoint_interval; /* C >= 1: (x, v) is stored every C steps and the C steps
                                    after a checkpoint are recomputed in the pull-back */
    double dt;                   /* time step (one substep) */
    const double* fluid_scale;   /* [T] factor on U per step (host), or NULL for 1 */
} st_adjoint_desc;
/* Runs the forward pass, keeps its checkpoints in the handle and writes Sbar (host
 * [nCells][3], FP64, deterministic fixed-point reduction with one scale for the run). */
ST_API int st_mean_source_forward(st_handle* h, int cloud, const st_adjoint_desc* desc,
                                  double* mean_source);
/* Pull-back of the last st_mean_source_forward with the same desc: given the cotangent
 * dJ/dSbar (host [nCells][3]) returns dJ/d(drag_multiplier), dJ/d(diameter_scale) and
 * dJ/dv0 (host [3][n], order of st_set_parcels; may be NULL).  Velocity cotangents are in
 * the velocity precision, parameter sums in FP64 (reproducible reduction order). */
ST_API int st_mean_source_pullback(st_handle* h, int cloud, const st_adjoint_desc* desc,
                                   const double* cotangent, double* d_drag_multiplier,
                                   double* d_diameter_scale, double* d_velocity0);

/* Sets the drag multiplier and the diameter scale of an existing handle (the st_params
 * fields of the same names), so that the parameters of the adjoint above can be arguments of
 * the differentiated function.  Takes effect at the next step or forward pass; invalidates
 * the last st_mean_source_forward.  Both must be finite and > 0. */
ST_API int st_set_drag_parameters(st_handle* h, double drag_multiplier, double diameter_scale);

/* ---- sharded steps: one cloud split over ranks (one handle per rank or GPU) ---------- */
/* The reference sums the per-rank sources over MPI (asyncParallelTracking.jl:1156-1183);
 * here the ranks combine the fixed-point accumulators before they are converted, so the
 * source is bit-identical to one handle stepping every parcel, for any split and any
 * reduction order (integer sums are exact).  Per step, on every rank:
 *   if st_shard_needs_probe(h, dt):  st_shard_probe(h, dt, fs); max-reduce the exponents
 *   st_shard_deposit(h, dt, fs);     sum-reduce the accumulators, max-reduce the exponents
 *   st_shard_finish(h);              the source (identical on every rank), next scale
 * The reductions act on the device buffers of st_shard_buffers (int64 accumulators, int32
 * exponents) and must be ordered on the handle's stream (e.g. NCCL all-reduce on it).
 * st_shard_set_total gives the parcel count of the cloud over all ranks, so that every rank
 * uses the same fixed-point headroom; it needs the deterministic deposit.  No counterpart in
 * the reference's one-GPU path. */
ST_API int st_shard_set_total(st_handle* h, int cloud, int64_t n_parcels_all_ranks);
ST_API int st_shard_buffers(st_handle* h, void** accumulators, int64_t* n_accumulators,
                            int32_t** exponents, int32_t* n_exponents);
/* 1 when the next step at this dt needs the probe phase, 0 when not, < 0 on error. */
ST_API int st_shard_needs_probe(st_handle* h, double dt);
ST_API int st_shard_probe(st_handle* h, double dt, double fluid_scale);
ST_API int st_shard_deposit(st_handle* h, double dt, double fluid_scale);
ST_API int st_shard_finish(st_handle* h);

/* ---- shims with the reference's names and semantics -------------------------------- */
/* Creates (or replaces) the process-wide default handle used by the two calls below, on
 * the current CUDA device; then st_default_handle() gives it to st_set_parcels & co. */
ST_API int st_setup(const st_params* p, const st_mesh_desc* mesh);
ST_API st_handle* st_default_handle(void);
/* allocate_array_ptr (A:1436-1483; called from F/juliaWrapper.H:129-141): returns library
 * owned, pinned host storage [size][nComponents] for "U" or "UTrans" that the caller
 * adopts as its field storage.  typeByteSize is 4 or 8, size must equal the cell count and
 * nComponents must be 3; otherwise NULL (the reference throws).  Repeated calls with the
 * same name return the same pointer while the size and type agree. */
ST_API void* st_allocate_array(const char* name, int size, int nComponents, int typeByteSize);
/* evolve_cloud (A:1485-1528; called at F/icoJuliaParcelFoam.C:123): copies the adopted
 * "U" to the device, runs st_step(dt, 1) on the default handle and writes the source of
 * cloud 0 into the adopted "UTrans" before returning (the synchronous variant of the
 * reference's coupling, syncSerialTracking.jl:547-567). */
ST_API int st_evolve_cloud(double dt);
/* The reference's asynchronous coupling (A:1062-1190 with its ConstExtrapolator, A:300-316,
 * A:742-747): call k takes U_k (the caller may overwrite it on return) and leaves in UTrans
 * the estimate est_k = 2 S_{k-1} - est_{k-1} (est_0 = 0, carried in FP64), where S_{k-1} is
 * the true source of the step the previous call launched; step k runs on the GPU while the
 * caller solves the next fluid step, and its source feeds the next call's estimate.  Device
 * errors of a step are reported by the call after it.  Do not mix with st_evolve_cloud
 * between st_setup and st_finalize. */
ST_API int st_evolve_cloud_async(double dt);
/* How st_evolve_cloud moves U and UTrans.  The arrays of st_allocate_array are pinned host
 * pages mapped into the device's address space.  ST_EXCHANGE_COPY (default): DMA copies
 * (plus a conversion pass on the device when the element size differs from the handle's
 * precision).  ST_EXCHANGE_MAPPED: zero copy, the library's kernels read U from and write
 * the source to those pages directly (F/juliaWrapper.H:105-172 with device-visible storage;
 * no counterpart in the reference, which copies, A:1081, A:1149-1152). */
enum { ST_EXCHANGE_COPY = 0, ST_EXCHANGE_MAPPED = 1 };
ST_API int st_set_exchange_mode(int mode);
/* Releases the default handle and the adopted arrays (F/juliaWrapper.C:33-50 detaches
 * the caller's fields first). */
ST_API int st_finalize(void);

/* ---- allocation-free step (no counterpart in the reference) ------------------------- */
/* Largest mesh (cells) that st_step_noalloc accepts: the size of its fixed device scratch
 * array, 3 x 8 bytes per cell (6 MiB), which every GPU that loads the library holds until
 * the process exits. */
#define ST_NOALLOC_MAX_CELLS 262144
/* One call of the mixed-precision parcel step (ST_PREC_MIXED, deterministic deposit, one
 * cloud, Morton re-sort not applied) for callers that cannot allocate device memory: a
 * host that hands all device memory to its own pool, or a plugin that must not grow the
 * process's device footprint after set-up.  Every array is caller-owned device memory:
 * positions x,y,z (double[n]), velocities u,v,w and diameters d (float[n]), cell velocity
 * U (float[nCells][3]) and the output source (double[nCells][3]); the parcel state is
 * updated in place.  The only scratch (fixed-point accumulator and control block) is a
 * fixed-size device array inside the library; no cudaMalloc, cudaFree or allocating
 * library routine is called.  Meshes above ST_NOALLOC_MAX_CELLS cells are rejected with
 * ST_ERR_INVALID_ARGUMENT.  Runs on the current device and `stream` (a cudaStream_t, NULL
 * for the default stream) and returns after the stream has finished, with device-side
 * errors reported: it synchronises the stream, so it cannot be captured into a CUDA graph,
 * and a call on a capturing stream is rejected with ST_ERR_INVALID_ARGUMENT before anything
 * is launched.  The first call on a device looks up the scratch array's address and keeps
 * it for the life of the process: do not call it on a device after cudaDeviceReset.  All
 * calls share the one array: calls that overlap on the GPU race.  Each call chooses its
 * fixed-point scale from its own deposits, so the source agrees with st_step's to the
 * fixed-point resolution and positions and velocities are bit-identical. */
ST_API int st_step_noalloc(const st_params* p, const st_mesh_desc* mesh, int64_t n, double* x,
                           double* y, double* z, float* u, float* v, float* w, const float* d,
                           const float* U, double* source, double dt, double fluid_scale,
                           void* stream);
/* ST_NOALLOC_MAX_CELLS, for callers that bind the library at run time. */
ST_API int64_t st_noalloc_max_cells(void);

#ifdef __cplusplus
}
#endif

#endif /* SCALETRACK_H */
