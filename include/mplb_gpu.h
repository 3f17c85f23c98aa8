/*
 * mplb_gpu.h -- C-ABI of the B200 lattice update for multiphaseLB.
 *
 * The reference advances its lattice with a fixed sequence of C calls on
 * host structures (src/applications/solvers/multiPhasePP/multiPhasePP.c:157-240):
 *
 *     collision(f) lbstream(f) updateBoundaries(f)
 *     collision(g) lbstream(g) updateBoundaries(g)
 *     macroDensity  heatSource  macroTemperature  interForce  macroVelocity
 *
 * This header replaces that sequence with one device-resident handle.  The
 * reference's readers, dictionaries and writers stay on the host; the driver
 * packs what they produced into the plain descriptors below (flat arrays,
 * sizes, no pointers-to-rows, no CUDA or torch types) and calls
 * mplb_gpu_create once, mplb_gpu_step in its time loop, and
 * mplb_gpu_download at write steps.  include/mplb_gpu_reference.h does the
 * packing from the reference's own structs.
 *
 * Conventions
 *  - Every function returns 0 on success and a negative MPLB_E* code on
 *    failure; mplb_gpu_last_error() then describes the failure (per thread).
 *    The library never exits, aborts or traps; the reference's errorMsg()
 *    (src/basic/errorMsg.c:6-12, print + exit(1)) becomes a return code the
 *    driver may pass to errorMsg itself.
 *  - Host arrays use the reference's row-major layouts: PDFs [node][k]
 *    (lbeField.value, src/dataTypes/lbeField.h:53), vectors [node][3]
 *    (macroFields.U/Fi/Ft, src/dataTypes/macroFields.h:33-48), scalars [node].
 *  - Arithmetic is IEEE binary64, the reference's DP build
 *    (src/dataTypes/dataTypes.h:19-21).
 *  - A handle is bound to one device and one CUDA stream and is not
 *    thread-safe, like one reference MPI rank.
 */
#ifndef MPLB_GPU_H
#define MPLB_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPLB_ABI_VERSION 6  /* 2: mplb_field_desc.alpha_1/alpha_2, mplb_opts.rank; 3: mplb_gpu_copy_nodes;
                               4: mplb_info.tile_ms[16], MPLB_E_TIMEOUT;
                               5: mplb_batch_filter, mplb_batch_average, mplb_mlp_init_column(_mass);
                               6: mplb_gpu_set_owned, mplb_gpu_add_mirror, mplb_gpu_clear_mirrors */
#define MPLB_MAX_Q 15
#define MPLB_MAX_PATCHES 64

/* Lattice models; same order as DdQq (src/dataTypes/latticeInfo.h:21-24). */
enum { MPLB_D2Q9 = 0, MPLB_D3Q15 = 1 };

/* Collision models; same values as lbeModel (src/lbEquation/lbeModel.h:4-22). */
enum { MPLB_LIMRT = 0, MPLB_MYMRT = 1, MPLB_XUMRT = 2, MPLB_LITEMPMRT = 3, MPLB_NO_MODEL = -1 };

/* Equations of state; same values as eosType (src/EOS/EOSInfo.h:17-31). */
enum { MPLB_EOS_IDEAL = 0, MPLB_EOS_CS = 1, MPLB_EOS_PR = 2, MPLB_EOS_VDW = 3 };

/* Boundary types; same values as bdType (src/boundary/bdType.h:4-33). */
enum {
    MPLB_BC_BOUNCEBACK = 0, MPLB_BC_FIXEDT = 1, MPLB_BC_FIXEDRANDOMT = 2,
    MPLB_BC_FIXEDGRADT = 3, MPLB_BC_FIXEDU = 4, MPLB_BC_UHF = 5,
    MPLB_BC_FIXEDEOSP = 6, MPLB_BC_OUTFLOW = 7, MPLB_BC_PERIODIC = 8
};

/* Field selectors for the per-operator entry points. */
enum { MPLB_FIELD_F = 0, MPLB_FIELD_G = 1 };

/* Storage precision of the PDFs.  MPLB_FP32_DEV stores them in FP32 as
 * deviations from the rest state (f - w rho_ref, g - wg T_ref), collides in
 * FP32 and keeps the density / temperature sums, EOS, psi, force, heat source
 * and T, U, S in FP64; fused box path only; not bit-identical to the
 * reference (its error against FP64 is measured). */
enum { MPLB_FP64 = 0, MPLB_FP32_DEV = 1 };

/* Execution path. */
enum {
    MPLB_PATH_AUTO = 0,      /* fused box kernels when the mesh is a box, else operators */
    MPLB_PATH_OPERATORS = 1, /* one kernel per reference operator, neighbour-table driven */
    MPLB_PATH_FUSED = 2      /* fused box kernels; create fails if the mesh is not a box */
};

/* Error codes. */
enum {
    MPLB_OK = 0,
    MPLB_E_ARG = -1,         /* invalid argument or descriptor */
    MPLB_E_UNSUPPORTED = -2, /* model / boundary / option outside the path */
    MPLB_E_CUDA = -3,        /* CUDA runtime error */
    MPLB_E_STATE = -4,       /* call not valid in the handle's current state */
    MPLB_E_NONFINITE = -5,   /* NaN/Inf found by a check */
    MPLB_E_IO = -6,          /* a field file or its folder could not be made or written */
    MPLB_E_TIMEOUT = -7      /* a bounded wait inside a kernel ran out: the steps since the last
                                synchronising call are not valid (reported by mplb_gpu_sync and
                                mplb_gpu_download) */
};

/*
 * Mesh of the single GPU domain.  Replaces latticeMesh.mesh
 * (src/dataTypes/basicMesh.h:39-70) for one rank with no ghosts
 * (nPoints == nlocal).
 */
typedef struct mplb_mesh_desc {
    int32_t lattice;              /* MPLB_D2Q9 or MPLB_D3Q15 */
    uint32_t n_points;            /* number of nodes */
    const int32_t* nb;            /* [n_points][Q]: node at x - c_k (pull source), -1 = none */
    const int32_t* points;        /* [n_points][3] integer coordinates, or NULL */
    uint32_t n_patches;           /* boundary patches, in file order (basicBoundary.nbd) */
    const uint32_t* patch_count;  /* [n_patches] nodes per patch (nbdelem) */
    const uint32_t* patch_nodes;  /* concatenation of the patches' node lists (bdPoints) */
} mplb_mesh_desc;

/* Equation of state and body forces; replaces EOSInfo (src/EOS/EOSInfo.h:80-102). */
typedef struct mplb_eos_desc {
    int32_t type;   /* MPLB_EOS_* */
    double a, b;    /* a_cs|a_pr|a_vdw, b_cs|b_pr|b_vdw */
    double w;       /* w_pr (Peng-Robinson acentric factor) */
    double R, G, M, Cv;
    double g[3];    /* gravity */
    double fext[3]; /* constant external force, applied off-boundary only */
    double rho_0;   /* buoyancy reference density */
} mplb_eos_desc;

/*
 * One population field; replaces lbeField's model, constants, update flag
 * and boundary table (src/dataTypes/lbeField.h:49-108,
 * src/lbEquation/lbParameters.h:16-31).
 */
typedef struct mplb_field_desc {
    int32_t model;            /* MPLB_LIMRT, MPLB_XUMRT (flow); MPLB_LITEMPMRT, MPLB_MYMRT (thermal); MPLB_NO_MODEL */
    int32_t update;           /* 0 = frozen (reference --frozen / --nht) */
    double Lambda[MPLB_MAX_Q];
    double sigma;             /* liMRT / xuMRT force coefficient */
    int32_t surface_tension;  /* 1 = liMRT / xuMRT surface-tension term (liMRTSurfaceTension.c, xuMRTSurfaceTension.c); FP64 only */
    double kappa_st;
    const int32_t* bc_type;   /* [n_patches] MPLB_BC_* for this field */
    const double* bc_value;   /* [n_patches][3]: fixedT uses [0], fixedU uses [0..2]; fixedRandomT:
                                 [0] T, [1] perturbation in percent, [2] boundary updates still
                                 perturbed (psteps - localTStep, fixedRandomTParam.h); outflow: none */
    double alpha_1, alpha_2;  /* myMRT equilibrium constants (myMRTConstants.h) */
} mplb_field_desc;

typedef struct mplb_opts {
    int32_t precision;   /* MPLB_FP64 */
    int32_t path;        /* MPLB_PATH_* */
    int32_t device;      /* CUDA device ordinal; -1 = the calling thread's current device */
    void* stream;        /* cudaStream_t to launch on; NULL = a stream owned by the handle */
    uint32_t start_time; /* reference timeInfo.start: the time the first step leaves */
    int32_t tile_config; /* fused path: 0 = time the tile candidates on the first step and keep
                            the fastest; k > 0 = use candidate k-1; -1 = candidate 0, no timing */
    int32_t rank;        /* parallel.pid of this domain: fixedRandomT seeds rand() with it
                            (fixedRandomT.c:37) */
} mplb_opts;

/* What create decided; filled by mplb_gpu_info. */
typedef struct mplb_info {
    int32_t path;            /* MPLB_PATH_OPERATORS or MPLB_PATH_FUSED */
    int32_t box_dims[3];     /* box extents when the mesh is a box, else 0 */
    int32_t box_periodic[3]; /* 1 = axis wraps */
    int32_t bc_sequential;   /* 1 = boundary updates run in the reference's serial order */
    uint32_t current_time;   /* reference timeInfo.current */
    uint64_t device_bytes;   /* device memory held by the handle */
    uint64_t kernel_launches;/* kernels this handle has launched so far */
    int32_t tile_config;     /* fused path: candidate in use (0-based), -1 before the first step */
    float tile_ms[16];       /* fused path: autotuner time per candidate (ms per step), 0 = not timed,
                                -1 = the candidate does not take this lattice */
} mplb_info;

typedef struct mplb_gpu mplb_gpu_t;

const char* mplb_gpu_version(void);
const char* mplb_gpu_last_error(void);

/* Build the device lattice.  Fields start at zero; upload them next. */
int mplb_gpu_create(const mplb_mesh_desc* mesh, const mplb_eos_desc* eos,
                    const mplb_field_desc* f, const mplb_field_desc* g,
                    const mplb_opts* opts, mplb_gpu_t** out);
int mplb_gpu_destroy(mplb_gpu_t* h);
int mplb_gpu_info(mplb_gpu_t* h, mplb_info* info);

/* Host -> device.  Any pointer may be NULL (field left as is).
 * rho/T/S/p: [n]; U/Fi/Ft: [n][3]; f: [n][Q]; g: [n][Q]. */
int mplb_gpu_upload(mplb_gpu_t* h, const double* rho, const double* U, const double* T,
                    const double* f, const double* g, const double* S,
                    const double* Fi, const double* Ft);
/* Device -> host, same layouts; any pointer may be NULL. */
int mplb_gpu_download(mplb_gpu_t* h, double* rho, double* U, double* T,
                      double* Fi, double* Ft, double* S, double* f, double* g);

/* Reference start-up (multiPhasePP.c:122-147): equilibrium(f), equilibrium(g),
 * interForce, heatSource at time.current == start_time. */
int mplb_gpu_initialize(mplb_gpu_t* h);

/* Advance nsteps time steps, each exactly multiPhasePP.c:157-240 without the
 * write block.  The handle's state is the reference's state after every call. */
int mplb_gpu_step(mplb_gpu_t* h, uint32_t nsteps);

/* Per-operator entry points, same names and semantics as
 * src/lbEquation/general/generalLbe.h and src/lbEquation/pseudoPot/interForce.c.
 * Each honours the field's update flag like the reference does. */
int mplb_gpu_equilibrium(mplb_gpu_t* h, int32_t field);                 /* general/equilibrium.c:6-90 */
int mplb_gpu_collision(mplb_gpu_t* h, int32_t field);                   /* general/collision.c:6-67 */
int mplb_gpu_lbstream(mplb_gpu_t* h, int32_t field);                    /* general/lbstream.c:5-72 */
int mplb_gpu_update_boundaries(mplb_gpu_t* h, int32_t field);           /* general/updateBoundaries.c:6-75 */
int mplb_gpu_macro_density(mplb_gpu_t* h, uint32_t start, uint32_t end);    /* general/macroDensity.c:7-75 */
int mplb_gpu_macro_velocity(mplb_gpu_t* h, uint32_t start, uint32_t end);   /* general/macroVelocity.c:6-65 */
int mplb_gpu_macro_temperature(mplb_gpu_t* h, uint32_t start, uint32_t end);/* general/macroTemperature.c:7-68 */
int mplb_gpu_inter_force(mplb_gpu_t* h);                                /* pseudoPot/interForce.c:7-52 */
int mplb_gpu_heat_source(mplb_gpu_t* h);                                /* general/heatSource.c:7-202 */
/* Write-time pressure (multiPhasePP.c:264): macroPressure on the device
 * (general/macroPressure.c:8-69, liMRTPressure.c:6-253, xuMRTPressure.c:6-22),
 * then the field to the host ([n] doubles). */
int mplb_gpu_macro_pressure(mplb_gpu_t* h);
int mplb_gpu_download_pressure(mplb_gpu_t* h, double* p);

/* Write step without stalling the time loop (the driver's write block,
 * multiPhasePP.c:249-310, downloads synchronously).  mplb_gpu_snapshot
 * queues on the handle's stream: the reference state of the current step
 * (and, with MPLB_SNAP_PRESSURE, macroPressure), a device copy of rho, T, p
 * and U (and, with MPLB_SNAP_PDFS, f and g),
 * then starts its transfer to pinned host memory on a side stream and
 * returns; the caller can go on stepping while it crosses PCIe.
 * mplb_gpu_snapshot_wait waits for the last snapshot and copies it out in the
 * reference's layouts (rho, T, p [node], U [node][3]; any pointer may be NULL;
 * p needs MPLB_SNAP_PRESSURE).  A second snapshot before the wait replaces
 * the first.  The handle holds 6 n doubles (6 n + 2 Q n with MPLB_SNAP_PDFS)
 * on the device and as many pinned on the host from the first call until
 * destroy. */
enum {
    MPLB_SNAP_PRESSURE = 1,  /* also run macroPressure and keep p */
    MPLB_SNAP_PDFS = 2       /* also keep f and g ([node][Q] each) for the writer */
};
int mplb_gpu_snapshot(mplb_gpu_t* h, int32_t flags);
int mplb_gpu_snapshot_wait(mplb_gpu_t* h, double* rho, double* U, double* T, double* p);
/* Write the last snapshot as the driver's write block does
 * (multiPhasePP.c:289-301): rho, T, p (if taken), U (3 components), f and g
 * (if taken with MPLB_SNAP_PDFS), in that order, with mplb_write_*_field's
 * formats and folders, at the time the snapshot was taken.  The files are
 * written by a host thread that first waits for the snapshot's transfer, so
 * the call returns at once and stepping goes on.  mplb_gpu_snapshot_join
 * waits for that thread and returns the first error of the writes started
 * since the last join (MPLB_E_NONFINITE for a NaN field: the fields before it
 * are written, as in the reference).  A new snapshot, or destroy, waits for a
 * running writer first.  For pvtu the driver writes the mesh part
 * (writeMeshToVTK) before this call and writePvtuExtra after the join. */
int mplb_gpu_snapshot_write(mplb_gpu_t* h, const char* root, int32_t pid, int32_t format);
int mplb_gpu_snapshot_join(mplb_gpu_t* h);

/* Time and buoyancy reference density (timeInfo.current, EOSInfo.rho_0). */
int mplb_gpu_set_time(mplb_gpu_t* h, uint32_t current);
int mplb_gpu_set_rho0(mplb_gpu_t* h, double rho_0);
/* averageScalarField(rho) on the device (src/basic/averageScalarField.c:4-78):
 * 0 if the current rho_0 <= 0, else the mean density summed in node order.
 * The result is stored as the new rho_0 and returned in *rho_0. */
int mplb_gpu_average_rho0(mplb_gpu_t* h, double* rho_0);

/* Conservation checks: total mass sum(rho) and thermal energy sum(T) over all
 * nodes, FP64 warp-shuffle tree reduction (not the reference's summation order). */
int mplb_gpu_mass_energy(mplb_gpu_t* h, double* mass, double* energy);

/* Equilibrium and mass monitor without leaving the fused state (no rebuild
 * of the reference state, unlike mass_energy): node density = mass of the
 * current populations (FP64 sum; for MPLB_FP32_DEV the FP32 sum of
 * deviations + the reference density).  *max_drho: largest change of a node
 * density since the previous monitor call (0 when reset != 0 or at the first
 * call); *mass: sum over nodes in a fixed order (deterministic).  Either
 * pointer may be NULL.  Needs an updated flow field. */
int mplb_gpu_monitor(mplb_gpu_t* h, int32_t reset, double* max_drho, double* mass);

/* Step to equilibrium.  The reference's driver (src/applications/solvers/multiPhasePP/multiPhasePP.c)
 * runs a fixed number of steps; this runs whole intervals of check_interval
 * steps until max over nodes |rho(t) - rho(t - K)| / K < tol, or max_steps
 * (rounded up to a whole interval).  rho is monitored as by mplb_gpu_monitor,
 * one read pass per check.  *steps: steps taken; *rate: the last
 * max |drho/dt| (either may be NULL).  A non-finite density stops the run
 * with MPLB_E_NONFINITE (*steps and *rate = inf filled in).  FP32-deviation
 * form: the lattice's total momentum is reset to its starting value at every
 * check when the lattice is fully periodic without net body force.  Needs an
 * updated flow field. */
int mplb_gpu_run_to_equilibrium(mplb_gpu_t* h, uint32_t max_steps, uint32_t check_interval, double tol,
                                uint32_t* steps, double* rate);

/* Wait for the handle's stream. */
int mplb_gpu_sync(mplb_gpu_t* h);

/* Ghost-node exchange between lattices, on the devices.  Replaces the
 * reference's host-side exchanges of a multi-rank run (sendPdfField /
 * recvPdfField, src/basic/sendPdfField.c:6-102 and recvPdfField.c:6-54, for
 * f and g; syncScalarField.c and syncVectorField.c for S, Fi and Ft) when
 * the ranks' lattices are handles of this library, on one GPU or on several.
 * Copies nodes [src_start, src_start + count) of src into nodes
 * [dst_start, dst_start + count) of dst, for every field named in `fields`
 * (MPLB_NODES_* bits), in the reference state of both handles.  The copy is
 * queued on src's stream after all work already queued on dst's stream, and
 * dst's stream waits for it; the call does not block the host.  Between
 * devices the copy goes peer to peer (peer access is enabled on first use
 * where the devices allow it).  Both handles hold the same lattice in FP64;
 * on one handle the two ranges must not overlap. */
enum {
    MPLB_NODES_RHO = 1,
    MPLB_NODES_U = 2,
    MPLB_NODES_T = 4,
    MPLB_NODES_FI = 8,
    MPLB_NODES_FT = 16,
    MPLB_NODES_S = 32,
    MPLB_NODES_F = 64,
    MPLB_NODES_G = 128
};
int mplb_gpu_copy_nodes(mplb_gpu_t* dst, uint32_t dst_start, mplb_gpu_t* src, uint32_t src_start,
                        uint32_t count, int32_t fields);

/* Copy the fused-path state of nodes [src_start, src_start + count) of src
 * to [dst_start, dst_start + count) of dst: the post-collision populations
 * of every updated field (the input of the next fused step), and T and U of
 * the last step.  No counterpart in the reference; it is the halo exchange
 * of slabs run on the fused path (the reference's sendPdfField /
 * recvPdfField, src/lbEquation/general/sendPdfField.c:7-102 and
 * recvPdfField.c:7-54, move the post-stream PDFs of ghost nodes instead,
 * inside its operator sequence).  Both handles must be on the fused FP64
 * path with the same lattice and field options; a handle still in the
 * reference's state (after initialize) first takes the loop's first
 * collision, as mplb_gpu_step does.  Device to device, ordered on the
 * handles' streams as mplb_gpu_copy_nodes. */
int mplb_gpu_copy_state(mplb_gpu_t* dst, uint32_t dst_start, mplb_gpu_t* src, uint32_t src_start, uint32_t count);

/* Slabs on the fused path with the halo written by the step kernels
 * themselves.  No counterpart in the reference; they replace its
 * sendPdfField / recvPdfField exchange (src/lbEquation/general/
 * sendPdfField.c:7-102, recvPdfField.c:7-54) for slabs on the fused path.
 *
 * mplb_gpu_set_owned: a fused step stores the outputs of nodes
 * [start, start + count) only (count 0: every node, the default); the other
 * nodes are this handle's halo, written by its neighbours.
 *
 * mplb_gpu_add_mirror: every fused step of h also stores the outputs of its
 * owned nodes [src_start, src_start + count) (the post-collision populations
 * of every updated field, and T and U where the step writes them) into nodes
 * [dst_start, dst_start + count) of dst's next-step input buffers -- the
 * state mplb_gpu_copy_state copies, written by the kernel instead of by
 * copies between the steps.  At most two ranges per handle; the target
 * range must lie outside dst's owned range (set that first); dst on another
 * GPU takes plain peer stores (peer access is enabled here).  dst must
 * outlive h's mirrors (mplb_gpu_clear_mirrors drops them).
 *
 * Rules for the stepping: a handle with mirrors takes one step per
 * mplb_gpu_step call; linked handles take their steps in turn (a neighbour
 * must be at the same time or one step ahead, else MPLB_E_STATE); each step
 * is queued after the neighbours' queued work and before their next step
 * (events between the handles' streams; nothing on one stream).  The halo
 * must hold the neighbours' fused state before the first mirrored step, and
 * again after any call that brings a handle back to the reference's state
 * (a download, an operator): exchange it once with mplb_gpu_copy_state. */
int mplb_gpu_set_owned(mplb_gpu_t* h, uint32_t start, uint32_t count);
int mplb_gpu_add_mirror(mplb_gpu_t* h, uint32_t src_start, uint32_t count, mplb_gpu_t* dst, uint32_t dst_start);
int mplb_gpu_clear_mirrors(mplb_gpu_t* h);

/* Several ranks' lattices driven from one process (one handle per rank, on
 * one GPU or several), each holding its owned nodes and its ghost nodes (no
 * neighbours, on no patch: the layout of the reference's partitioned meshes).
 * runs[] lists the ghost exchange once: nodes [src_start, src_start + count)
 * of handle h[src] fill nodes [dst_start, ...) of handle h[dst].
 * mplb_ranks_initialize is multiPhasePP.c:122-147 on every rank (after the
 * caller's uploads of rho, U, T) with the ghosts of rho, U, T, then Fi, Ft,
 * then S exchanged; mplb_ranks_step is nsteps of multiPhasePP.c:157-240 on
 * every rank, exchanging the ghosts with mplb_gpu_copy_nodes where the
 * reference exchanges them: f after its boundaries (and after its collision
 * when surface tension is on, liMRTCollision.c:126-131), g after its
 * boundaries, S after heatSource, Fi and Ft after interForce.  All handles
 * hold the same lattice and field options. */
typedef struct mplb_ghost_run {
    uint32_t dst, dst_start;
    uint32_t src, src_start;
    uint32_t count;
} mplb_ghost_run;
int mplb_ranks_initialize(mplb_gpu_t* const* h, uint32_t count, const mplb_ghost_run* runs, uint32_t nruns);
int mplb_ranks_step(mplb_gpu_t* const* h, uint32_t count, const mplb_ghost_run* runs, uint32_t nruns,
                    uint32_t nsteps);

/* Total mass sum(rho[i]) and energy sum(T[i]) of plain device arrays, without
 * allocating device memory.  No counterpart in the reference: it is for
 * callers that may not call cudaMalloc where they want this check (a
 * framework allocator that owns device memory, a time loop with a
 * no-allocation policy, code that must not synchronise the device).
 * rho, T (may be NULL: energy 0) and out (2 doubles: mass, energy) are device
 * pointers on the current device; work is queued on `stream` (a cudaStream_t,
 * NULL = the default stream) and not waited for.
 * Scratch is a fixed 64 KiB array inside the library, held by every GPU that
 * loads it until exit; n is limited to 16,777,216 nodes (larger n returns
 * MPLB_E_ARG).  The first call on a device looks up that array's device
 * address; make that first call before any stream capture.  Calls that
 * overlap on the GPU share the array and race; order them on one stream. */
int mplb_mass_energy_noalloc(const double* rho, const double* T, uint32_t n, double* out, void* stream);

/* ------------------------------------------------------------------------
 * Batched ensemble.  No counterpart in the reference, whose driver
 * (src/applications/solvers/multiPhasePP/multiPhasePP.c) advances one lattice per process: here many
 * independent lattices -- each an ordinary handle created above -- advance
 * together, one kernel launch per time step for all of them, a block taking
 * (lattice, tile) pairs from a work table.  Each lattice's steps are the
 * same arithmetic as mplb_gpu_step on that handle.
 *
 * Eligible handles: D2Q9, precision MPLB_FP32_DEV, fused path, a fully
 * periodic box without boundary patches, isothermal (g frozen or absent),
 * all on one device.  The handles stay owned by the caller and must outlive
 * the batch; between batch calls they can be used (download, pressure, ...)
 * as usual.  Work runs on the first handle's stream; every call returns with
 * the handles' state current and their streams ordered after it.
 * ---------------------------------------------------------------------- */
typedef struct mplb_batch mplb_batch_t;

typedef struct {
    int32_t tile_config;      /* 0: time every tile candidate on the real
                                 state at the first call, keep the fastest;
                                 k > 0: candidate k-1 */
    uint32_t check_interval;  /* steps between convergence checks (even, >= 2) */
    double tol;               /* converged when max |rho(t) - rho(t-K)| / K < tol */
} mplb_batch_opts;

typedef struct {
    uint32_t n_lattices;
    uint64_t nodes;           /* sum over lattices */
    int32_t tile_config;      /* candidate in use (-1 before the first call) */
    int32_t n_candidates;
    int32_t tile_x[8], tile_y[8];
    float tile_ms[8];         /* autotuner: ms per step of each candidate */
    int32_t grid;             /* persistent blocks per step launch */
    uint64_t kernel_launches;
    uint64_t graph_launches;  /* check intervals replayed from the captured graph */
} mplb_batch_info;

int mplb_batch_create(mplb_gpu_t* const* lattices, uint32_t count, const mplb_batch_opts* opts,
                      mplb_batch_t** out);
int mplb_batch_destroy(mplb_batch_t* b);
int mplb_batch_info_get(mplb_batch_t* b, mplb_batch_info* info);
/* nsteps time steps of every lattice, no convergence checks. */
int mplb_batch_step(mplb_batch_t* b, uint32_t nsteps);
/* Advance lattices in check intervals of K = check_interval steps until each
 * has max |drho/dt| < tol (rho as the next step sums it, over one interval),
 * or has taken max_steps (rounded up to a whole interval), or has a
 * non-finite density (retired, rate = inf, not counted as converged).  Each
 * check also resets every lattice's total momentum to its starting value
 * (lattices without net body force).  A converged
 * lattice leaves the work table and stops.  Each interval -- K step launches
 * and one check launch -- replays one captured CUDA graph.
 * steps_out[i]: steps lattice i took; rate_out[i]: its last max |drho/dt|
 * (may be NULL); *n_converged: lattices that met tol. */
int mplb_batch_run(mplb_batch_t* b, uint32_t max_steps, uint32_t* steps_out, double* rate_out,
                   uint32_t* n_converged);

/* Time-averaging filter (off until set).  A static lattice settles to a
 * fixed point of the time step; near it the state is that fixed point plus
 * decaying oscillations, the slowest being the acoustic modes of the box,
 * whose damping (viscosity x (2 pi / L)^2) makes large lattices slow to
 * settle.  A filter window replaces lattice i's populations by their mean
 * over its last window[i] steps: the fixed point is unchanged (the mean is
 * linear in the state and every state of an equilibrium is the same), an
 * oscillation of period P shrinks by about |sin(pi window / P)| / (pi window
 * / P) -- nearly to zero for window = P, where plain stepping would take
 * many periods.  window[i] = 0 leaves lattice i unfiltered; window = NULL
 * turns the filter off.  mplb_batch_run then runs a window once `first`
 * steps are done and again `every` steps after the end of each window
 * (every = 0: only on request, mplb_batch_average), at the end of a check
 * interval, followed by a check of its own (steps_out counts window steps).
 * A window is M steps, M the smallest even number above the longest window
 * among the lattices still running: lattice i averages the states after
 * its steps M-1-window[i] .. M-2, and the window's last step runs from
 * that mean (so the populations the reference state is emitted from and
 * those the next step reads are both filtered).  Sums are FP64 (exact for
 * FP32 states), the mean is rounded once.  Device memory: 9 n doubles per
 * filtered lattice. */
#define MPLB_BATCH_MAX_WINDOW 1048576u
int mplb_batch_filter(mplb_batch_t* b, const uint32_t* window, uint32_t first, uint32_t every);
/* One filter window on every lattice now; *steps_out = its length in steps
 * (0 when no lattice is filtered). */
int mplb_batch_average(mplb_batch_t* b, uint32_t* steps_out);

/* ------------------------------------------------------------------------
 * Learned warm start.  No counterpart in the reference, whose initial fields
 * come from its dictionaries (a tanh/Maxwell bubble in the workloads here).
 * A 5-64-64-64-1 tanh network maps (T/Tc, a, b, r/R, R) -- Carnahan-Starling
 * constants a, b, distance r of a node to the bubble centre, radius R -- to
 * b * rho at equilibrium.  r/R and R enter as the pair ((r - R)/5, 5/R)
 * (interface at 0 with a width independent of R, curvature for the Laplace
 * shift).  Weights and activations BF16, accumulation FP32, FP32 master
 * weights and Adam state; trained on the device by this library's own
 * forward and backward kernels on density samples the caller takes from
 * converged lattices.
 *
 * Parameter vector (MPLB_MLP_PARAMS floats): W1[64][5], b1[64], W2[64][64],
 * b2[64], W3[64][64], b3[64], W4[64], b4 -- each W row-major [out][in].
 * ---------------------------------------------------------------------- */
#define MPLB_MLP_PARAMS 8769
typedef struct mplb_mlp mplb_mlp_t;

/* Glorot-uniform weights from `seed`, zero biases. */
int mplb_mlp_create(int32_t device, uint64_t seed, mplb_mlp_t** out);
int mplb_mlp_destroy(mplb_mlp_t* m);
int mplb_mlp_get_params(mplb_mlp_t* m, float* params);
/* Replaces the master weights (and their BF16 copy); resets Adam. */
int mplb_mlp_set_params(mplb_mlp_t* m, const float* params);
/* The network's normalised, BF16-rounded inputs for one sample (host). */
void mplb_mlp_features(double t_ratio, double a, double b, double r, double R, float* out5);
/* Training set: n samples (target b * rho), copied to the device. */
int mplb_mlp_set_samples(mplb_mlp_t* m, const double* t_ratio, const double* a, const double* b, const double* r,
                         const double* R, const double* rho, uint32_t n);
/* Gradient of the mean squared error over the whole training set, no update. */
int mplb_mlp_gradient(mplb_mlp_t* m, float* grad, double* loss);
/* `steps` Adam steps (beta 0.9 / 0.999) on minibatches of `batch` samples
 * drawn by a counter-based hash; *loss = the last minibatch's MSE. */
int mplb_mlp_train(mplb_mlp_t* m, uint32_t steps, uint32_t batch, float lr, double* loss);
/* rho for n samples. */
int mplb_mlp_predict(mplb_mlp_t* m, const double* t_ratio, const double* a, const double* b, const double* r,
                     const double* R, uint32_t n, double* rho);
/* Initial state of a box lattice with a Carnahan-Starling EOS: rho of every
 * node from the network (r = distance of the node's box coordinates to
 * `center`), U = 0, T = T.  Call mplb_gpu_initialize next, as after
 * mplb_gpu_upload.  The handle and the network must be on one device. */
int mplb_mlp_init_bubble(mplb_mlp_t* m, mplb_gpu_t* h, double t_ratio, const double* center, double radius,
                         double T);
/* As mplb_mlp_init_bubble, with the lattice's total density made equal to
 * target_mass (e.g. the mass of the tanh/Maxwell state being replaced, so
 * that both relax to the same equilibrium).  The network's inputs are BF16,
 * so its mass is a step function of the radius: the radius is bracketed to
 * one step (secant, then bisection) and the two fields are blended to hold
 * the target mass -- the bulk densities stay the network's, the interface
 * moves by a fraction of a step.  *radius_used (may be NULL) receives the
 * effective radius.  Allocates one scratch array of n doubles. */
int mplb_mlp_init_bubble_mass(mplb_mlp_t* m, mplb_gpu_t* h, double t_ratio, const double* center, double radius,
                              double T, double target_mass, double* radius_used);
/* Axial profile: a liquid band (a column or layer) of thickness `height`
 * along `axis` (0 = x, 1 = y, 2 = z), centred at coordinate `center`
 * (periodic distance over the box), in vapour: rho of every node from the
 * network with a flat interface (features with R = +inf, r = height/2 minus
 * the node's distance to the band centre), U = 0, T = T.  Use a network
 * trained on flat interfaces (the packaged column weights).  Call
 * mplb_gpu_initialize next.  No counterpart in the reference, whose column
 * starts from its tanh profile (tgProfileScalarField.c). */
int mplb_mlp_init_column(mplb_mlp_t* m, mplb_gpu_t* h, double t_ratio, int32_t axis, double center, double height,
                         double T);
/* As mplb_mlp_init_column, with the lattice's total density made equal to
 * target_mass in the same way as mplb_mlp_init_bubble_mass (the band height
 * bracketed and two fields blended); *height_used (may be NULL) receives the
 * effective height.  Allocates one scratch array of n doubles. */
int mplb_mlp_init_column_mass(mplb_mlp_t* m, mplb_gpu_t* h, double t_ratio, int32_t axis, double center,
                              double height, double T, double target_mass, double* height_used);

/*
 * Field files in the reference's per-rank formats, the data format chosen as
 * timeInfo.data does (include/dataTypes.h:53).  Replace writeScalarField
 * (src/IO/writeScalarField.c:10-59) and writeVectorField
 * (src/IO/writeVectorField.c:9-70) for the asciiRaw, binaryRaw and pvtu
 * formats with the same bytes: asciiRaw "%g" text, binaryRaw float values in
 * node order, both in <root>/processor<pid>/<time>/<name> (folders made as
 * needed); pvtu appends a DataArray block to
 * <root>/processor<pid>/<time>/fields.vtu.  root NULL or "" is the current
 * folder, as in the reference.  field is [n] (scalar) or [n][vsize] doubles
 * on the host.  A NaN anywhere returns MPLB_E_NONFINITE and writes nothing
 * (the reference stops the run there).  EnSight returns MPLB_E_UNSUPPORTED.
 * Host code only: no GPU is needed.  Text is formatted by several host
 * threads (MPLB_IO_THREADS, default: the hardware threads up to 32); the
 * bytes do not depend on their number.
 */
enum {
    MPLB_FMT_ASCII_RAW = 0,
    MPLB_FMT_BINARY_RAW = 1,
    MPLB_FMT_PVTU = 2,
    MPLB_FMT_ENSIGHT = 3
};
int mplb_write_scalar_field(const char* root, int32_t pid, uint32_t time, int32_t format, const char* name,
                            const double* field, uint64_t n);
int mplb_write_vector_field(const char* root, int32_t pid, uint32_t time, int32_t format, const char* name,
                            const double* field, uint64_t n, uint32_t vsize);

#ifdef __cplusplus
}
#endif

#endif /* MPLB_GPU_H */
