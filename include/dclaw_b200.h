/*
 * dclaw_b200.h -- C ABI of the B200 (sm_100a) D-Claw uniform-patch time step.
 *
 * The step is D-Claw's single-level patch update: b4step2 (admissibility,
 * speed limit, static-friction directions), step2/flux2 (augmented f-wave
 * Riemann solves, MC wave limiting, transverse propagation, flux
 * accumulation, Courant number) and src2 (Coulomb/viscous friction,
 * pore-pressure and solid-fraction relaxation), all in FP64.
 *
 * Conventions shared by every entry point
 *   - All array arguments are DEVICE pointers unless stated otherwise;
 *     `const dclaw_params*` is always a HOST pointer (copied into the launch).
 *   - State is structure-of-arrays, 5 planes in the order h, hu, hv, hm, pb.
 *     The segregation (h*chi) and bed-change fields of the 7-field Fortran
 *     state are identically zero when segregation = 0 and entrainment = 0,
 *     which is the only configuration accepted, so they are not stored.
 *   - Patch-call layout ("padded"): each plane holds (mx+2*mbc)*(my+2*mbc)
 *     doubles, x fastest; cell (i,j) with Fortran index i in 1-mbc..mx+mbc,
 *     j in 1-mbc..my+mbc lives at [(j-1+mbc)*(mx+2*mbc) + (i-1+mbc)].
 *     mbc must be 2.
 *   - Fused layout ("interior"): each plane holds mx*my doubles, x fastest;
 *     ghost cells are produced on the fly from the boundary conditions.
 *   - aux planes (padded layout): 0 b (bed), 1 phi, 2 theta, 3 fsphi,
 *     4 taudir_x, 5 taudir_y -- the first six D-Claw aux fields of a
 *     Cartesian run (digclaw_module.f90:96-110).
 *   - Every call is asynchronous on `stream` (a cudaStream_t, NULL = legacy
 *     default stream). The return code reports argument errors found on the
 *     host and CUDA launch errors; numerical errors (NaN in the state) are
 *     reported through the device status word of dclaw_clock.
 *   - The library never allocates device memory on these paths: callers
 *     pass a workspace of dclaw_workspace_bytes() bytes.
 */
#ifndef DCLAW_B200_H
#define DCLAW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DCLAW_ABI_VERSION 2

/* return / status codes */
#define DCLAW_OK 0
#define DCLAW_ERR_ARG 1          /* bad size, pointer or parameter */
#define DCLAW_ERR_UNSUPPORTED 2  /* option not implemented (bed_normal=1, ...) */
#define DCLAW_ERR_NAN 3          /* NaN found in the state (check4nans) */
#define DCLAW_ERR_CUDA 4         /* CUDA launch / runtime error */
#define DCLAW_ERR_WORKSPACE 5    /* workspace too small */
#define DCLAW_ERR_TOO_LARGE 6    /* size beyond a fixed limit */

/* boundary condition codes (clawdata.bc_lower / bc_upper) */
#define DCLAW_BC_EXTRAP 1
#define DCLAW_BC_WALL 3

/*
 * Parameters. Names follow the reference's setrun data classes:
 * geo_data (grav, dry_tolerance, speed_limit, friction_*), DClawInputData
 * (src/python/dclaw/data.py:315-351) and clawdata (order, transverse_waves,
 * limiter, cfl_*, dt_*, bc_*). Angles are in RADIANS here (set_dig converts
 * degrees, digclaw_module.f90:135-136).
 */
typedef struct dclaw_params {
    /* geo_data */
    double grav;
    double dry_tolerance;
    double speed_limit;
    int32_t friction_forcing;     /* Manning friction in src2 (src2.f90:271-289) */
    int32_t dd_manning;
    double manning_coefficient;
    double friction_depth;
    double manning_max;
    /* dclaw_data */
    double rho_s, rho_f, m_crit, m0, mref, kref;
    double phi;                   /* basal friction angle, radians */
    double delta, mu, alpha_c, c1, sigma_0;
    double theta_input;           /* radians; only used with bed_normal = 1 */
    int32_t src2method;           /* -1 (no m/p source), 0, 1 (mp_update_relax_Dclaw4) or 2 (mp_update_FE_4quad) */
    int32_t alphamethod;          /* 0 or 1 */
    int32_t rarecorrectortest;    /* 0/1 */
    int32_t bed_normal;           /* must be 0 */
    int32_t entrainment;          /* 0, or 1 on the full-state step only (dclaw_step_full) */
    int32_t segregation;          /* 0, or 1 on the full-state step only (dclaw_step_full) */
    int32_t curvature;            /* must be 0 */
    /* clawdata */
    int32_t order;                /* method(2): 1 or 2 */
    int32_t transverse_waves;     /* method(3): 0, 1 or 2 */
    int32_t limiter;              /* mthlim for every wave: 0 none,1 minmod,2 superbee,3 van Leer,4 MC,5 Beam-Warming */
    int32_t bc_lower[2];          /* x, y */
    int32_t bc_upper[2];          /* x, y */
    double cfl_desired;
    double cfl_max;
    double dt_max;
    /* segregation and entrainment (dclaw_data, src/python/dclaw/data.py:338-347);
     * read only by dclaw_step_full */
    double beta_seg;              /* species flux: alpha_seg = 1 - beta_seg (riemannsolvers_dclaw.f:88,464-468) */
    double delta_kr_order;        /* segregation = 1: kperm times 10^(delta_kr_order 2 (chi - 1/2))
                                     (digclaw_module.f90:418-431) */
    double chie;                  /* species fraction of entrained material (entrainment.f90:87) */
    double me;                    /* solid fraction of the erodible layer (entrainment.f90:59) */
    double entrainment_rate;      /* entrainment.f90:66-73 */
    int32_t entrainment_method;   /* 0: ent_dclaw4 (entrainment.f90:27-100); 1: none, as the
                                     reference's method 1 (src2.f90:256-262) */
    int32_t pad_;
} dclaw_params;

/*
 * Device-resident clock of a run: the Courant number of the last step and
 * the dt chosen for the next one by the tick rule
 *   dt_next = min(dt * cfl_desired / cfl, dt_max)   (cfl > 0; dt_max else),
 * clipped so that t never passes t_final when t_final > 0
 * (tick.f:490-526 and the time clamp of the step-function API).
 */
typedef struct dclaw_clock {
    double t;            /* simulated time after the last step */
    double dt;           /* dt the next step will use */
    double cfl;          /* Courant number of the last step (cflgrid) */
    double dt_last;      /* dt the last step used */
    double t_final;      /* <= 0: no clamp */
    uint64_t cfl_bits;   /* internal accumulator (order-preserving bits) */
    uint32_t nsteps;     /* steps taken */
    uint32_t blocks_done;/* internal counter */
    int32_t status;      /* DCLAW_OK or DCLAW_ERR_NAN */
    int32_t fixed_dt;    /* 1: keep dt constant (no tick rule) */
    double t_obs;        /* > 0 (with the tick rule): every dt is also clipped at
                            the next multiple of t_obs, so t lands on each
                            observation time: dt <= (floor(t / t_obs + 1e-9) + 1)
                            t_obs - t, the port's flume loop
                            (pf_flume/flume_model.py:152-153); 0: off */
} dclaw_clock;

/* ---- library info and parameters ---------------------------------------- */
int dclaw_abi_version(void);
const char* dclaw_error_string(int code);
/* reference defaults (data.py:315-351, geo_data, clawdata) with config-0 style numerics */
void dclaw_params_default(dclaw_params* p);
/* host-side validation; returns DCLAW_OK, DCLAW_ERR_ARG or DCLAW_ERR_UNSUPPORTED */
int dclaw_params_check(const dclaw_params* p);
/* dclaw_params_check, and DCLAW_ERR_UNSUPPORTED for segregation or
 * entrainment: the entry points on the five-field state (h, hu, hv, hm, pb)
 * carry no species fraction hchi and no bed change; those options need the
 * full-state step dclaw_step_full. (Ensemble members of dclaw_step_batched
 * must pass this check too.) */
int dclaw_params_check_5(const dclaw_params* p);
/* bytes of device workspace the step entry points need for an mx x my patch */
size_t dclaw_workspace_bytes(int mx, int my);

/* ---- step2-style patch calls (padded layout, mbc = 2) -------------------
 * Replace the Fortran patch step of stepgrid: bc2amr (GeoClaw, called before
 * the step), b4step2 (src/2d/dig/b4step2.f90:7), step2 + stepgrid's
 * flux-differencing update (GeoClaw step2.f90, driving flux2fw.f:8-11 with
 * rpn2_dclaw.f:24 / rpt2_dclaw.f:16) and src2 (src/2d/dig/src2.f90:27).
 */
/* fill the two ghost rings of q from the boundary conditions (bc2amr) */
int dclaw_bc2amr(double* q, int mx, int my, int mbc, const dclaw_params* p, void* stream);
/* fill aux for a new patch: ghost bed = nearest interior bed (setaux.f90:155-184),
 * phi/theta uniform, fsphi/taudir zero (setaux.f90:195-198,268-281) */
int dclaw_setaux(double* aux, int mx, int my, int mbc, const dclaw_params* p, void* stream);
/* b4step2: qfix + bdif clamp on all cells, speed limit, calc_taudir (aux 3..5) */
int dclaw_b4step2(double* q, double* aux, int mx, int my, int mbc, double dx, double dy,
                  double t, double dt, const dclaw_params* p, dclaw_clock* clock, void* stream);
/* step2 + update: q <- q - dt/dx (fm(i+1)-fp(i)) - dt/dy (gm(j+1)-gp(j)) on the interior;
 * the patch Courant number is max-reduced into clock->cfl_bits/cfl.
 * fluxes (nullable): 20 padded planes fm[5], fp[5], gm[5], gp[5]. */
int dclaw_step2(double* q, const double* aux, int mx, int my, int mbc, double dx, double dy,
                double dt, const dclaw_params* p, dclaw_clock* clock, double* fluxes,
                void* work, size_t work_bytes, void* stream);
/* src2: friction + m/pb relaxation on interior cells */
int dclaw_src2(double* q, const double* aux, int mx, int my, int mbc, double dx, double dy,
               double t, double dt, const dclaw_params* p, void* stream);

/* ---- fused uniform-patch step (interior layout) -------------------------
 * One full step (bc2amr + b4step2 + step2 + update + src2 + Courant number)
 * from q_in to q_out (distinct buffers). dt is read from clock->dt; after
 * the step clock holds t += dt, cfl, nsteps += 1 and the next dt (tick rule
 * unless clock->fixed_dt). phi is the uniform basal friction angle
 * (p->phi). branch_log (nullable) receives per-interface branch bits:
 * x interfaces [(my+2) rows][(mx+1)], then y interfaces [(mx+2) cols][(my+1)].
 */
int dclaw_step(const double* q_in, double* q_out, const double* b, int mx, int my,
               double dx, double dy, const dclaw_params* p, dclaw_clock* clock,
               void* work, size_t work_bytes, uint32_t* branch_log, void* stream);
/* The step on the reference's whole state, for segregation and entrainment.
 * The reference carries q(7) = (h, hu, hv, hm, pb, hchi, bdif)
 * (digclaw_module.f90:96-102); this entry point takes and returns those
 * seven fields as (7, my, mx) planes (interior, x fastest, device):
 * hchi = h chi (species fraction chi, clipped to [0, 1] by qfix), bdif = the
 * bed eroded so far (the step sees the bed b - bdif). It is stepgrid's patch
 * step like dclaw_step (b4step2.f90:7, step2 and src2.f90:27 with tick's dt
 * rule) with every option of dclaw_step plus
 *   segregation = 1: kperm times 10^(delta_kr_order 2 (chi - 1/2)) in setvars
 *                    (digclaw_module.f90:418-431); the species waves use
 *                    alpha_seg = 1 - beta_seg (riemannsolvers_dclaw.f:88,463-468)
 *                    whatever segregation is, as the reference's do;
 *   entrainment = 1, entrainment_method = 0: ent_dclaw4 in src2
 *                    (src2.f90:252-262, entrainment.f90:27-100), eroding
 *                    up to h_e - bdif, h_e (my, mx) on the device = the
 *                    erodible depth aux(i_ent) (required then; nullable
 *                    otherwise).
 * With hchi = bdif = 0 and both options off it returns dclaw_step's bits for
 * the first five fields. work holds dclaw_step_full_workspace_bytes(mx, my);
 * branch_log as for dclaw_step. One launch per stage (seven). */
int dclaw_step_full(const double* q_in, double* q_out, const double* b, const double* h_e, int mx, int my,
                    double dx, double dy, const dclaw_params* p, dclaw_clock* clock, void* work,
                    size_t work_bytes, uint32_t* branch_log, void* stream);
size_t dclaw_step_full_workspace_bytes(int mx, int my);
/* Allocation-free variant of dclaw_step. No counterpart in the reference:
 * it exists for callers that drive the step from code with no device
 * allocator of their own -- a Fortran time loop bound through iso_c_binding
 * (gfortran has no CUDA allocation API), or a host application that owns all
 * device memory and hands the step only the state it already holds -- and so
 * cannot size and keep the workspace dclaw_step needs. Its scratch (the
 * per-cell records) lives in a fixed 28 MiB device array inside the library,
 * which every GPU that loads the library keeps until the process exits; the
 * patch is limited to (mx+4)*(my+4) <= 262144 padded cells (e.g. 508 x 508),
 * larger patches return DCLAW_ERR_TOO_LARGE without launching anything.
 * It never calls cudaMalloc/cudaFree. The first call on a device looks up
 * the array's device address (with that device current) and should come
 * before any stream capture on that device; first calls from several host
 * threads at once are safe (the look-up runs under a lock, once per
 * device). All calls on a device share the
 * one array: calls whose work overlaps on the GPU (different streams, or
 * different host threads without ordering) race and must not be issued.
 * Arguments and results are those of dclaw_step without the workspace and
 * the branch log. */
int dclaw_step_noalloc(const double* q_in, double* q_out, const double* b, int mx, int my,
                       double dx, double dy, const dclaw_params* p, dclaw_clock* clock,
                       void* stream);
/* largest patch (padded cells) dclaw_step_noalloc accepts */
size_t dclaw_step_noalloc_max_cells(void);
/* dclaw_step on a state held in HOST memory: the reference's patch step
 * works on host arrays (stepgrid passes q and aux to step2, step2.f90:9-10,
 * then src2, src2.f90:27), and a host time loop that keeps the state there
 * calls this once per step. q_in and q_out are (5, my, mx) host arrays (they
 * may be the same array: the step then updates it in place); b, clock and
 * work are on the device, work holding dclaw_step_host_workspace_bytes()
 * (the step's workspace and a device copy of the state in and out). The
 * step is pipelined by bands of tile rows: each band's input rows go up on
 * one copy stream, its records, tiles and src2 run on `stream`, and its
 * output rows come down on another copy stream, so that both copy
 * directions and the compute overlap. Host memory must be page-locked
 * (cudaHostAlloc / cudaHostRegister) for the copies to overlap; pageable
 * memory gives the same result without the overlap. nbands = 0 picks the
 * band count (about 28 MB of state per band, at most 64); a positive value
 * asks for that many (capped by the tile rows and 64). The call returns once
 * the work is queued; `stream` waits for the last download, so a
 * synchronize on it (or on an event recorded after the call) means q_out and
 * the clock are complete. Results are those of dclaw_step, bit for bit. */
int dclaw_step_host(const double* q_in, double* q_out, const double* b, int mx, int my,
                    double dx, double dy, const dclaw_params* p, dclaw_clock* clock,
                    void* work, size_t work_bytes, int nbands, void* stream);
size_t dclaw_step_host_workspace_bytes(int mx, int my);
/* ---- one patch over several GPUs (row slabs) ------------------------------
 * A patch too large for one GPU splits into slabs of whole tile rows, one per
 * GPU. Each GPU holds its rows plus a halo of dclaw_rows_granule() rows on
 * each side that lies inside the patch (the step reads at most 4 rows away),
 * as a patch of its own: its own mx x my_local state, bed and workspace, its
 * edges at the patch's edges keeping the patch's boundary conditions. Per
 * step every GPU receives its halo rows from its neighbours, calls
 * dclaw_step_rows for its own rows, max-reduces clock->cfl_bits over the GPUs
 * (the order-preserving bit pattern of the non-negative Courant number, so
 * an integer max), and calls dclaw_clock_tick. The result equals dclaw_step
 * on the whole patch, bit for bit, with the same dt: the reference's patch
 * advance likewise computes cflgrid per patch and takes the largest for the
 * level's next dt (GeoClaw's advanc, called from tick.f:333). */
/* rows per tile row: row ranges of dclaw_step_rows start and end on multiples */
int dclaw_rows_granule(void);
/* dclaw_step for rows row_first .. row_first+row_count-1 (1-based) of the
 * patch only: row_first - 1 is a multiple of dclaw_rows_granule(), and the
 * range ends on one or at the last row. Those rows of q_out are written (the
 * others are left as they are), their tiles' Courant number is max-reduced
 * into clock->cfl_bits, and the clock is NOT ticked. Workspace: as dclaw_step. */
int dclaw_step_rows(const double* q_in, double* q_out, const double* b, int mx, int my,
                    double dx, double dy, const dclaw_params* p, dclaw_clock* clock,
                    void* work, size_t work_bytes, int row_first, int row_count, void* stream);
/* the tick rule after dclaw_step_rows: t += dt, cfl from cfl_bits, the next dt
 * (tick.f:490-526), cfl_bits cleared */
int dclaw_clock_tick(dclaw_clock* clock, const dclaw_params* p, void* stream);
/* the band plan dclaw_step_host uses: returns the band count nb and writes
 * the first tile row of each band to first[0..nb] (first[nb] = tile rows),
 * at most `max` entries; 0 for an invalid size */
int dclaw_step_host_bands(int mx, int my, int nbands, int32_t* first, int max);
/* ---- batched ensemble -------------------------------------------------------
 * An ensemble of independent uniform patches of uneven sizes, each with its
 * own parameters and its own clock (the particle-filter use of the
 * reference's differentiable port: one simulation per particle,
 * gradient_particle_filter/pf_flume/flume_model.py:129-179, vmapped in
 * pf_flume/inference.py:96-108). All members advance together: one step of
 * the ensemble is six launches (a scan of every cell that marks the active
 * tiles, a list of the active tiles and of the tiles whose records they
 * read, those records, a persistent kernel pulling the active tiles of
 * every member from one work queue, src2, each member's tick), so a
 * sequence of ensemble steps captures into one CUDA graph. Tiles with no wet
 * cell within 3 cells are skipped (src2 writes their zeros).
 * Member m's state is 5 planes [5][my][mx] at q_off in the state arenas; its
 * bed is [my][mx] at b_off in the bed arena. */
typedef struct dclaw_member {
    int32_t mx, my;
    double dx, dy;
    uint64_t q_off;       /* doubles into the state arenas */
    uint64_t b_off;       /* doubles into the bed arena */
    uint64_t rec_off;     /* doubles into the workspace: per-cell records */
    uint64_t qs_off;      /* doubles into the workspace: state before src2 */
    uint32_t tile0;       /* first tile of the member in the ensemble's tile list */
    uint32_t ntiles_x;    /* tiles along x */
    uint32_t ntiles;      /* tiles of the member */
    uint32_t rchunk0;     /* first 256-cell chunk of the member's padded cells */
    uint32_t nrchunks;
    uint32_t schunk0;     /* first 256-cell chunk of the member's interior cells */
    uint32_t nschunks;
    uint32_t pad_;
} dclaw_member;

typedef struct dclaw_batch {
    int32_t nmembers;
    int32_t tile_shape;        /* index into dclaw_batch_tile_shapes() */
    int32_t tile_ctas_per_sm;  /* persistent tile CTAs per SM (1 or 2) */
    int32_t cell_ctas_per_sm;  /* persistent CTAs per SM of the cell kernels */
    uint32_t ntiles;           /* tiles of all members (for tile_shape) */
    uint32_t nrchunks, nschunks;
    uint32_t pad_;
    uint64_t q_doubles;        /* size of one state arena */
    uint64_t b_doubles;        /* size of the bed arena */
    uint64_t work_bytes;       /* workspace size */
} dclaw_batch;

/* tile shapes compiled for the ensemble kernels; returns how many (<= max) */
int dclaw_batch_tile_shapes(int32_t* tx, int32_t* ty, int max);
/* host-side layout of n members (sizes and spacings in host arrays): fills
 * members[0..n) (host array) and *batch for the given tile shape */
int dclaw_batch_layout(int n, const int32_t* mx, const int32_t* my, const double* dx, const double* dy,
                       int tile_shape, dclaw_member* members, dclaw_batch* batch);
/* one step of every member. batch: host; members, params, clocks: DEVICE
 * arrays of nmembers; q_in / q_out: distinct state arenas; b: bed arena;
 * work: batch->work_bytes (the tile queue counter inside it must be zero
 * before the first step: dclaw_batch_reset). */
int dclaw_step_batched(const dclaw_batch* batch, const dclaw_member* members, const dclaw_params* params,
                       dclaw_clock* clocks, const double* q_in, double* q_out, const double* b, void* work,
                       void* stream);
/* zero the ensemble's work-queue counters (before the first step) */
int dclaw_batch_reset(const dclaw_batch* batch, void* work, void* stream);

/* ---- adjoint of one step ----------------------------------------------------
 * The reference has no adjoint of the Fortran step; its differentiable port
 * takes gradients with jax.grad through checkpointed scans
 * (differentiable_dclaw/dclaw_jax/solver.py:357-388,
 * differentiable_dclaw/tests/test_reverse_mode.py:37-49). This is the
 * hand-written reverse of the same step as dclaw_step, for the gradient of
 * a loss over a run of steps.
 *
 * lam_in = (dS/dq)^T lam_out, where S is one step of size *dt (a DEVICE
 * double; dt is data, not differentiated) from q_in (interior layout, 5
 * planes) over bed b. pbar (DEVICE, 4 doubles, ACCUMULATED) receives
 * (dS/dtheta)^T lam_out for theta = (phi [radians], kref, alpha_c, mu).
 * bbar (DEVICE, mx*my doubles, ACCUMULATED, nullable) receives (dS/db)^T
 * lam_out, the adjoint of the bed (through calc_taudir's surface slopes and
 * the solver's bed step; the ghost beds are copies of the nearest cells).
 * At branches (dry tolerance, limiter regimes, wall and static-friction
 * tests, min/max picks) the adjoint follows the branch the forward step
 * took. Results are bit-reproducible (no atomics in the sums). status
 * (DEVICE int32, nullable) receives DCLAW_ERR_NAN if q_in holds a NaN.
 * work: dclaw_adjoint_workspace_bytes(mx, my) bytes. */
size_t dclaw_adjoint_workspace_bytes(int mx, int my);
/* DCLAW_OK when the options have an adjoint form; DCLAW_ERR_UNSUPPORTED for
 * the rare-wave corrector test and for src2method 2 (FE_4quad's data-dependent
 * substeps); Manning friction (constant or dd_manning) has its reverse */
int dclaw_adjoint_supported(const dclaw_params* p);
int dclaw_step_adjoint(const double* q_in, const double* b, int mx, int my, double dx, double dy,
                       const double* dt, const dclaw_params* p, const double* lam_out, double* lam_in,
                       double* pbar, double* bbar, void* work, size_t work_bytes, int32_t* status, void* stream);
/* dclaw_step_adjoint in two parts. prepare queues what does not depend on
 * lam_out (the activity blocks, the forward recompute of the step's
 * intermediates into work); reverse, given the same q_in, b, dt, p and work
 * after prepare, queues the reverse stages. A backward pass over many steps
 * can prepare step n-1 in a second workspace (on another stream) while step
 * n's reverse runs; the results are those of dclaw_step_adjoint, bit for bit. */
int dclaw_step_adjoint_prepare(const double* q_in, const double* b, int mx, int my, double dx, double dy,
                               const double* dt, const dclaw_params* p, void* work, size_t work_bytes,
                               int32_t* status, void* stream);
int dclaw_step_adjoint_reverse(const double* q_in, const double* b, int mx, int my, double dx, double dy,
                               const double* dt, const dclaw_params* p, const double* lam_out, double* lam_in,
                               double* pbar, double* bbar, void* work, size_t work_bytes, int32_t* status,
                               void* stream);

/* ---- adjoint of one step of an ensemble ---------------------------------------
 * The reference differentiates its particle filters member by member with
 * jax.jacfwd / jax.grad under jax.vmap (gradient_particle_filter/pf_flume/
 * inference.py:96-108). Here the adjoint of one step of every member of an
 * ensemble of uneven patches runs as one sequence of 20 launches that work
 * only where members are wet: a scan marks each member's 16 x 16 activity
 * blocks (a wet cell within 4), a list kernel gathers the active blocks and
 * the blocks beside them, the forward recompute and the zeroing of the
 * reverse planes run over the second list and the reverse stages over the
 * first, each a grid-stride loop of one CTA per listed block. Each member
 * has its own parameters, dt and parameter adjoints; member k's lam_in
 * equals dclaw_step_adjoint's on member k alone bit for bit, and its
 * parameter adjoints agree to rounding (the block sums are grouped by
 * activity block, not by 128-item chunk).
 * Item spaces (chunk0 / nchunk index): 0 padded cells, 1 interior cells,
 * 2 x-interface solves, 3 y-interface solves, 4 x-interface fluxes, 5 y-interface
 * fluxes. */
typedef struct dclaw_adj_member {
    int32_t mx, my;
    double dx, dy;
    uint64_t q_off;        /* doubles into the state and adjoint arenas ([5][my][mx]) */
    uint64_t b_off;        /* doubles into the bed arena */
    uint64_t work_off;     /* bytes into the batch's adjoint workspace (256-aligned) */
    uint32_t chunk0[6];    /* first chunk of the member in each item space */
    uint32_t nchunk[6];    /* chunks of the member in each item space */
} dclaw_adj_member;

typedef struct dclaw_adj_batch {
    int32_t nmembers;
    uint32_t chunk_items;  /* items per chunk (threads per block) */
    uint32_t nchunks[6];   /* chunks of all members per item space */
    uint32_t nblocks;      /* 16 x 16 activity blocks of all members */
    uint32_t pad_;
    uint64_t work_bytes;   /* adjoint workspace of the whole batch (+ block lists) */
} dclaw_adj_batch;

/* host-side layout: members[0..n) (host array) from sizes, spacings and the
 * members' offsets in the state / bed arenas (host arrays, in doubles) */
int dclaw_adjoint_batch_layout(int n, const int32_t* mx, const int32_t* my, const double* dx, const double* dy,
                               const uint64_t* q_off, const uint64_t* b_off, dclaw_adj_member* members,
                               dclaw_adj_batch* batch);
/* batch: host; members, params, dt (one per member), status (one int32 per
 * member, nullable), pbar (4 per member, accumulated): DEVICE arrays.
 * q_in, lam_out, lam_in: state-shaped arenas; b: bed arena; bbar (nullable,
 * accumulated): bed-shaped arena of the beds' adjoints; work:
 * batch->work_bytes. Members whose options have no adjoint form get
 * DCLAW_ERR_UNSUPPORTED in their status word. */
int dclaw_step_adjoint_batched(const dclaw_adj_batch* batch, const dclaw_adj_member* members,
                               const dclaw_params* params, const double* dt, const double* q_in, const double* b,
                               const double* lam_out, double* lam_in, double* pbar, double* bbar, void* work,
                               int32_t* status, void* stream);
/* the two parts of dclaw_step_adjoint_batched, as for the single patch */
int dclaw_step_adjoint_batched_prepare(const dclaw_adj_batch* batch, const dclaw_adj_member* members,
                                       const dclaw_params* params, const double* dt, const double* q_in,
                                       const double* b, void* work, int32_t* status, void* stream);
int dclaw_step_adjoint_batched_reverse(const dclaw_adj_batch* batch, const dclaw_adj_member* members,
                                       const dclaw_params* params, const double* dt, const double* q_in,
                                       const double* b, const double* lam_out, double* lam_in, double* pbar,
                                       double* bbar, void* work, int32_t* status, void* stream);

/* initialise a device clock: t, dt, t_final, fixed_dt; counters cleared, t_obs 0 */
int dclaw_clock_init(dclaw_clock* clock, double t, double dt, double t_final, int fixed_dt,
                     void* stream);
/* set the clock's observation interval (0: off) and clip its next dt by it */
int dclaw_clock_set_obs(dclaw_clock* clock, double t_obs, void* stream);
/* Observation record after a step (the flume loop of the differentiable port,
   pf_flume/flume_model.py:154-158): for each clock c of n_clocks whose t lands on
   an observation time, |t - (k+1) t_obs| < 1e-9 with k = rint(t / t_obs) - 1 in
   0..n_obs-1, and whose last dt was positive, slot k of `out` (n_obs rows of
   n_select doubles) receives the state entries q[select[e]] of the entries e of
   that clock (member[e]; member NULL: all entries belong to clock 0; select
   NULL: entry e is q[e]), and out_step[k * n_clocks + c] = step. Other slots
   are left as they are. Clocks with t_obs = 0 record nothing. */
int dclaw_obs_record(const dclaw_clock* clocks, int n_clocks, const int32_t* member, const double* q,
                     const int64_t* select, int64_t n_select, int n_obs, int step, double* out,
                     int32_t* out_step, void* stream);
/* Running peak of a plane for the differentiable peak-depth run (the port's
   rollout_peak, differentiable_dclaw/dclaw_jax/solver.py:357-388): where
   h[i] > hmax[i], hmax[i] = h[i] and argstep[i] = step. peak_adjoint adds
   g[i] to lam_h[i] where argstep[i] == step (the gradient of a maximum goes
   to the step that set it; ties to the earliest). n entries, device pointers. */
int dclaw_peak_update(const double* h, double* hmax, int32_t* argstep, int64_t n, int step, void* stream);
int dclaw_peak_adjoint(const double* g, const int32_t* argstep, int64_t n, int step, double* lam_h,
                       void* stream);
/* Fortran-layout adapters for the patch calls. A Fortran patch array
   a(nf_fortran, 1-mbc:mx+mbc, 1-mbc:my+mbc) (field fastest; D-Claw's
   q(meqn=7, ...) and aux(maux, ...), digclaw_module.f90:96-110) and the patch
   calls' padded structure-of-arrays form (nf planes of (my+2mbc)(mx+2mbc), x
   fastest) hold the same cells. from_fortran copies fields 1..nf of each cell
   into the planes; to_fortran copies the planes back into fields 1..nf and
   leaves fields nf+1..nf_fortran as they are (for q: hchi and bdif, which stay
   zero without segregation and entrainment). Device pointers;
   nf <= nf_fortran. */
int dclaw_fields_from_fortran(const double* fortran, int nf_fortran, int nf, int mx, int my, int mbc,
                              double* planes, void* stream);
int dclaw_fields_to_fortran(const double* planes, int nf, int nf_fortran, int mx, int my, int mbc,
                            double* fortran, void* stream);
/* max over cells of |u|+sqrt(g h) (interior layout) written to *smax (device double) */
int dclaw_max_wave_speed(const double* q, int mx, int my, const dclaw_params* p, double* smax,
                         void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DCLAW_B200_H */
