/*
 * multifil_b200 -- C ABI of the B200 (sm_100a) half-sarcomere timestep engine.
 *
 * The reference (travistune3/multifil_jax) has no FFI: its seam is the Python
 * call run(topology, duration_ms, dt, pCa, z_line, lattice_spacing, K_lat, nu,
 * dynamic_params, static_params, replicates, rng_seed, ...) -> SimulationResult
 * (multifil_jax/simulation.py:754-771), which dispatches the jitted
 * _run_sim_kernel(topology, batched_params, z_batched, pCa_batched,
 * ls_batched, rng_keys, dt, ..., n_cg_steps, n_newton_steps) -> 52 metrics of
 * shape [batch, time] (simulation.py:584-747).  The entry points below replace
 * that kernel; the Python package multifil_jax_b200 keeps the run() API on
 * top of them through ctypes.
 *
 * Conventions
 *   - Every function returns 0 on success or a negative MF_ERR_* code; the
 *     message of the last failure on a context is mf_last_error(ctx).
 *   - No exceptions cross this boundary; no device trap is ever raised.
 *   - "device" pointers are CUDA device addresses owned by the caller; the
 *     library never frees them.  "host" pointers are read during the call.
 *   - A context is driven by one host thread at a time.  Several contexts
 *     may coexist.  Outputs are valid once the given stream has synchronised.
 */
#ifndef MULTIFIL_B200_H
#define MULTIFIL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MF_ABI_VERSION 2

/* error codes */
#define MF_OK 0
#define MF_ERR_INVALID (-1)   /* bad argument / shape */
#define MF_ERR_CUDA (-2)      /* a CUDA runtime call failed */
#define MF_ERR_NOMEM (-3)     /* device memory exhausted / admission refused */
#define MF_ERR_NOTFOUND (-4)  /* unknown topology id or request id */
#define MF_ERR_TIMEOUT (-5)   /* a bounded device wait gave up */
#define MF_ERR_BUSY (-6)      /* request still running */

/* per-condition status bits written to status_out */
#define MF_STATUS_NONFINITE 1      /* a Newton update or residual was not finite (the update
                                      was zeroed, as kernels/solver.py:415 does) */
#define MF_STATUS_NOT_CONVERGED 2  /* residual above solver_residual_tol at some step */
/* bit 4 is unused: every index the kernel forms is validated on the host when
 * the lattice is uploaded, and no data-dependent index leaves its range */
#define MF_STATUS_MULTIBIND 8      /* a site carried 3+ force-carrying heads at some step (the
                                      reference's double binding, transitions.py:1199-1219;
                                      their forces are summed in head order) */

/* batch flags */
#define MF_FLAG_DYNAMIC_LS 1       /* lattice spacing solved as an unknown (K_lat given) */
#define MF_FLAG_PRECISE 2          /* displacement formulation + FP64 residual test/squaring */
#define MF_FLAG_ORIGINAL_PRNG 4    /* pre-0.5 jax.random counter layout */
#define MF_FLAG_PLAIN 8            /* one condition per launch, one launch per step */
#define MF_FLAG_NO_GRAPH 16        /* batched path without CUDA-graph capture */
#define MF_FLAG_CONST_DRIVERS 32   /* z, pCa and ls are [B]: one value per condition for every
                                      step (a scalar sweep), instead of [B*T_max] traces */

#define MF_N_PARAMS 44
#define MF_N_METRICS 52

/* subpopulations (mf_batch.pop_*): reference core/subpopulation.py */
#define MF_MAX_POPS 4              /* populations per condition */
#define MF_POP_EXPLICIT 1          /* per-unit labels select a population's tables ('random',
                                      'c_zone'); without it the K generators are blended
                                      with the fractions ('mean_field') */
#define MF_POP_XB 2                /* the populations change crossbridge rates (xb_* fields) */
#define MF_POP_TM 4                /* the populations change tropomyosin rates (tm_* fields) */

typedef struct mf_ctx mf_ctx;

/* Lattice arrays as produced by SarcTopology.create
 * (reference core/sarc_geometry.py:112-176, 379-645).  Host pointers. */
typedef struct {
    int32_t n_thick, n_crowns, n_thin, n_sites;
    int32_t n_xb_per_crown, max_sites_per_face, n_xb_bins;
    const int32_t* xb_to_thin_id;      /* [n_thick*n_crowns*n_xb_per_crown] */
    const int32_t* xb_to_thin_face;    /* same */
    const uint8_t* xb_valid;           /* same */
    const int32_t* face_to_sites;      /* [n_thin*3*max_sites_per_face], -1 padded */
    const int32_t* n_sites_per_face;   /* [n_thin*3] */
    const int32_t* tm_prev_neighbor;   /* [n_thin*n_sites] */
    const int32_t* tm_next_neighbor;   /* [n_thin*n_sites] */
    const float* crown_offsets;        /* [n_thick*n_crowns] */
    const float* crown_rests;          /* [n_thick*n_crowns] */
    const float* binding_offsets;      /* [n_thin*n_sites] */
    const float* binding_rests;        /* [n_thin*n_sites] */
    const float* thin_rest_cumsum;     /* [n_thin*n_sites] cumsum(binding_rests) per filament */
    const float* xb_bin_edges;         /* [n_xb_bins+1] */
    const float* xb_bin_centers;       /* [n_xb_bins] */
} mf_topo_desc;

/* One batch of independent conditions (one row of the reference's vmap each). */
typedef struct {
    int32_t B;              /* number of conditions */
    int32_t T_max;          /* row stride of the per-step arrays */
    const int32_t* topo_id; /* [B] host: lattice of each condition (mf_upload_topology ids) */
    const float* params;    /* [B*44] device: DynamicParams rows, reference field order */
    const float* z;         /* [B*T_max] device: z_line trace ([B] with MF_FLAG_CONST_DRIVERS) */
    const float* pCa;       /* [B*T_max] device (same) */
    const float* ls;        /* [B*T_max] device: lattice_spacing trace, driver / d_ref basis (same) */
    const int32_t* n_steps; /* [B] device: steps of each condition (<= T_max) */
    const uint32_t* keys;   /* [B*2] device: jax.random key of each condition */
    const float* K_lat;     /* [B] device: lattice stiffness already x n_thick (dynamic LS) */
    const float* nu;        /* [B] device: Poisson exponent (dynamic LS) */
    const float* dt;        /* [B] device: timestep (ms) of each condition */
    int32_t n_newton;       /* StaticParams.n_newton_steps (4) */
    int32_t n_cg;           /* StaticParams.n_cg_steps (6) */
    int32_t flags;          /* MF_FLAG_* */
    int32_t chunk_steps;    /* steps per launch in the batched path (0 = all) */
    float residual_warn;    /* StaticParams.solver_residual_tol (status bit only) */
    float* metrics_out;     /* [B*52*T_max] device, or page-locked host memory mapped at the
                               same address (cudaHostAlloc under unified addressing): the
                               kernels then write the metrics over the bus and no copy
                               follows; pageable memory is refused (MF_ERR_INVALID) */
    int32_t* status_out;    /* [B] device */
    uint32_t* keys_out;     /* [B*2] device or NULL: key after the last step */
    /* test hooks (NULL in production) */
    const float* u_thin;    /* [B*T_max*n_sites_total] injected uniforms or NULL */
    const float* u_xb;      /* [B*T_max*total_xbs] injected uniforms or NULL */
    float* x_trace;         /* [B*T_max*max_dof] node positions after each step or NULL */
    int8_t* state_trace;    /* [B*T_max*(max_xbs + max_sites)] xb then tm states or NULL */
    int32_t* bound_trace;   /* [B*T_max*(max_xbs + max_sites)] xb then thin bound_to or NULL */
    /* Subpopulations (simulation.py:485-577 and the per-population branches of
     * kernels/transitions.py:580-596, 925-994); n_pops <= 1: one population and
     * the pop_* fields are ignored.  Mechanics always use `params`. */
    int32_t n_pops;           /* K populations, 2..MF_MAX_POPS (population 0 = wild type) */
    int32_t pop_flags;        /* MF_POP_EXPLICIT | MF_POP_XB | MF_POP_TM */
    int32_t label_stride;     /* row stride of xb_label / tm_label (>= every condition's
                                 total_xbs and n_sites_total) */
    const float* pop_params;  /* [B*n_pops*44] device: each population's DynamicParams row */
    const float* pop_frac;    /* [B*n_pops] device: blend weights (mean field) */
    const int8_t* xb_label;   /* [B*label_stride] device: population of each head
                                 (MF_POP_EXPLICIT with MF_POP_XB; values are clamped to [0, K)) */
    const int8_t* tm_label;   /* [B*label_stride] device: population of each binding site
                                 (MF_POP_EXPLICIT with MF_POP_TM) */
} mf_batch;

int mf_abi_version(void);
int mf_create(int device, mf_ctx** out);
int mf_destroy(mf_ctx* ctx);
const char* mf_last_error(mf_ctx* ctx);

/* Copy a lattice to the device; the library owns the copy until mf_destroy. */
int mf_upload_topology(mf_ctx* ctx, const mf_topo_desc* desc, int32_t* topo_id);

/* Run every condition of the batch to its n_steps.  Batched path: one CTA per
 * condition, whole time loop resident in shared memory, launches of
 * chunk_steps steps replayed from a captured CUDA graph.  With MF_FLAG_PLAIN:
 * one condition per launch and one launch per step (the baseline form). */
int mf_run_batch(mf_ctx* ctx, const mf_batch* batch, void* stream);

/* CTA size of a lattice's conditions: 128, 256, 384, 512 or 1024 threads
 * (no counterpart in the reference, whose XLA compiler picks the launch
 * shapes).  mf_tune_threads_mode sets it for one precision mode (precise = 1:
 * MF_FLAG_PRECISE batches), mf_tune_threads for both.  Defaults up to 1200
 * nodes: 384 threads (precise mode: 256 when the lattice has more than 12
 * filaments); 512 up to 4000 nodes, else 1024; batches with MF_FLAG_DYNAMIC_LS
 * use at least 512 unless the size was set here;
 * multifil_jax_b200.autotune measures and sets the best one; threads = 0
 * restores the default.  MF_ERR_INVALID when the lattice does not fit in
 * shared memory at that size. */
int mf_tune_threads_mode(mf_ctx* ctx, int32_t topo_id, int32_t precise, int32_t threads);
int mf_tune_threads(mf_ctx* ctx, int32_t topo_id, int32_t threads);

/* Device bytes the library needs for a batch (admission control). */
int mf_workspace_bytes(mf_ctx* ctx, const mf_batch* batch, uint64_t* bytes);

/* Allocation-free variant of mf_run_batch (no counterpart in the reference:
 * it exists for callers of this library, not of the reference API).
 * For callers that must not have the library allocate device memory on the
 * call path: a framework that owns all HBM through its own allocator and
 * budget.  All per-call scratch (per-condition workspaces and the launch
 * descriptor table) comes from one 8 MiB array compiled into the library
 * (present on every device that loads it, until process exit); the call
 * never allocates.  A batch whose scratch exceeds 8 MiB is rejected with
 * MF_ERR_NOMEM and a message naming both sizes (at 2x2 about 70 conditions
 * fit).  Batched single-launch path only: MF_FLAG_PLAIN and chunk_steps > 0
 * are rejected, as are negative n_newton / n_cg (MF_ERR_INVALID).
 * The call blocks the calling host thread: it reads n_steps, K_lat, nu and dt
 * from the device with synchronous copies before launching (so those four
 * arrays must hold their values when the call is made, not merely be ordered
 * on `stream`), and it returns only after `stream` has synchronised.  It can
 * therefore not be recorded inside a stream capture.  The array's device
 * address is resolved once per device per process, on the first call with
 * that device current; a process that resets the device (cudaDeviceReset)
 * must not call this entry point afterwards.  Every call reuses the same
 * array (the region a call uses is zeroed before its kernels run); calls that
 * overlap on the GPU race on it and must be serialised by the caller. */
int mf_run_batch_static(mf_ctx* ctx, const mf_batch* batch, void* stream);

/* ---- one step of caller-owned states (the public timestep split) ------- */
/* Phases of mf_step_states (reference timestep.py:65-199 and the functions it
 * calls).  MF_PHASE_KINETICS is kinetics_step (nearest sites, tropomyosin and
 * crossbridge transitions); MF_PHASE_TIMESTEP is timestep (kinetics, then the
 * equilibrium solve); MF_PHASE_EQUILIBRIUM alone is solve_equilibrium
 * (kernels/solver.py:663-771); MF_PHASE_NEAREST alone is
 * update_nearest_neighbors (kernels/geometry.py:186-262). */
#define MF_PHASE_NEAREST 1
#define MF_PHASE_TRANSITIONS 2
#define MF_PHASE_EQUILIBRIUM 4
#define MF_PHASE_KINETICS (MF_PHASE_NEAREST | MF_PHASE_TRANSITIONS)
#define MF_PHASE_TIMESTEP (MF_PHASE_KINETICS | MF_PHASE_EQUILIBRIUM)

/* B states of one lattice held by the caller in the reference's State layout
 * (core/state.py:69-113), row-major [B, ...] device arrays, updated in place.
 * Float32 arithmetic (the reference's).  Drivers follow resolve_value
 * (core/state.py:331-343): NULL or NaN entries take the constant from the
 * parameter row. */
typedef struct {
    int32_t B;
    int32_t topo_id;
    int32_t phases;            /* MF_PHASE_* bits */
    int32_t flags;             /* 0 or MF_FLAG_ORIGINAL_PRNG */
    float dt;                  /* timestep (ms) of the transition tables */
    int32_t n_newton;          /* Newton cap (solve_equilibrium's n_newton_steps) */
    int32_t n_cg;              /* CG iterations per Newton step */
    float* thick_axial;        /* [B*n_thick*n_crowns] thick.axial */
    int8_t* xb_states;         /* [B*X] thick.xb_states */
    int32_t* xb_bound_to;      /* [B*X] thick.xb_bound_to (-1 unbound) */
    int32_t* xb_nearest_bs;    /* [B*X] thick.xb_nearest_bs */
    float* xb_distances;       /* [B*X*2] thick.xb_distances (axial, radial) */
    float* thin_axial;         /* [B*S] thin.axial */
    int8_t* tm_states;         /* [B*S] thin.tm_states */
    int32_t* thin_bound_to;    /* [B*S] thin.bound_to (-1 unbound) */
    uint32_t* keys;            /* [B*2] jax.random key; advanced by the transitions phase */
    const float* params;       /* [B*44] DynamicParams rows (the constants) */
    const float* pCa;          /* [B] drivers or NULL */
    const float* z_line;       /* [B] or NULL */
    const float* lattice_spacing; /* [B] or NULL */
    const float* K_lat;        /* [B] effective lattice stiffness (x n_thick) or NULL: fixed spacing */
    const float* d_ref;        /* [B] reference spacing (with K_lat) */
    float* residual_out;       /* [B] or NULL: max |F| after the solve (pN) */
    float* ls_out;             /* [B] or NULL: lattice spacing after the solve */
    int32_t* iters_out;        /* [B] or NULL: Newton iterations */
    int32_t* status_out;       /* [B] or NULL: MF_STATUS_* bits */
    int32_t n_pops, pop_flags, label_stride; /* subpopulations, as in mf_batch */
    const float* pop_params;
    const float* pop_frac;
    const int8_t* xb_label;
    const int8_t* tm_label;
    const float* u_thin;       /* test hook: [B*S] injected uniforms or NULL */
    const float* u_xb;         /* test hook: [B*X] injected uniforms or NULL */
} mf_state_batch;

/* Run the selected phases on every state of the batch (one CTA per state).
 * Replaces the reference's kinetics_step / timestep / solve_equilibrium /
 * update_nearest_neighbors (timestep.py:65-199, kernels/solver.py:663-771,
 * kernels/geometry.py:186-262) for B states at once.  The transition
 * tables are built on every call that samples.  Returns after `stream` has
 * synchronised. */
int mf_step_states(mf_ctx* ctx, const mf_state_batch* sb, void* stream);

/* Test hook: the transition tables a condition's kernel builds for one
 * DynamicParams row `params` (host, 44 floats) at (pCa, lattice spacing d)
 * and timestep dt (ms), with the arithmetic of the precision mode in `flags`
 * (MF_FLAG_PRECISE or 0).  They are the reference's expm_pade6_batch results
 * (kernels/transitions.py:99-190) on its tropomyosin generators (:434-513),
 * crossbridge bin grid (:807-922) and absorbing-chain grid (:1029-1078),
 * in the form the kernel keeps them.  Outputs (host, any may be NULL):
 *   cum_tm [27*4*4]        cumulative rows (jnp.cumsum order) of the 27
 *                          tropomyosin tables, configuration-major;
 *   cum_xb [2*n_bins*6*6]  cumulative rows of the crossbridge tables, row
 *                          block = permissiveness * n_bins + bin;
 *   pabs   [2*n_bins*3]    P_abs[3,4], P_abs[2,0], P_abs[3,0] of each block.
 * Allocates and synchronises the device (a test hook, not a hot path). */
int mf_transition_tables(mf_ctx* ctx, int32_t topo_id, const float* params, float pCa, float d, float dt,
                         int32_t flags, float* cum_tm, float* cum_xb, float* pabs);

/* jax.random on the host: key = PRNGKey(seed); keys_out[2*i..] = split(key, n)[i].
 * partitionable=1: JAX >= 0.5 layout; 0: original layout. */
int mf_prng_split(uint32_t k0, uint32_t k1, int32_t n, int32_t partitionable, uint32_t* keys_out);
/* uniform(key, (n,)) float32 on the host (for tests of the device generator). */
int mf_prng_uniform(uint32_t k0, uint32_t k1, int32_t n, int32_t partitionable, float* out);

/* ---- continuous-batching server (serving form) ------------------------ */
typedef struct {
    int32_t topo_id;
    int32_t n_steps;
    float dt;
    uint32_t key[2];
    float params[MF_N_PARAMS];
    float pCa, z_line, lattice_spacing;   /* constant drivers */
} mf_request;

/* Start a server on ctx with a device-memory budget (bytes) for resident
 * slots and a chunk of steps per scheduling tick.  mf_server_start runs every
 * request in float32 mode (the reference's arithmetic); mf_server_start_mode
 * with precise = 1 runs them with MF_FLAG_PRECISE. */
int mf_server_start(mf_ctx* ctx, uint64_t mem_budget, int32_t chunk_steps, int32_t max_slots);
int mf_server_start_mode(mf_ctx* ctx, uint64_t mem_budget, int32_t chunk_steps, int32_t max_slots,
                         int32_t precise);
/* Queue a request; returns its id.  MF_ERR_NOMEM if it can never fit. */
int mf_server_submit(mf_ctx* ctx, const mf_request* req, uint64_t* req_id);
/* Run up to max_ticks scheduling ticks (admit, launch one chunk, retire). */
int mf_server_step(mf_ctx* ctx, int32_t max_ticks, int32_t* n_active, int32_t* n_queued);
/* Fetch a finished request's metrics (host [52*n_steps]); MF_ERR_BUSY if not done. */
int mf_server_poll(mf_ctx* ctx, uint64_t req_id, float* metrics_host, int32_t* status, double* t_submit,
                   double* t_done);
int mf_server_cancel(mf_ctx* ctx, uint64_t req_id);
int mf_server_stop(mf_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* MULTIFIL_B200_H */
