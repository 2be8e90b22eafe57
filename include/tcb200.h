/*
 * tcb200.h - C ABI of libtcb200.so, the B200 (sm_100a) kernels behind the
 * torchcor_b200 package: TorchCor's monodomain time step (ionic update with
 * stimulus injection and activation/repolarisation tracking, P1 assembly into
 * CSR, Jacobi-preconditioned CG).
 *
 * Conventions
 *  - Every entry point returns an int status: TCB_OK (0) or a negative
 *    TCB_E* code; tcb_status_string() names it and tcb_last_error() returns
 *    the message of the last failure on the calling thread.
 *  - Device pointers are plain pointers to memory the caller allocated (the
 *    Python layer uses torch tensors); the library never frees caller memory.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *  - Per-node arrays have `n_pad` entries (n_nodes rounded up to 128); the
 *    sparse matrices are stored as CSR (patterns bit-identical to the
 *    reference's coalesced COO -> CSR) and, for the solver, as sliced ELL with
 *    slice height 32 (TCB_SLICE) sharing one column array.
 *
 * Each declaration names the reference (TorchCor 0.1.8) interface it replaces.
 */
#ifndef TCB200_H
#define TCB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TCB_OK 0
#define TCB_EINVAL (-1)     /* invalid argument (size, pointer, model id) */
#define TCB_ECUDA (-2)      /* a CUDA runtime call failed */
#define TCB_ETIMEOUT (-3)   /* a bounded device-side wait gave up */
#define TCB_ENOMEM (-4)     /* host allocation failed */
#define TCB_ERANGE (-5)     /* size beyond a stated limit */

#define TCB_SLICE 32        /* sliced-ELL slice height (one warp) */
#define TCB_MAX_STIMULI 32  /* stimuli per simulation (one bit each) */

/* ionic model ids */
#define TCB_MODEL_MS 1      /* ModifiedMS2v / MitchellSchaeffer (dimensional, mV) */
#define TCB_MODEL_TTP 2     /* TenTusscherPanfilov */
#define TCB_MODEL_CRN 3     /* CourtemancheRamirezNattel */

int tcb_version(void);
const char* tcb_status_string(int status);
/* Copies the last error message of this thread into buf (truncated). */
int tcb_last_error(char* buf, int64_t len);

/* ---------------------------------------------------------------- pattern
 * CSR pattern of the assembled P1 operator plus a deterministic scatter map.
 * Replaces the Python-list COO build + coalesce of
 * torchcor/core/assemble.py:217-248 (tets) and :67-96 (triangles): the CSR
 * (rowptr, col) equals coalesce(COO).to_sparse_csr() of the reference; each
 * slot's contributions are listed in the reference's COO order
 * ((a*k+b)*E + e ascending), as flat indices e*k*k + a*k + b into the
 * (E, k, k) local-matrix array.  Host code (elems in host memory).
 */
int tcb_pattern_size(const int32_t* elems, int64_t n_elems, int32_t k, int64_t n_nodes, int64_t* nnz);
int tcb_pattern_build(const int32_t* elems, int64_t n_elems, int32_t k, int64_t n_nodes,
                      int32_t* rowptr /* n_nodes+1 */, int32_t* col /* nnz */,
                      int32_t* slot_ptr /* nnz+1 */, int32_t* slot_src /* k*k*n_elems */,
                      int32_t* diag /* n_nodes: slot of (i,i) */);
/* Sliced-ELL layout of a CSR pattern: slice_ptr[n_slices+1] entry offsets
 * (each slice holds 32 * its widest row entries).  Host code. */
int tcb_sell_layout(const int32_t* rowptr, int64_t n_rows, int64_t* slice_ptr, int64_t* n_entries);

/* ---------------------------------------------------------------- device ingest
 * Mesh ingest on the device (replaces MeshReader's np.loadtxt, mesh.py:26-63, and
 * the COO build + coalesce of assemble.py:217-248 for device-resident elements).
 * Text: tcb_text_scratch(n) int64 words of scratch; tcb_text_newlines gives the
 * newline count (pos == NULL) or positions; tcb_text_parse parses `rows` lines from
 * line `first_line` (0-based), skipping `skip` fields and reading `cols` fields as
 * int64 (as_int) or correctly rounded float64 into out[rows][cols]; rows it cannot
 * parse exactly are counted in *bad (device int64, caller-zeroed).
 * Pattern: tcb_pattern_device with work = 2*(N+1) int64, keys = k*k*E uint64,
 * iwork = 2*N+1 int32 returns nnz; tcb_pattern_device_emit writes the same arrays
 * as tcb_pattern_build (device pointers). */
int64_t tcb_text_scratch(int64_t n_bytes);
int tcb_text_newlines(const char* text, int64_t n_bytes, int64_t* scratch, int64_t* pos, int64_t cap, int64_t* count,
                      void* stream);
int tcb_text_parse(const char* text, int64_t n_bytes, const int64_t* newlines, int64_t n_newlines, int64_t first_line,
                   int64_t rows, int32_t skip, int32_t cols, int32_t as_int, void* out, int64_t* bad, void* stream);
int tcb_pattern_device(const int32_t* elems, int64_t n_elems, int32_t k, int64_t n_nodes, int64_t* work,
                       uint64_t* keys, int32_t* iwork, int64_t* nnz, void* stream);
int tcb_pattern_device_emit(const int64_t* work, const uint64_t* keys, int64_t n_elems, int32_t k, int64_t n_nodes,
                            int32_t* rowptr, int32_t* col, int32_t* slot_ptr, int32_t* slot_src, int32_t* diag,
                            void* stream);

/* ---------------------------------------------------------------- assembly
 * Element matrices of P1 tetrahedra (k=4) or surface triangles (k=3).
 * Replaces Matrices3D.construct_local_matrices (assemble.py:202-215) and
 * Matrices3DSurface (assemble.py:99-145), with the conductivity tensor of
 * Conductivity.calculate_sigma (conductivity.py:64-67) formed in the kernel:
 * sigma = st*I + (sl-st) f f^T per element.
 * Outputs: ke[E*k*k] stiffness, mw[E] = volume/20 (tets) or area/12 (tris).
 */
int tcb_assemble_local(int32_t k, const float* nodes /* N*3, mm */, const int32_t* elems, int64_t n_elems,
                       const float* sl, const float* st, const float* fibres /* E*3 */,
                       float* ke, float* mw, void* stream);
/* Sum element contributions into CSR values in the scatter map's order
 * (replaces the coalesce of assemble.py:233-248). m_val gets mw*pattern. */
int tcb_assemble_gather(int32_t k, const int32_t* slot_ptr, const int32_t* slot_src, int64_t nnz,
                        const float* ke, const float* mw, float* k_val, float* m_val, void* stream);
/* Monodomain.assemble system values (monodomain.py:93-106, preconditioner.py:9-27):
 * k_val /= chi (in place); a_val = m*cm + (k*dt)*theta; k_rhs = ((1-theta)*dt)*k;
 * d_inv[i] = 1/a(i,i) (0 for i >= n_nodes up to n_pad).  *a_split (device int32, caller sets 1)
 * is cleared if any a_val differs from fp32(fp32(m*cm) + k_rhs); it stays 1 for theta = 0.5, and the
 * solver then rebuilds A from M and k_rhs instead of streaming it. */
int tcb_assemble_system(int64_t nnz, int64_t n_nodes, int64_t n_pad, const int32_t* diag, float* k_val,
                        const float* m_val, double chi, double cm, double dt, double theta,
                        float* a_val, float* k_rhs, float* d_inv, int32_t* a_split, void* stream);
/* int16 column offsets (col - row) of a sliced-ELL column array; *max_abs
 * (device int32, caller-zeroed) receives max |col - row|.  The offsets are
 * usable when that maximum is below 32768.  Replaces nothing in the
 * reference (index compression of the solver's matrix stream). */
int tcb_sell_delta(int64_t n_rows, const int64_t* slice_ptr, int64_t n_slices, const int32_t* sell_col,
                   int16_t* delta, int32_t* max_abs, void* stream);
/* Repack up to 4 CSR value arrays (and the columns) into sliced ELL; padding
 * entries get column = own row and value 0. */
int tcb_sell_pack(int64_t n_rows, const int32_t* rowptr, const int32_t* col, const int64_t* slice_ptr,
                  int64_t n_slices, int32_t n_vals, const float* const* vals /* host array of device ptrs */,
                  int32_t* sell_col, float* const* sell_vals, void* stream);

/* ---------------------------------------------------------------- ionic
 * Ionic models.  `params` is a host array of doubles in the order of
 * tcb_model_params(model) (the Python-level attributes of the reference
 * class, plus dt); state is (n_states x n_pad) structure-of-arrays.
 * Replaces ModifiedMS2v (ionic/ModifiedMS2v.py:4-44), TenTusscherPanfilov
 * (ionic/TenTusscherPanfilov.py:6-454), CourtemancheRamirezNattel
 * (ionic/CourtemancheRamirezNattel.py:5-444).
 */
const char* tcb_model_params(int32_t model);       /* comma-separated parameter names */
const char* tcb_model_states(int32_t model);       /* comma-separated state names (row order) */
int tcb_model_layout(int32_t model, const double* params, int64_t* n_states, int64_t* table_floats);
/* Layout of lookup table `index` (0, 1, 2 in the reference's construction
 * order: TTP V, CaSS, V-Ek; CRN Cai... listed as V, Cai, fn) inside the model's
 * table array: rows x stride floats (stride = ncol rounded up to 4, or 1)
 * starting at float offset `offset`.  TCB_ERANGE past the last table. */
int tcb_model_table_info(int32_t model, int32_t index, int64_t* rows, int32_t* ncol, int32_t* stride,
                         int64_t* offset);
/* Instances of the fused per-step ionic kernel for `model` (no counterpart in the reference: launch
 * shapes an autotuner chooses between, all in the reference's per-node order of operations): *count
 * instances; instance `variant` (1..count, 0 = the default) handles *nodes_per_thread consecutive
 * nodes per thread (structure-of-arrays state moved as 4-, 8- or 16-byte vectors) with the register
 * budget of *blocks_per_sm 256-thread blocks per SM; *fast_math = 1 if it divides and takes
 * logarithms with the hardware approximations (a few ulp), 0 for IEEE division and logf;
 * *staged = 1 for the persistent form that bulk-copies the next tile of nodes into shared memory
 * while it computes the current one.  TCB_ERANGE past the last instance. */
int tcb_ionic_variant(int32_t model, int32_t variant, int32_t* count, int32_t* nodes_per_thread,
                      int32_t* blocks_per_sm, int32_t* fast_math, int32_t* staged);
/* construct_tables (TTP :197-318, CRN :212-328); no-op for MS.  `tables` must be
 * 16-byte aligned (TCB_EINVAL otherwise), as in every call that reads it. */
int tcb_model_tables(int32_t model, const double* params, float* tables, void* stream);
/* initialize(n_nodes): fill state rows and V with the initial values */
int tcb_model_init(int32_t model, const double* params, float* state, int64_t n_pad, float* v, void* stream);
/* Per-node parameters of `model` (comma-separated names, "" if none): TTP "GCaL,GKr,GKs,Gto" — the
 * reference's per-node conductance tensors (TenTusscherPanfilov.py:327-330), which initialize() fills
 * uniformly and a caller may overwrite node by node.  A node_params array holds them as rows of
 * n_pad floats in this order; NULL means the uniform values of the *_init parameters. */
const char* tcb_model_node_params(int32_t model);
/* differentiate(V): dv = -Iion and the state update, for n nodes (`tables` 16-byte aligned;
 * node_params as above, or NULL) */
int tcb_model_differentiate(int32_t model, const double* params, const float* tables, const float* node_params,
                            float* state, int64_t n_pad, int64_t n, const float* v, float* dv, void* stream);

/* ---------------------------------------------------------------- time loop
 * One simulation on the device.  Replaces Monodomain.step / solve's loop
 * (monodomain.py:109-196) with ConjugateGradient.solve (solver.py:40-76).
 * Step n (1-based) reads the membrane potential ring x[(n-1)%3] (solution of
 * step n-1) and x[(n+1)%3] (the one before) and writes x[n%3].
 */
typedef struct tcb_mono {
    int64_t n_nodes, n_pad, n_slices, nt;
    int32_t model, n_states;
    /* matrix (sliced ELL, TCB_SLICE rows per slice) */
    const int64_t* slice_ptr;
    const int32_t* col;
    const int16_t* col_delta; /* optional: col - row as int16 (all |col-row| < 32768), or NULL */
    const float* m_val;      /* M */
    const float* k_val;      /* ((1-theta)*dt) * K/chi */
    const float* a_val;      /* Cm*M + theta*dt*K/chi */
    const float* d_inv;      /* 1/diag(A) */
    /* ionic */
    float* state;
    const float* tables;     /* 16-byte aligned (TCB_EINVAL otherwise); unused for MS */
    /* vectors (n_pad each; x is 3*n_pad) */
    float* x;
    float* bprime;
    float* r;
    float* p;
    float* ap;
    float* z;                /* batch solver only: z = D r of every row, n_pad */
    float* p2;               /* batch solver only: second search-direction buffer, n_pad */
    float* at;
    float* rt;
    float* snapshots;        /* row j = solution of step j*per_frame, n_nodes per row; may be NULL;
                                with snap_ring > 0 a ring of snap_ring rows: frame j goes to row j % snap_ring */
    /* stimuli and schedule */
    const uint32_t* stim_bits;   /* per node: bit s set if the node is in stimulus s */
    const float* step_t;         /* [nt+1]: fp32 of the accumulated time t_n */
    const uint32_t* step_stim;   /* [nt+1]: bit s set if stimulus s is on at step n */
    float stim_amp[TCB_MAX_STIMULI];
    /* solver */
    double a_tol, r_tol;
    int32_t max_iter, linear_guess, at_rt, per_frame;
    int32_t a_split;         /* 1 if every a_val == fp32(fp32(m_val*cm) + k_val) (tcb_assemble_system's check) */
    float cm, dt;
    int32_t snap_ring;       /* 0: snapshots holds every frame; > 0: rows in the snapshot ring (the
                                caller copies each frame out before it is overwritten) */
    /* launch shapes (no counterpart in the reference; chosen by measurement) */
    int32_t ionic_variant;   /* ionic kernel instance, 1..count of tcb_ionic_variant(); 0 = the default.
                                Instances with more than one node per thread need x, state, bprime, at, rt
                                and stim_bits aligned to the vector (else the first one-node instance runs) */
    int32_t cg_per_sm;       /* blocks per SM of the CG kernel that keeps rows in shared memory: 0 = the
                                most whose rows fit (2, else 1); 1 or 2 pins it */
    int32_t fused_step;      /* 1: each step is one launch, the ionic update fused into the CG kernel that
                                keeps rows in shared memory (where that kernel applies: int16 column
                                offsets, rows that fit); 0: the ionic and CG kernels as two launches.
                                The values are the same either way */
    /* device bookkeeping (caller-allocated, zero-initialised) */
    int32_t* step_iters;     /* [nt+1] CG iterations of each step */
    int32_t* counter;        /* [4]: next step, error code, 2 spare */
    double* scratch;         /* >= tcb_mono_scratch_doubles() */
    uint32_t* barrier;       /* [4] grid-barrier words, zeroed, 8-byte aligned */
    /* model parameters (host) */
    const double* params;
    /* per-node model parameters (tcb_model_node_params), n_pad floats per row, or NULL */
    const float* node_params;
} tcb_mono;

int64_t tcb_mono_scratch_doubles(void);
/* Run steps [step_begin, step_end) (1-based, step_begin must equal the device
 * counter).  Non-convergence is not an error (n_iter == max_iter), as in the
 * reference. */
int tcb_mono_run(const tcb_mono* m, int64_t step_begin, int64_t step_end, void* stream);
/* The linear solves alone for steps [step_begin, step_end): right-hand side
 * M b' - K' u, linear-extrapolation guess from the solution ring, Jacobi-PCG
 * (replaces ConjugateGradient.solve, solver.py:40-76, where the caller supplies
 * b' and the matrices); the ionic kernel is not run.  Used for the extracellular
 * potential recovery (monodomain.py:254-286) with M := K(sigma_i), b' := -Vm,
 * K' := 0, A := K(sigma_i + sigma_e). */
int tcb_mono_cg_run(const tcb_mono* m, int64_t step_begin, int64_t step_end, void* stream);
/* Like tcb_mono_run, recording CUDA events around every kernel on `stream`;
 * adds the summed device times (ms) of the ionic and CG kernels to
 * ms_ionic / ms_cg (for roofline accounting; costs one event pair per launch).
 * A fused step's single kernel counts as CG time (ms_ionic gets nothing). */
int tcb_mono_profile(const tcb_mono* m, int64_t step_begin, int64_t step_end, void* stream, double* ms_ionic,
                     double* ms_cg);
/* Which CG kernel tcb_mono_run launches for this simulation on the current
 * device: 2 = the fused step (ionic update inside the CG kernel that keeps rows
 * in shared memory), 1 = that CG kernel after a separate ionic launch, 0 = the
 * streaming kernel; negative = error status.  No counterpart in the reference
 * (used to label measurements). */
int tcb_mono_cg_kernel(const tcb_mono* m);
/* tcb_mono_run without scratch arguments (no counterpart in the reference):
 * for callers that cannot allocate device memory at the call site (a host
 * application that owns the device memory pool and forbids allocations after
 * start-up, or a latency-critical caller that cannot afford cudaMalloc's
 * implicit synchronisation).  The CG kernel's reduction partials and barrier
 * words live in a static device array of the library (64 KiB + 16 B per GPU,
 * held until exit); m->scratch and m->barrier are ignored.  Allocates nothing.
 * The first call on a device looks up the array's address (make it before any
 * stream capture).  Calls whose kernels overlap on the GPU share the array and
 * race: serialise them.  A launch needing more than 2048 CG blocks is
 * rejected with TCB_ERANGE. */
int tcb_mono_run_noalloc(const tcb_mono* m, int64_t step_begin, int64_t step_end, void* stream);
/* Activation/repolarisation update and snapshot for the final step. */
int tcb_mono_finish(const tcb_mono* m, void* stream);
/* Device error word after a run (TCB_OK or TCB_ETIMEOUT); synchronises the stream. */
int tcb_mono_check(const tcb_mono* m, void* stream);

/* ---------------------------------------------------------------- batches
 * Many simulations stepping together (no counterpart in the reference, which
 * runs one simulation per process): one ionic launch per model and one
 * persistent CG launch per step cover every simulation; each keeps its own
 * arrays (a tcb_mono each, with the z and p2 buffers set), step counter,
 * schedule, tolerances and iteration count (per-simulation convergence).
 * Simulations may be at different steps; one whose counter is outside
 * [1, nt] is skipped.  The plan is rebuilt (tcb_batch_prepare) whenever the
 * set of simulations changes; the workspace is caller-allocated device memory
 * of tcb_batch_workspace_bytes(n) bytes (n <= 1024).
 */
typedef struct tcb_batch_plan {
    void* workspace;
    int32_t n_sims, cg_blocks, cg_smem, n_groups;
    int32_t group_model[3];
    int32_t group_shared[3];
    int32_t cg_variant;       /* CG kernel: 1 / 2 = streaming sized for 1 / 2 blocks per SM,
                                 3 = ELL streams staged in shared memory by bulk copies */
    int32_t cg_stage_bytes;   /* staging bytes per warp and stage (variant 3) */
    int32_t cg_stage_ok;      /* 1 if every ELL array allows bulk copies (16-byte aligned) */
    int32_t cg_flags;         /* combination (int16 columns 4, A rebuilt 2, linear guess 1) all
                                 simulations share, or -1: the CG kernel is specialised on it */
    int64_t group_tiles[3];
    int64_t total_slices;
    char group_consts[3][1024];
    int32_t ionic_tiles_per_block;   /* batched ionic kernel: 128-node tiles each block walks;
                                        0 = sized from each model group (at most 8, at least
                                        16 blocks per SM where the group is large enough) */
    int32_t ionic_blocks_per_sm;     /* its register budget: 4, 6, 8 or 12 blocks of 128
                                        threads per SM; 0 = 8 with CRN groups, else 12 (the
                                        staged form: 4, 6 or 8; 0 = 6) */
    int32_t ionic_staged;            /* 1: the staged form (each block's next tile copied into
                                        shared memory by bulk copies while it computes one) */
    int32_t ionic_stage_ok;          /* 1 if every per-node array allows bulk copies (16-byte
                                        aligned) */
} tcb_batch_plan;

int64_t tcb_batch_workspace_bytes(int32_t n_sims);
int tcb_batch_prepare(const tcb_mono* sims, int32_t n_sims, void* workspace, int64_t bytes, tcb_batch_plan* plan);
/* Switch a prepared plan to CG kernel variant 1, 2 or 3 (see cg_variant) and the
 * matching grid; TCB_ERANGE if that variant cannot be resident or (3) the arrays
 * do not allow bulk copies.  No counterpart in the reference (a tuning knob of
 * this implementation). */
int tcb_batch_set_cg(tcb_batch_plan* plan, int32_t variant);
/* The plan's batched ionic launch: tiles per block, 0 (sized from the groups, the
 * default after tcb_batch_prepare) or 1..64 for every group; the kernel instance's
 * register budget, 0 (default) or 4, 6, 8, 12 blocks per SM (4, 6, 8 staged); staged
 * 0 or 1 (TCB_ERANGE if the arrays do not allow it, see ionic_stage_ok).  TCB_EINVAL for
 * other values.  The staged form takes the single-simulation default's division policy
 * (hardware division for TTP and CRN), so its results differ from the unstaged form's
 * by rounding only; tiles and budget do not change results.  No counterpart in the
 * reference (tuning knobs of this implementation). */
int tcb_batch_set_ionic(tcb_batch_plan* plan, int32_t tiles_per_block, int32_t blocks_per_sm, int32_t staged);
/* `steps` batch steps: every listed simulation whose counter is in [1, nt] advances one step each. */
int tcb_batch_run(const tcb_batch_plan* plan, int64_t steps, void* stream);
/* Device error word of the batch (synchronises the stream). */
int tcb_batch_check(const tcb_batch_plan* plan, void* stream);

#ifdef __cplusplus
}
#endif
#endif
