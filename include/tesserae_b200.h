/*
 * tesserae_b200.h -- C ABI of libtesserae_b200.so, the B200 (sm_100a) explicit
 * material-point-method step of Tesserae.jl.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and returns
 * an int status (TB_OK = 0, negative on error; tb_last_error() gives the message).
 * No C++ exception crosses this boundary.
 *
 * All particle, grid, partition and weight arrays are CALLER-OWNED device memory
 * (Julia CuArrays via `pointer`, or cudaMalloc/torch in tests). The library owns
 * only its scratch (sort buffers, scan partials, host-staging buffers), kept in
 * the tb_ctx, and never frees caller memory.
 *
 * Precision forms (the `_f64` / `_f32` suffix):
 *   _f64  "plain": every array is double. Drop-in for `gpu_preserve` data.
 *   _f32  "mixed": every array is float EXCEPT the deformation gradient F,
 *         which stays double; weights, P2G and G2P run in FP32 (each P2G lane
 *         sums its particles' contributions to a node in plain FP32 registers;
 *         the at most 9 partial sums that reach a node are added, in FP32 on
 *         the 3D paths and in FP64 on the 2D and boundary-block ones, before
 *         the one global atomic per node), and F update, det F and log J run in
 *         FP64. Drop-in for `gpu` (Float32-cast) data plus an FP64 F array.
 *
 * Index conventions follow the reference (Julia, column-major, 1-based):
 *   block ids are 1-based linear ids over nblocks(mesh), 0 = outside the mesh
 *     (Tesserae.jl src/Parallel/gpu_block_strategy.jl:46-53);
 *   particleindices hold 1-based particle ids, block-contiguous, ascending
 *     block id then ascending particle id (the reference CPU strategy's order,
 *     src/Parallel/cpu_block_strategy.jl:174-190; its GPU strategy leaves the
 *     order inside a block unspecified, gpu_block_strategy.jl:133-140);
 *   offsets are 0-based exclusive prefix sums of counts, length nblocks+1.
 *
 * Tensor components are column-major: 3D grad_v/F/B = (11,21,31,12,22,32,13,23,33),
 * 2D = (11,21,12,22). Symmetric sigma = (11,21,31,22,32,33) in 3D, (11,21,22) in 2D
 * (Tensorial.jl SymmetricSecondOrderTensor independent-component order).
 */
#ifndef TESSERAE_B200_H
#define TESSERAE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TB_OK 0
#define TB_ERR_ARG (-1)         /* invalid argument (null pointer, bad size, bad enum) */
#define TB_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define TB_ERR_CAPACITY (-3)    /* a size exceeds the Int32 capacity of the partition */
#define TB_ERR_UNSUPPORTED (-4) /* combination not supported (e.g. dim 1) */
#define TB_ERR_DEVICE (-5)      /* a kernel reported an error status (e.g. a window left its block tile) */

/* Uniform Cartesian mesh (reference: src/Mesh/cartesian.jl:38-102).
 * xmin, h and h_inv are given in FP64 exactly as the caller's mesh stores them;
 * the _f32 entry points cast each to float (src/adapt.jl:53-57: Float32(h_inv),
 * not inv(Float32(h))), so block ids match the Float32 reference bit for bit. */
typedef struct tb_mesh {
    int32_t dim;          /* 2 or 3 */
    int32_t block_log2;   /* cells per block edge = 1 << block_log2 (reference default 2) */
    int64_t n_nodes[3];   /* nodes per axis (cells + 1); unused axes = 1 */
    double xmin[3];       /* first node coordinate per axis */
    double h;             /* spacing */
    double h_inv;         /* stored inverse spacing */
} tb_mesh;

/* Basis kinds on the hot path (src/Basis/bspline.jl, gimp.jl, wls.jl). */
enum tb_basis_kind {
    TB_BSPLINE_QUADRATIC = 0,     /* BSpline(Quadratic()) */
    TB_UGIMP = 1,                 /* uGIMP() */
    TB_WLS_BSPLINE_QUADRATIC = 2, /* WLS(BSpline(Quadratic())), MLS-MPM */
    TB_WLS_UGIMP = 3,             /* WLS(uGIMP()) */
    TB_KC_BSPLINE_QUADRATIC = 4,  /* KernelCorrection(BSpline(Quadratic())) (src/Basis/kernelcorrection.jl) */
    TB_KC_UGIMP = 5               /* KernelCorrection(uGIMP()) */
};

/* Constitutive models of the recognised G2P equation sets (tb_step_params.material). */
enum tb_material_kind {
    TB_MATERIAL_NEOHOOKEAN = 0, /* README.md:85: sigma = (mu (F F^T - I) + lambda log J I) / J, V = V0 det F */
    TB_MATERIAL_FLUID = 1,      /* weakly compressible fluid p = -K (J - 1), K = lambda, V = V0 det F */
    TB_MATERIAL_VONMISES = 2    /* docs/src/gpu.md:202-392 (Taylor impact): Hencky elasticity, von Mises
                                   yield with linear hardening, return map in principal logarithmic
                                   stretches; V = det(dF) V */
};

/* Transfer schemes of the recognised @P2G/@G2P equation sets. */
enum tb_transfer_kind {
    TB_TRANSFER_FLIP = 0, /* README.md:71-87: v += sum w (v_i - vn_i) (flip_alpha blends PIC) */
    TB_TRANSFER_APIC = 1  /* docs/src/transfer.md:166-186: v = sum w v_i, B = sum w v_i (x) (x_i - x_p) */
};

/* Particle state as structure-of-arrays component pointers. Scalar type is T
 * (double for _f64, float for _f32) except F, which is always double.
 * Optional arrays may be NULL; the matching scalar in tb_step_params is used. */
typedef struct tb_particles {
    int64_t n;
    void* x[3];       /* position (required) */
    void* v[3];       /* velocity */
    void* V;          /* current volume */
    void* m;          /* optional per-particle mass */
    void* l;          /* optional per-particle uGIMP length (absolute units) */
    void* grad_v[9];  /* velocity gradient, column-major */
    void* sigma[6];   /* symmetric Cauchy stress */
    void* F[9];       /* deformation gradient, column-major, ALWAYS double */
    void* B[9];       /* APIC affine matrix, column-major (TB_TRANSFER_APIC only) */
    void* V0;         /* optional per-particle initial volume */
    void* mu;         /* optional per-particle Lame mu */
    void* lambda;     /* optional per-particle Lame lambda */
    void* eps_p;      /* equivalent plastic strain (TB_MATERIAL_VONMISES only) */
    void* Cp_inv[6];  /* inverse plastic right Cauchy-Green tensor, symmetric (TB_MATERIAL_VONMISES only) */
} tb_particles;

/* Grid fields as SoA component pointers (scalar type T), each of length
 * prod(n_nodes), column-major node order (src/Grids/grid.jl:70-78).
 *
 * Block-sparse grid (SpGrid, src/Grids/sparray.jl, spindices.jl): with
 * block_numbering set, the fields store only the active node blocks (blocks of
 * (1 << mesh.block_log2)^dim nodes, node block of node i = i >> block_log2 per
 * axis, nblocks(mesh) of them): node I of block B lives at
 *   (block_numbering[B] - 1) * blocklength + (I's column-major index inside B)
 * (the reference's storageindex), and a node of an inactive block
 * (block_numbering[B] == 0) reads as zero and takes no scatter.
 * tb_update_sparsity_* fills block_numbering, active_blocks and *nactive from
 * the particle positions; the fused steps update them every step. Leave the
 * four fields zero for a dense grid. */
typedef struct tb_grid {
    void* m;
    void* mv[3];
    void* f[3];
    void* v[3];
    void* vn[3];
    int32_t* block_numbering; /* [nblocks(mesh)] device: 0 inactive, k >= 1 storage block k */
    int32_t* active_blocks;   /* [nblocks(mesh)] device: 1-based id of the node block stored as block k at [k-1] */
    int32_t* nactive;         /* [2] device: active node blocks at [0] (scratch at [1]) */
    int64_t capacity;         /* nodes each field array holds (a multiple of blocklength) */
} tb_grid;

/* The GPUBlockStrategy arrays (src/Parallel/gpu_block_strategy.jl:10-22). */
typedef struct tb_partition {
    int32_t* blockids;        /* [n] */
    int32_t* counts;          /* [nblocks] */
    int32_t* offsets;         /* [nblocks + 1] */
    int32_t* blocklist;       /* [nblocks] non-empty block ids ascending; first nactive valid */
    int32_t* particleindices; /* [n] 1-based; first nassigned valid */
    int64_t nblocks;          /* prod(nblocks(mesh)), checked against the mesh */
} tb_partition;

/* Stored basis weights, the BasisWeightArray layout of the reference
 * (src/Basis/basis_weight.jl:345-358,413-432): w is Array{T,4}(3,3,3,n) (2D:
 * (3,3,n)), grad_w is Array{Vec{dim,T}}(3,3,3,n) (AoS, dim per node), window is
 * the CartesianIndices{dim} per particle as (start_1, stop_1, start_2, stop_2, ...)
 * 1-based inclusive Int64 (an empty window is start = 1, stop = 0). Values at
 * local slots outside a truncated window are left as zero. */
typedef struct tb_weights {
    void* w;
    void* grad_w;
    int64_t* window;
} tb_weights;

/* Scalars of the recognised step (README.md:71-87, docs/src/gpu.md:296-331). */
typedef struct tb_step_params {
    double dt;
    double mass;        /* per-particle mass when particles.m == NULL */
    double V0;          /* initial volume when particles.V0 == NULL */
    double mu;          /* Lame mu when particles.mu == NULL */
    double lambda;      /* Lame lambda when particles.lambda == NULL */
    double gravity[3];  /* body acceleration added to f as w m g */
    double gimp_l;      /* uGIMP particle length when particles.l == NULL */
    double flip_alpha;  /* FLIP blend: v_p = (1-a) sum w v_i + a (v_p + sum w (v_i - vn_i)), the blend of
                           test/transfer.jl:111-133; 1 = README FLIP (v_p += sum w (v_i - vn_i)) */
    int32_t basis;      /* enum tb_basis_kind */
    int32_t transfer;   /* enum tb_transfer_kind */
    int32_t material;   /* enum tb_material_kind */
    int32_t wall_mask;  /* slip walls: bit 2d = low face of axis d, bit 2d+1 = high face */
    int32_t wall_layers;/* node layers next to each walled face whose normal velocity is zeroed */
    int32_t reserved;
    double hardening;   /* TB_MATERIAL_VONMISES: linear hardening modulus H */
    double yield_stress;/* TB_MATERIAL_VONMISES: initial yield stress */
} tb_step_params;

typedef struct tb_ctx tb_ctx;

/* ---- context ---------------------------------------------------------- */

/* Create a context bound to `device` and `stream` (a cudaStream_t, NULL = the
 * legacy default stream). One context per stream; a context is not re-entrant. */
tb_ctx* tb_create(int32_t device, void* stream);
void tb_destroy(tb_ctx* ctx);
const char* tb_last_error(const tb_ctx* ctx);
int32_t tb_set_stream(tb_ctx* ctx, void* stream);
int32_t tb_synchronize(tb_ctx* ctx);
/* Number of this library's kernel launches issued through ctx so far. */
int64_t tb_launch_count(const tb_ctx* ctx);

/* Per-kernel device time: while enabled, every launch of this library through
 * ctx is bracketed by CUDA events on ctx's stream (the per-phase timer table of
 * the reference's tutorials, docs/literate/tutorials/taylor_impact.jl:107-185). */
typedef struct tb_kernel_time {
    char name[32];     /* kernel family: bin_count, bin_scan, bin_scatter, bin_fixup,
                          grid_mark, grid_zero, p2g, grid_update, g2p, g2p_outside, ... */
    int64_t launches;
    double ms;         /* summed device time */
} tb_kernel_time;
int32_t tb_profile_enable(tb_ctx* ctx, int32_t on);
/* Synchronises, writes up to `cap` entries accumulated since the last read,
 * sets *count to the number of kernel families, and resets the totals. */
int32_t tb_profile_read(tb_ctx* ctx, tb_kernel_time* out, int32_t cap, int32_t* count);

/* ---- basis weights: update!(weights, particles, mesh) -----------------
 * reference: src/Basis/basis_weight.jl:714-752 (GPU kernel :686-689). */
int32_t tb_update_weights_f64(tb_ctx* ctx, const tb_mesh* mesh, const tb_particles* particles,
                              const tb_step_params* params, tb_weights* weights);
int32_t tb_update_weights_f32(tb_ctx* ctx, const tb_mesh* mesh, const tb_particles* particles,
                              const tb_step_params* params, tb_weights* weights);

/* ---- binning: update!(partition::GPUBlockStrategy, particles.x) ---------
 * reference: src/Parallel/gpu_block_strategy.jl:142-166. Synchronises the
 * stream once and returns the totals (the reference's one readback, :161-164). */
int32_t tb_bin_particles_f64(tb_ctx* ctx, const tb_mesh* mesh, const tb_particles* particles,
                             tb_partition* partition, int64_t* nactive, int64_t* nassigned);
int32_t tb_bin_particles_f32(tb_ctx* ctx, const tb_mesh* mesh, const tb_particles* particles,
                             tb_partition* partition, int64_t* nactive, int64_t* nassigned);

/* ---- update_sparsity!(grid::SpGrid, particles.x) -----------------------
 * reference: src/Grids/sparsity.jl:19-60 (particle-driven update: blocks that
 * hold a particle inside the mesh, each with its 3^dim neighbourhood of node
 * blocks, numbered in ascending block order). Bins the particles into
 * `partition` (as tb_bin_particles_*), then numbers the active node blocks of
 * the sparse `grid`. Synchronises once and returns in *nstored the nodes each
 * field must hold (active blocks x blocklength); TB_ERR_CAPACITY if that exceeds
 * grid.capacity (the numbering is written all the same, so a caller can grow
 * the fields and go on). */
int32_t tb_update_sparsity_f64(tb_ctx* ctx, const tb_mesh* mesh, const tb_particles* particles,
                               tb_partition* partition, tb_grid* grid, int64_t* nstored);
int32_t tb_update_sparsity_f32(tb_ctx* ctx, const tb_mesh* mesh, const tb_particles* particles,
                               tb_partition* partition, tb_grid* grid, int64_t* nstored);
int32_t tb_update_sparsity_f32x64(tb_ctx* ctx, const tb_mesh* mesh, const tb_particles* particles,
                                  tb_partition* partition, tb_grid* grid, int64_t* nstored);

/* ---- @P2G scatter half: m, mv, f (assigned targets are zeroed first) ----
 * reference: src/Transfer/gpu.jl:196-223 (block-scheduled) with the sums of
 * README.md:72-74 plus gravity f += w m g (test/transfer.jl:96). Requires a
 * partition from tb_bin_particles_* for the same positions. Asynchronous. */
int32_t tb_p2g_f64(tb_ctx* ctx, const tb_mesh* mesh, const tb_particles* particles,
                   const tb_partition* partition, tb_grid* grid, const tb_step_params* params);
int32_t tb_p2g_f32(tb_ctx* ctx, const tb_mesh* mesh, const tb_particles* particles,
                   const tb_partition* partition, tb_grid* grid, const tb_step_params* params);

/* ---- @P2G grid half: vn = mv/m, v = vn + dt f/m (guarded), slip walls ----
 * reference: foreach_loop -> gpukernel_foreach (src/Transfer/foreach.jl:276-339),
 * equations docs/src/gpu.md:309-316. Asynchronous. */
int32_t tb_grid_update_f64(tb_ctx* ctx, const tb_mesh* mesh, tb_grid* grid, const tb_step_params* params);
int32_t tb_grid_update_f32(tb_ctx* ctx, const tb_mesh* mesh, tb_grid* grid, const tb_step_params* params);

/* ---- @G2P gather + particle update (FLIP or APIC, Neo-Hookean) ----------
 * reference: src/Transfer/gpu.jl:226-232 with README.md:79-86. Asynchronous. */
int32_t tb_g2p_f64(tb_ctx* ctx, const tb_mesh* mesh, const tb_grid* grid, tb_particles* particles,
                   const tb_step_params* params);
int32_t tb_g2p_f32(tb_ctx* ctx, const tb_mesh* mesh, const tb_grid* grid, tb_particles* particles,
                   const tb_step_params* params);

/* ---- fused step: bin -> P2G -> grid update -> G2P, `nsteps` times --------
 * The canonical loop of README.md:66-87 / docs/src/gpu.md:296-331 on device
 * data, with no host synchronisation between steps. */
int32_t tb_step_f64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                    tb_grid* grid, const tb_step_params* params, int32_t nsteps);
int32_t tb_step_f32(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                    tb_grid* grid, const tb_step_params* params, int32_t nsteps);
/* FP64-position form of tb_step_f32: particles->x[d] are double arrays, every
 * other field as in tb_step_f32 (F double). Windows and in-cell offsets are
 * computed from the FP64 positions, binning uses the Float64 findblock rule,
 * and G2P adds the FP32 displacement to the FP64 position. A Float32 position
 * near 0.5 carries an ulp of 6e-8, larger than a step's displacement rounding
 * allows for 1e-5 accuracy over 100 steps; this form removes that error.
 * In 3D every basis and transfer of the step; in 2D the B-spline / uGIMP
 * FLIP/PIC step only (TB_ERR_UNSUPPORTED otherwise). The reference's
 * counterpart is the same step under
 * gpu_preserve (src/adapt.jl:15-17), which leaves chosen arrays in Float64. */
int32_t tb_step_f32x64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                       tb_grid* grid, const tb_step_params* params, int32_t nsteps);

/* ---- reorder_particles! -------------------------------------------------
 * reference: reorder_particles!(particles, partition; threshold) and
 * block_ordered_particle_contiguity (src/Parallel/gpu_block_strategy.jl:172-238,
 * src/Parallel/cpu_block_strategy.jl:221-269). The partition must come from
 * binning these particles. The score is the fraction of neighbouring particles
 * in memory that share a block (1 when fully block-grouped); with `threshold` in
 * [0, 1] the particles are reordered when the score is below it (always at 1,
 * never at 0): every field present in `particles` is permuted into block order,
 * partition->blockids follow and partition->particleindices become 1..n. Fields
 * are 4 or 8 bytes per the precision form (x double in _f32x64, F always double).
 * Synchronous; `reordered` (may be NULL) receives 1 if it reordered. Particles
 * outside the mesh are an error when a reorder is due (TB_ERR_ARG), as on the
 * reference's GPU path. */
int32_t tb_reorder_particles_f64(tb_ctx* ctx, int32_t dim, tb_particles* particles, tb_partition* partition,
                                 double threshold, int32_t* reordered);
int32_t tb_reorder_particles_f32(tb_ctx* ctx, int32_t dim, tb_particles* particles, tb_partition* partition,
                                 double threshold, int32_t* reordered);
int32_t tb_reorder_particles_f32x64(tb_ctx* ctx, int32_t dim, tb_particles* particles, tb_partition* partition,
                                    double threshold, int32_t* reordered);
/* max over the particles of sqrt((lambda + 2 mu) / (m / V)) + |v| (lambda, mu and
 * m per particle when the arrays are given, else from params): the speed of the
 * Taylor impact's time step CFL h / c_max (docs/src/gpu.md:283-284), reduced on
 * the device. Synchronous. `particles` may be in the FP64-position form (x is
 * not read). */
int32_t tb_max_wave_speed_f64(tb_ctx* ctx, int32_t dim, const tb_particles* particles,
                              const tb_step_params* params, double* c_max);
int32_t tb_max_wave_speed_f32(tb_ctx* ctx, int32_t dim, const tb_particles* particles,
                              const tb_step_params* params, double* c_max);
/* block_ordered_particle_contiguity of `n` particles binned into `partition`. Synchronous. */
int32_t tb_particle_contiguity(tb_ctx* ctx, const tb_partition* partition, int64_t n, double* score);
/* tb_step_* with reorder_particles!(particles, partition; threshold) after every
 * binning, decided on the device (no host synchronisation): the loop of
 * docs/literate/tutorials/taylor_impact.jl:120-127. A reorder that is due while
 * particles lie outside the mesh is skipped and reported as TB_ERR_DEVICE at the
 * next synchronising call. */
int32_t tb_step_reorder_f64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                            tb_grid* grid, const tb_step_params* params, int32_t nsteps, double threshold);
int32_t tb_step_reorder_f32(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                            tb_grid* grid, const tb_step_params* params, int32_t nsteps, double threshold);
int32_t tb_step_reorder_f32x64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                               tb_grid* grid, const tb_step_params* params, int32_t nsteps, double threshold);

/* @G2P2G (src/Transfer/g2p2g.jl:98-159) for the FLIP/PIC equation set of the
 * plain step: one pass doing each particle's G2P (README.md:79-86) and then its
 * P2G of m, mv, f (README.md:72-74, zeroed first) with the weights of the
 * position the particle had before the G2P half moved it (the reference binds
 * one support window for both halves, g2p2g.jl:103-106); the P2G half reads the
 * updated v, sigma and V; the grid half (README.md:75-76, walls) follows. The
 * particles are binned into `partition` at their positions on entry. APIC is
 * refused (TB_ERR_UNSUPPORTED); the _f32x64 form takes FP64 positions as
 * tb_step_f32x64 does. Asynchronous on the context's stream. */
int32_t tb_g2p2g_f64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                     tb_grid* grid, const tb_step_params* params);
int32_t tb_g2p2g_f32(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                     tb_grid* grid, const tb_step_params* params);
int32_t tb_g2p2g_f32x64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                        tb_grid* grid, const tb_step_params* params);

/* ---- host-buffer rollout (end-to-end form of tb_step_*) ----------------
 * `host` holds HOST pointers (pinned memory recommended) for the particle state;
 * the context stages it into its own device buffers, runs `nsteps` steps and
 * copies the state back. Grid and partition live in context-owned device memory.
 * Synchronous. This is the call a host program without device arrays makes. */
int32_t tb_rollout_host_f64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* host,
                            const tb_step_params* params, int32_t nsteps);
int32_t tb_rollout_host_f32(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* host,
                            const tb_step_params* params, int32_t nsteps);
/* host-buffer form of tb_step_f32x64 (x double on the host as well). */
int32_t tb_rollout_host_f32x64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* host,
                               const tb_step_params* params, int32_t nsteps);

/* ---- reverse mode: sensitivities of a rollout ---------------------------
 * No counterpart in the reference: Tesserae.jl differentiates only constitutive
 * laws and basis jets (through Tensorial's dual numbers) and has no adjoint of
 * its transfers. These entry points give the sensitivities of a scalar loss to
 * the particle state that tb_step_* advances -- positions x, velocities v and
 * the deformation gradient F (sigma and V are functions of F) -- and to the
 * per-particle Lame parameters. The adjoint arithmetic is FP64 in both forms
 * (the _f32 entry points differentiate the mixed FP32 step).
 * Supported: quadratic B-spline and uGIMP bases, FLIP/PIC transfer (any
 * flip_alpha), Neo-Hookean and fluid materials, slip walls. WLS bases and APIC
 * return TB_ERR_UNSUPPORTED. */
typedef struct tb_adjoint {
    double* x[3];     /* d loss / d x_p per component */
    double* v[3];     /* d loss / d v_p */
    double* F[9];     /* d loss / d F_p, column-major like particles.F */
    double* mu;       /* d loss / d mu_p, accumulated (+=); NULL = not wanted */
    double* lambda;   /* d loss / d lambda_p (the bulk modulus K for fluids), accumulated; NULL = not wanted */
    double* B[9];     /* d loss / d B_p, column-major like particles.B (TB_TRANSFER_APIC only; NULL otherwise) */
} tb_adjoint;

/* One step backwards. `particles` holds the state at the START of the step as
 * tb_step_* reads it (x, v, F, sigma, V). On entry `adj` holds the sensitivities
 * to the state at the END of the step; on return, to the state at its start
 * (adj.mu and adj.lambda accumulate). The step's partition and forward grid
 * are recomputed into `partition` and `grid`. Asynchronous. */
int32_t tb_adjoint_step_f64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                            tb_grid* grid, const tb_step_params* params, tb_adjoint* adj);
int32_t tb_adjoint_step_f32(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                            tb_grid* grid, const tb_step_params* params, tb_adjoint* adj);

/* Checkpointed rollout. tb_tape_forward_* advances `particles` by `nsteps`
 * steps exactly like tb_step_* and keeps the state at steps 0, K, 2K, ...
 * (K = checkpoint_every) in context-owned device memory. tb_tape_backward_*
 * takes in `adj` the sensitivities to the final state and returns the
 * sensitivities to the state at step 0 (mu and lambda accumulate over all
 * steps); for each segment of K steps it restores the checkpoint, re-runs the
 * segment keeping every step's input state, grid and partition, and steps
 * backwards through it, so the device memory held is nsteps/K particle states
 * plus K (state + grid + partition) slots. With K = 1 the forward pass keeps
 * every step's (state + grid + partition) slot instead (nsteps slots) and the
 * backward pass runs no forward step at all. `particles` is the working state
 * and holds the step-0 state again on return; the backward pass uses its own
 * grids and partitions (`partition` and `grid` are not touched). It must
 * follow the forward pass on the same context with the same particle count,
 * mesh and params. Asynchronous. */
int32_t tb_tape_forward_f64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                            tb_grid* grid, const tb_step_params* params, int32_t nsteps, int32_t checkpoint_every);
int32_t tb_tape_forward_f32(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                            tb_grid* grid, const tb_step_params* params, int32_t nsteps, int32_t checkpoint_every);
int32_t tb_tape_backward_f64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                             tb_grid* grid, const tb_step_params* params, tb_adjoint* adj);
int32_t tb_tape_backward_f32(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                             tb_grid* grid, const tb_step_params* params, tb_adjoint* adj);
/* The FP64-position form (particles.x double, the rest as _f32; the cases of
 * tb_step_f32x64): the forward steps, the windows and the in-window offsets of
 * the reverse step come from the FP64 positions. */
int32_t tb_adjoint_step_f32x64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                               tb_grid* grid, const tb_step_params* params, tb_adjoint* adj);
int32_t tb_tape_forward_f32x64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles, tb_partition* partition,
                               tb_grid* grid, const tb_step_params* params, int32_t nsteps, int32_t checkpoint_every);
int32_t tb_tape_backward_f32x64(tb_ctx* ctx, const tb_mesh* mesh, tb_particles* particles,
                                tb_partition* partition, tb_grid* grid, const tb_step_params* params,
                                tb_adjoint* adj);
/* Device bytes a tape of `nsteps` steps over `n` particles holds (forward and
 * backward pass together) for element size `elem` (4 or 8; F is FP64 in both),
 * with the APIC matrix B when `apic` != 0, FP64 positions when `x64` != 0
 * (elem 4 only), checkpointed every
 * `checkpoint_every` steps (1: the whole tape). Pure arithmetic, no device call:
 * lets a caller pick the interval against its free device memory. Returns -1 on
 * invalid arguments. */
int64_t tb_tape_bytes(const tb_mesh* mesh, int64_t n, int32_t elem, int32_t apic, int32_t x64, int32_t nsteps,
                      int32_t checkpoint_every);
/* Frees the context's tape buffers (the next tb_tape_forward_* allocates them
 * again); the tape is invalid afterwards. Synchronises the context's stream. */
int32_t tb_tape_release(tb_ctx* ctx);

/* ---- binning without allocation ---------------------------------------
 * No counterpart in the reference: Tesserae.jl always allocates its partition
 * scratch through KernelAbstractions. This entry point is for callers that
 * cannot call cudaMalloc (code inside another framework's memory pool or a
 * runtime that forbids device allocation after start-up, loops that must not
 * stall on the allocator) and have no tb_ctx. It bins like tb_bin_particles_f32
 * (precision = 1) or _f64 (precision = 0), with the same bit-exact output, but
 * its scratch is one fixed array compiled into the library, held by every GPU
 * that loads the library until exit. It allocates nothing: inputs above
 * TB_NOALLOC_MAX_PARTICLES particles or TB_NOALLOC_MAX_BLOCKS grid blocks are
 * rejected with TB_ERR_CAPACITY. It runs on the current device and `stream`,
 * synchronises `stream` once to read the totals, and writes a message into
 * `errbuf` (may be NULL) on error. Every call looks the scratch up with
 * cudaGetSymbolAddress on the current device (so a device reset, which may move
 * it, is harmless). The first call on a device may load the library's device
 * code (lazy loading), which is when the driver reserves the array: make one
 * warm-up call per device during start-up, before any stream capture; later
 * calls allocate nothing. All calls share the scratch: calls that overlap on
 * the GPU race, so serialise them. */
#define TB_NOALLOC_MAX_PARTICLES (1 << 20)
#define TB_NOALLOC_MAX_BLOCKS (1 << 20)
int32_t tb_bin_particles_noalloc(const tb_mesh* mesh, const tb_particles* particles, int32_t precision,
                                 tb_partition* partition, void* stream, int64_t* nactive, int64_t* nassigned,
                                 char* errbuf, int32_t errlen);

#ifdef __cplusplus
}
#endif

#endif /* TESSERAE_B200_H */
