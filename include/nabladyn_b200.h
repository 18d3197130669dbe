/*
 * nabladyn_b200: the C-ABI of the B200 MD step hot path.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream (cudaStream_t passed
 * as nd_stream_t), launches its kernels on that stream and returns ND_OK or an error code;
 * nd_last_error() gives the calling thread's last message. No entry point allocates device
 * memory, synchronizes the device or reads device memory on the host, so every call can be
 * captured in a CUDA Graph. Callers own every buffer.
 *
 * Data errors (a cell too small, a non-finite coordinate, more pairs than the capacity) are
 * not call errors: they are bits of a device status word, decoded by the host when it reads
 * the status, exactly as in the reference's neighbor operator.
 */
#ifndef NABLADYN_B200_H
#define NABLADYN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ND_OK 0
#define ND_EINVAL 1 /* an argument is out of range; nothing was launched */
#define ND_ECUDA 2  /* the CUDA runtime reported an error */

#define ND_FLOAT32 0
#define ND_FLOAT64 1

/* Status bits of status[0]; they latch until the list is allocated again. */
#define ND_STATUS_INVALID_CELL 1
#define ND_STATUS_NON_FINITE 2
#define ND_STATUS_OVERFLOW 8

typedef void* nd_stream_t; /* a cudaStream_t */

/* The calling thread's message for its last failed call. */
const char* nd_last_error(void);

/* The ABI version of this header: 1. */
int nd_abi_version(void);

/* ------------------------------------------------------------------------------------------
 * The neighbor operator.
 *
 * Replaces the torch.library namespace nabladyn_neighbors of the reference
 * (src/nabladyn/neighbors/csrc/ops.cpp:11-41, ops.h:12-89). The 15 buffers keep the
 * reference's order and meaning; the host allocates them as
 * src/nabladyn/neighbors/_neighbor_list.py:229-254 does (scan_temp sized by
 * nd_neighbors_scan_temp_bytes). Positions and cell are [N, 3] and [3] of one dtype, with
 * positions wrapped into [0, L).
 * ---------------------------------------------------------------------------------------- */
typedef struct nd_neighbor_buffers {
    int32_t* dims;           /* [3] bins per axis */
    void* widths;            /* [3] bin widths, the positions' dtype */
    int32_t* atom_bin;       /* [N] */
    int32_t* bin_counts;     /* [B + 1], zero between builds */
    int32_t* bin_offsets;    /* [B + 1] */
    int64_t num_bin_slots;   /* B + 1 */
    int32_t* unordered_ids;  /* [N] */
    int32_t* sorted_ids;     /* [N] */
    void* sorted_positions;  /* [N, 3], the positions' dtype */
    uint8_t* scan_temp;      /* scratch of the scans */
    int64_t scan_temp_bytes; /* its size */
    int32_t* pair_counts;    /* [N] */
    int32_t* pair_offsets;   /* [N] */
    int32_t* pair_total;     /* [1] */
    int32_t* status;         /* [2]: flags, pairs needed */
    int32_t* pairs;          /* [2, C] */
    int64_t capacity;        /* C */
    int32_t* bits;           /* [N * ceil(N / 32)] on the all-pairs path, else NULL */
    int64_t bits_numel;      /* 0 on the grid path */
} nd_neighbor_buffers;

/* The update's own buffers (src/nabladyn/neighbors/_neighbor_list.py:43-56, 265-272). */
typedef struct nd_reuse_buffers {
    void* reference_positions; /* [N, 3]: the frame of the last build */
    void* reference_cell;      /* [3] */
    const int32_t* limits;     /* [3]: the first grid's bins per axis */
    void* reuse;               /* [4]: threshold^2, then the scale per axis */
    int32_t* rebuild;          /* [1] */
    int32_t* rebuild_count;    /* [1] */
} nd_reuse_buffers;

/* scan_temp_bytes(Tensor reference, int items) -> int
 * (src/nabladyn/neighbors/csrc/runtime/entry_points.cu:284-301): the scratch bytes of a scan
 * over `items` int32 values. */
int nd_neighbors_scan_temp_bytes(int64_t items, int64_t* bytes);

/* count_first_frame(positions, cell, radius, <15 buffers>)
 * (src/nabladyn/neighbors/csrc/runtime/entry_points.cu:303-352): the grid and each atom's pair
 * count, so the host can size the pairs. */
int nd_neighbors_count_first_frame(int dtype, const void* positions, const void* cell,
                                   int64_t num_atoms, double radius,
                                   const nd_neighbor_buffers* buffers, nd_stream_t stream);

/* fill_first_frame(positions, cell, radius, <15 buffers>)
 * (src/nabladyn/neighbors/csrc/runtime/entry_points.cu:354-399): the pairs, into the capacity
 * the host chose, then the total, the overflow check and the padding. */
int nd_neighbors_fill_first_frame(int dtype, const void* positions, const void* cell,
                                  int64_t num_atoms, double radius,
                                  const nd_neighbor_buffers* buffers, nd_stream_t stream);

/* update(positions, cell, cutoff, radius, reference_positions, reference_cell, limits, reuse,
 *        rebuild, rebuild_count, <15 buffers>)
 * (src/nabladyn/neighbors/csrc/runtime/entry_points.cu:401-508): check the cell, decide reuse
 * on the GPU, rebuild behind the device flag and store the new reference frame. */
int nd_neighbors_update(int dtype, const void* positions, const void* cell, int64_t num_atoms,
                        double cutoff, double radius, const nd_reuse_buffers* reuse,
                        const nd_neighbor_buffers* buffers, nd_stream_t stream);

/* Builds one frame's pair list, as count_first_frame then fill_first_frame would, without
 * allocating: for callers that cannot call cudaMalloc (code inside another framework's graph
 * capture or memory pool, hosts that forbid allocation, fixed memory maps). It has no
 * counterpart in the reference. Every intermediate buffer lives in one file-scope device array
 * of about 1.3 MB that each GPU loading this library holds until the process exits; the caller
 * passes only the inputs and the outputs: positions [N, 3] wrapped into [0, L) and cell [3]
 * (device), the grid dims[3] and bin widths[3] (host values, as allocate chooses them), and
 * pairs [2, capacity], pair_total [1], status [2] (device). Limits: N <= 16384 and at most
 * 16384 bins; with at most three bins per axis (the all-pairs path) N <= 2048; larger inputs,
 * and widths that are not finite, not positive or narrower than the radius, return ND_EINVAL.
 * The kernels bin with width L / dims (the cell on the device) and, should that be narrower
 * than the radius, build nothing and set ND_STATUS_INVALID_CELL. The first call on a device looks up the array's address with
 * cudaGetSymbolAddress, so make it before any stream capture. Every call shares the array and
 * leaves the last call's contents in it: calls that overlap on the GPU (other streams, other
 * threads) race and must be serialized by the caller. */
int nd_neighbors_build_no_alloc(int dtype, const void* positions, const void* cell,
                                int64_t num_atoms, double radius, const int32_t* dims,
                                const double* widths, int32_t* pairs, int64_t capacity,
                                int32_t* pair_total, int32_t* status, nd_stream_t stream);

/* ------------------------------------------------------------------------------------------
 * Lennard-Jones over a [2, C] pair index.
 *
 * Replaces, for the Lennard-Jones model, the torch.func evaluation
 * quantity.energy_force_virial(model)(positions, cell, pairs)
 * (src/nabladyn/quantity.py:160-184 over src/nabladyn/potential/_lennard_jones/_potential.py:
 * 209-234): E, F = -dE/dx and W = -dE/dstrain in one pass, plus dE/dsigma and dE/depsilon
 * per type-pair row when sigma_grad is given. energy, virial and the gradients are float64.
 * With a strain, every pair vector is deformed by (I + strain) first and F, W are the
 * derivatives of that strained energy (src/nabladyn/space.py:51-64).
 * ---------------------------------------------------------------------------------------- */
typedef struct nd_lj_pairs_args {
    int dtype;
    const void* positions;    /* [N, 3], wrapped into [0, L) */
    const void* cell;         /* [3] */
    int64_t num_atoms;        /* N */
    const int32_t* pairs;     /* [2, C] */
    int64_t capacity;         /* C */
    const int32_t* atom_types; /* [N] in [0, T); ignored when T == 1 */
    int32_t num_types;        /* T, 1..8 */
    const void* sigma;        /* [T(T+1)/2] */
    const void* epsilon;      /* [T(T+1)/2] */
    double cutoff;
    const void* strain;       /* [3, 3] strain, row-major; NULL for none */
    double* energy;           /* [1] out */
    void* forces;             /* [N, 3] out */
    double* virial;           /* [3, 3] out */
    double* sigma_grad;       /* [T(T+1)/2] out, or NULL */
    double* epsilon_grad;     /* [T(T+1)/2] out, or NULL */
} nd_lj_pairs_args;

int nd_lj_energy_force_virial(const nd_lj_pairs_args* args, nd_stream_t stream);

/* A batch of F frames of one system (config: the parameter fit of
 * src/nabladyn/training/_fit.py:245-271). Positions [F, N, 3] wrapped into [0, L), cells [F, 3],
 * pairs [F, 2, C] (each frame's index padded with self-pairs to the common C). */
typedef struct nd_lj_batch_args {
    int dtype;
    int64_t frames;             /* F */
    const void* positions;      /* [F, N, 3] */
    const void* cells;          /* [F, 3] */
    int64_t num_atoms;          /* N */
    const int32_t* pairs;       /* [F, 2, C] */
    int64_t capacity;           /* C */
    const int32_t* atom_types;  /* [N]; ignored when T == 1 */
    int32_t num_types;          /* T, 1..8 */
    const void* sigma;          /* [T(T+1)/2] */
    const void* epsilon;        /* [T(T+1)/2] */
    double cutoff;
    double* energy;             /* forward out: [F] */
    void* forces;               /* forward out: [F, N, 3] */
    double* virial;             /* forward out: [F, 3, 3] */
    const double* energy_grad;  /* backward in: dLoss/dE [F] */
    const void* forces_grad;    /* backward in: dLoss/dF [F, N, 3] */
    const double* virial_grad;  /* backward in: dLoss/dW [F, 3, 3] */
    double* sigma_grad;         /* backward out: dLoss/dsigma [T(T+1)/2], summed over frames */
    double* epsilon_grad;       /* backward out: dLoss/depsilon [T(T+1)/2] */
} nd_lj_batch_args;

/* E, F, W of every frame. */
int nd_lj_batch_forward(const nd_lj_batch_args* args, nd_stream_t stream);

/* The hand-written parameter backward: dLoss/dsigma and dLoss/depsilon from the gradients of
 * the loss with respect to every frame's E, F and W (the reference takes it by torch.func
 * double backward). */
int nd_lj_batch_parameter_backward(const nd_lj_batch_args* args, nd_stream_t stream);

/* ------------------------------------------------------------------------------------------
 * The MD engine: velocity-Verlet (NVE) and Nose-Hoover chain (NVT) steps of a Lennard-Jones
 * system with the neighbor rebuild decided on the GPU.
 *
 * Replaces the step the reference assembles from three compiled programs around the neighbor
 * operator and captures in a CUDA Graph (src/nabladyn/md/_simulation.py:316-364,
 * src/nabladyn/md/_ensembles/_nve.py:39-58, _nvt.py:88-129, _verlet.py:8-31, _chain.py:36-83).
 * Per-atom state lives in cell order (sorted by cell, then atom id, at each rebuild); `ids`
 * maps a slot to the caller's atom. T is the system's dtype; positions are [N, 4] (x, y, z,
 * type). The caller allocates every buffer; nd_md_partial_slots gives the size of partials.
 * ---------------------------------------------------------------------------------------- */
typedef struct nd_md_system {
    int dtype;
    int64_t num_atoms;
    int32_t num_types;       /* 1..8; types ride in positions[:, 3] */
    int32_t small;           /* 1: one tile holds the whole system, minimum image per pair */
    int32_t dims[3];         /* cells per axis (>= 3 each unless small) */
    int32_t bricks_x;        /* bricks per row of cells along x */
    int32_t width;           /* neighbor-list slots per list row, a multiple of 8 */
    int32_t tile_capacity;   /* atoms per brick tile, at most */
    double cell[3];          /* orthorhombic cell lengths, fixed */
    double widths[3];        /* cell widths, L / dims, rounded to T */
    double cutoff;           /* LJ cutoff r_c */
    double radius;           /* list radius R = r_c + skin */
    double timestep;         /* dt */
    double threshold_squared; /* reuse while every |x - x_ref|^2 is below this */
    void* positions;         /* [N, 4] T */
    void* velocities;        /* [N, 3] T */
    void* forces;            /* [N, 3] T */
    void* inverse_masses;    /* [N] T */
    void* masses;            /* [N] T */
    int64_t* images;         /* [N, 3] */
    int32_t* ids;            /* [N] */
    void* reference_positions; /* [N, 4] T */
    void* shadow_positions;  /* the permutation's copies of the arrays above, forces excepted */
    void* shadow_velocities;
    void* shadow_inverse_masses;
    void* shadow_masses;
    int64_t* shadow_images;
    int32_t* shadow_ids;
    int32_t* cell_counts;    /* [cells + 1], zero between rebuilds */
    int32_t* cell_offsets;   /* [cells + 1] */
    int32_t* atom_cell;      /* [N] */
    int32_t* slots;          /* [N] */
    int32_t* unordered;      /* [N] */
    int32_t* order;          /* [N] */
    void* scan_temp;         /* nd_neighbors_scan_temp_bytes(cells + 1) bytes */
    uint16_t* neighbors;     /* [ceil(rows / 32) * 32 * width]; rows = N when small, else
                              * N + 2 * cells + 2: two rows per pair of centers of one cell,
                              * the halves of the pair's list */
    int32_t* neighbor_counts; /* [rows] */
    int32_t* pair_order;     /* [2 * (rows / 2 + 1)]: per brick its center pairs, longest
                              * lists first, as (pair, first center << 1 | has a second) */
    int32_t* rebuild;        /* [2]: the reuse check's flag; a count the step graph's drift
                              * kernel keeps (zero between steps) */
    int32_t* rebuild_count;  /* [1] */
    int32_t* status;         /* [4]: flags, most neighbors needed, largest tile needed, largest tile built */
    double* partials;        /* [nd_md_partial_slots]: per-block float64 sums */
    double* totals;          /* [16]: E, K, W xx yy zz xy xz yz; then K of nd_md_kinetic */
    double* thermostat;      /* [24] float64 chain block */
    const void* sigma;       /* [T(T+1)/2] T */
    const void* epsilon;     /* [T(T+1)/2] T */
} nd_md_system;

/* Loads a frame in the caller's order: positions [N, 3] wrapped into [0, L), velocities,
 * masses [N], images [N, 3] int64, types [N] int32 (NULL for one type). */
int nd_md_import(const nd_md_system* system, const void* positions, const void* velocities,
                 const void* masses, const int64_t* images, const int32_t* types,
                 nd_stream_t stream);

/* Wraps, re-sorts, permutes the state and builds the neighbor list, unconditionally. */
int nd_md_rebuild(const nd_md_system* system, nd_stream_t stream);

/* Forces and energy (and the virial) at the current positions; totals[0], totals[2..7]. */
int nd_md_forces(const nd_md_system* system, int virial, nd_stream_t stream);

/* One step: [NVT: chain half step] half kick, drift, reuse check; the rebuild behind the
 * device flag; forces, half kick, [NVT: K and the closing chain half step]. */
int nd_md_step(const nd_md_system* system, int thermostat, int virial, nd_stream_t stream);

/* One phase of nd_md_step: 0 the drift and reuse check, 1 the gated rebuild, 2 the forces with
 * the second half kick and the tail; -1 all three. Running 0, 1, 2 in order is one step. */
int nd_md_step_phase(const nd_md_system* system, int phase, int thermostat, int virial,
                     nd_stream_t stream);

/* `steps` whole steps of a small-box system (fewer than three cells on an axis, at most 4,096
 * atoms), as many calls of nd_md_step without the virial would make them, in one launch of one
 * thread-block cluster (up to 8 CTAs, each owning a range of atoms, phases separated by cluster
 * barriers): a small box's step is a few microseconds of work over six launches, so the
 * launches bound it. After a failure (a status bit) the list is no longer rebuilt, as in
 * nd_md_step. The totals' float64 sums run in another fixed order than nd_md_step's. No
 * counterpart in the reference (its small-box step is the same graph as any other). */
int nd_md_run_small(const nd_md_system* system, int thermostat, int steps, nd_stream_t stream);

/* The number of kernels one NVE nd_md_step without the virial launches (the drift, the
 * rebuild's kernels, the forces); an NVT step or one with the virial adds a finalize. */
int nd_md_step_launches(const nd_md_system* system, int64_t* launches);

/* Writes the frame in the caller's order; any output may be NULL. */
int nd_md_export(const nd_md_system* system, void* positions, void* velocities, void* forces,
                 int64_t* images, int thermostat, nd_stream_t stream);

/* K of the current velocities in float64, into totals[9]. */
int nd_md_kinetic(const nd_md_system* system, int thermostat, nd_stream_t stream);

/* The float64 slots the partials buffer needs. */
int nd_md_partial_slots(const nd_md_system* system, int64_t* slots);

/* ------------------------------------------------------------------------------------------
 * The replica server: many independent float32, one-type Lennard-Jones NVT replicas resident
 * in one pool, each advanced by one CTA for a budget of steps per launch (the serving workload
 * of the reference's md.nvt, src/nabladyn/md/_ensembles/_nvt.py:132-179, run for many small
 * systems at once). A replica's atoms occupy [atom_offset, atom_offset + N) of every per-atom
 * pool array; its list occupies ceil(N / 32) * 32 * width uint16 from list_offset; its cell
 * table cells + 1 ints from cell_offset.
 * ---------------------------------------------------------------------------------------- */
typedef struct nd_replica {
    int64_t atom_offset;
    int64_t list_offset;      /* a multiple of 8 */
    int64_t cell_offset;
    int32_t num_atoms;        /* 2 .. 65535 */
    int32_t width;            /* list slots per atom, a multiple of 8 */
    int32_t dims[3];          /* cells per axis, each >= 1, product <= 4096 */
    int32_t steps_left;       /* decremented by every step run */
    int32_t status;           /* ND_STATUS_* bits */
    int32_t rebuild_count;
    float cell[3];
    float widths[3];
    float cutoff;
    float radius;             /* cutoff + skin */
    float threshold_squared;  /* the reuse threshold, as the engine's */
    float timestep;
    float sigma;
    float epsilon;
    double energy;            /* E after the last step run (or at admission) */
    double thermostat[24];    /* the engine's float64 chain block */
} nd_replica;

typedef struct nd_replica_pool {
    nd_replica* replicas;      /* [slots] */
    void* positions;           /* [atoms, 4] float32 */
    void* velocities;          /* [atoms, 3] float32 */
    void* forces;              /* [atoms, 3] float32 */
    void* masses;              /* [atoms] float32 */
    void* inverse_masses;      /* [atoms] float32 */
    int64_t* images;           /* [atoms, 3] */
    void* reference_positions; /* [atoms, 4] float32 */
    uint16_t* neighbors;       /* the lists */
    int32_t* neighbor_counts;  /* [atoms] */
    int32_t* sorted;           /* [atoms] */
    int32_t* scratch;          /* [atoms] */
    int32_t* cell_starts;      /* the cell tables */
    void* ordered_positions;   /* [atoms, 4] float32: the last rebuild's positions in cell order */
} nd_replica_pool;

/* A CUDA graph of `steps` steps of the system (no virial) whose rebuild kernels run in the body
 * of a conditional IF node, set on the device from the reuse check's flag: a step that reuses
 * the list launches four kernels. The graph bakes in the system's buffers. Replaces the
 * reference's capture of its whole step into one CUDA Graph (src/nabladyn/md/_simulation.py:
 * 366-402), whose rebuild is gated inside the operator's kernels. */
int nd_md_graph_create(const nd_md_system* system, int thermostat, int steps, void** graph_out);
int nd_md_graph_launch(void* graph, nd_stream_t stream);
int nd_md_graph_destroy(void* graph);

/* mode 0: admit the listed slots (wrap, build, first forces). mode 1: run each listed slot for
 * min(budgets[k], steps_left) steps. One CTA per listed slot; slots never interact. */
int nd_serve_run(const nd_replica_pool* pool, const int32_t* slots, const int32_t* budgets,
                 int32_t count, int32_t mode, nd_stream_t stream);

/* ---- SchNet (src/nabladyn/potential/_schnet/_potential.py:45-208) ---------------------------
 * E, F and W of a SchNet model with 64 features and 2..64 Gaussians over a [2, C] pair list,
 * float32 positions, BF16 tcgen05 tensor cores with FP32 accumulation for every 64 x 64 product,
 * the reverse pass by hand, E and W in float64. Replaces the reference's autograd evaluation
 * of SchNet._energy_wrapped under quantity.energy_force_virial (src/nabladyn/quantity.py:93-117);
 * the reference has no native counterpart. */
typedef struct nd_schnet_args {
    int64_t num_atoms;          /* N */
    int64_t num_columns;        /* C: columns of pairs */
    int32_t interactions;       /* blocks */
    int32_t num_types;          /* T */
    int32_t gaussians;          /* K, 2..64 */
    int32_t reserved;
    double cutoff;              /* nm */
    const float* positions;     /* [N, 3], wrapped into [0, L) */
    const float* cell;          /* [3] */
    const int32_t* pairs;       /* [2, C]: first atoms, then second atoms; equal = padding */
    const int64_t* atom_types;  /* [N] in [0, T) */
    const void* weights;        /* nd_schnet_weight_bytes bytes, 256-byte aligned (packed by
                                   the host: per block ten 64 x 64 BF16 operand images, then
                                   float32 biases, readout and the embedding tables) */
    void* workspace;            /* nd_schnet_workspace_bytes bytes, 256-byte aligned */
    double* energy;             /* [1] */
    float* forces;              /* [N, 3] or NULL */
    double* virial;             /* [9] or NULL */
    int32_t* status;            /* [4]: pairs within the cutoff, status bits (1: a pair index
                                   out of range; 16: a tensor-core product did not complete
                                   within its bounded wait), and for that case the first
                                   kernel stage (16 * kernel + product) and tile that gave up */
} nd_schnet_args;

int64_t nd_schnet_weight_bytes(int32_t interactions, int32_t num_types);
int64_t nd_schnet_workspace_bytes(int64_t num_atoms, int64_t num_columns, int32_t interactions);
int nd_schnet_energy_force_virial(const nd_schnet_args* args, nd_stream_t stream);

/* The per-pair passes of SchNet's parameter gradient of a training loss over E, F and W, by
 * forward-over-reverse along the loss's adjoints: one block's filter network with its
 * derivative along each pair's rate rdot = (d . (dL/dF_a - dL/dF_b) + d^T dL/dW d) / r.
 * direction 0 (forward) writes the block's messages m (those of the E/F/W call, from its
 * workspace) and adds their tangent m_dot; direction 1 (reverse) adds
 * v_bar and v_dot_bar and writes every pair's BF16 rows (g, g_dot, s, s_dot, z_bar, z_dot_bar,
 * u_bar, u_dot_bar), from which the filter weights' gradients are sums over pairs. Reads the
 * compacted pairs in `workspace` of the nd_schnet_energy_force_virial call just made with the
 * same weights, positions, pairs and sizes. Replaces the double backward of the reference's
 * torch.func gradient program (src/nabladyn/training/_fit.py:245-271) for the pair terms; the
 * reference has no native counterpart. */
typedef struct nd_schnet_tangent_args {
    int64_t num_atoms;              /* N, as in the E/F/W call */
    int64_t num_columns;            /* C, as in the E/F/W call */
    int32_t interactions;
    int32_t num_types;
    int32_t gaussians;
    int32_t block;                  /* the interaction block, 0 .. interactions - 1 */
    double cutoff;
    const void* weights;            /* the packed parameter block of the E/F/W call */
    void* workspace;                /* the workspace that call filled */
    const float* force_adjoint;     /* [N, 3] dL/dF */
    const double* virial_adjoint;   /* [9] dL/dW, row-major */
    const void* v;                  /* [N, 64] BF16: this block's x A^T */
    const void* v_dot;              /* [N, 64] BF16: its derivative along the direction */
    float* m;                       /* forward: [N, 64], written */
    float* m_dot;                   /* forward: [N, 64], added to */
    const void* m_bar;              /* reverse: [N, 64] BF16 */
    const void* m_dot_bar;          /* reverse: [N, 64] BF16 */
    float* v_bar;                   /* reverse: [N, 64], added to */
    float* v_dot_bar;               /* reverse: [N, 64], added to */
    void* pair_rows;                /* reverse: [8, capacity, 64] BF16, rows of pairs in the
                                       compacted order; rows past the pair count set to zero */
    int64_t capacity;               /* at least num_columns */
    int32_t* status;                /* [4], as for nd_schnet_energy_force_virial */
} nd_schnet_tangent_args;

int nd_schnet_tangent(const nd_schnet_tangent_args* args, int32_t direction, nd_stream_t stream);

/* The atom-wise layers of the same parameter gradient (the embedding, each block's A, D1, d1,
 * D2, d2 and the readout, src/nabladyn/potential/_schnet/_potential.py:76-88, 190-208) with
 * their tangents and reverse, in FP32, and the sums over atoms that give those parameters'
 * gradients (added to `gradient`). Stages, with nd_schnet_tangent between them:
 *   0 start (x_0 from the table, v_0; clears every block's message and scatter buffers),
 *   1 block forward after its tangent forward pass (h, x', v' and their tangents),
 *   2 readout (x_bar, x_dot_bar and the readout's gradients),
 *   3 block reverse before its tangent reverse pass (m_bar, m_dot_bar; D2, d2, D1, d1),
 *   4 block reverse after it (x_bar += v_bar A, x_dot_bar += v_dot_bar A; A).
 * The per-atom arrays live in `workspace` at nd_schnet_atom_offset(N, blocks, kind, block):
 * FP32 [N, 64] per block: 0 x, 1 x_dot, 2 h, 3 h_dot, 4 m, 5 m_dot, 6 v_bar, 7 v_dot_bar;
 * FP32: 8 x and 9 x_dot after the last block, 10 x_bar, 11 x_dot_bar (after stage 4 of
 * block 0: dL/d(embedding rows)); BF16 [N, 64]: 12 v, 13 v_dot per block, 14 m_bar,
 * 15 m_dot_bar; 16 the per-tile partial sums. No counterpart in the reference. */
typedef struct nd_schnet_atom_args {
    int64_t num_atoms;              /* N */
    int32_t interactions;           /* blocks */
    int32_t num_types;              /* T */
    const int64_t* atom_types;      /* [N] in [0, T) */
    const float* parameters;        /* nd_schnet_atom_parameter_floats floats: per block
                                       A [64][64], D1 [64][64], d1 [64], D2 [64][64], d2 [64];
                                       then R1 [32][64], e1 [32], R2 [32], e2 (padded to 32);
                                       then the embedding [T][64] */
    float* gradient;                /* the same layout, added to */
    const double* energy_adjoint;   /* [1] dL/dE */
    void* workspace;                /* nd_schnet_atom_workspace_bytes, 256-byte aligned */
} nd_schnet_atom_args;

int64_t nd_schnet_atom_parameter_floats(int32_t interactions, int32_t num_types);
int64_t nd_schnet_atom_workspace_bytes(int64_t num_atoms, int32_t interactions);
int64_t nd_schnet_atom_offset(int64_t num_atoms, int32_t interactions, int32_t kind,
                              int32_t block);
int nd_schnet_atoms(const nd_schnet_atom_args* args, int32_t stage, int32_t block,
                    nd_stream_t stream);

/* ---- Integrator of frames in the caller's order ------------------------------------------
 * Velocity Verlet with the Nose-Hoover chain of three (src/nabladyn/md/_ensembles/_nve.py:39-58,
 * _nvt.py:88-129, _chain.py:23-105) and isotropic MTK NPT with chains on the particles and the
 * barostat (_npt.py:66-251) for any potential: the caller runs its neighbor update and forces
 * (with the virial for NPT) between nd_integrate_open and nd_integrate_close. `mode` is 0 NVE,
 * 1 NVT, 2 NPT. The thermostat block has the MD engine's layout (nd_md_system.thermostat);
 * totals[1] gets the step's K, totals[9] the K of nd_integrate_kinetic. Replaces the ensemble
 * halves the reference compiles with Inductor. */
typedef struct nd_integrator {
    int dtype;               /* ND_FLOAT32 or ND_FLOAT64 */
    int64_t num_atoms;
    void* positions;         /* [N, 3], wrapped into [0, L) */
    void* velocities;        /* [N, 3] (the pending chain factor not yet applied) */
    const void* forces;      /* [N, 3] */
    const void* masses;      /* [N] */
    int64_t* images;         /* [N, 3] */
    void* cell;              /* [3]; NPT rescales it */
    double* thermostat;      /* [24] */
    double* partials;        /* [nd_integrate_partial_slots] */
    double* totals;          /* [16] */
    int32_t* status;         /* [1]: bit 2 a non-finite coordinate */
    double timestep;         /* ps */
    double* barostat;        /* [32] for NPT (else NULL): p_eps, its chain q[3] p[3] and masses
                                [3], box mass, pressure, alpha = 1 + 1/N, the float64 cell [3],
                                this step's drag and growth */
    const double* virial;    /* [9] W of the last forces, for NPT (else NULL) */
} nd_integrator;

int nd_integrate_partial_slots(int64_t num_atoms, int64_t* slots);
int nd_integrate_open(const nd_integrator* s, int mode, nd_stream_t stream);
int nd_integrate_close(const nd_integrator* s, int mode, nd_stream_t stream);
int nd_integrate_kinetic(const nd_integrator* s, int mode, nd_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* NABLADYN_B200_H */
