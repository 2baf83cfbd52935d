/*
 * dfft.h - C ABI of the B200-native distributed 3D FFT execute path.
 *
 * One process drives one GPU.  The ranks of a slab or pencil topology are
 * virtual: every buffer handed to dfft_execute holds the local blocks of all
 * ranks of the topology, concatenated in rank order (rank 0 first), each block
 * in exactly the shape and memory order that rank holds in the reference
 * library (see dfft_get_local_extents / dfft_get_local_offset).  The
 * all-to-all exchanges between the FFT stages become on-device permutations.
 *
 * Every entry point returns a dfft_status; nothing throws across the ABI.
 * dfft_last_error_string() gives the message of the last failure on the
 * calling thread.
 *
 * Reference interfaces replaced (paths relative to the reference's
 * distributed/src/):
 *   KokkosFFT::Distributed::Plan ctor        KokkosFFT_Distributed_Plan.hpp:154-181
 *   internal_plan_factory                    KokkosFFT_Distributed_Plan.hpp:46-113
 *   KokkosFFT::Distributed::execute          KokkosFFT_Distributed_Plan.hpp:212-238
 *   Plan::name                               KokkosFFT_Distributed_Plan.hpp:200
 *   compute_local_extents_and_starts         KokkosFFT_Distributed_MPI_Extents.hpp:546-577
 *   BlockInfo / block analyses               KokkosFFT_Distributed_Types.hpp:61-154,
 *                                            KokkosFFT_Distributed_BlockAnalyses.hpp:391-506
 *   get_all_slab/pencil_topologies           KokkosFFT_Distributed_Topologies.hpp:421-811
 *   TransBlock pack/all2all/unpack buffers   KokkosFFT_Distributed_TransBlock.hpp:76-107
 */
#ifndef DFFT_H
#define DFFT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DFFT_MAX_RANK 4

typedef enum {
  DFFT_SUCCESS = 0,
  DFFT_ERROR_INVALID_ARGUMENT = 1,
  DFFT_ERROR_INVALID_TOPOLOGY = 2,
  DFFT_ERROR_INVALID_EXTENTS = 3,
  DFFT_ERROR_UNSUPPORTED = 4,
  DFFT_ERROR_CUDA = 5,
  DFFT_ERROR_ALLOC = 6,
  DFFT_ERROR_INTERNAL = 7,
  DFFT_ERROR_TIMEOUT = 8
} dfft_status;

/* Transform kind.  R2C plans run C2R on dfft_execute(..., DFFT_BACKWARD). */
typedef enum { DFFT_KIND_C2C = 0, DFFT_KIND_R2C = 1 } dfft_kind;

/* Storage and arithmetic precision: complex128/float64 or complex64/float32.
 * DFFT_PREC_F32_COMPENSATED stores and computes like DFFT_PREC_F32, except
 * that the last radix pass of every two-line C2C stage (power-of-two lines
 * on 16-byte aligned buffers: the stages of 3D C2C pencils and slabs) runs in
 * compensated arithmetic: exact twiddle products through fused multiply-adds,
 * error-free two-sum additions carried as hi + lo float pairs, one rounding
 * per output.  Other stages run the plain FP32 kernels.  No counterpart in the
 * reference (which has no FP32 path with compensation). */
typedef enum { DFFT_PREC_F64 = 0, DFFT_PREC_F32 = 1, DFFT_PREC_F32_COMPENSATED = 2 } dfft_precision;

/* KokkosFFT::Normalization (default backward: 1/N on the backward transform). */
typedef enum {
  DFFT_NORM_BACKWARD = 0,
  DFFT_NORM_FORWARD = 1,
  DFFT_NORM_ORTHO = 2,
  DFFT_NORM_NONE = 3
} dfft_normalization;

typedef enum { DFFT_FORWARD = 0, DFFT_BACKWARD = 1 } dfft_direction;

/* Execution strategy.
 *   DFFT_EXEC_FUSED           : one kernel per FFT axis; pack, all-to-all,
 *                               unpack, local transposes and normalisation are
 *                               folded into the loads and stores of those
 *                               kernels (default).
 *   DFFT_EXEC_LITERAL         : the reference's block sequence kernel by kernel
 *                               (local transposes, per-axis FFTs, pack,
 *                               all-to-all permutation, unpack, normalisation).
 *   DFFT_EXEC_LITERAL_CAPTURE : as DFFT_EXEC_LITERAL, and every transpose
 *                               block's pack input, send and recv buffers and
 *                               unpack output are kept for
 *                               dfft_debug_export_buffers. */
typedef enum { DFFT_EXEC_FUSED = 0, DFFT_EXEC_LITERAL = 1, DFFT_EXEC_LITERAL_CAPTURE = 2 } dfft_exec_mode;

typedef struct {
  int32_t rank;                         /* view rank, 2..4 */
  int32_t fft_rank;                     /* number of FFT axes, 1..3 */
  int32_t axes[3];                      /* FFT axes (negative values count from the end) */
  uint64_t in_extents[DFFT_MAX_RANK];   /* global extents of the input (real extents for R2C) */
  uint64_t out_extents[DFFT_MAX_RANK];  /* global extents of the (complex) output */
  uint64_t in_topology[DFFT_MAX_RANK];  /* ranks along each axis for the input */
  uint64_t out_topology[DFFT_MAX_RANK]; /* ranks along each axis for the output */
  int32_t in_topology_layout_right;     /* rank order of in_topology: 1 LayoutRight (default), 0 LayoutLeft */
  int32_t out_topology_layout_right;    /* rank order of out_topology */
  int32_t view_layout_right;            /* memory order of the local blocks: 1 C order, 0 Fortran order */
  int32_t kind;                         /* dfft_kind */
  int32_t precision;                    /* dfft_precision */
  int32_t normalization;                /* dfft_normalization */
  int32_t exec_mode;                    /* dfft_exec_mode */
  void* stream;                         /* cudaStream_t the plan launches on (NULL: legacy default stream) */
} dfft_plan_desc;

/* One entry of the reference's block list for one virtual rank
 * (BlockInfo, KokkosFFT_Distributed_Types.hpp:61-154). */
typedef struct {
  int32_t block_type; /* 0 Transpose, 1 FFT */
  int32_t block_idx;
  int32_t fft_dim;
  int32_t in_axis, out_axis, comm_axis;
  uint64_t in_topology[DFFT_MAX_RANK];
  uint64_t out_topology[DFFT_MAX_RANK];
  uint64_t in_extents[DFFT_MAX_RANK];
  uint64_t out_extents[DFFT_MAX_RANK];
  uint64_t buffer_extents[DFFT_MAX_RANK + 1];
  uint64_t in_map[DFFT_MAX_RANK];
  uint64_t out_map[DFFT_MAX_RANK];
} dfft_block_info;

typedef struct dfft_plan_s dfft_plan;

/* Fill a descriptor with the reference defaults (LayoutRight everywhere,
 * C2C, F64, backward normalisation, fused execution, legacy stream). */
void dfft_plan_desc_init(dfft_plan_desc* d);

/* Plan construction (Plan ctor + internal_plan_factory).  Validates the
 * topologies and extents like the reference and allocates the plan's device
 * scratch and tables on the current CUDA device. */
dfft_status dfft_plan_create(dfft_plan** plan, const dfft_plan_desc* desc);

/* Host-only planning: validation and block analyses without touching the GPU.
 * The returned plan answers the query functions below but cannot execute. */
dfft_status dfft_plan_analyze(dfft_plan** plan, const dfft_plan_desc* desc);

dfft_status dfft_plan_destroy(dfft_plan* plan);

/* execute(plan, in, out, direction).  Device pointers to concatenated per-rank
 * blocks.  DFFT_FORWARD reads the input layout from `in` and writes the output
 * layout to `out`; DFFT_BACKWARD reads the (complex) output layout from `in`
 * and writes the input layout to `out`.  `in` is not modified.  Asynchronous
 * on the plan's stream.  Each buffer must be aligned to its element type
 * (real or complex of the plan's precision); a misaligned pointer is rejected
 * with DFFT_ERROR_INVALID_ARGUMENT before any launch. */
dfft_status dfft_execute(const dfft_plan* plan, const void* in, void* out, int32_t direction);

/* Same as dfft_execute with an explicit stream (overrides the plan's). */
dfft_status dfft_execute_on_stream(const dfft_plan* plan, const void* in, void* out, int32_t direction,
                                   void* stream);

/* Adjoint (conjugate transpose, normalisation included) of the plan's forward
 * (direction = DFFT_FORWARD: reads the complex output layout, writes the input
 * layout) or backward transform (DFFT_BACKWARD: reads the input layout, writes
 * the complex output layout).  For R2C plans the real-input adjoint weights
 * the interior modes of the R2C axis (1/2 before C2R, 2 after R2C), so that
 * <F x, y> = <x, F^H y> with the real inner product.  No counterpart in the
 * reference (used for gradients through the transform). */
dfft_status dfft_execute_adjoint(const dfft_plan* plan, const void* in, void* out, int32_t direction, void* stream);

/* "SlabPlan", "PencilPlan" or "SharedPlan" (Plan::name). */
const char* dfft_plan_name(const dfft_plan* plan);

/* Number of virtual ranks (total size of the topology). */
dfft_status dfft_get_nprocs(const dfft_plan* plan, int64_t* nprocs);

/* Local extents and starts (logical axis order) of a rank's block; which = 0
 * input layout, 1 output layout (compute_local_extents_and_starts). */
dfft_status dfft_get_local_extents(const dfft_plan* plan, int64_t rank, int32_t which, uint64_t* extents,
                                   uint64_t* starts);

/* Element offset of a rank's block inside the concatenated buffer. */
dfft_status dfft_get_local_offset(const dfft_plan* plan, int64_t rank, int32_t which, uint64_t* offset);

/* Number of elements (real for an R2C input, complex otherwise) of the
 * concatenated input (which = 0) or output (which = 1) buffer. */
dfft_status dfft_get_buffer_elements(const dfft_plan* plan, int32_t which, uint64_t* count);

/* The reference's block list for one virtual rank. */
dfft_status dfft_get_num_blocks(const dfft_plan* plan, int64_t* nblocks);
dfft_status dfft_get_block_info(const dfft_plan* plan, int64_t rank, int64_t block, dfft_block_info* info);

/* Max buffer size over ranks in elements of the real type (m_max_buffer_size). */
dfft_status dfft_get_max_buffer_size(const dfft_plan* plan, uint64_t* size);

/* Topology chain of the slab / pencil analyses.  On entry *n is the capacity
 * (number of topologies) of the arrays; on return the chain length.
 * topologies is [n][rank]; trans_axes [n-1] and layouts [n] are pencil-only
 * (zeros for slabs). */
dfft_status dfft_get_topology_chain(const dfft_plan* plan, int64_t* n, uint64_t* topologies, int64_t* trans_axes,
                                    int64_t* layouts);

/* ---- One process per GPU: per-rank plans ----
 * The reference's distributed Plan on one MPI / NCCL rank
 * (KokkosFFT_Distributed_Plan.hpp:154-238 with a communicator of
 * nprocs = prod(in_topology) ranks): the plan holds only rank `rank`'s
 * program, reads its local input block and writes its local output block
 * (dfft_get_local_extents with that rank, logical axis order, contiguous in
 * the view's memory order), and leaves every all-to-all of a TransBlock
 * (KokkosFFT_Distributed_TransBlock.hpp:76-107) to the caller's communicator,
 * as the reference's backends do with MPI_Alltoall or ncclSend / ncclRecv
 * pairs (KokkosFFT_Distributed_MPI_All2All.hpp:23-58,
 * KokkosFFT_Distributed_NCCL_All2All.hpp:21-89).
 *
 * A direction runs as dfft_get_num_exchanges + 1 segments.  Segment 0 reads
 * `in`; every segment but the last ends with exchange k's send buffer
 * written in the reference's pack order ([group size, buffer extents] for
 * LayoutRight views, [buffer extents, group size] for LayoutLeft: the pack
 * folded into the last FFT stage's stores); the caller's all-to-all over the
 * exchange's group then sends chunk j (element_bytes * elements / group_size
 * bytes) to group member j and receives chunk j from member j; segment k + 1
 * reads the recv buffer in place (the unpack folded into the next stage's
 * loads); the last segment writes `out`.  The group of exchange k is the
 * whole communicator (slab plans) or the row / column communicator of the
 * Cartesian grid over the split entries of in_topology
 * (KokkosFFT_Distributed_PencilPlan.hpp:32-71), members in rank order.  When
 * `padded` is set, entries of the send buffer past the pack bins are never
 * written: keep them zero (clear the buffer once) so that the exchanged bytes
 * equal the reference's. */
dfft_status dfft_plan_create_rank(dfft_plan** plan, const dfft_plan_desc* desc, int64_t rank);
/* Host-only form (queries only). */
dfft_status dfft_plan_analyze_rank(dfft_plan** plan, const dfft_plan_desc* desc, int64_t rank);

typedef struct {
  int64_t block;          /* index of the transpose block in the block list */
  int32_t comm_axis;      /* -1 whole communicator, 0 row, 1 column communicator */
  int32_t padded;         /* 1: the send buffer has entries no segment writes (keep them zero) */
  uint64_t elements;      /* elements of the send buffer (= recv buffer), all peers' chunks */
  uint64_t element_bytes; /* bytes of one element (real before the first R2C stage, complex after) */
  int64_t group_size;     /* members of the exchange group (chunks of the buffers) */
} dfft_exchange_info;

dfft_status dfft_get_num_exchanges(const dfft_plan* plan, int32_t direction, int64_t* n);
dfft_status dfft_get_exchange_info(const dfft_plan* plan, int32_t direction, int64_t k, dfft_exchange_info* info);
/* Group of exchange k as seen by world rank `rank` (any rank, so that every
 * process can create every sub-communicator collectively): its index in the
 * group and the group's world ranks by group index (group_size entries). */
dfft_status dfft_get_exchange_group(const dfft_plan* plan, int32_t direction, int64_t k, int64_t rank,
                                    int64_t* sub_rank, int64_t* members);
/* Run one segment on `stream`.  in: segment 0; out: the last segment; send:
 * every segment but the last (exchange `segment`'s send buffer); recv: every
 * segment but the first (exchange `segment - 1`'s recv buffer). */
dfft_status dfft_execute_segment(const dfft_plan* plan, int32_t direction, int64_t segment, const void* in,
                                 void* out, void* send, void* recv, void* stream);

/* All segments of a direction with the caller's all-to-all in between:
 * exchange(user, k, send, recv, bytes_per_peer, stream) must move exchange
 * k's chunks (ordered on `stream`, or complete before returning) and return
 * 0, or non-zero to abort (DFFT_ERROR_CUDA with that code in the message).
 * send and recv must hold the largest exchange. */
typedef int32_t (*dfft_exchange_fn)(void* user, int64_t k, const void* send, void* recv, uint64_t bytes_per_peer,
                                    void* stream);
dfft_status dfft_execute_exchanged(const dfft_plan* plan, const void* in, void* out, int32_t direction, void* send,
                                   void* recv, dfft_exchange_fn exchange, void* user, void* stream);

/* ---- Batched execution under a CUDA graph ----
 * Captures, once, the execution of `count` transforms (plans[i] applied to
 * ins[i] -> outs[i] in directions[i]) into one CUDA graph.  Transforms with
 * the same branches[i] run in order on one branch; different branches run
 * concurrently (branches = NULL: every transform on its own branch), so fields
 * of different sizes overlap.  The buffers are baked into the graph:
 * every dfft_graph_launch repeats the same transforms on the same pointers.
 * Plans must outlive the graph.  All transforms of one plan must be on the
 * same branch (they share the plan's scratch arrays); a plan on two branches
 * is rejected with DFFT_ERROR_INVALID_ARGUMENT.  No counterpart in the reference (its
 * batched Navier-Stokes example loops over execute calls). */
typedef struct dfft_graph_s dfft_graph;
dfft_status dfft_graph_create(dfft_graph** graph, const dfft_plan* const* plans, const void* const* ins,
                              void* const* outs, const int32_t* directions, const int32_t* branches, int64_t count);
dfft_status dfft_graph_launch(const dfft_graph* graph, void* stream);
dfft_status dfft_graph_destroy(dfft_graph* graph);

/* ---- Batched execution of many plans (fields of uneven sizes) ----
 * A batch holds distinct, executable fused plans of one precision (the same
 * plan twice is rejected: its scratch arrays would be shared).  One execute
 * transforms ins[i] -> outs[i] with plans[i] for every field, in the given
 * direction, on one stream: each stage index of the fields' programs runs as
 * one persistent launch per group of stages of the same kind, direction and
 * row orientation (a work table of every field's tiles, any supported line
 * lengths: 2^k up to 2048 and 3 * 2^k up to 768, register kernels), instead
 * of one launch per field; stages outside that set launch per field.  Buffers
 * follow dfft_execute.  Capture dfft_batch_execute in a CUDA graph to replay
 * it.  No counterpart in the reference (its batched Navier-Stokes example
 * drives one plan over 4D views per field,
 * examples/navier-stokes-MPI-batched/main.cpp:465-468). */
typedef struct dfft_batch_s dfft_batch;
dfft_status dfft_batch_create(dfft_batch** batch, const dfft_plan* const* plans, int64_t count);
dfft_status dfft_batch_execute(const dfft_batch* batch, const void* const* ins, void* const* outs, int32_t direction,
                               void* stream);
/* kernel launches of one dfft_batch_execute in a direction */
dfft_status dfft_batch_get_launch_count(const dfft_batch* batch, int32_t direction, int64_t* launches);
dfft_status dfft_batch_destroy(dfft_batch* batch);

/* ---- Pseudo-spectral Navier-Stokes step of the reference's batched example
 * (examples/navier-stokes-MPI-batched/main.cpp:518-669, RK4 of
 * examples/utils/math_utils.hpp:90-141) on a plan's buffers.  The plan must be
 * an R2C plan over LayoutRight 4D views (3, nx, ny, nz) with FFT axes {1,2,3};
 * uk is its output (spectral) buffer.  nu = 1/Re, dt the time step, the
 * domain is [0, lx*pi)^3 (lx = 2 for [0, 2 pi)). */
typedef struct dfft_ns_s dfft_ns;
dfft_status dfft_ns_create(dfft_ns** ns, const dfft_plan* plan, double nu, double dt, double lx);
/* Taylor-Green vortex (main.cpp:322-363): u = (v0 sin x cos y cos z,
 * -v0 cos x sin y cos z, 0) on x = lx pi i / nx, uk = its forward transform,
 * dealiased and projected onto the divergence-free space */
dfft_status dfft_ns_init_taylor_green(dfft_ns* ns, void* uk, double v0, void* stream);
/* dukdt = right-hand side at uk (uk is dealiased in place, as in the reference) */
dfft_status dfft_ns_rhs(dfft_ns* ns, void* uk, void* dukdt, void* stream);
/* one RK4 time step of uk in place (4 right-hand sides: 20 transforms) */
dfft_status dfft_ns_step(dfft_ns* ns, void* uk, void* stream);
/* total kinetic energy of main.cpp:746-766, (lx pi)^3 / N^2 * sum 0.5 factor |uk|^2
 * (factor 1 on kz = 0, else 2), FP64 reduction; synchronises the stream */
dfft_status dfft_ns_energy(dfft_ns* ns, const void* uk, double* energy, void* stream);
/* One RK4 time step of `count` fields (distinct states, uks[i] the spectral
 * buffer of states[i]) captured once into a library-owned CUDA graph.
 *   batched = 1: per RK stage the pointwise phases per field and every
 *     transform of all fields through one batched execution (one launch per
 *     stage of the transform; the states' plans must be distinct);
 *   batched = 0: each field's step on one of up to four concurrent graph
 *     branches with its plan's tuned kernels (fields sharing a plan on one
 *     branch).
 * dfft_graph_launch advances every field by one step; dfft_graph_destroy
 * frees it.  States and plans must outlive the graph.  No counterpart in the
 * reference (main.cpp:518-586 loops over the fields' RK4 stages). */
dfft_status dfft_ns_graph_create(dfft_graph** graph, dfft_ns* const* states, void* const* uks, int64_t count,
                                 int32_t batched);
/* Physical velocity of a spectrum (the backward transform of diag_fields,
 * main.cpp:711-724) into a buffer of the plan's input layout; uk is not
 * modified. */
dfft_status dfft_ns_velocity(dfft_ns* ns, const void* uk, void* u, void* stream);
/* Physical vorticity curl u (compute_vorticity, main.cpp:677-698: i k x uk
 * with the full, not dealiased, wavenumbers, then the backward transform)
 * into a buffer of the plan's input layout; uk is not modified. */
dfft_status dfft_ns_vorticity(dfft_ns* ns, const void* uk, void* vor, void* stream);
/* Diagnostics of a spectrum, reduced in FP64 whatever the plan's precision:
 *   energy         as dfft_ns_energy (main.cpp:746-766);
 *   enstrophy      (1/2) integral |curl u|^2 = coef sum 0.5 f |k x uk|^2;
 *   divergence_l2  (integral |div u|^2)^(1/2) = (coef sum f |k . uk|^2)^(1/2);
 * with f = 1 on the kz = 0 plane, 2 elsewhere, coef = (lx pi)^3 / N^2.
 * With num_bins > 0, e_spec[i] = sum of 0.5 f |uk|^2 over the modes with
 * k_bins[i] <= |k| < k_bins[i + 1], k_bins = linspace(0, k_max, num_bins + 1)
 * (k_max the largest |k| of the grid) and k_vals[i] the bin midpoints
 * (diag_energy, main.cpp:471-500, :741-794; the reference uses 50 bins).
 * num_bins <= DFFT_NS_MAX_BINS.  Synchronises the stream. */
#define DFFT_NS_MAX_BINS 2048
typedef struct {
  double energy;
  double enstrophy;
  double divergence_l2;
} dfft_ns_diag;
dfft_status dfft_ns_diagnostics(dfft_ns* ns, const void* uk, int32_t num_bins, double* e_spec, double* k_vals,
                                dfft_ns_diag* out, void* stream);
/* The reference's diagnostic files of one iteration (diag_fields +
 * diag_energy, main.cpp:705-818): for every virtual rank, the components of
 * its local block of the velocity (u, v, w) and of the vorticity (vor_x,
 * vor_y, vor_z) as raw arrays of the plan's real type in C order, named
 * "<out_dir>/<label>_rx<rx:03>_ry<ry:03>_<iter:010>.dat" with (rx, ry) the
 * rank's coordinates in the in_topology (1, px, py, 1); and E_spec / k_vals
 * (num_bins doubles each) under the coordinates of rank 0.  The directory must
 * exist.  `out` (may be NULL) receives the diagnostics of dfft_ns_diagnostics.
 * Synchronises the stream. */
dfft_status dfft_ns_write_diagnostics(dfft_ns* ns, const void* uk, const char* out_dir, int32_t iter,
                                      int32_t num_bins, dfft_ns_diag* out, void* stream);
/* Adjoints of the right-hand side and of the RK4 step, for gradients
 * through the solver.  Cotangents live in the spectral (output) layout and
 * pair with tangents through the real inner product Re sum conj(a) b over the
 * stored half spectrum, the inner product of dfft_execute_adjoint.
 *   dfft_ns_rhs_adjoint:  grad = (d f / d uk)^T lambda for f(uk) = the
 *     right-hand side of dfft_ns_rhs at uk (which first dealiases uk); the
 *     physical velocity and its gradients are recomputed from uk (nine
 *     transforms), nothing of a forward call is stored;
 *   dfft_ns_step_adjoint: lambda <- (d S / d uk)^T lambda for one RK4 step S
 *     of dfft_ns_step from state uk; the four stage states are recomputed from
 *     uk (three right-hand sides), then the four stage VJPs run backwards.
 * uk and lambda are not modified (except lambda's update in the step
 * adjoint).  The first call allocates the adjoint workspace (five spectral
 * and one physical buffer).  No counterpart in the reference. */
dfft_status dfft_ns_rhs_adjoint(dfft_ns* ns, const void* uk, const void* lambda, void* grad, void* stream);
dfft_status dfft_ns_step_adjoint(dfft_ns* ns, const void* uk, void* lambda, void* stream);
dfft_status dfft_ns_destroy(dfft_ns* ns);

/* get_all_slab_topologies (pencil = 0) / get_all_pencil_topologies (pencil = 1),
 * KokkosFFT_Distributed_Topologies.hpp:421-618 / :645-811, on their own.  On
 * entry *n is the capacity (number of topologies) of the output arrays; on
 * return the chain length.  topologies is [n][rank], trans_axes [n-1] and
 * layouts [n] (pencil only).  Fails with DFFT_ERROR_INVALID_TOPOLOGY where the
 * reference throws. */
dfft_status dfft_get_all_topologies(int32_t pencil, int32_t rank, const uint64_t* in_topology,
                                    int32_t in_layout_right, const uint64_t* out_topology, int32_t out_layout_right,
                                    int32_t fft_rank, const int32_t* axes, int64_t* n, uint64_t* topologies,
                                    int64_t* trans_axes, int64_t* layouts);

/* ---- The data-movement layer on its own ----
 * The reference's pack / unpack of one rank's view
 * (KokkosFFT::Distributed::Impl::pack / unpack,
 * KokkosFFT_Distributed_PackUnpack.hpp:439-499), its all-to-all
 * (Impl::all2all, KokkosFFT_Distributed_MPI_All2All.hpp:23-58) here over every
 * virtual rank at once, and the TransBlock that chains them
 * (KokkosFFT_Distributed_TransBlock.hpp:38-107).  They run the same kernels as
 * the plans' literal programs.
 *   - views and buffers are device arrays of elements of element_bytes (4, 8
 *     or 16; the kernels copy whole elements, so float, double, complex64 and
 *     complex128 all work) aligned to element_bytes;
 *   - a view of rank D gives its extents in its own dimension order (the
 *     rank's local extents permuted by its map: dimension i holds logical
 *     axis map[i]); a buffer has rank D + 1, the process dimension first for
 *     layout_right = 1 (LayoutRight) and last for 0 (LayoutLeft), which is
 *     also the memory order of views and buffers;
 *   - pack splits logical axis `axis` into the buffer's process bins (the
 *     first n % P bins one larger, zeros outside a bin); unpack merges it;
 *   - asynchronous on `stream`; pack / unpack / all2all use a few hundred
 *     bytes of stream-ordered device memory for their index tables. */
dfft_status dfft_pack(int32_t rank, const uint64_t* src_extents, const int32_t* src_map, int32_t axis,
                      const uint64_t* buffer_extents, int32_t layout_right, int32_t element_bytes, const void* src,
                      void* dst, void* stream);
dfft_status dfft_unpack(int32_t rank, const uint64_t* buffer_extents, const int32_t* dst_map, int32_t axis,
                        const uint64_t* dst_extents, int32_t layout_right, int32_t element_bytes, const void* src,
                        void* dst, void* stream);
/* MPI_Alltoall of every virtual rank: send and recv hold nprocs buffers of
 * buffer_extents (rank buffer_rank), rank after rank; recv of rank r, chunk j
 * = send of the j-th member of r's communicator, chunk (r's rank in it).
 * comm_axis -1: one communicator of all ranks; 0 / 1: the row / column
 * communicators MPI_Cart_sub keeps from MPI_Cart_create over the entries of
 * cart_topology (cart_rank entries) larger than one (row-major, no
 * reordering), as the pencil plans build them
 * (KokkosFFT_Distributed_PencilPlan.hpp:32-71).  The buffer's process extent
 * must equal the communicator size. */
dfft_status dfft_all2all(int64_t nprocs, int32_t buffer_rank, const uint64_t* buffer_extents, int32_t layout_right,
                         int32_t comm_axis, int32_t cart_rank, const uint64_t* cart_topology, int32_t element_bytes,
                         const void* send, void* recv, void* stream);

/* TransBlock over every rank of a topology pair.  Forward packs the input
 * blocks (in_topology, src_map) along src_axis, exchanges, and unpacks into
 * the output blocks (out_topology, dst_map) merging dst_axis; backward is the
 * reverse.  The buffer extents are compute_buffer_extents(global_extents,
 * in_topology, out_topology) (dfft_trans_block_buffer_extents). */
typedef struct {
  int32_t rank;                           /* view rank, 2..4 */
  uint64_t global_extents[DFFT_MAX_RANK];
  uint64_t in_topology[DFFT_MAX_RANK];
  uint64_t out_topology[DFFT_MAX_RANK];
  int32_t in_topology_layout_right;       /* rank order of in_topology (1 LayoutRight) */
  int32_t out_topology_layout_right;
  int32_t src_map[DFFT_MAX_RANK];         /* map of the input views */
  int32_t dst_map[DFFT_MAX_RANK];         /* map of the output views */
  int32_t src_axis;                       /* forward: split on send */
  int32_t dst_axis;                       /* forward: merged on receive */
  int32_t view_layout_right;              /* memory order of views and buffers */
  int32_t element_bytes;                  /* 4, 8 or 16 */
  int32_t comm_axis;                      /* as dfft_all2all */
  uint64_t cart_topology[DFFT_MAX_RANK];  /* as dfft_all2all; all zeros: in_topology */
} dfft_trans_block_desc;
typedef struct dfft_trans_block_s dfft_trans_block;
dfft_status dfft_trans_block_create(dfft_trans_block** tb, const dfft_trans_block_desc* desc);
/* rank + 1 entries */
dfft_status dfft_trans_block_buffer_extents(const dfft_trans_block* tb, uint64_t* extents);
/* in / out: every rank's block concatenated in rank order; send / recv: nprocs
 * buffers.  Views and buffers must not alias (TransBlock::good). */
dfft_status dfft_trans_block_execute(const dfft_trans_block* tb, const void* in, void* out, void* send, void* recv,
                                     int32_t direction, void* stream);
dfft_status dfft_trans_block_destroy(dfft_trans_block* tb);

/* ---- Layout math on the host (no GPU) ----
 * rank_to_coord (KokkosFFT_Distributed_MPI_Extents.hpp:492-529). */
dfft_status dfft_rank_to_coord(int32_t rank, const uint64_t* topology, int32_t layout_right, int64_t rank_id,
                               uint64_t* coord);
/* compute_local_extents_and_starts of one rank (MPI_Extents.hpp:546-577). */
dfft_status dfft_compute_local_extents_and_starts(int32_t rank, const uint64_t* global_extents,
                                                  const uint64_t* topology, int32_t layout_right, int64_t rank_id,
                                                  uint64_t* extents, uint64_t* starts);
/* compute_buffer_extents<Layout> (KokkosFFT_Distributed_Extents.hpp:35-90):
 * rank + 1 entries. */
dfft_status dfft_compute_buffer_extents(int32_t rank, const uint64_t* global_extents, const uint64_t* in_topology,
                                        const uint64_t* out_topology, int32_t layout_right,
                                        uint64_t* buffer_extents);
/* permute_map_by_axes<Layout> (KokkosFFT_Distributed_Mapping.hpp:39-110). */
dfft_status dfft_permute_map_by_axes(int32_t rank, const int32_t* src_map, int32_t naxes, const int32_t* axes,
                                     int32_t layout_right, int32_t* out_map);
/* propose_transpose_block (KokkosFFT_Distributed_BlockAnalyses.hpp:93-136):
 * the block of rank `rank_id` and its max buffer size. */
dfft_status dfft_propose_transpose_block(int32_t rank, const int32_t* map, const uint64_t* in_topology,
                                         const uint64_t* out_topology, const uint64_t* in_extents,
                                         const uint64_t* global_extents, int32_t naxes, const int32_t* axes,
                                         int64_t rank_id, int32_t is_layout_right, int32_t is_last, int32_t in_axis,
                                         int32_t out_axis, int32_t comm_axis, int64_t block_idx,
                                         int64_t size_factor, int32_t view_layout_right, dfft_block_info* info,
                                         uint64_t* max_buffer_size);

/* Copy data recorded by the last DFFT_EXEC_LITERAL_CAPTURE execution in
 * `direction` for transpose block `block` (index in the block list) to host:
 *   which = 0 send buffers, 1 recv buffers: nprocs x prod(buffer_extents)
 *             elements, rank-major, each in the reference's buffer order;
 *   which = 2 pack input, 3 unpack output: the concatenated per-rank blocks of
 *             the block's input / output layout. */
dfft_status dfft_debug_export_buffers(const dfft_plan* plan, int32_t direction, int64_t block, int32_t which,
                                      void* host_dst, uint64_t capacity_bytes);

/* Device error word of the plan: 0, or the code a kernel left when one of
 * its bounded waits ran out (1: a TMA tile load of a stage did not complete
 * within about one second; that stage returned early and the transform's
 * output is invalid).  Synchronises the device; reset = 1 clears the word.
 * No counterpart in the reference. */
dfft_status dfft_get_device_error(const dfft_plan* plan, int32_t reset, int32_t* code);

/* Number of kernel launches one dfft_execute issues in a direction. */
dfft_status dfft_get_launch_count(const dfft_plan* plan, int32_t direction, int64_t* launches);

/* Bytes of device memory the plan holds (scratch, tables, debug buffers). */
dfft_status dfft_get_workspace_bytes(const dfft_plan* plan, uint64_t* bytes);

/* Local 3D C2C FFT that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc: programs whose device
 * memory is already owned by another allocator (for example a framework's
 * caching pool that reserved the GPU up front), and latency-critical loops
 * that must not hit cudaMalloc / cudaFree, which can synchronise the device.
 *
 * Transforms all three axes of one C-order array of n0 x n1 x n2 complex
 * elements (complex128 for DFFT_PREC_F64, complex64 for DFFT_PREC_F32), the
 * local transform each rank of the reference runs; in / out are device
 * pointers to distinct arrays and `stream` is a cudaStream_t (NULL: legacy
 * default stream).  The intermediate array between the axis stages lives in a
 * library-owned __device__ array of DFFT_NOALLOC_MAX_BYTES, which every GPU
 * that loads the library holds until the process exits.
 *   - every extent must be a power of two in [16, 4096] and the array at most
 *     DFFT_NOALLOC_MAX_BYTES; otherwise DFFT_ERROR_UNSUPPORTED;
 *   - in and out must be aligned to one complex element (8 bytes for
 *     complex64, 16 for complex128); otherwise DFFT_ERROR_INVALID_ARGUMENT;
 *   - the first call on a device sets the device up (synchronous copies of
 *     the twiddle tables): make it before any stream capture;
 *   - all calls share the library-owned arrays: calls that overlap on the GPU
 *     race with each other. */
#define DFFT_NOALLOC_MAX_BYTES (64ull * 1024ull * 1024ull)
dfft_status dfft_execute_local_c2c_noalloc(const void* in, void* out, int64_t n0, int64_t n1, int64_t n2,
                                           int32_t precision, int32_t direction, int32_t normalization,
                                           void* stream);

/* Message of the last failure on this thread ("" if none). */
const char* dfft_last_error_string(void);

/* Library version string. */
const char* dfft_version(void);

#ifdef __cplusplus
}
#endif

#endif /* DFFT_H */
