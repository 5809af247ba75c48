/*
 * jaccpot_b200 — C ABI of the Blackwell (sm_100a) FMM evaluation pass.
 *
 * The reference (jaccpot, Python/JAX) has no native seam: its kernels are JAX
 * functions called from the engine.  Each entry point below replaces one of
 * those functions and is what a jax.ffi custom call (or the ctypes host code in
 * jaccpot_b200/) binds.  Reference paths are relative to the jaccpot project.
 *
 * Conventions (all GPU entry points):
 *   - every array argument is a DEVICE pointer owned by the caller; nothing
 *     here allocates device memory;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream);
 *   - calls are asynchronous and stream-ordered; the return value reports only
 *     argument validation and launch errors (JB_OK = 0);
 *   - particles are Morton-sorted float4 (x, y, z, mass); node centres are
 *     float4 (x, y, z, total mass);
 *   - coefficient rows (multipoles, locals) hold (p+1)^2 floats in the packed
 *     real (Dehnen, no-sqrt2) layout, degree n at [n^2, n^2+2n+1) with
 *     m = -n..n (operators/_sh_indexing.py:36-118), padded to a row stride of
 *     jb_coeff_stride(p) floats;
 *   - topology arrays are the ones jb_tree_build produces (int32 node ids,
 *     int64 CSR offsets), see jaccpot_b200/tree.py.
 */
#ifndef JACCPOT_B200_H
#define JACCPOT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JB_API __attribute__((visibility("default")))

enum {
  JB_OK = 0,
  JB_ERR_ARG = 1,         /* null pointer, negative size, bad enum */
  JB_ERR_ORDER = 2,       /* expansion order outside [1, JB_MAX_ORDER] */
  JB_ERR_CUDA = 3,        /* launch or runtime error (see jb_last_cuda_error) */
  JB_ERR_INDEX = 4,       /* a list entry is out of range (jb_validate_lists) */
  JB_ERR_WORKSPACE = 5,   /* caller buffer too small */
  JB_ERR_ALLOC = 6,       /* host allocation failed (tree build) */
  JB_ERR_NONFINITE = 7,   /* non-finite input (tree build) */
  JB_ERR_UNSUPPORTED = 8  /* mode not built for this order */
};

#define JB_MAX_ORDER 10

/* M2L arithmetic modes (jb_m2l). */
enum {
  JB_M2L_FP32 = 0,       /* rotate + scale, FP32 CUDA cores */
  JB_M2L_SPLIT_BF16 = 1  /* constant factors on tcgen05, BF16 hi/lo 3-product */
};

/* Near-field accumulation flags (jb_leaf_eval), OR-able. */
enum {
  JB_P2P_FP32 = 0,
  JB_P2P_KAHAN = 1,     /* compensated per-target sums */
  JB_P2P_POTENTIAL = 2, /* also accumulate the potential (else out.w holds only the far part) */
  JB_P2P_FAR_ONLY = 4,  /* jb_leaf_eval: the far field (L2P) alone, no P2P */
  JB_P2P_NEAR_ONLY = 8, /* jb_leaf_eval: the near field (P2P) alone, no L2P */
  /* jb_leaf_eval in two halves, so the near field can run on one stream while
   * the upward sweep, M2L and L2L run on another: NEAR_FIRST writes the near
   * field (split leaves' partials left unsummed), FAR_AFTER then adds the L2P
   * and sums the partials.  The two calls together give the bits of one call
   * without either flag. */
  JB_P2P_NEAR_FIRST = 16,
  JB_P2P_FAR_AFTER = 32
};

/* Most particles one leaf may hold in the leaf kernels (jb_leaf_eval*,
 * jb_adj_near; a leaf of more than 32 is evaluated in two passes of at most
 * 32 targets); also the partial-row length (float4 per slot) of split
 * leaves.  Bits of the leaf error word (jb_leaf_eval_errors). */
#define JB_MAX_LEAF_OCCUPANCY 64
enum {
  JB_LEAF_ERR_OCCUPANCY = 1, /* a unit's leaf holds more than JB_MAX_LEAF_OCCUPANCY particles: skipped */
  JB_LEAF_ERR_SLOT = 2       /* a partial-row slot at or beyond the slot count: not written / not read */
};

/* ------------------------------------------------------------------------ */
/* Host-side prepare: tree + interaction lists (stand-in for yggdrax).      */
/* ------------------------------------------------------------------------ */
typedef struct jb_tree jb_tree;

typedef struct {
  int64_t num_particles;
  int32_t num_nodes, num_internal, num_leaves, num_levels;
  int64_t num_far_pairs, num_near_pairs;
  int32_t max_leaf_occupancy;
} jb_tree_info_t;

enum {
  JB_TREE_PERMUTATION = 0,      /* int64[N]: sorted slot -> input index */
  JB_TREE_NODE_RANGES = 1,      /* int32[2*num_nodes], inclusive */
  JB_TREE_LEFT_CHILD = 2,       /* int32[num_internal] */
  JB_TREE_RIGHT_CHILD = 3,      /* int32[num_internal] */
  JB_TREE_PARENT = 4,           /* int32[num_nodes], root -1 */
  JB_TREE_NODE_LEVEL = 5,       /* int32[num_nodes] */
  JB_TREE_LEVEL_OFFSETS = 6,    /* int32[num_levels+1], internal nodes by depth */
  JB_TREE_LEAF_OF_PARTICLE = 7, /* int32[N] (sorted slot -> leaf index) */
  JB_TREE_FAR_OFFSETS = 8,      /* int64[num_nodes+1] */
  JB_TREE_FAR_SOURCES = 9,      /* int32[num_far_pairs] */
  JB_TREE_NEAR_OFFSETS = 10,    /* int64[num_leaves+1] */
  JB_TREE_NEAR_SOURCES = 11,    /* int32[num_near_pairs] (leaf indices) */
  JB_TREE_CENTERS_F64 = 12,     /* double[3*num_nodes], COM */
  JB_TREE_RADII_F64 = 13,       /* double[num_nodes], bounding radius about COM */
  JB_TREE_FAR_GEARS = 14        /* int32[num_far_pairs]: gear of each far pair (jb_dtree_adaptive_walk only) */
};

/* Morton sort + radix tree with leaves of <= leaf_size particles + dual
 * traversal with opening angle theta.  Replaces yggdrax's tree build and
 * build_well_separated_interactions / neighbour lists as called from
 * runtime/fmm_prepare.py:823 (_build_tree_with_config) and :1411
 * (_build_dual_tree_artifacts). Host memory; pos is (n,3), mass (n,). */
JB_API int jb_tree_build(int64_t n, const double* pos, const double* mass, int leaf_size,
                         double theta, jb_tree** out);
JB_API int jb_tree_info(const jb_tree* t, jb_tree_info_t* info);
JB_API int jb_tree_copy(const jb_tree* t, int field, void* dst);
JB_API void jb_tree_free(jb_tree* t);

/* The same tree and lists built on the GPU (csrc/tree_gpu.cu), bit for bit
 * the arrays jb_tree_build returns for the same float64 inputs: Morton codes
 * + LSD radix sort, breadth-first radix split, FP64 COM / radii, breadth-first
 * dual walk, CSR by key sort.  Replaces the same yggdrax calls
 * (runtime/fmm_prepare.py:823, :1411).  pos (n,3) and mass (n,) are DEVICE
 * float64 arrays; the handle owns device copies of every JB_TREE_* field.
 * Device memory comes stream-ordered from a library pool per device that
 * keeps up to 4 GiB cached between builds; the handle's arrays are freed on
 * the build's stream by jb_dtree_free (free it before destroying the
 * stream).  Synchronises the stream (the split and the walk size their next
 * step from counts read back level by level).                              */
typedef struct jb_dtree jb_dtree;
JB_API int jb_tree_build_device(int64_t n, const double* pos, const double* mass, int leaf_size,
                                double theta, void* stream, jb_dtree** out);
JB_API int jb_dtree_info(const jb_dtree* t, jb_tree_info_t* info);
/* Device pointer of a JB_TREE_* field (NULL for a bad field); valid until
 * jb_dtree_free. */
JB_API const void* jb_dtree_field(const jb_dtree* t, int field);
/* Synchronous device-to-host copy of a field (sizes as for jb_tree_copy). */
JB_API int jb_dtree_copy(const jb_dtree* t, int field, void* dst);
JB_API void jb_dtree_free(jb_dtree* t);

/* Replaces the far and near lists of a device tree by those of the
 * error-controlled walk: the reference's Dehnen eq. (15)/(16a) acceptance
 * (adaptive_error_model="dehnen_paper", runtime/_adaptive_policy.py:267-376,
 * :2216-2376) taken target-centric.  An ordered node pair (t <- s) is far
 * when (rho_s + rho_t) < theta_max d and the force-error estimate
 *   dF_p = 8 max(rho_s, rho_t) / (rho_s + rho_t) * G
 *          * sum_{l<=p} C(p,l) P_l(s) rho_t^(p-l) / d^(p+2)
 * of the highest gear is below max(eps * force_scale[t], 1e-24); it is then
 * tagged with the lowest passing gear (JB_TREE_FAR_GEARS).  Otherwise two
 * leaves are a near pair (t's list only) and anything else splits the node of
 * larger radius.  Lists come out target-major CSR like the theta walk's, but
 * need not be symmetric.  Inputs (device): power = Dehnen's per-degree source
 * power P_l (num_nodes x num_degrees, double; jb_node_dehnen_power),
 * force_scale = per-node force scale (float; jb_node_force_scale); host:
 * gear_orders ascending, num_gears <= 8, each < num_degrees.  Synchronises. */
/* Inputs of jb_dtree_adaptive_walk.  jb_node_dehnen_power: Dehnen's
 * per-degree source power P_l = sqrt(sum_m (l-|m|)! (l+|m|)! w_m M_l^m^2), w_m =
 * 2 for m != 0 in the real packing, l = 0..p, double, num_nodes x (p+1)
 * (runtime/_adaptive_policy.py:161-214 dehnen_multipole_power_by_degree).
 * jb_node_force_scale: the smallest |a| over each node's particles (sorted
 * acc4 of a prepass), leaves first, then internal nodes level by level,
 * deepest first -- the "min" reduction the reference uses with
 * dehnen_paper (_adaptive_policy.py:402-470). */
JB_API int jb_node_dehnen_power(int p, int num_nodes, const float* mult, int row_stride, double* out, void* stream);
JB_API int jb_node_force_scale(int num_nodes, int num_internal, const int* left, const int* right,
                               const int* level_offsets_host, int num_levels, const int* node_ranges,
                               const float* acc4, float* scale, void* stream);
/* The analytic per-pair gear of a fixed far list: for every pair e =
 * (pair_tgt[e] <- far_src[e]) the lowest gear whose eq. (15) estimate (as in
 * jb_dtree_adaptive_walk) is below max(eps * force_scale[t], 1e-24); the
 * highest gear where none passes (the reference's order tags for its gear
 * buckets under dehnen_paper, runtime/_adaptive_policy.py:2352-2358).
 * com / radius: double, the tree's (JB_TREE_CENTERS_F64 / RADII_F64). */
JB_API int jb_far_dehnen_gears(int64_t num_pairs, const int* pair_tgt, const int* far_src, const double* com,
                               const double* radius, int num_degrees, const double* power, const float* force_scale,
                               double G, double eps, int num_gears, const int* gear_orders, int* gears,
                               void* stream);
JB_API int jb_dtree_adaptive_walk(jb_dtree* t, int num_degrees, const double* power, const float* force_scale,
                                  double G, double eps, double theta_max, int num_gears, const int* gear_orders,
                                  void* stream);

/* Work-unit schedules built on the GPU (csrc/schedule_gpu.cu) from device
 * lists, entry for entry the arrays of the host builders in schedule.py
 * (m2l_schedule, leaf_schedule, gear_m2l_schedule); the prepare-time
 * planning that the reference does for its M2L chunks
 * (runtime/kernels/_m2l.py:1667) and near-field schedules
 * (nearfield/_schedules.py:271).  All pointers are DEVICE memory; the handle
 * owns its outputs (pool memory, freed on the build stream).  The calls
 * synchronise the stream.                                                   */
typedef struct jb_dsched jb_dsched;
typedef struct {
  int64_t num_units, num_split, num_slots, num_runs, num_targets;
} jb_sched_info_t;
enum {
  JB_SCHED_UNITS = 0,          /* int32[num_units][4] */
  JB_SCHED_AUX = 1,            /* int32[num_units][2] (leaf schedule); int32[num_units][4]
                                  segment bounds (mixed gear schedule) */
  JB_SCHED_RUNS = 2,           /* int32[num_runs][2] (leaf schedule) */
  JB_SCHED_SPLIT = 3,          /* int32[num_split][4] */
  JB_SCHED_FAR_SOURCES = 4,    /* int32[num_far] regrouped by gear (gear schedule) */
  JB_SCHED_GEAR_OFFSETS = 5,   /* int64[num_gears+1] (gear schedule) */
  JB_SCHED_TARGETS = 6,        /* int32[num_targets] (M2L schedule) */
  JB_SCHED_PAIRS_PER_GEAR = 7  /* int64[num_gears] (gear schedule) */
};
/* targets == NULL: every node with far pairs, longest list first. */
JB_API int jb_m2l_schedule_device(int num_nodes, const int64_t* far_off, int max_pairs, int num_targets,
                                  const int* targets, void* stream, jb_dsched** out);
/* Leaves [leaf_lo, leaf_hi); max_sources >= 1. */
JB_API int jb_leaf_schedule_device(int num_internal, int num_leaves, const int* node_ranges, const int64_t* near_off,
                                   const int* near_src, int leaf_lo, int leaf_hi, int max_sources, void* stream,
                                   jb_dsched** out);
/* gears: int32 per far pair in [0, num_gears) (JB_ERR_INDEX otherwise). */
JB_API int jb_gear_schedule_device(int num_nodes, const int64_t* far_off, const int* far_src, const int* gears,
                                   int num_gears, int max_pairs, void* stream, jb_dsched** out);
/* The schedule of jb_m2l_mixed: each target's pairs sorted by order, highest
 * first (stable inside), cut into units of at most max_pairs (<= 65535);
 * slots numbered per target; units sorted by decreasing segment lengths,
 * highest order first.  gear_orders (HOST, num_gears entries) must each be
 * one of p_max - 2j, j < JB_MIXED_GEAR_SEGMENTS, >= 1 (JB_ERR_ARG
 * otherwise); a gear outside [0, num_gears) gives JB_ERR_INDEX.  Fields:
 * UNITS, AUX (bounds), SPLIT, FAR_SOURCES, PAIRS_PER_GEAR.                  */
JB_API int jb_gear_mixed_schedule_device(int num_nodes, const int64_t* far_off, const int* far_src, const int* gears,
                                         int num_gears, const int* gear_orders, int p_max, int max_pairs,
                                         void* stream, jb_dsched** out);
/* rev[e] = index of the reverse pair (s <- t) of every far pair e = (t <- s)
 * of a symmetric CSR far list (device arrays; rows sorted, as jb_tree_build
 * emits them); JB_ERR_INDEX when some pair has no reverse.  The host twin is
 * Topology.far_reverse_index in tree.py.  Synchronises the stream.           */
JB_API int jb_far_reverse_index(int num_nodes, const int64_t* far_off, const int* far_src, int* rev, void* stream);
JB_API int jb_dsched_info(const jb_dsched* d, jb_sched_info_t* info);
JB_API const void* jb_dsched_field(const jb_dsched* d, int field);
JB_API void jb_dsched_free(jb_dsched* d);

/* ------------------------------------------------------------------------ */
/* Device pass.                                                             */
/* ------------------------------------------------------------------------ */

/* Level sweeps: levels with at most m2m_max_parents (l2l_max_parents)
 * parents run the M2M (L2L) translations with each translation's degrees
 * split over four warps (shorter chains), wider levels with one thread per
 * translation.  Same operations either way.  Process-wide setting.          */
JB_API int jb_set_level_split(int m2m_max_parents, int l2l_max_parents);

/* Near field of jb_leaf_eval: 1 (default) walks the target x source-chunk
 * work of leaves with more than 16 particles chunk-major over all 32 lanes
 * of a warp and takes 1/r from the flush-to-zero instruction; 0 gives each
 * target one lane (idle lanes for the rest).  The sums are bit-identical
 * either way while every squared distance (+ eps2) is 0 or at least 2^-126.
 * Process-wide setting.                                                   */
JB_API int jb_set_leaf_form(int chunk_major);

/* Source-row fetch of the single-order FP32 M2L (jb_m2l, jb_m2l_gears,
 * jb_m2l_weighted, jb_adj_m2l; jb_m2l_mixed always fetches per thread):
 * 1 (default) copies the rows of a warp's 32
 * work units together, one cp.async instruction per row (lane k takes
 * 16-byte word k); 0 lets each thread copy its own row word by word (every
 * warp instruction then touches 32 rows).  The same arithmetic either way;
 * the compiler may fuse a multiply and an add differently in the two
 * kernels, so results agree to FP32 rounding.  Process-wide setting.       */
JB_API int jb_set_m2l_fetch(int warp_rows);

/* CUDA-graph plumbing for a captured pass (graph: a cudaGraph_t taken from a
 * stream capture).  node_priority = 1 instantiates it so that each kernel
 * node keeps the priority of the stream it was captured on, which lets a
 * pass whose far-field chain was captured on a high-priority stream and whose
 * near field on a low-priority one overlap the two as the eager launches do;
 * 0 runs every node at the priority of the stream it is launched into. */
JB_API int jb_graph_instantiate(void* graph, int node_priority, void** exec);
JB_API int jb_graph_launch(void* exec, void* stream);
JB_API int jb_graph_exec_destroy(void* exec);

/* Row stride (floats) of a coefficient array of order p: (p+1)^2 rounded up
 * to a multiple of 4.  Returns 0 for an unsupported order. */
JB_API int jb_coeff_stride(int p);

/* Last CUDA error string seen by this thread (empty if none). */
JB_API const char* jb_last_cuda_error(void);

/* Builds sorted float4 particles from the caller's (N,3) positions and (N,)
 * masses: out[i] = (pos[perm[i]], mass[perm[i]]).  The Morton-order gather
 * at runtime/fmm_prepare.py (positions_sorted / masses_sorted). */
JB_API int jb_gather_sorted(int64_t n, const float* pos, const float* mass, const int64_t* perm,
                            float* out_pos4, void* stream);

/* Checks every list entry against its range on the device (one-off, at
 * prepare time); writes the number of bad entries to *bad_count_dev (int32).
 * The hot kernels below trust validated lists. */
JB_API int jb_validate_lists(int num_nodes, int num_internal, const int* left, const int* right,
                             const int64_t* far_off, const int* far_src, int64_t num_far,
                             const int64_t* near_off, const int* near_src, int64_t num_near,
                             int* bad_count_dev, void* stream);

/* Leaf-occupancy precondition of the leaf kernels: writes to *bad_count_dev
 * (int32, device) the number of leaves whose inclusive node range is empty,
 * reversed or holds more than max_occupancy particles (max_occupancy in
 * [1, JB_MAX_LEAF_OCCUPANCY]).  No reference counterpart: yggdrax's leaf
 * blocks are padded to the tree's max leaf size by construction
 * (nearfield/_schedules.py:271). */
JB_API int jb_validate_leaves(int num_nodes, int num_internal, const int* node_ranges, int max_occupancy,
                              int* bad_count_dev, void* stream);

/* Upward sweep, leaf stage: COM centre (yggdrax compute_tree_mass_moments,
 * upward/real_tree_expansions.py:439) and P2M (:89-213, p2m_real_direct,
 * operators/real_p2m_l2p.py:51) for every leaf.  Writes centers[leaf] and
 * mult[leaf]. */
JB_API int jb_p2m(int p, const float* pos4, int num_nodes, int num_internal, const int* node_ranges,
                  float* centers, float* mult, void* stream);

/* Upward sweep, one level: COM of each internal node in [first, last) from
 * its children and M2M (m2m_real, operators/real_translations.py:531;
 * aggregate_m2m_real_by_level, upward/real_tree_expansions.py:216-364). */
JB_API int jb_m2m_level(int p, int first, int last, const int* left, const int* right, const int* node_ranges,
                        float* centers, float* mult, void* stream);

/* Far field (M2L + accumulation) over work units.  units is int4[num_units]:
 * (target node, first pair, end pair, slot) with pairs indexing far_src (the
 * CSR source list of the target); a unit covers at most a bounded number of
 * consecutive pairs.  slot < 0: the unit covers the target's whole list and
 * writes locals[target]; slot >= 0: it writes row `slot` of `partials`
 * (num_slots x jb_coeff_stride(p) floats, caller-provided scratch), and the
 * split list int4[num_split] = (target, first slot, slot count, 0) is then
 * summed into locals in slot order.  Rows of targets without pairs are not
 * written (zero them first).  Replaces _accumulate_m2l_fullbatch/_chunked_scan
 * + m2l_rot_scale_real_batch (runtime/kernels/_m2l.py:1483-1793,
 * operators/m2l_real_rot_scale.py:392-486). */
JB_API int jb_m2l(int p, int mode, int num_units, const int* units, const float* mult, const float* centers,
                  const int* far_src, float* locals, float* partials, int num_split, const int* split,
                  void* stream);

/* jb_m2l with far pair e's contribution scaled by far_w[e] (device float per
 * CSR far entry): the block-step weighted far field of the mutual lane
 * (jaccpot/mutual/force.py:920 _far_pair_weights there: a pair's weight is
 * that of its finer node's level, the same for both directions). FP32.    */
JB_API int jb_m2l_weighted(int p, int num_units, const int* units, const float* mult, const float* centers,
                           const int* far_src, const float* far_w, float* locals, float* partials, int num_split,
                           const int* split, void* stream);

/* Far field with a per-pair expansion order (gear): the reference's
 * adaptive-order downward sweep, which buckets far pairs by gear and runs
 * each bucket's M2L at that gear's order (runtime/fmm_prepare.py:2400-2480,
 * _bucket_far_pairs_by_level_split).  Units (as jb_m2l) are grouped by gear:
 * units[gear_unit_offsets[g] .. gear_unit_offsets[g+1]) run at order
 * gear_orders[g] <= p_max (HOST arrays, num_gears entries / num_gears+1);
 * far_src is the source list regrouped so no unit mixes gears.  Rows of
 * mult / locals / partials have stride jb_coeff_stride(p_max); a gear reads
 * the degrees <= its order and writes zeros above them. */
JB_API int jb_m2l_gears(int p_max, int mode, int num_gears, const int* gear_orders, const int64_t* gear_unit_offsets,
                        const int* units, const float* mult, const float* centers, const int* far_src,
                        float* locals, float* partials, int num_split, const int* split, void* stream);

/* The same far field in one launch, for gears whose orders lie on the ladder
 * p_max, p_max-2, p_max-4, p_max-6 (those >= 1; JB_MIXED_GEAR_SEGMENTS at
 * most): a unit (target, first, end, slot) is a slice of one target's list
 * with its pairs sorted by order, highest first, and bounds[u] = (b1, b2, b3,
 * end) cuts it into segments [b_j, b_j+1) (b_0 = first) evaluated at order
 * p_max - 2j, all into one accumulator, so a target split over gears needs
 * no partial rows.  units / bounds / far_src / split come from
 * jb_gear_mixed_schedule_device (device arrays).  FP32.                     */
#define JB_MIXED_GEAR_SEGMENTS 4
JB_API int jb_m2l_mixed(int p_max, int num_units, const int* units, const int* bounds, const float* mult,
                        const float* centers, const int* far_src, float* locals, float* partials, int num_split,
                        const int* split, void* stream);

/* Split-BF16 far field on the tensor cores (tcgen05.mma kind::f16, FP32
 * accumulation in TMEM): the M2L chain Dz(az) B Dz(-ax) r^-k K r^-(n+1) Dz(ax)
 * B^T Dz(-az) (operators/m2l_real_rot_scale.py:288-386 with B^T Z B folded into
 * K) with the three constant products done as A_hi W_hi + A_lo W_hi + A_hi W_lo
 * on BF16 hi/lo splits.  Pairs in CSR order (pair_tgt[e] <- far_src[e]) are
 * taken 128 per tile; seg_off / segs (int4: target, first row, end row, slot)
 * describe each tile's target runs; slot >= 0 rows go to partials and the split
 * list sums them as in jb_m2l.  *status (device int, zero it first) becomes 1
 * if a tensor-core barrier wait timed out.  products = 3: B, K and B^T all run
 * on the tensor cores (three MMA round trips per tile); products = 1: only K
 * does, B and B^T run as literal-constant FMAs in registers (one round
 * trip).  Orders 2..8. */
JB_API int jb_m2l_split(int p, int products, int num_tiles, int64_t num_pairs, const int* pair_tgt,
                        const int* far_src, const int* seg_off, const int* segs, const float* mult,
                        const float* centers, float* locals, float* partials, int num_split, const int* split,
                        int* status, void* stream);

/* Split-BF16 far field, unit layout: the same work units / partials / split
 * list as jb_m2l (thread = unit); step j takes the j-th pair of 128 units as
 * one tensor-core tile for the K product (B and B^T in registers) and each
 * thread accumulates its local in registers.  *status as jb_m2l_split.
 * Orders 2..8. */
JB_API int jb_m2l_split_units(int p, int num_units, const int* units, const float* mult, const float* centers,
                              const int* far_src, float* locals, float* partials, int num_split, const int* split,
                              int* status, void* stream);

/* Downward sweep, one level: for each internal node in [first, last), adds
 * l2l(parent) to both children (l2l_real, operators/real_translations.py:604;
 * _propagate_solidfmm_locals_by_level, runtime/kernels/_l2l.py:210-404). */
JB_API int jb_l2l_level(int p, int first, int last, const int* left, const int* right,
                        const float* centers, float* locals, void* stream);

/* The downward sweep straight to the leaves (the same operator, l2l_real,
 * operators/real_translations.py:604, composed): units[u] = (leaf node,
 * first, end, unused) over anc[], the leaf's ancestors that received far
 * pairs (nearest first); locals[leaf] += sum_a L2L(a -> leaf)(locals[a]).
 * Call after the M2L, on locals holding each node's own M2L sum, instead of
 * the jb_l2l_level sweep.  Shifting a degree-p expansion is exact, so the
 * leaves' locals equal the cascade's up to rounding; the internal nodes keep
 * their own M2L sums (the adjoint, which reads them, uses the cascade).
 * Device pointers; units and anc come from the caller's schedule.          */
JB_API int jb_l2l_leaves(int p, int num_units, const int* units, const int* anc, const float* centers,
                         float* locals, void* stream);

/* Leaf evaluation over work units: L2P of each leaf's local at its particles
 * (runtime/kernels/_evaluate.py:2106-2484, evaluate_local_real_with_grad) plus
 * the near field over the self leaf and the leaf's neighbour list
 * (nearfield/near_field.py:916, nearfield/_kernels.py:40-338), assembled as
 * acc = near - G * grad (runtime/kernels/_evaluate.py:1157-1172).
 *   units int4[num_units] = (leaf index, first run, end run, source count)
 *   aux   int2[num_units] = (slot, flags); flags & 1: this unit also does the
 *                           self block and the far field of the leaf
 *   runs  int2[...]       = (first sorted particle, count): contiguous source
 *                           ranges (runs of consecutive neighbour leaves)
 * slot < 0: writes out_acc4 for the leaf's particles; slot >= 0: writes 64
 * float4 at partials[64*slot] (scratch), then split int4[num_split] = (leaf,
 * first slot, slot count, 0) is summed into out_acc4.  out_acc4[i] = (ax, ay,
 * az, potential) in sorted order; p2p_mode is a JB_P2P_* flag set.
 * Preconditions: every leaf a unit names holds at most JB_MAX_LEAF_OCCUPANCY
 * particles (check once with jb_validate_leaves; a unit breaking it writes
 * nothing and sets JB_LEAF_ERR_OCCUPANCY), and partials holds
 * JB_MAX_LEAF_OCCUPANCY float4 per slot for every slot in aux / split. */
/* jb_leaf_eval with every particle pair scaled by
 * level_weights[max(rung_i, rung_j)] (rung: int32 per SORTED particle,
 * clamped to [0, num_level_weights); num_level_weights <= 32; device
 * arrays): the block-step weighted near field of the mutual lane
 * (jaccpot/mutual/nearfield.py:140 _pair_weights there).  The far part is
 * whatever the locals hold (weighted by jb_m2l_weighted).                  */
JB_API int jb_leaf_eval_weighted(int p, int p2p_mode, const float* pos4, const int* rung, int num_level_weights,
                                 const float* level_weights, int num_internal, int num_units, const int* units,
                                 const int* aux, const int* runs, const int* node_ranges, const float* centers,
                                 const float* locals, float G, float eps2, float* out_acc4, float* partials,
                                 int num_split, const int* split, void* stream);
JB_API int jb_leaf_eval(int p, int p2p_mode, const float* pos4, int num_internal, int num_units, const int* units,
                        const int* aux, const int* runs, const int* node_ranges, const float* centers,
                        const float* locals, float G, float eps2, float* out_acc4, float* partials, int num_split,
                        const int* split, void* stream);

/* Reads the leaf error word of the current device (JB_LEAF_ERR_* bits set by
 * jb_leaf_eval, jb_leaf_eval_weighted and jb_leaf_eval_noalloc launches so
 * far) into *flags after the work queued on `stream` has finished, and clears
 * it when `clear` is nonzero.  Synchronises the stream.  No reference
 * counterpart (the reference raises at trace time instead). */
JB_API int jb_leaf_eval_errors(int* flags, int clear, void* stream);

/* jb_leaf_eval for callers that cannot allocate device memory: no reference
 * counterpart (the reference's XLA runtime owns all buffers).  A jax.ffi /
 * XLA custom-call handler only receives the buffers XLA planned for it and
 * must not cudaMalloc in the middle of XLA's asynchronous schedule, and code
 * running under CUDA stream capture may not cudaMalloc at all; both can still
 * pass inputs and outputs.  Same arguments as jb_leaf_eval except that
 * `partials` is replaced by num_slots, which must be at least 1 + the largest
 * slot in aux and split (the schedule's slot count): the scratch is a static
 * device array of JB_LEAF_EVAL_NOALLOC_MAX_SLOTS x JB_MAX_LEAF_OCCUPANCY
 * float4 (16 MiB) that every GPU loading the library holds until exit.  num_slots above the
 * maximum returns JB_ERR_WORKSPACE; a slot at or beyond num_slots is neither
 * written nor read and sets JB_LEAF_ERR_SLOT (jb_leaf_eval_errors).  Leaves
 * as jb_leaf_eval (at most JB_MAX_LEAF_OCCUPANCY particles).  Allocates
 * nothing.  The first call on a device (and the first after the device's
 * context was reset) looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the one array: calls that overlap on the GPU (different
 * streams, no ordering between them) race. */
#define JB_LEAF_EVAL_NOALLOC_MAX_SLOTS 16384
JB_API int jb_leaf_eval_noalloc(int p, int p2p_mode, const float* pos4, int num_internal, int num_units,
                                const int* units, const int* aux, const int* runs, const int* node_ranges,
                                const float* centers, const float* locals, float G, float eps2, float* out_acc4,
                                int num_slots, int num_split, const int* split, void* stream);

/* Target subset (runtime/kernels/_evaluate.py:1941-2095): targets_sorted are
 * sorted-slot indices; out_acc4[q] in target order. */
JB_API int jb_eval_targets(int p, const float* pos4, int num_internal, const int* node_ranges,
                           const float* centers, const float* locals, const int64_t* near_off,
                           const int* near_src, const int* leaf_of, int64_t num_targets,
                           const int* targets_sorted, float G, float eps2, float* out_acc4,
                           void* stream);

/* Un-permute (runtime/fmm_evaluate.py:526-538): out_acc[perm[i]] = acc4[i].xyz,
 * out_pot (optional) likewise. */
JB_API int jb_scatter_unsorted(int64_t n, const float* acc4, const int64_t* perm, float* out_acc,
                               float* out_pot, void* stream);

/* The same un-permute from the inverse permutation (inv_perm[perm[i]] = i):
 * out_acc[j] = acc4[inv_perm[j]].xyz, out_pot (optional) likewise.  The
 * output is written in order (coalesced) and only the reads scatter: 0.043
 * against 0.113 ms at N = 4M.  The values are the same
 * (runtime/fmm_evaluate.py:526-538).                                      */
JB_API int jb_gather_unsorted(int64_t n, const float* acc4, const int64_t* inv_perm, float* out_acc,
                              float* out_pot, void* stream);

/* ------------------------------------------------------------------------ */
/* Adjoint (vector-Jacobian product) at fixed topology.                     */
/*                                                                          */
/* Gradient of L = sum_i w_i . acc_i w.r.t. positions and masses, with the   */
/* COM centres differentiated: the VJP that jax.grad takes through the       */
/* reference's differentiable_accelerations (runtime/fmm_evaluate.py:542-731,*/
/* :1175-1250), with its analytic near-field rule (nearfield/grad.py:726-869)*/
/* and L2P rule (operators/real_p2m_l2p.py:402-491).  Run after a forward   */
/* pass (centres, multipoles, final locals in place), in this order:        */
/*   jb_adj_near, jb_adj_leaf_far, jb_adj_l2l_level (deepest level first),  */
/*   jb_adj_m2l, jb_adj_m2l_centers, jb_adj_m2m_level (root first),         */
/*   jb_adj_p2m.  cbar4 (num_nodes float4) and mbar (num_nodes x stride)    */
/*   start at zero; w4 is the sorted float4 cotangent (w, 0);               */
/*   xm4[i] = (dL/dx, dL/dy, dL/dz, dL/dm) sorted.  Needs symmetric near and */
/*   far lists (jb_tree_build emits both directions).  Orders 1..9.         */
/* ------------------------------------------------------------------------ */
#define JB_ADJ_MAX_ORDER_API 9
/* P2P VJP over the leaf-evaluation units (writes xm4; split leaves use
 * partials + split exactly as jb_leaf_eval). */
JB_API int jb_adj_near(const float* pos4, const float* w4, int num_internal, int num_units, const int* units,
                       const int* aux, const int* runs, const int* node_ranges, float G, float eps2, float* out_xm4,
                       float* partials, int num_split, const int* split, void* stream);
/* L2P VJP: lbar[leaf] = dL/dlocal, adds the particle and leaf-centre terms. */
JB_API int jb_adj_leaf_far(int p, const float* pos4, const float* w4, int num_nodes, int num_internal,
                           const int* node_ranges, const float* centers, const float* locals, float G, float* xm4,
                           float* lbar, float* cbar4, void* stream);
/* L2L VJP for parents in [first, last) (transpose of runtime/kernels/_l2l.py:210-404). */
JB_API int jb_adj_l2l_level(int p, int first, int last, const int* left, const int* right, const float* centers,
                            const float* locals, float* lbar, float* cbar4, void* stream);
/* M2L VJP w.r.t. the multipoles: mbar[u] = sum_v M2L(c_v - c_u) lbar[v] over u's
 * list, same units / partials / split as jb_m2l (transpose of _m2l.py:1483-1793). */
JB_API int jb_adj_m2l(int p, int num_units, const int* units, const float* lbar, const float* centers,
                      const int* far_src, float* mbar, float* partials, int num_split, const int* split,
                      void* stream);
/* M2L VJP w.r.t. the centres: per pair (pair_tgt[e] <- far_src[e]) the
 * displacement derivative into g4 (num_pairs float4 scratch), then gathered
 * into cbar4 with rev[e] = index of the reverse pair. */
JB_API int jb_adj_m2l_centers(int p, int num_nodes, int64_t num_pairs, const int* pair_tgt, const int* far_src,
                              const int64_t* far_off, const int* rev, const float* mult, const float* lbar,
                              const float* centers, float* g4, float* cbar4, void* stream);
/* M2M + COM VJP for parents in [first, last) (transpose of
 * upward/real_tree_expansions.py:216-364 and the COM of :439). */
JB_API int jb_adj_m2m_level(int p, int first, int last, const int* left, const int* right, const float* centers,
                            const float* mult, float* mbar, float* cbar4, void* stream);
/* P2M + leaf COM VJP (transpose of real_tree_expansions.py:89-213); adds into xm4. */
JB_API int jb_adj_p2m(int p, const float* pos4, int num_nodes, int num_internal, const int* node_ranges,
                      const float* centers, const float* mbar, const float* cbar4, float* xm4, void* stream);

/* ------------------------------------------------------------------------ */
/* Learned gear selector (replaces the analytic per-pair order policy of     */
/* runtime/_adaptive_policy.py:249-372 that feeds the gear buckets of         */
/* runtime/fmm_prepare.py:2400-2480).  MLP 12 -> 64 -> 64 -> 4, GELU, BF16    */
/* weights (FP32 values rounded to BF16), FP32 accumulation; gears are the    */
/* orders (2, 4, 6, 8).  Parameter vector layout: W1[64][12] b1[64]           */
/* W2[64][64] b2[64] W3[4][64] b3[4].                                         */
/* ------------------------------------------------------------------------ */
JB_API int jb_gear_param_count(void);
/* Per node: 8 log per-degree multipole powers (node_feat, num_nodes x 8) and
 * the smallest particle force magnitude under the node (scale) from a
 * previous pass's sorted acc4; level_offsets_host is a HOST array. */
JB_API int jb_gear_node_features(int p, int num_nodes, int num_internal, const int* left, const int* right,
                                 const int* level_offsets_host, int num_levels, const int* node_ranges,
                                 const float* mult, const float* centers, const float* radii, const float* acc4,
                                 float* node_feat, float* scale, void* stream);
/* 12 features per far pair (pair_ids NULL = all pairs, else n selected ids). */
JB_API int jb_gear_pair_features(int64_t n, const int64_t* pair_ids, const int* pair_tgt, const int* far_src,
                                 const float* centers, const float* radii, const float* node_feat,
                                 const float* scale, float G, float* out, void* stream);
/* Training labels: log10(force error / target force scale) of each gear's M2L
 * against the order-10 M2L (mult10: order-10 multipoles), n x 4. */
JB_API int jb_gear_errors(int64_t n, const int64_t* pair_ids, const int* pair_tgt, const int* far_src,
                          const float* mult10, const float* centers, const float* radii, const float* scale, float G,
                          float* out, void* stream);
/* One batch's parameter gradients (softmax cross-entropy on the gear label):
 * block b writes gpart[b][param_count] and lpart[b] (ceil(n/128) blocks). */
JB_API int jb_gear_train_grad(int n, const float* X, const int* labels, const float* Wq, float* gpart, float* lpart,
                              void* stream);
/* Adam step on FP32 master weights; Wq = BF16-rounded copy. */
JB_API int jb_gear_adam(int nblocks, const float* gpart, float inv_batch, float lr, float beta1, float beta2,
                        float eps, int step, float* master, float* m1, float* m2, float* Wq, void* stream);
/* Fused inference per far pair: features, normalisation ((x - norm[k]) *
 * norm[12 + k]), MLP, gear = lowest g with P(label <= g) >= conf, or the
 * highest gear when the top probability is below min_top. */
JB_API int jb_gear_select(int64_t n, const int* pair_tgt, const int* far_src, const float* centers,
                          const float* radii, const float* node_feat, const float* scale, float G, const float* Wq,
                          const float* norm, float conf, float min_top, int* gear_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Verification and measurement helpers (no reference counterpart in the    */
/* hot path; they back the error report and the roofline denominators).    */
/* ------------------------------------------------------------------------ */

/* FP64 direct sum on sampled targets over all n sorted particles, self pair
 * excluded: runtime/reference.py:292 (direct_sum) and
 * bench/validation/mac_error_distribution.py:140-186 (targets subset).
 * out4[4q..4q+3] = (ax, ay, az, potential) in float64. */
JB_API int jb_direct_f64(int64_t n, const float* pos4, int64_t num_targets, const int* targets_sorted, double G,
                         double eps2, double* out4, void* stream);

/* Pipe-throughput probe: blocks x 256 threads x iters x 8 dependent-chain
 * FMAs (use_mufu = 0), rsqrt (1) or packed f32x2 FMAs (2); or (3) the near
 * field's particle-pair arithmetic on register-resident data, 24 pairs per
 * thread and iteration (the pair rate the FP32 + MUFU pipes allow for that
 * instruction mix).  Time it with events. */
JB_API int jb_probe_throughput(int blocks, int iters, int use_mufu, float* sink, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* JACCPOT_B200_H */
