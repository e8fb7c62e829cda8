/*
 * n2w.h — C ABI of the B200-native Walk-on-Spheres engine (libn2w.so).
 *
 * Plain C types only: pointers, sizes, POD structs.  Every function returns an
 * int status (N2W_OK == 0) and records a human-readable message retrievable with
 * n2w_last_error() on the calling thread.  Device pointers (d_*) are CUDA
 * device addresses owned by the caller unless stated otherwise.  Stream
 * arguments are cudaStream_t values passed as n2w_stream_t (NULL = legacy
 * default stream).
 *
 * Reference interfaces replaced (paths inside Somatic-Cell/n2wos-cuda):
 *   mesh generators / loaders / normalize  include/n2wos/mesh.hpp:9-19
 *   CPU brute force closest point           include/n2wos/closest_point.hpp:9-17
 *   CudaBvh / CuBqlBvh ctor + query_device  include/n2wos/cuda_bvh.hpp:34-57,
 *                                           include/n2wos/cubql_bvh.hpp:33-65
 *   NC walker launchers                     include/n2wos/tcnn_nc_wos.hpp:79-134
 *   persistent WoS + reductions             src/cuda/cubql_bvh.cu:263-393,819-960
 */
#ifndef N2W_H_
#define N2W_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define N2W_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define N2W_OK 0
#define N2W_EINVAL 1    /* invalid argument (null pointer, bad size, bad mode) */
#define N2W_ECUDA 2     /* CUDA runtime error (message holds cudaGetErrorString) */
#define N2W_ENOMEM 3    /* host or device allocation failed / admission refused */
#define N2W_ETIMEOUT 4  /* a device-side budget or deadline expired */
#define N2W_EIO 5       /* file could not be read or parsed */
#define N2W_EINTERNAL 6 /* internal invariant violated */

typedef struct CUstream_st* n2w_stream_t; /* == cudaStream_t */

/* 12-byte AoS point, layout-identical to the reference's DeviceVec3
 * (src/cuda/bvh_types.cuh:17-21). */
typedef struct n2w_vec3 {
  float x, y, z;
} n2w_vec3;

typedef struct n2w_mesh n2w_mesh; /* host triangle mesh (opaque) */
typedef struct n2w_bvh n2w_bvh;   /* device-resident BVH + triangles (opaque) */
typedef struct n2w_comm n2w_comm; /* NCCL communicator of one rank (opaque) */

const char* n2w_last_error(void);
int n2w_abi_version(void);
/* Fills buf with "runtime=<v>,driver=<v>" (reference cuda_bvh.hpp:79). */
int n2w_cuda_runtime_version_string(char* buf, size_t cap);
/* Fills buf with "<name> sm_<maj><min> global_mem=<bytes>" (reference cuda_bvh.hpp:80). */
int n2w_cuda_device_summary(char* buf, size_t cap);

/* ---- meshes (host) ------------------------------------------------------ */
/* Copies nv vertices (xyz float triples) and nt triangles (uint32 triples). */
int n2w_mesh_create(const float* vertices, int64_t nv, const uint32_t* triangles, int64_t nt,
                    const char* name, n2w_mesh** out);
/* Reference bumpy-sphere surface (src/mesh/procedural_bumpy_sphere.cpp:12-90). */
int n2w_mesh_bumpy_sphere_ref(int stacks, int slices, float amplitude, n2w_mesh** out);
/* Same UV topology, radius r = 1 + amplitude*sin(k_theta*theta)*cos(k_phi*phi). */
int n2w_mesh_bumpy_sphere_trig(int stacks, int slices, float amplitude, int k_theta, int k_phi,
                               n2w_mesh** out);
/* Subdivided icosahedron (20*4^level triangles) radially displaced by seeded
 * multi-octave value noise: r = 1 + amplitude * noise(x). */
int n2w_mesh_icosphere_displaced(int level, float amplitude, float base_frequency, int octaves,
                                 float persistence, uint64_t seed, n2w_mesh** out);
int n2w_mesh_load_ply(const char* path, n2w_mesh** out);
int n2w_mesh_load_obj(const char* path, n2w_mesh** out);
/* AABB-centre translate + scale by max vertex radius (reference src/mesh/normalize.cpp:18-37).
 * center_out[3] and scale_out (=1/radius) may be NULL. */
int n2w_mesh_normalize(n2w_mesh* mesh, float* center_out, float* scale_out);
int n2w_mesh_counts(const n2w_mesh* mesh, int64_t* nv, int64_t* nt);
/* Copies vertices (3*nv floats) and triangles (3*nt uint32); either may be NULL. */
int n2w_mesh_copy_out(const n2w_mesh* mesh, float* vertices, uint32_t* triangles);
/* bounds_out[6] = min xyz, max xyz. */
int n2w_mesh_bounds(const n2w_mesh* mesh, float* bounds_out);
/* Number of triangles with |cross(b-a,c-a)|^2 <= area2_epsilon (reference closest_point.cpp:70-83). */
int n2w_mesh_count_degenerate(const n2w_mesh* mesh, float area2_epsilon, int64_t* out);
/* Host brute-force closest point over every triangle (reference
 * closest_point_bruteforce, src/geometry/closest_point.cpp:50-68): squared
 * distance, closest point (xyz) and triangle id (lowest id on exact ties) for n
 * host points, with the device kernel's arithmetic.  threads <= 0 uses all
 * hardware threads.  Any output may be NULL.  Used by the probes to validate. */
int n2w_mesh_closest_point_host(const n2w_mesh* mesh, const float* xyz, int64_t n, float* d2_out,
                                float* closest_out, int* tri_out, int threads);
/* Mesh name ("procedural_bumpy_sphere", file stem of a loaded mesh, ...); owned by the mesh. */
const char* n2w_mesh_name(const n2w_mesh* mesh);
void n2w_mesh_free(n2w_mesh* mesh);

/* ---- BVH + closest point ----------------------------------------------- */
typedef struct n2w_bvh_stats {
  int64_t triangles;      /* triangles stored (= mesh triangles) */
  int64_t nodes;          /* 4-wide nodes on the device */
  int64_t binary_nodes;   /* nodes of the binary tree before collapsing */
  int64_t leaves;         /* leaf references */
  int32_t leaf_size;      /* maximum triangles per leaf */
  int32_t max_depth;      /* depth of the 4-wide tree (root = 0) */
  double build_milliseconds; /* host build + upload wall time */
  double sah_cost;        /* SAH cost of the binary tree (traversal 1, intersection 1) */
  int64_t device_bytes;   /* bytes resident on the device */
} n2w_bvh_stats;

/* Host-only build of the same layout (no device needed): nodes (128 B each)
 * and leaf-ordered triangles (48 B each) for inspection and CPU restatements. */
typedef struct n2w_bvh_host n2w_bvh_host;
int n2w_bvh_host_build(const n2w_mesh* mesh, int leaf_size, const char* build_method,
                       n2w_bvh_host** out);
int n2w_bvh_host_stats(const n2w_bvh_host* h, n2w_bvh_stats* out);
int n2w_bvh_host_copy(const n2w_bvh_host* h, void* nodes_out, void* tris_out);
void n2w_bvh_host_free(n2w_bvh_host* h);

/* Builds on the host and uploads to the current device.  build_method:
 * "sah" (binned SAH, default when NULL) or "spatial_median" (largest-centroid-axis
 * median split, the reference's in-tree builder, bvh_build_host.cpp:74-120).
 * leaf_size in [1, 8]. */
int n2w_bvh_create(const n2w_mesh* mesh, int leaf_size, const char* build_method, n2w_bvh** out);
int n2w_bvh_stats_get(const n2w_bvh* bvh, n2w_bvh_stats* out);
void n2w_bvh_destroy(n2w_bvh* bvh);

/* Exact closest point on the mesh for each query point (reference
 * CudaBvh::query_device, include/n2wos/cuda_bvh.hpp:50-57; cubql_bvh.hpp:45-52).
 * Outputs: squared distance, closest point, triangle index (lowest index on exact
 * distance ties, identical to the CPU brute force), stack-overflow flag.
 * query_count == 0 is a no-op; < 0 or null pointers -> N2W_EINVAL;
 * block_size outside [1,1024] -> N2W_EINVAL.  No allocation, no host transfer. */
int n2w_bvh_query_device(const n2w_bvh* bvh, const n2w_vec3* d_points, int query_count,
                         float* d_distance2, n2w_vec3* d_closest, int* d_triangle_id,
                         int* d_overflow, int block_size, n2w_stream_t stream);
/* Masked variant (reference cubql_bvh.hpp:57-65): slots with d_active[i]==0 skip
 * traversal and write d2=0, closest=query point, tri=-1, overflow=0. */
int n2w_bvh_query_device_masked(const n2w_bvh* bvh, const n2w_vec3* d_points,
                                const uint8_t* d_active, int query_count, float* d_distance2,
                                n2w_vec3* d_closest, int* d_triangle_id, int* d_overflow,
                                int block_size, n2w_stream_t stream);
/* Diagnostic variant: also writes per-query node visits and triangle tests
 * (d_node_visits / d_tri_tests, int32 each) for algorithmic-byte accounting. */
int n2w_bvh_query_device_counted(const n2w_bvh* bvh, const n2w_vec3* d_points, int query_count,
                                 float* d_distance2, n2w_vec3* d_closest, int* d_triangle_id,
                                 int* d_overflow, int* d_node_visits, int* d_tri_tests,
                                 int block_size, n2w_stream_t stream);
/* Inside/outside classification of a closed mesh by +x ray parity, with the
 * reference's ray test and query offset (src/cuda/cubql_bvh.cu:407-455, which
 * runs it on the CPU for slice masks).  d_inside[i] = 1 inside, 0 outside;
 * *d_overflow (device int, caller-zeroed) is set to 1 if a stack overflowed. */
int n2w_bvh_inside_device(const n2w_bvh* bvh, const n2w_vec3* d_points, int query_count,
                          uint8_t* d_inside, int* d_overflow, int block_size, n2w_stream_t stream);
/* Slice grid of the reference renderer (src/cuda/cubql_bvh.cu:963-1025): view
 * "xy"|"xz"|"yz", frame from the mesh bounds grown by padding_fraction, widened
 * to the pixel aspect when preserve_aspect; pixel (ix, iy) -> points[iy*W+ix].
 * frame_out[4] = u_min, u_max, v_min, v_max (may be NULL). */
int n2w_slice_points(const float* bounds6, const char* view, float plane, int width, int height,
                     float padding_fraction, int preserve_aspect, float* points_out, float* frame_out);
/* Same grid with every choice explicit: frame_in[4] (u_min, u_max, v_min, v_max)
 * replaces the padded bounds when not NULL (bounds6 may then be NULL); rule picks
 * the pixel-coordinate rounding: N2W_SLICE_RULE_RENDER u_min + du * (i / (n-1))
 * (reference renderer, cubql_bvh.cu:1013-1017) or N2W_SLICE_RULE_EVAL
 * u_min + (du * i) / (n-1) (reference NC evaluator, eval_tcnn_nc_wos.cu:393). */
#define N2W_SLICE_RULE_RENDER 0
#define N2W_SLICE_RULE_EVAL 1
int n2w_slice_points_ex(const float* bounds6, const float* frame_in, const char* view, float plane, int width,
                        int height, float padding_fraction, int preserve_aspect, int rule, float* points_out,
                        float* frame_out);
/* Seed grid built with the BVH: (n+1)^3 lattice nodes lo + h*(i,j,k); slot of
 * the triangle nearest each node (leaf order).  Queries test that triangle first,
 * so their traversal starts with a tight bound.  Any output may be NULL. */
int n2w_bvh_seed_grid(const n2w_bvh* bvh, float* lo_out, float* h_out, int* n_out, int* slots_out);
/* Copies the device layout back to the host: nodes (128 B each) and leaf-ordered
 * triangles (48 B each).  Either pointer may be NULL.  Used by the CPU restatement
 * of the traversal to count visits. */
int n2w_bvh_copy_layout(const n2w_bvh* bvh, void* nodes_out, void* tris_out);

/* ---- boundary value problems ------------------------------------------- */
/* Boundary / source modes.  Values 0..16 and 30..32 keep the reference's
 * NcBoundaryMode ids (include/n2wos/tcnn_nc_wos.hpp:14-35); 100+ are new. */
#define N2W_BC_HARMONIC_X2_MINUS_Y2 0
#define N2W_BC_EXTERNAL_CHARGES_MEDIUM 1
#define N2W_BC_EXTERNAL_CHARGES_HIGH 2
#define N2W_BC_HARMONIC_ZEBRA_K4 3
#define N2W_BC_HARMONIC_ZEBRA_K8 4
#define N2W_BC_HARMONIC_ZEBRA_K12 5
#define N2W_BC_EXTERNAL_CHARGES_SHELL_K8 6
#define N2W_BC_EXTERNAL_CHARGES_SHELL_K16 7
#define N2W_BC_TEXTURE_STRIPES_K8 8
#define N2W_BC_TEXTURE_STRIPES_K16 9
#define N2W_BC_TEXTURE_CHECKER_K8 10
#define N2W_BC_TEXTURE_CHECKER_K16 11
#define N2W_BC_CONSTANT_ONE 12
#define N2W_BC_HARMONIC_MIXTURE_SMOOTH 13     /* reference include/n2wos/nc_harmonic_mixture.hpp */
#define N2W_BC_HARMONIC_MIXTURE_FIGLIKE 14
#define N2W_BC_HARMONIC_MIXTURE_MULTISCALE 15
#define N2W_BC_HARMONIC_MIXTURE_FIGLIKE_HF 16
#define N2W_BC_POISSON_MULTISCALE 30
#define N2W_BC_POISSON_FIGLIKE_HF 31
#define N2W_BC_POISSON_FIGLIKE_HF_X5 32
#define N2W_BC_CHARGES_SEEDED 100   /* sum_k a_k / |x - c_k| with a seeded charge set */
#define N2W_BC_POISSON_SINPROD 101  /* u = sin(w x) sin(w y) sin(w z), f = 3 w^2 u */

#define N2W_SOURCE_BALL 0    /* source sampled inside each ball from its Green's function */
#define N2W_SOURCE_CENTER 1  /* reference rule r^2/6 * f(ball centre), exact for harmonic f */

#define N2W_MAX_CHARGES 16

typedef struct n2w_problem {
  int32_t mode;             /* N2W_BC_* */
  int32_t source_sampling;  /* N2W_SOURCE_* (ignored for harmonic problems) */
  int32_t charge_count;     /* for N2W_BC_CHARGES_SEEDED */
  float omega;              /* for N2W_BC_POISSON_SINPROD */
  float charges[N2W_MAX_CHARGES][4]; /* x, y, z, amplitude */
  int32_t source_samples;   /* N2W_SOURCE_BALL: points averaged per ball (0 or 1 = one, max 64) */
  int32_t reserved;
} n2w_problem;

/* Seeded charge set: centres uniform in the spherical shell r in [r_min, r_max]
 * (uniform in volume), amplitudes uniform in [-1, 1]; stream = splitmix64(seed). */
int n2w_problem_charges_seeded(int count, float r_min, float r_max, uint64_t seed,
                               n2w_problem* out);
int n2w_problem_sinprod(float omega, int source_sampling, n2w_problem* out);
int n2w_problem_reference_mode(int mode, int source_sampling, n2w_problem* out);
/* Exact solution u(x) (FP64 where analytic) for n points (host arrays). */
int n2w_problem_exact(const n2w_problem* problem, const double* xyz, int64_t n, double* u_out);
/* Dirichlet data g and source f as the device evaluates them (FP32), host side. */
int n2w_problem_eval_f32(const n2w_problem* problem, const float* xyz, int64_t n, float* g_out,
                         float* f_out);
/* Case-insensitive name -> mode id (reference parse_nc_boundary_mode aliases,
 * src/cuda/cubql_bvh.cu:1739-1800, plus "charges_seeded", "poisson_sinprod"). */
int n2w_problem_mode_from_name(const char* name, int* mode_out);
const char* n2w_problem_mode_name(int mode);

/* ---- walkers ------------------------------------------------------------ */
#define N2W_WALK_PURE 0      /* walk to the epsilon shell */
#define N2W_WALK_PREFIX 1    /* stop at depth_m, emit X_m for the cache (coarse level) */
#define N2W_WALK_RESIDUAL 2  /* record X_m at depth_m, continue to the boundary */

typedef struct n2w_walk_options {
  int32_t walks_per_point;
  int32_t max_steps;     /* reference default 256 */
  int32_t depth_m;       /* truncation depth for PREFIX / RESIDUAL */
  float epsilon;         /* stopping shell width */
  float step_scale;      /* ball radius = step_scale * distance (reference 0.999) */
  uint64_t seed;         /* Philox key */
  int32_t block_size;    /* threads per block of the persistent walker (0 = tuned default) */
  int32_t blocks_per_sm; /* resident blocks per SM (0 = occupancy maximum) */
  int32_t chunk;         /* walks a lane takes per queue pop (0 = tuned default) */
  int32_t accumulate;    /* 0: outputs are overwritten; 1: results are added */
  int64_t deadline_ns;   /* 0 = none; else walkers stop this many ns after launch */
  int32_t regen_threshold; /* lanes of a warp that must be waiting before walk
                              updates / regeneration run (1..32; 0 = tuned default) */
} n2w_walk_options;

/* Per-point FP64 estimator accumulators (device arrays, one entry per point). */
typedef struct n2w_point_stats {
  double* d_sum;          /* sum of sample values */
  double* d_sum_sq;       /* sum of squared sample values */
  uint32_t* d_count;      /* samples accumulated */
  uint64_t* d_steps;      /* sum of walk steps (ball moves) */
  uint32_t* d_forced;     /* walks stopped by max_steps */
} n2w_point_stats;

/* Run-level counters written by the walker (device struct, zeroed by the call). */
typedef struct n2w_walk_counters {
  unsigned long long walks;        /* walks finished */
  unsigned long long steps;        /* ball moves (walk-steps) */
  unsigned long long queries;      /* closest-point queries */
  unsigned long long node_visits;  /* 4-wide node fetches */
  unsigned long long tri_tests;    /* triangle tests */
  unsigned long long overflow;     /* traversal stack overflows */
  unsigned long long forced;       /* walks stopped by max_steps */
  unsigned long long timed_out;    /* walks abandoned by the deadline */
} n2w_walk_counters;

/* Host evaluation of the walkers' generator: Philox4x32-10 of counter ctr[4]
 * under the key the walkers derive from (seed, tag); tag 0 = plain walks,
 * 1 = coarse (PREFIX) walks, 2 = residual walks.  Lets a caller reproduce the
 * random numbers of walk w = point*W + j at step s: ctr = {w, w>>32, s, 0|1}. */
int n2w_rng_philox4x32_10(const uint32_t* ctr, uint64_t seed, uint32_t tag, uint32_t* out);

/* Workspace bytes a walker call over point_count points needs: the work-queue
 * counter, run counters and each point's first closest-point query (24 B). */
size_t n2w_wos_workspace_bytes(int64_t point_count);

/* Plain WoS estimate of u at each point with per-point FP64 reductions on the
 * device: persistent walker, counter-based Philox RNG, queue regeneration.
 * d_workspace may be NULL (then stream-ordered memory is taken from the CUDA
 * pool for the call).  d_counters (device) may be NULL. */
int n2w_wos_estimate(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_vec3* d_points,
                     int64_t point_count, const n2w_walk_options* options,
                     n2w_point_stats stats, n2w_walk_counters* d_counters, void* d_workspace,
                     n2w_stream_t stream);

/* Allocation-free n2w_wos_estimate.  No counterpart in the reference.
 * For callers that may not allocate device memory while they solve (a host
 * application that hands the library a fixed share of HBM and forbids other
 * allocations; a serving loop that must not call cudaMalloc on its request
 * path, since cudaMalloc can synchronise the device).  The walker scratch lives
 * in one static device array of N2W_NOALLOC_SCRATCH_BYTES (4 MiB), held by every
 * GPU that loads the library until exit; point_count above N2W_NOALLOC_MAX_POINTS
 * returns N2W_EINVAL.  The caller still passes points and outputs.  Every
 * call looks up the array's device address (cudaGetSymbolAddress, with the
 * current device; it allocates nothing, and stays right after a
 * cudaDeviceReset); the first call on a device also loads the module, so make
 * that first call before any stream capture.
 * All calls on a device share the one array, so calls that overlap on the GPU
 * (other streams, other threads) race: serialise them.  No cudaMalloc /
 * cudaFree or other allocating routine is called. */
#define N2W_NOALLOC_SCRATCH_BYTES (4u << 20)
#define N2W_NOALLOC_MAX_POINTS ((N2W_NOALLOC_SCRATCH_BYTES - 512u) / 24u)
int n2w_wos_estimate_noalloc(const n2w_bvh* bvh, const n2w_problem* problem,
                             const n2w_vec3* d_points, int64_t point_count,
                             const n2w_walk_options* options, n2w_point_stats stats,
                             n2w_walk_counters* d_counters, n2w_stream_t stream);

/* Per-sample outputs, mirroring launch_nc_pure_wos_samples
 * (include/n2wos/tcnn_nc_wos.hpp:87-93): sample j of point i is at i*W+j. */
int n2w_wos_pure_samples(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_vec3* d_points,
                         int64_t point_count, const n2w_walk_options* options,
                         float* d_sample_values, int* d_step_count, int* d_forced_max_steps,
                         int* d_query_overflow, n2w_stream_t stream);

/* Coarse (PREFIX) and residual (RESIDUAL) walks for NC / 2LMC, mirroring
 * launch_nc_hybrid_prefix and launch_nc_2lmc_prefix_continue
 * (include/n2wos/tcnn_nc_wos.hpp:95-124).  Per sample: X_m mapped to the unit
 * cube by (x - input_min) / input_extent (reference cubql_bvh.cu:1311-1315),
 * the prefix value A_m (source accumulated to depth m, plus boundary value if
 * the walk stopped earlier), needs_cache flag, and for RESIDUAL the value of the
 * continuation (A_m + continuation).  d_continuation_values may be NULL for PREFIX. */
int n2w_wos_prefix_samples(const n2w_bvh* bvh, const n2w_problem* problem,
                           const n2w_vec3* d_points, int64_t point_count,
                           const n2w_walk_options* options, int mode, const float* input_min,
                           const float* input_extent, float* d_prefix_inputs,
                           float* d_boundary_values, float* d_continuation_values,
                           uint8_t* d_needs_cache, int* d_step_count, int* d_forced_max_steps,
                           int* d_query_overflow, n2w_stream_t stream);

/* nc = A + C*needs, residual = needs ? W - C : 0 (reference cubql_bvh.cu:1608-1627). */
int n2w_wos_combine(const float* d_cache_outputs, const float* d_boundary_values,
                    const float* d_continuation_values, const uint8_t* d_needs_cache,
                    int64_t sample_count, float* d_nc_values, float* d_residual_values,
                    int block_size, n2w_stream_t stream);

/* Per-point FP64 reduction of per-sample arrays (sample j of point i at i*W+j):
 * warp shuffles + FP64 atomics (replaces the host summaries of
 * src/tools/eval_tcnn_nc_wos.cu:525-569). */
int n2w_reduce_samples(const float* d_values, const int* d_step_count, const int* d_forced,
                       int64_t point_count, int walks_per_point, n2w_point_stats stats,
                       int accumulate, n2w_stream_t stream);

/* ---- neural cache (hash grid + MLP), replaces the reference's tiny-cuda-nn
 *      HashGrid + FullyFusedMLP + Adam (src/tools/eval_tcnn_nc_wos.cu:747-759) -- */
typedef struct n2w_cache n2w_cache;
typedef struct n2w_cache_config {
  int32_t n_levels;             /* 1..16 */
  int32_t n_features_per_level; /* 2 */
  int32_t log2_hashmap_size;    /* T = 2^log2 entries per hashed level */
  float base_resolution;        /* N_min */
  float per_level_scale;        /* b; 0 = derive from max_resolution */
  float max_resolution;         /* N_max (used when per_level_scale == 0) */
  int32_t n_neurons;            /* 16, 32 or 64 */
  int32_t n_hidden_layers;      /* 1..4 */
  float learning_rate;          /* Adam */
  float beta1, beta2, epsilon;
  uint64_t seed;                /* parameter initialisation */
} n2w_cache_config;

/* 16 levels x 2 features, 2^19 entries, resolutions 16..2048, 64 x 2 hidden,
 * Adam lr 1e-2, beta (0.9, 0.99), eps 1e-15. */
int n2w_cache_config_default(n2w_cache_config* out);
/* Host-only: parameter counts and per-level resolution / table size of a config. */
int n2w_cache_describe(const n2w_cache_config* cfg, int64_t* grid_params, int64_t* mlp_params,
                       int32_t* level_resolution, int32_t* level_table_size);
int n2w_cache_create(const n2w_cache_config* cfg, n2w_cache** out);
void n2w_cache_destroy(n2w_cache* cache);
/* Parameter counts (floats) and per-level resolution / table size (arrays of n_levels). */
int n2w_cache_info(const n2w_cache* cache, n2w_cache_config* cfg_out, int64_t* grid_params,
                   int64_t* mlp_params, int32_t* level_resolution, int32_t* level_table_size);
/* C(x) for n inputs in the unit cube (float[3n]) -> d_outputs[n]. */
int n2w_cache_infer(const n2w_cache* cache, const float* d_inputs, int64_t n, float* d_outputs,
                    n2w_stream_t stream);
/* Adds d(mean (C(x)-t)^2)/d(params) into the cache's gradient buffer (no update);
 * d_outputs (may be NULL) receives C(x).  Used by gradient checks. */
int n2w_cache_gradients(n2w_cache* cache, const float* d_inputs, const float* d_targets, int64_t n,
                        float* d_outputs, n2w_stream_t stream);
/* One Adam step on the L2 loss mean (C(x)-t)^2 over the batch; *h_loss_out (may be
 * NULL; synchronises when given) receives the batch loss before the update. */
int n2w_cache_train_step(n2w_cache* cache, const float* d_inputs, const float* d_targets, int64_t n,
                         float* h_loss_out, n2w_stream_t stream);
int n2w_cache_zero_grad(n2w_cache* cache, n2w_stream_t stream);
/* The cache's FP32 gradient buffer (count floats, [grid | mlp]) and its device
 * loss sum, for callers that reduce gradients with their own communicator:
 * n2w_cache_gradients -> reduce the buffer in place -> n2w_cache_apply_gradients. */
int n2w_cache_gradient_buffer(n2w_cache* cache, float** d_grad, int64_t* count, float** d_loss_sum);
/* One Adam step on grad_scale * (the gradient buffer); clears the buffer. */
int n2w_cache_apply_gradients(n2w_cache* cache, float grad_scale, n2w_stream_t stream);
/* Stream-ordered device copy of the parameters (FP32 master and FP16 working
 * copy) of src into dst, which must have the same configuration: the snapshot
 * step of progressive estimation.  Adam state and gradients are not copied. */
int n2w_cache_copy_params(n2w_cache* dst, const n2w_cache* src, n2w_stream_t stream);
/* Host copies of the FP32 master parameters, the FP16 working copy and the FP32
 * gradient ([grid | mlp] order; any pointer may be NULL). */
int n2w_cache_get_params(const n2w_cache* cache, float* h_fp32, uint16_t* h_fp16, float* h_grad);
int n2w_cache_set_params(n2w_cache* cache, const float* h_fp32);
/* Versioned binary checkpoint: config, step, parameters, Adam moments. */
int n2w_cache_save(const n2w_cache* cache, const char* path);
int n2w_cache_load(const char* path, n2w_cache** out);

/* ---- neural-cache estimators -------------------------------------------- */
/* n points uniform in the interior of the closed mesh: Philox candidates in
 * [box_lo, box_hi] kept by +x ray parity (the reference samples its training
 * set the same way on the CPU, src/tools/eval_tcnn_nc_wos.cu:437-491).
 * Synchronises; *h_accepted_out (may be NULL) = points produced. */
int n2w_sample_interior(const n2w_bvh* bvh, const float* box_lo, const float* box_hi, int64_t n,
                        uint64_t seed, n2w_vec3* d_points_out, int64_t* h_accepted_out,
                        n2w_stream_t stream);
/* Same, also reporting *h_candidates_out (may be NULL): the candidates the n
 * accepted points consumed, n * draws / hits over every draw of the launch, so
 * n / *h_candidates_out estimates the interior volume fraction of the box. */
int n2w_sample_interior_ex(const n2w_bvh* bvh, const float* box_lo, const float* box_hi, int64_t n,
                           uint64_t seed, n2w_vec3* d_points_out, int64_t* h_accepted_out,
                           int64_t* h_candidates_out, n2w_stream_t stream);
/* Unit-cube cache inputs: clamp((x - input_min) / input_extent, 0, 1)
 * (reference nc_fill_inputs_kernel, src/cuda/cubql_bvh.cu:1359-1370). */
int n2w_map_to_unit(const n2w_vec3* d_points, int64_t n, const float* input_min,
                    const float* input_extent, float* d_inputs, n2w_stream_t stream);

typedef struct n2w_nc_train_options {
  int32_t steps;            /* training steps */
  int32_t batch;            /* fresh interior points per step */
  int32_t walks_per_label;  /* WoS walks averaged into each label */
  int32_t max_steps;
  float epsilon;
  float step_scale;
  uint64_t seed;
  float input_min[3];
  float input_extent[3];
  float sample_lo[3];       /* box for interior sampling */
  float sample_hi[3];
} n2w_nc_train_options;
/* Online training: per step, fresh interior points, WoS labels (mean of
 * walks_per_label walks, per-point FP64 on the device), one Adam step on the L2
 * loss.  h_losses (may be NULL) receives each step's batch loss (synchronises
 * every step when given). */
int n2w_nc_train(n2w_cache* cache, const n2w_bvh* bvh, const n2w_problem* problem,
                 const n2w_nc_train_options* options, float* h_losses, n2w_stream_t stream);

/* Data-parallel online training, one process per GPU: every rank draws its own
 * fresh points (rank r keyed by seed + r * 0xD6E8FEB86659FD93) and WoS labels,
 * computes the mean gradient of its batch, the gradients are summed over the
 * communicator's ranks (NCCL all-reduce) and every rank applies the same Adam
 * step to the mean of the rank means -- the gradient of the union batch, since
 * every rank's batch has options->batch points.  Caches start from the same
 * parameters on every rank (same config and seed) and stay identical.  With a
 * one-rank communicator this is n2w_nc_train.  h_losses: the union batch's loss
 * per step (synchronises every step when given).  No counterpart in the
 * reference (one process, one GPU). */
int n2w_nc_train_dp(n2w_cache* cache, const n2w_bvh* bvh, const n2w_problem* problem,
                    const n2w_nc_train_options* options, n2w_comm* comm, float* h_losses, n2w_stream_t stream);

typedef struct n2w_nc2lmc_options {
  int32_t coarse_walks;     /* walks per point truncated at depth_m, closed by the cache */
  int32_t residual_walks;   /* walks per point continued to the boundary (0 = NC-WoS only) */
  int32_t depth_m;
  int32_t max_steps;
  float epsilon;
  float step_scale;
  uint64_t seed;
  float input_min[3];
  float input_extent[3];
  int32_t point_batch;      /* points per internal batch (0 = auto) */
} n2w_nc2lmc_options;
/* NC+2LMC: coarse stats accumulate A_m + C(X_m) (or the full walk value when it
 * stops before depth m); residual stats accumulate W(X_m) - C(X_m) (0 when it
 * stopped before m).  Estimate = mean(coarse) + mean(residual); estimator
 * variance = var_c / N_c + var_r / N_r. */
int n2w_nc2lmc_estimate(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_cache* cache,
                        const n2w_vec3* d_points, int64_t n, const n2w_nc2lmc_options* options,
                        n2w_point_stats coarse, n2w_point_stats residual, n2w_stream_t stream);

/* Sample counts of an NC+2LMC run (device struct; the call ADDS to it, the
 * caller zeroes it).  Mirrors the NC evaluator's host-side counting
 * (src/tools/eval_tcnn_nc_wos.cu:527-533, 548-549). */
typedef struct n2w_nc2lmc_counters {
  unsigned long long coarse_cache_queries;   /* coarse walks closed by the cache */
  unsigned long long coarse_forced;          /* coarse walks stopped by max_steps */
  unsigned long long coarse_overflow;        /* coarse walks with a traversal overflow */
  unsigned long long residual_cache_queries; /* residual walks that reached depth m */
  unsigned long long residual_forced;
  unsigned long long residual_overflow;
} n2w_nc2lmc_counters;
/* n2w_nc2lmc_estimate plus counters (d_counters may be NULL).  cache == NULL
 * selects the analytic cache C(x) = u(x), the exact solution of the problem:
 * the reference's debug-only oracle levels (src/cuda/wos_wavefront.cu:140-149,
 * methods oracle_coarse / oracle_residual / oracle_2lmc). */
int n2w_nc2lmc_estimate_ex(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_cache* cache,
                           const n2w_vec3* d_points, int64_t n, const n2w_nc2lmc_options* options,
                           n2w_point_stats coarse, n2w_point_stats residual, n2w_nc2lmc_counters* d_counters,
                           n2w_stream_t stream);

/* Progressive NC+2LMC with snapshot overlap (reference
 * docs/progressive_snapshot_accounting_policy.md:30-52: evaluate snapshot k
 * while training snapshot k+1, two cache instances, swap only at block
 * boundaries).  For block k = 0 .. blocks-1:
 *   1. freeze theta_infer = theta_train (n2w_cache_copy_params);
 *   2. run one NC+2LMC block with theta_infer on eval_stream (estimate options;
 *      block seed derived from estimate.seed and k) and add its per-point
 *      coarse and residual sums into `coarse` / `residual`;
 *   3. unless k is the last block, train theta_train for train_steps_per_block
 *      steps (train options; per-block seed) on train_stream when overlap = 1,
 *      or on eval_stream after the block when overlap = 0;
 *   4. wait for both streams.
 * Every block has the same coarse and residual walks per point, so the pooled
 * estimate mean(coarse) + mean(residual) is unbiased for any sequence of
 * snapshots, and its variance is var_c / N_c + var_r / N_r over the pooled
 * samples.  The result does not depend on `overlap` (up to FP64 addition
 * order).  `coarse` and `residual` are zeroed first.  h_blocks (may be NULL)
 * receives per-block CUDA-event times.  Synchronises at every block boundary. */
typedef struct n2w_nc_progressive_options {
  int32_t blocks;                /* estimation blocks (one frozen snapshot each) */
  int32_t train_steps_per_block; /* training steps theta_train takes during a block */
  int32_t overlap;               /* 1: estimate and train on two streams; 0: serial */
  int32_t reserved;
  n2w_nc_train_options train;    /* `steps` is ignored */
  n2w_nc2lmc_options estimate;   /* per-block walks */
} n2w_nc_progressive_options;
typedef struct n2w_nc_progressive_block {
  float eval_ms;   /* the block's estimate on eval_stream */
  float train_ms;  /* the block's training (0 for the last block) */
  float wall_ms;   /* block start (snapshot copy) to both streams done */
  float reserved;
} n2w_nc_progressive_block;
int n2w_nc_progressive(n2w_cache* theta_train, n2w_cache* theta_infer, const n2w_bvh* bvh,
                       const n2w_problem* problem, const n2w_vec3* d_points, int64_t n,
                       const n2w_nc_progressive_options* options, n2w_point_stats coarse,
                       n2w_point_stats residual, n2w_nc_progressive_block* h_blocks,
                       n2w_stream_t eval_stream, n2w_stream_t train_stream);

/* Training labels over a fixed point set, mirroring launch_nc_update_labels
 * (include/n2wos/tcnn_nc_wos.hpp:79-86, kernel src/cuda/cubql_bvh.cu:1372-1420).
 * Each call is one refresh: N2W_LABEL_WOS runs walks_per_point more walks per
 * point into the caller-owned running accumulators `accum` (zero them before
 * refresh 0) and writes targets = running mean of every walk so far;
 * N2W_LABEL_EXACT writes the exact solution.  Inputs are the points mapped to
 * the unit cube.  d_workspace: n2w_wos_workspace_bytes(n) bytes or NULL. */
#define N2W_LABEL_EXACT 0 /* reference NcLabelSource::ExactAnalytic */
#define N2W_LABEL_WOS 1   /* reference NcLabelSource::WosSupervision */
typedef struct n2w_nc_label_options {
  int32_t walks_per_point;
  int32_t max_steps;
  float epsilon;
  float step_scale;
  uint64_t seed;
  int32_t refresh_index;
  int32_t label_source;
  float input_min[3];
  float input_extent[3];
  int32_t block_size;       /* walker block size (0 = tuned default) */
  int32_t reserved;
} n2w_nc_label_options;
int n2w_nc_update_labels(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_vec3* d_points, int64_t n,
                         const n2w_nc_label_options* options, n2w_point_stats accum, float* d_inputs,
                         float* d_targets, void* d_workspace, n2w_stream_t stream);

/* ---- batched instances (one persistent launch) --------------------------- */
/* A scene merges several BVHs into one device layout (indices rebased) so one
 * launch can walk many meshes.  The BVHs may be destroyed afterwards.  No
 * counterpart in the reference, which runs one problem per launch. */
typedef struct n2w_scene n2w_scene;
int n2w_scene_create(const n2w_bvh* const* bvhs, int count, n2w_scene** out);
int n2w_scene_info(const n2w_scene* scene, int* mesh_count, int64_t* nodes, int64_t* triangles,
                   int64_t* device_bytes);
void n2w_scene_destroy(n2w_scene* scene);

/* One PDE instance of a batch: plain WoS at point_count device points of scene
 * mesh `mesh` for problem `problem` (index into the batch's problem array),
 * walks_per_point walks each, Philox key `seed`.  Walks are keyed exactly as
 * n2w_wos_estimate keys them, so an instance's estimates equal a single-problem
 * call with the same seed up to the order of FP64 additions, whatever else the
 * batch holds.  Results go to the instance's per-point accumulators. */
typedef struct n2w_batch_item {
  int32_t mesh;
  int32_t problem;
  const n2w_vec3* d_points;
  int64_t point_count;
  int32_t walks_per_point;
  int32_t reserved;
  uint64_t seed;
  n2w_point_stats stats;
} n2w_batch_item;

/* Launch shape of a batch (the autotuner's search space). */
typedef struct n2w_batch_tuning {
  int32_t block_size;      /* walker threads per block: 64, 128 or 256 */
  int32_t blocks_per_sm;   /* 0 = occupancy maximum */
  int32_t chunk;           /* walks a lane takes per queue pop */
  int32_t regen_threshold; /* waiting lanes that trigger walk updates */
  int32_t reg_variant;     /* 0: 64 registers / 4 blocks per SM; 1: 80 registers / 3 blocks */
  float ms;                /* autotuner: best time of this shape on the probe batch */
} n2w_batch_tuning;

typedef struct n2w_batch n2w_batch;
/* Copies the problems and the instance table to the device.  options supplies
 * max_steps, epsilon, step_scale, accumulate (0: each launch first zeroes every
 * instance's accumulators) and the launch shape; walks_per_point and seed are
 * per item. */
int n2w_batch_create(const n2w_scene* scene, const n2w_problem* problems, int problem_count,
                     const n2w_batch_item* items, int item_count, const n2w_walk_options* options,
                     n2w_batch** out);
int n2w_batch_info(const n2w_batch* batch, int64_t* total_points, int64_t* total_walks,
                   n2w_walk_options* options_out, int* reg_variant_out);
/* New Philox keys for every item (e.g. the next round of an adaptive estimate);
 * synchronises the stream.  A captured graph picks them up. */
int n2w_batch_set_seeds(n2w_batch* batch, const uint64_t* seeds, n2w_stream_t stream);
/* One launch over every instance: memsets and kernels only, no allocation and
 * no host synchronisation, so it can be captured into a CUDA graph.
 * d_counters (device, may be NULL) receives run counters over all instances. */
int n2w_batch_launch(n2w_batch* batch, n2w_walk_counters* d_counters, n2w_stream_t stream);
/* Captures n2w_batch_launch on `stream` (not the legacy default stream) into a
 * graph the batch owns; n2w_batch_graph_launch replays it. */
int n2w_batch_capture_graph(n2w_batch* batch, n2w_walk_counters* d_counters, n2w_stream_t stream);
int n2w_batch_graph_launch(n2w_batch* batch, n2w_stream_t stream);
/* Times launch shapes on a probe batch (the first max(min(n,64), f*n) points of
 * every item, scratch accumulators) and applies the fastest to the batch:
 * threads per block x register budget, then chunk, then regeneration
 * threshold.  Trials are copied to trials_out (up to trials_cap).  Drops a
 * captured graph (capture again after tuning). */
int n2w_batch_autotune(n2w_batch* batch, double sample_fraction, n2w_batch_tuning* best_out,
                       n2w_batch_tuning* trials_out, int trials_cap, int* trials_count, n2w_stream_t stream);
int n2w_batch_set_tuning(n2w_batch* batch, const n2w_batch_tuning* tuning, n2w_stream_t stream);
void n2w_batch_destroy(n2w_batch* batch);

/* ---- serving loop (continuous batching) ---------------------------------- */
/* A device-resident request loop: meshes (as one scene), problems and walker
 * buffers stay on the GPU; requests of uneven point counts are admitted while
 * a device pool allocated at start-up has room, and every tick runs ONE
 * persistent walker launch over all in-flight requests, so requests that
 * arrive while others run join the next launch.  Each request runs sweeps of
 * walks until the maximum per-point standard error is <= its target (or its
 * walk cap).  A request's result does not depend on the other requests (up
 * to the order of FP64 additions).  No counterpart in the reference. */
#define N2W_REQUEST_PENDING 0 /* waiting for admission (pool memory / in-flight slots) */
#define N2W_REQUEST_ACTIVE 1  /* admitted, walking */
#define N2W_REQUEST_DONE 2    /* target standard error reached */
#define N2W_REQUEST_CAPPED 3  /* stopped at max_walks_per_point */
#define N2W_REQUEST_FAILED 4

typedef struct n2w_server_options {
  int64_t pool_bytes;      /* device pool for requests; 0 = pool_fraction of free memory */
  float pool_fraction;     /* used when pool_bytes == 0 (default 0.25) */
  int32_t max_inflight;    /* requests admitted at once (default 256) */
  int64_t tick_walks;      /* walks shared out per tick (default 2^21) */
  int32_t max_steps;       /* walk cap (default 256) */
  float epsilon;           /* stopping shell (default 1e-3) */
  float step_scale;        /* default 0.999 */
  int32_t block_size;      /* walker threads per block (default 256) */
  int32_t regen_threshold; /* default 8 */
  int32_t chunk;           /* walks a lane takes per queue pop in a tick (default 1: a tick holds
                              few walks per lane, so single walks balance the lanes best) */
  int64_t tick_walks_max;  /* budget of a tick in which no request in flight could finish its
                              sweep within tick_walks walks (default 2^23; <= tick_walks: always tick_walks):
                              larger ticks run more efficiently but delay small requests */
} n2w_server_options;

#define N2W_STDERR_MAX 0 /* every point's standard error <= target */
#define N2W_STDERR_RMS 1 /* root mean square over points of the standard errors <= target */

typedef struct n2w_request {
  int32_t mesh;                /* index into the server's meshes */
  int32_t problem;             /* index into the server's problems */
  int64_t point_count;
  float target_stderr;         /* stop when the standard error (see stderr_norm) <= this */
  int32_t min_walks_per_point; /* first sweep size floor (>= 32 walks are used) */
  int32_t max_walks_per_point; /* walk cap per point */
  uint64_t seed;
  int32_t stderr_norm;         /* N2W_STDERR_MAX (default) or N2W_STDERR_RMS */
  int32_t mode;                /* N2W_REQUEST_MODE_PLAIN or N2W_REQUEST_MODE_NC2LMC */
} n2w_request;

#define N2W_REQUEST_MODE_PLAIN 0  /* plain WoS, batched with every plain request of the tick */
#define N2W_REQUEST_MODE_NC2LMC 1 /* NC+2LMC with the cache registered for (mesh, problem) */

/* A pre-trained cache for NC+2LMC requests on one (mesh, problem) pair.  The
 * cache must outlive the server.  Each sweep of such a request runs
 * coarse_walks walks truncated at depth_m and closed by the cache plus
 * ceil(residual_fraction * coarse_walks) residual walks per point, in chunks
 * of 4,096 points between the plain ticks (n2w_nc2lmc_estimate_ex; its sample
 * buffers come from the stream-ordered allocator), so NC walks do not share
 * the plain requests' launch.  The standard error is sqrt(var_c/N_c + var_r/N_r). */
typedef struct n2w_server_nc {
  const n2w_cache* cache;
  float input_min[3];
  float input_extent[3];
  int32_t depth_m;
  float residual_fraction;
} n2w_server_nc;

typedef struct n2w_request_info {
  int32_t state;            /* N2W_REQUEST_* */
  int32_t sweeps;
  int64_t walks_per_point;  /* walks each point received (NC+2LMC: coarse walks) */
  int64_t ticks;            /* launches the request took part in (NC+2LMC: chunks) */
  float max_stderr;         /* max per-point standard error at the end */
  float rms_stderr;         /* root mean square of the per-point standard errors at the end */
  double queue_seconds;     /* submission -> admission */
  double latency_seconds;   /* submission -> result ready */
  int64_t residual_walks_per_point; /* NC+2LMC: residual walks each point received */
} n2w_request_info;

typedef struct n2w_server_stats {
  int64_t submitted, completed, inflight, pending, peak_inflight;
  int64_t ticks, walks, walk_steps, overflow;
  int64_t pool_bytes, pool_used, peak_pool_bytes;
  int64_t nc_chunks, nc_walks; /* NC+2LMC chunks run and their coarse + residual walks */
  int64_t tick_us, nc_us;      /* worker wall time in plain ticks / NC+2LMC steps (incl. syncs) */
  int64_t tick_gpu_us;         /* device time of the ticks' first-query + walker launches (CUDA events) */
} n2w_server_stats;

typedef struct n2w_server n2w_server;
int n2w_server_options_default(n2w_server_options* out);
/* Builds the scene from the BVHs, copies the problems, allocates the pool and
 * starts the worker thread on the current device.  The BVHs must outlive the
 * server (NC+2LMC requests walk them directly). */
int n2w_server_create(const n2w_bvh* const* bvhs, int mesh_count, const n2w_problem* problems, int problem_count,
                      const n2w_server_options* options, n2w_server** out);
/* Registers (or replaces) the cache used by NC+2LMC requests on (mesh, problem).
 * nc->cache == NULL selects the analytic cache C(x) = u(x) (a check of the
 * estimator, as n2w_nc2lmc_estimate_ex).  depth_m >= 0, residual_fraction in (0, 1]. */
int n2w_server_set_nc(n2w_server* server, int mesh, int problem, const n2w_server_nc* nc);
/* Thread-safe.  Copies the host points (3 * point_count floats).  Requests
 * larger than the whole pool fail with N2W_ENOMEM; NC+2LMC requests need a
 * cache registered for their (mesh, problem). */
int n2w_server_submit(n2w_server* server, const n2w_request* request, const float* h_points, int64_t* id_out);
int n2w_server_poll(n2w_server* server, int64_t id, int* state_out);
/* Blocks until the request finishes (timeout_seconds < 0: no limit; on
 * timeout N2W_ETIMEOUT and the request stays), then copies per-point means and
 * standard errors (point_count doubles each; either may be NULL) and releases
 * the request. */
int n2w_server_wait(n2w_server* server, int64_t id, double timeout_seconds, double* h_mean, double* h_stderr,
                    n2w_request_info* info);
int n2w_server_get_stats(n2w_server* server, n2w_server_stats* out);
/* Stops the worker (unfinished requests fail) and frees everything. */
void n2w_server_destroy(n2w_server* server);

/* ---- device utilities ---------------------------------------------------- */
/* u(x) of the problem at n device points, evaluated in FP64 and stored as FP32. */
int n2w_problem_exact_device(const n2w_problem* problem, const n2w_vec3* d_points, int64_t n, float* d_u_out,
                             n2w_stream_t stream);
/* Analytic cache: outputs = u(input_min + inputs * input_extent) for unit-cube
 * inputs (float[3n]), the stand-in for C(x) in the oracle levels. */
int n2w_oracle_cache_infer(const n2w_problem* problem, const float* d_inputs, int64_t n, const float* input_min,
                           const float* input_extent, float* d_outputs, n2w_stream_t stream);
/* n unit-cube samples from Philox(seed; sample, step) and, when d_targets is
 * not NULL, targets u(input_min + x * input_extent).  The cache probe's batch
 * generator (src/tools/probe_tcnn_cache.cu:233-250) with a counter-based RNG. */
int n2w_fill_unit_samples(const n2w_problem* problem, int64_t n, uint64_t seed, uint32_t step,
                          const float* input_min, const float* input_extent, float* d_inputs, float* d_targets,
                          n2w_stream_t stream);
/* d_acc4[0..3] += sum pred, sum exact, sum (pred-exact)^2, sum |pred-exact|
 * (FP64): the cache probe's downstream consumer (probe_tcnn_cache.cu:251-262). */
int n2w_compare_accumulate(const float* d_pred, const float* d_exact, int64_t n, double* d_acc4,
                           n2w_stream_t stream);
/* d_counts3[0..2] += number of nonzero entries of needs_cache (u8), forced and
 * overflow (int32); any input may be NULL. */
int n2w_count_samples(const uint8_t* d_needs_cache, const int* d_forced, const int* d_overflow, int64_t n,
                      unsigned long long* d_counts3, n2w_stream_t stream);

/* ---- thin device-memory helpers for callers without a CUDA binding ------ */
/* ---- multi-GPU exchange (NCCL, one process per GPU) --------------------- */
/* Walks and points shard with no communication; ranks exchange only sums of
 * per-point statistics, timings and (data-parallel training) gradients, as
 * all-reduces of caller-owned device buffers on the caller's stream.  Rank 0
 * creates the id with n2w_comm_unique_id and hands its N2W_COMM_ID_BYTES bytes
 * to every rank (any host channel); each rank then calls n2w_comm_create with
 * its own device current.  No counterpart in the reference. */
#define N2W_COMM_ID_BYTES 128
#define N2W_DTYPE_F32 0
#define N2W_DTYPE_F64 1
#define N2W_DTYPE_U32 2
#define N2W_DTYPE_U64 3
#define N2W_DTYPE_I32 4
#define N2W_OP_SUM 0
#define N2W_OP_MAX 1
#define N2W_OP_MIN 2
int n2w_comm_unique_id(uint8_t* id_out);
int n2w_comm_create(const uint8_t* id, int world, int rank, n2w_comm** out);
int n2w_comm_info(const n2w_comm* comm, int* rank, int* world);
int n2w_comm_allreduce(n2w_comm* comm, const void* d_send, void* d_recv, int64_t count, int dtype, int op,
                       n2w_stream_t stream);
/* In place: FP64 sum and sum of squares, u32 count, and steps / forced when
 * non-null, summed over ranks (combines walk shards of the same points). */
int n2w_comm_allreduce_point_stats(n2w_comm* comm, n2w_point_stats stats, int64_t n, n2w_stream_t stream);
/* All ranks reach this call before any returns (synchronises `stream`). */
int n2w_comm_barrier(n2w_comm* comm, n2w_stream_t stream);
void n2w_comm_destroy(n2w_comm* comm);

int n2w_device_count(int* out);
int n2w_set_device(int device);
int n2w_malloc(void** d_ptr, size_t bytes);
int n2w_free(void* d_ptr);
int n2w_malloc_host(void** h_ptr, size_t bytes); /* pinned */
int n2w_free_host(void* h_ptr);
int n2w_memcpy_h2d(void* d_dst, const void* h_src, size_t bytes, n2w_stream_t stream);
int n2w_memcpy_d2h(void* h_dst, const void* d_src, size_t bytes, n2w_stream_t stream);
int n2w_memset(void* d_ptr, int value, size_t bytes, n2w_stream_t stream);
int n2w_stream_create(n2w_stream_t* out);
int n2w_stream_destroy(n2w_stream_t stream);
int n2w_stream_sync(n2w_stream_t stream);
int n2w_device_sync(void);
/* Records a pair of events around nothing: timer handle for callers. */
typedef struct n2w_timer n2w_timer;
int n2w_timer_create(n2w_timer** out);
int n2w_timer_start(n2w_timer* t, n2w_stream_t stream);
int n2w_timer_stop(n2w_timer* t, n2w_stream_t stream);
int n2w_timer_elapsed_ms(n2w_timer* t, float* ms_out); /* synchronises on the stop event */
void n2w_timer_destroy(n2w_timer* t);
int n2w_sm_count(int* out);
int n2w_mem_info(size_t* free_bytes, size_t* total_bytes);
/* Sustained read bandwidth (GB/s) of one on-chip level, measured by the
 * library's own probe kernels on the current device: level 1 = each block
 * re-reads its own 16 KiB slice (L1 hits), level 2 = a `bytes` buffer that fits
 * in L2 streamed with loads that bypass L1.  The roofline denominator for the
 * L1/L2-resident traversal.  Allocates its buffers.  No counterpart in the
 * reference. */
int n2w_probe_read_bandwidth(int level, size_t bytes, int iterations, double* gbs_out);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* N2W_H_ */
