/*
 * blacktracer.h -- C ABI of the B200-native BlackTracer hot path.
 *
 * Plain C types only (pointers, sizes, PODs).  CUDA streams are passed as
 * void* (a cudaStream_t; NULL = the legacy default stream).  Unless stated
 * otherwise, array arguments of the *_dev functions are DEVICE pointers owned
 * by the caller; *_host functions take HOST pointers and do the copies.
 *
 * Every entry point returns 0 (BT_OK) or a BT_ERR_* code; bt_last_error()
 * gives a message for the last failure on the calling thread.
 *
 * Each declaration names the reference interface it replaces
 * (annemiekie/BlackTracer; "BT/" = BlackTracer2/BlackTracer/).
 */
#ifndef BLACKTRACER_H
#define BLACKTRACER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BT_ABI_VERSION 1

enum {
  BT_OK = 0,
  BT_ERR_ARG = 1,      /* invalid argument (size, level, NULL pointer)      */
  BT_ERR_CUDA = 2,     /* a CUDA runtime call failed                        */
  BT_ERR_NOMEM = 3,    /* device allocation failed / budget exceeded        */
  BT_ERR_NUMERIC = 4,  /* a bounded iteration did not converge              */
  BT_ERR_STATE = 5     /* handle used in the wrong state                    */
};

/* Per-ray status written by the integrators. */
enum {
  BT_RAY_ESCAPED = 0,     /* integrated to the end of the affine range     */
  BT_RAY_CAPTURED = 1,    /* capture test said "falls in": (-1, -1, 0)     */
  BT_RAY_MAXSTEP = 2,     /* MAXSTP attempts without reaching the end: the
                             reference then returns the camera's own angles */
  BT_RAY_NONCONVERGED = 3 /* capture-test Newton loop hit its cap (the
                             reference loop is unbounded, BT/Metric.h:152)  */
};

/* Arithmetic of the geodesic integrator. */
enum {
  BT_PRECISION_PLAIN = 0, /* FP64, reference operation order, no FMA      */
  BT_PRECISION_MIXED = 1, /* FP32 bulk, FP64 near the photon sphere, at
                             turning points, for capture and for phi.
                             Does NOT meet 1e-6 rad against the reference:
                             p99 ~1.6e-4 rad on the C2 grid, with a
                             different grid topology.  The reference's step
                             controller reads an error estimate whose FP32
                             rounding noise (1e-4..1e-1 relative where the
                             FP64 one is 1e-9..5e-4) changes its accept /
                             grow decisions, so the rays follow other step
                             sequences; FAST is the form that meets 1e-6.  */
  BT_PRECISION_FAST = 2   /* FP64, the same method with the equations of
                             motion reassociated (3 reciprocals instead of
                             16 divisions, by Newton-refined approximate
                             reciprocals), stage sin/cos by angle addition,
                             error ratio and step-size factor in FP32, FMA:
                             same grid topology as PLAIN, p99 ~1e-10 rad    */
};

/* Field-for-field the reference Camera (BT/Camera.h:8-11). */
typedef struct bt_camera {
  double theta, phi, r;
  double speed, br, btheta, bphi;
  double alpha, w, wbar, Delta, ro;
} bt_camera;

/* Camera(theta, phi, r, speed): static / user-speed camera.
 * Replaces BT/Camera.h:27-38 (+ initforms :54-61).  Spin a replaces the
 * process-global metric::a set by BlackHole::setA (BT/BlackHole.h:12-15). */
int bt_camera_static(double a, double theta, double phi, double r,
                     double speed, bt_camera* out);

/* Camera(theta, phi, r, br, btheta, bphi): Keplerian circular-orbit camera
 * boosted along (br, btheta, bphi).  Replaces BT/Camera.h:40-52 with
 * metric::calcSpeed (BT/Metric.h:104-108). */
int bt_camera_orbit(double a, double theta, double phi, double r, double br,
                    double btheta, double bphi, bt_camera* out);

/* Camera::getParamArray (BT/Camera.h:67-78): the 7 floats the map uses. */
int bt_camera_params(const bt_camera* cam, float out7[7]);

/* Integrator options.  Defaults (bt_integ_opts_default) are the reference's
 * rkckIntegrate1 constants, BT/Metric.h:311-314 and MAXSTP :31. */
typedef struct bt_integ_opts {
  double eps;        /* relative tolerance            (1e-5)   */
  double h1;         /* initial step magnitude        (0.01)   */
  double z_end;      /* affine end point, negative    (-1e7)   */
  int32_t maxstp;    /* attempt cap                   (1000)   */
  int32_t precision; /* BT_PRECISION_*                (PLAIN)  */
  double fp64_band;  /* MIXED: |r - r_ph| band kept in FP64, in M (0.05) */
} bt_integ_opts;

void bt_integ_opts_default(bt_integ_opts* o);

/* Backward null-geodesic integration of n camera-sky directions.
 * Replaces Grid::integration_wrapper (BT/Grid.h:514-556; called from
 * Grid::callKernel :382-401), which works in place on vector<double>& theta,
 * phi and vector<int>& step with the camera and spin taken from globals.
 * Here inputs and outputs are separate DEVICE arrays of n elements; outputs
 * follow the reference: captured rays give (-1, -1, 0); a ray that reaches
 * MAXSTP keeps the camera's angles (wrapped) with steps = maxstp-1.
 * status (may be NULL) receives BT_RAY_* per ray.  o may be NULL (defaults). */
int bt_integrate_rays(const bt_camera* cam, double a, const double* theta,
                      const double* phi, size_t n, double* theta_out,
                      double* phi_out, int32_t* steps, uint8_t* status,
                      const bt_integ_opts* o, void* stream);

/* The same with HOST arrays: copies in, integrates, copies out, synchronises
 * the stream.  Uses a per-thread device staging area grown on demand. */
int bt_integrate_rays_host(const bt_camera* cam, double a, const double* theta,
                           const double* phi, size_t n, double* theta_out,
                           double* phi_out, int32_t* steps, uint8_t* status,
                           const bt_integ_opts* o, void* stream);

/* bt_integrate_rays_host without any allocation.  No counterpart in the
 * reference.  For callers that cannot let the library allocate device
 * memory: a render or serving thread that must not stall on the implicit
 * device synchronisation of cudaMalloc/cudaFree, a plugin host with a fixed
 * device-memory budget, middleware whose device memory belongs to another
 * runtime.  The rays are staged in a fixed static device array of
 * bt_integrate_rays_host_static_capacity() rays (65536), held by every GPU
 * that loads this library until the process exits; larger n is rejected
 * with BT_ERR_ARG.  The first call on a device looks up that array's
 * address (with the device current) and keeps it for that device's current
 * context; a call after cudaDeviceReset, in the new context, looks it up
 * again.  Make the first call on a device before any stream capture.
 * status may be NULL.  All calls share the one array: calls that
 * overlap on the GPU (other threads or streams of the same device) race on
 * it and must be serialised by the caller.  Synchronises `stream`. */
int bt_integrate_rays_host_static(const bt_camera* cam, double a,
                                  const double* theta, const double* phi,
                                  size_t n, double* theta_out, double* phi_out,
                                  int32_t* steps, uint8_t* status,
                                  const bt_integ_opts* o, void* stream);
size_t bt_integrate_rays_host_static_capacity(void);

/* ------------------------------------------------------------------ grid */

/* Lattice size of a grid with max level L: N = 2^L/(2-eq)+1 rows,
 * M = (2-eq)*2*(N-1) columns, eq = angle ? 1 : 0.  BT/Grid.h:612-615. */
int bt_grid_dims(int maxlevel, int angle, int32_t* N, int32_t* M);

/* A device-resident adaptive grid: the reference's Grid object
 * (BT/Grid.h:27-660) with CamToCel / steps / blockLevels held as a dense
 * N x M lattice in HBM instead of hash maps.  Created once per (maxlevel,
 * angle) and rebuilt in place for any camera / spin. */
typedef struct bt_grid bt_grid;

int bt_grid_create(int maxlevel, int angle, bt_grid** out);
void bt_grid_destroy(bt_grid* g);

/* Builds the grid: Grid::Grid(maxLevelPrec, startLevel, angle, camera, bh)
 * (BT/Grid.h:605-624) -- start-level trace, level-synchronous refinement
 * (refineCheck, PRECCELEST = 0.015), T-vertex fix.  Asynchronous on
 * `stream`; no host synchronisation inside (graph-capturable).  The
 * T-vertex fix runs in the canonical order (level, then key i<<32|j) --
 * the reference iterates an unordered_map there, whose order is
 * implementation-defined.  o may be NULL (reference defaults); o->precision
 * selects the plain or mixed integrator. */
int bt_grid_build(bt_grid* g, const bt_camera* cam, double a, int startlevel,
                  const bt_integ_opts* o, void* stream);

typedef struct bt_grid_info {
  int32_t N, M, maxlevel, startlevel, angle;
  int64_t traced;         /* rays integrated by the build            */
  int64_t n_leaf_blocks;  /* leaf blocks below the max level          */
  uint32_t flags;         /* nonzero: a bounded iteration gave up
                             (1: T-vertex fix not converged, 2: fix
                             stack, 4: work list overflow, 8: the
                             one-launch build gave up waiting) or 16:
                             an early refinement the level form would
                             not make (bt_grid_set_flow)             */
  /* device pointers into the lattice (valid until the next build) */
  const double* thphi;    /* N*M (theta, phi) pairs                  */
  const int32_t* steps;   /* N*M                                     */
  const uint8_t* exists;  /* N*M, 1 where CamToCel holds the key     */
  const int8_t* blevel;   /* N*M, blockLevels at the block origin    */
  const uint8_t* status;  /* N*M, BT_RAY_* of traced vertices        */
  float trace_ms;         /* with bt_grid_set_timing: device time of
                             the ray-tracing launches of the build   */
  int32_t trace_launches;
  int32_t launches;       /* kernels the last build launched          */
} bt_grid_info;

/* Records CUDA events around the ray-tracing launches of later builds
 * (reported by bt_grid_query as trace_ms; eager builds only). */
int bt_grid_set_timing(bt_grid* g, int on);

/* on = 1: later builds are captured once into a CUDA graph (per start
 * level, precision and trace launch shape) and replayed.  No counterpart in
 * the reference (its build is host-driven). */
int bt_grid_set_graph(bt_grid* g, int on);

/* on >= 1: later builds run the refinement levels as one persistent launch
 * of `on` blocks of 256 threads per SM (capped by the occupancy limit, 2)
 * instead of one trace launch per level; 0 = off.  A block is checked
 * (refineCheck, BT/Grid.h:410-445) as soon as its own four corners are
 * traced, or refined as soon as one traced diagonal alone is far enough
 * apart (maxlevel - startlevel <= 7), and a new vertex is traced as soon as a
 * check creates it, so no level waits for the previous level's longest rays.
 * The grids are the same bit for bit, except where a block refined on its
 * (1, 2) diagonal has a NaN separation on the other, which refineCheck's
 * std::max turns into a leaf: that build reports flag 16 (rebuild in the
 * level form).  Reserves 12 + min(maxlevel - 2, 6) bytes per lattice vertex
 * of the set; used when the set's lattices hold fewer than 2^28 vertices in
 * all (otherwise builds take the level form).  No counterpart in the
 * reference (its build is host-driven, level by level). */
int bt_grid_set_flow(bt_grid* g, int on);

/* Diagnostic: the number of Jacobi passes of the T-vertex fix per level of
 * later builds, 1..8 (default 8, the most any grid needs; 2-3 is typical).
 * A level whose last pass still changed a vertex is reported as not
 * converged: flag 1 in bt_grid_info.flags and BT_ERR_NUMERIC from
 * bt_grid_query.  Lowering it exists to exercise that report.  No
 * counterpart in the reference (its fixTvertices is sequential). */
int bt_grid_set_tfix_passes(bt_grid* g, int passes);

/* Diagnostic: cooperative = 1 (default) runs the T-vertex fix of a level as
 * one cooperative launch when the set's blocks fit the device at once;
 * 0 launches each pass, the commit and the check separately (the path sets
 * too large for one cooperative launch take).  Same grids either way. */
int bt_grid_set_tfix_launch(bt_grid* g, int cooperative);

/* Diagnostic for the one-launch build's failure path: the next build (flow
 * on, eager) loses one ray -- counted as in flight, never traced -- so that
 * nothing can end the flow; its warps give up after about two seconds
 * without progress and the build reports flag 8 (BT_ERR_NUMERIC, "the flow
 * gave up waiting").  The grid is then incomplete; later builds are normal. */
int bt_grid_set_flow_drop(bt_grid* g);

/* Synchronises `stream` and reports the build.  Returns BT_ERR_NUMERIC when
 * a bounded loop (T-vertex fixed point) gave up. */
int bt_grid_query(bt_grid* g, bt_grid_info* info, void* stream);

/* Dense export into caller DEVICE arrays of N*M elements (any may be NULL):
 * theta/phi (-2 where no vertex exists), exists, steps, blevel (-1 = none),
 * status. */
int bt_grid_export_dense(const bt_grid* g, double* theta, double* phi,
                         uint8_t* exists, int32_t* steps, int8_t* blevel,
                         uint8_t* status, void* stream);

/* Compact export of the grid in key order (i, then j) -- the reference's
 * CamToCel (BT/Grid.h:575), steps (:577) and blockLevels (:588) as sorted
 * lists.  Destination pointers may be HOST (pageable or pinned) or DEVICE
 * memory, or NULL to skip an array; cap_* give their capacities.  The
 * function synchronises `stream` once (to learn the counts) and enqueues the
 * copies; the caller synchronises before reading host buffers.  Returns
 * BT_ERR_ARG (with n_* set) when a capacity is too small. */
typedef struct bt_grid_export_t {
  uint32_t* vi;          /* vertex row i                      */
  uint32_t* vj;          /* vertex column j                   */
  double* theta;         /* celestial theta                   */
  double* phi;           /* celestial phi                     */
  int32_t* steps;        /* integration steps                 */
  size_t cap_vertices;
  uint32_t* bi;          /* leaf-block origin row             */
  uint32_t* bj;          /* leaf-block origin column          */
  int8_t* level;         /* block level                       */
  size_t cap_blocks;
  size_t n_vertices;     /* out                               */
  size_t n_blocks;       /* out                               */
} bt_grid_export_t;
int bt_grid_export(bt_grid* g, bt_grid_export_t* out, void* stream);

/* The float2 grid the per-pixel map reads: replaces saveAsGpuHash
 * (BT/Grid.h:642-654) + the PSH tables + makeGrid
 * (BT/MakeImageKernel.cu:369-384).  (-2,-2) = no vertex, (-1,-1) =
 * captured; for half grids (GM/GN > 3) the lower hemisphere is mirrored
 * (rows = 2N-1).  Returns a device pointer owned by the grid. */
int bt_grid_map_export(bt_grid* g, const float** grid_out, int32_t* rows,
                       int32_t* cols, int32_t* sym, void* stream);

/* ------------------------------------------------------------ grid sets */

/* A set of `count` grids of the same (maxlevel, angle), each built for its
 * own camera and spin, together: the reference builds its grids one after
 * the other (BT/BlackTracer.cpp:220-262, one Grid per camera of `cams`);
 * here every level of all grids is refined by one launch and traced by one
 * persistent launch with a shared work queue, so the long rays of one grid
 * overlap the work of the others.  Members are bt_grid handles for
 * bt_grid_query / export / map_export; they are released with the set
 * (bt_grid_destroy on a member does nothing, bt_grid_build on a member
 * returns BT_ERR_ARG).  Builds of one set must be ordered on one stream. */
typedef struct bt_batch bt_batch;

int bt_batch_create(int maxlevel, int angle, int count, bt_batch** out);
void bt_batch_destroy(bt_batch* b);

/* Builds all grids: grid k from cams[k] with spin spins[k] (count each),
 * from `startlevel`, options o for all.  Asynchronous on `stream`. */
int bt_batch_build(bt_batch* b, const bt_camera* cams, const double* spins,
                   int startlevel, const bt_integ_opts* o, void* stream);

/* Builds only members 0..n-1 (1 <= n <= count) from cams[0..n-1] and
 * spins[0..n-1]; the other members are left unbuilt.  For callers that
 * gather a varying number of grids per build (a serving loop). */
int bt_batch_build_first(bt_batch* b, int n, const bt_camera* cams,
                         const double* spins, int startlevel,
                         const bt_integ_opts* o, void* stream);

/* Member k (0 <= k < count), or NULL. */
bt_grid* bt_batch_grid(bt_batch* b, int k);

/* As bt_grid_set_graph / bt_grid_set_timing / bt_grid_set_flow, for the whole set. */
int bt_batch_set_graph(bt_batch* b, int on);
int bt_batch_set_timing(bt_batch* b, int on);
int bt_batch_set_flow(bt_batch* b, int on);

/* Launch shape of the persistent ray-tracing kernel: threads per block
 * (64, 128 or 256) and resident blocks per SM (0 = as many as fit). */
typedef struct bt_trace_shape {
  int32_t threads;        /* 64, 128 or 256                                 */
  int32_t blocks_per_sm;  /* 0: as many as fit                             */
  int32_t refill;         /* idle lanes a warp refills at once (0: 8)      */
} bt_trace_shape;
int bt_batch_set_shape(bt_batch* b, const bt_trace_shape* shape);

typedef struct bt_batch_info {
  int32_t count;           /* members built by the last build              */
  int64_t traced;          /* rays integrated by the last build, all grids */
  uint32_t flags;          /* OR of the members' flags                     */
  float trace_ms;          /* with timing on, eager builds                 */
  int32_t trace_launches;
  int32_t launches;        /* kernels per build                            */
  int32_t graph;           /* builds replay a CUDA graph                   */
  bt_trace_shape shape;
} bt_batch_info;
int bt_batch_query(bt_batch* b, bt_batch_info* info, void* stream);

/* Autotuner: times `repeats` builds of these cameras for each candidate
 * trace launch shape, keeps the fastest in the set and reports it (best,
 * best_ms may be NULL).  Synchronises `stream`. */
int bt_batch_autotune(bt_batch* b, const bt_camera* cams, const double* spins,
                      int startlevel, const bt_integ_opts* o, int repeats,
                      bt_trace_shape* best, float* best_ms, void* stream);

typedef struct bt_tune_result {
  bt_trace_shape shape;  /* level builds: trace launch shape and refill size  */
  int32_t flow;          /* 0: level builds; k >= 1: one launch, k blocks/SM  */
  int32_t band_met;      /* MIXED: 1 when fp64_band meets the p99 target      */
  double fp64_band;      /* MIXED: the band chosen; otherwise the option's    */
  double band_p99_rad;   /* MIXED: its p99 error against PLAIN on the sample
                            rays; otherwise -1                                */
  float best_ms;         /* per build of the set, chosen configuration        */
  float level_ms;        /* fastest level-build configuration                 */
  float flow_ms;         /* fastest one-launch configuration (0: none ran)    */
  int32_t candidates;    /* configurations timed                              */
} bt_tune_result;

/* The full autotuner.  For the MIXED form it first picks the FP64 band
 * (fp64_band, the FP64-fallback threshold around the photon orbit): the
 * narrowest of 0.05, 0.1, 0.2, 0.5, 1, 2, 5 M whose p99 angular error
 * against the PLAIN form, on 2048 seeded directions of each of the first
 * (up to) 8 cameras, is at most p99_target_rad; when none is, the one with
 * the smallest error (band_met = 0).  Then it times `repeats` builds of the
 * set with that band for every configuration: level builds over the trace
 * launch shapes of bt_batch_autotune plus 128 threads at 1 and 2 blocks per
 * SM, and refill sizes 4, 8 and 16 (the rays
 * per warp step that a warp waits to start together; each lane holds one
 * ray), and one-launch builds (bt_batch_set_flow) of 1 and 2 blocks per SM.
 * The set keeps the fastest (shape, refill and form); pass out->fp64_band
 * in the options of later MIXED builds.  Synchronises `stream`.  No
 * counterpart in the reference. */
int bt_batch_tune(bt_batch* b, const bt_camera* cams, const double* spins, int startlevel,
                  const bt_integ_opts* o, double p99_target_rad, int repeats,
                  bt_tune_result* out, void* stream);

/* As bt_batch_set_shape / bt_batch_tune for a lone grid (bt_grid_create),
 * on its last build's camera, spin and start level; the tuned configuration
 * is kept for later builds. */
int bt_grid_set_shape(bt_grid* g, const bt_trace_shape* shape);
int bt_grid_tune(bt_grid* g, const bt_integ_opts* o, double p99_target_rad, int repeats,
                 bt_tune_result* out, void* stream);

/* ------------------------------------------------------- per-pixel map */

/* Camera-sky corner directions of an equirectangular W x H output:
 * Viewer::makeSphereView (BT/Viewer.h:82-88).  view: DEVICE float2 array of
 * (H+1)*(W+1) (theta, phi) pairs. */
int bt_view_sphere(float* view, int width, int height, void* stream);

/* A resident environment map: its summed-area table (float4 per pixel,
 * channels B^2.2*A, G^2.2*A, R^2.2*A, A), built on the device from a BGR8
 * image of rows x cols (cv::imread order).  Replaces the host OpenMP table
 * of cudaPrep (BT/MakeImageKernel.cu:1312-1330) and its per-call upload. */
typedef struct bt_env bt_env;
int bt_env_create(const uint8_t* bgr, int rows, int cols, int bgr_on_device,
                  bt_env** out, void* stream);
void bt_env_destroy(bt_env* e);
int bt_env_sat(const bt_env* e, const float** sat, int32_t* rows, int32_t* cols);

/* A resident star set in the reference's StarProcessor layout
 * (BT/StarProcessor.h:25-31): star_pos = 2n (theta, phi), star_mag = 2n
 * (magnitude, B-V), tree = 2^(treeLevel+1)-1 cumulative counts (binaryStarTree).
 * psf_rgb (optional) is the diffraction sprite, psf_size^2 RGB8. */
typedef struct bt_stars bt_stars;
int bt_stars_tree_size(int treeLevel);
/* StarProcessor's tree (makeTree, BT/StarProcessor.h:172-212) from a star
 * list: HOST arrays; stars with mag > magnitude_cut are left out
 * (BT/StarProcessor.h:37-46).  Outputs sized 2n, 2n, tree_size. */
int bt_stars_build_tree(const float* theta, const float* phi, const float* mag,
                        const float* bv, int n, int treeLevel,
                        float magnitude_cut, float* star_pos, float* star_mag,
                        int* tree, int* n_kept);
int bt_stars_create(const float* star_pos, const float* star_mag, int n,
                    const int* tree, int treeLevel, const uint8_t* psf_rgb,
                    int psf_size, bt_stars** out, void* stream);
void bt_stars_destroy(bt_stars* s);

/* The blackbody colour tables of a star set, copied to HOST arrays of
 * 3 * count floats: per entry its RGBtoHSP (h, s, p) and 255 * HSPtoRGB of
 * that.  table 0: the reference's 391 entries (BT/Const.h:7, 1000-40000 K in
 * 100 K steps); table 1: the 1024-entry FP32 table (bt_frame.bb_table = 1;
 * no counterpart in the reference), entry k the linear interpolation of the
 * reference's entries at k * 390 / 1023.  *count = entries; nothing is
 * copied when capacity is smaller (or arrays NULL).  Synchronises stream. */
int bt_stars_blackbody(const bt_stars* s, int table, float* hsp, float* rgb, int capacity,
                       int* count, void* stream);

/* A renderer: per-resolution device scratch (the reference's dev_in,
 * dev_gap, dev_bh, dev_area, star buffers), created once per output size. */
typedef struct bt_map bt_map;
int bt_map_create(int width, int height, bt_map** out);
void bt_map_destroy(bt_map* m);

/* One frame.  Replaces makeImage / cudaPrep (BT/MakeImageKernel.cu:1206-1559,
 * called from Distorter::cudaCall, BT/Distorter.h:103-148) for one grid
 * (G = 1): pixInterpolation, findBlackPixels, findArea, smoothAreaH/V,
 * distortEnvironmentMap (map), distortStarMap + sumStarLight
 * (+ addDiffraction) + makePix (star), addStarsAndBackground (both).
 * All pointers are DEVICE pointers; nothing is copied to the host. */
typedef struct bt_frame {
  const float* grid;      /* bt_grid_map_export: grid_rows x grid_cols float2 */
  int32_t grid_rows, grid_cols, grid_level;  /* GN1, GM, MAXLEVEL            */
  const float* view;      /* (H+1)*(W+1) float2 camera-sky corners          */
  float hor, ver;         /* look-around offsets (pixInterpolation)         */
  float cam[7];           /* Camera::getParamArray                          */
  const bt_env* env;      /* required when map != 0                         */
  const bt_stars* stars;  /* required when star != 0                        */
  int32_t map, star, lr;  /* the reference's map / star / dev_lr toggles    */
  int32_t step;           /* splat half-width, 0..2 (the reference uses 1)  */
  int32_t diffraction;    /* scatter the sprite around saturated stars      */
  uint8_t* out;           /* H*W BGRA8                                      */
  /* Extensions (0 = the reference's behaviour): */
  int32_t bb_table;       /* 1: 1024-entry FP32 blackbody table (1000-40000 K,
                             interpolated from the reference's 391 entries)  */
  int32_t psf_scale;      /* 1: diffraction footprint scaled by the square
                             root of the lensing magnification at the
                             receiving pixel (clamped to [0.25, 4], rounded
                             to 33 levels 9% apart), total sprite light kept */
  /* Blending between two grids (the reference's Gr > 1 path): NULL grid2
   * renders `grid` alone. */
  const float* grid2;     /* second map grid, same shape as grid            */
  float alpha;            /* weight of grid2, in [0, 1]                     */
  float cam2[7];          /* getParamArray of grid2's camera: the frame uses
                             (1 - alpha) cam + alpha cam2 (camUpdate)       */
  const struct bt_blend* blend;  /* prepared on (grid, grid2)               */
  /* Star trails from the previous frame rendered with the same trails
   * object (NULL: none, as in the reference's first frame). */
  struct bt_trails* trails;
} bt_frame;

/* Blending between two grids computed for neighbouring camera poses (the
 * reference's movement between precomputed grids, BT/MakeImageKernel.cu
 * camUpdate / findBhCenter / findBhBorders / smoothBorder :386-456 and the
 * Gr > 1 branch of pixInterpolation :466-510).  bt_blend_prepare finds the
 * black hole's centre (box of the captured vertices of either grid) and its
 * border along 1000 directions in each grid, smoothed 4 times; a frame with
 * grid2 then blends the two grids, stretched towards their borders near the
 * shadow.  The reference's border walk has no bound; here it stops at the
 * lattice edge and bt_blend_info reports how many walks did. */
typedef struct bt_blend bt_blend;
int bt_blend_create(bt_blend** out);
void bt_blend_destroy(bt_blend* b);
int bt_blend_prepare(bt_blend* b, const float* grid_a, const float* grid_b, int rows,
                     int cols, void* stream);
/* Device pointer to the border (2 + 2*angles float2: the box, then per
 * direction grid a's and grid b's point); walks_at_edge is valid once the
 * prepare's stream has been synchronised. */
int bt_blend_info(const bt_blend* b, const float** border, int32_t* angles,
                  uint32_t* walks_at_edge);

/* Star trails between consecutive frames: addTrails, makeGradField and
 * clearArrays (BT/MakeImageKernel.cu:98-174, 517-537, 618-629).  A frame
 * rendered with bt_frame.trails draws, for every star seen in a pixel whose
 * kd-tree search holds fewer than n_stars / 100 stars, a fading line from
 * the position in the previous frame (of the same trails object) that best
 * follows the celestial gradient, within width / 25 pixels and 45 degrees;
 * the line is added to the star light.  A star's positions are cached per
 * frame in ascending pixel order, up to trailnum (the reference uses 30).
 * The first frame after create / reset draws none.  The reference's line
 * walk can step past its target and never end; here it stops there
 * (walks_cut counts those), and crossing lines keep the brighter value per
 * channel.  max_hits (0 = width * height) bounds the (pixel, star) pairs per
 * frame; pairs past it draw no trail (dropped). */
typedef struct bt_trails bt_trails;
int bt_trails_create(int n_stars, int width, int height, int trailnum, size_t max_hits,
                     bt_trails** out);
void bt_trails_destroy(bt_trails* t);
int bt_trails_reset(bt_trails* t);
typedef struct bt_trails_info {
  int64_t frame;        /* frames rendered since create / reset             */
  uint32_t hits;        /* (pixel, star) pairs of the last frame            */
  uint32_t dropped;     /* pairs beyond max_hits                            */
  uint32_t walks_cut;   /* line walks stopped at their target               */
  const float* trail;   /* DEVICE: the last frame's trail light, 3 per pixel */
} bt_trails_info;
/* Synchronises `stream` (the stream of the last frame). */
int bt_trails_query(bt_trails* t, bt_trails_info* info, void* stream);

/* An Airy diffraction sprite (size x size RGB8, the layout the reference
 * loads its diffraction image in, BT/MakeImageKernel.cu:1281-1286):
 * I = (2 J1(x)/x)^2 with the first dark ring at `first_zero` pixels for
 * 550 nm, scaled per channel by wavelength (R 610, G 550, B 465 nm), 255 at
 * the centre.  For bt_stars_create's psf_rgb. */
int bt_psf_airy(int size, float first_zero, uint8_t* rgb);

/* HOST only.  The sprite resampled for the magnification-scaled footprint
 * (bt_frame.psf_scale; no counterpart in the reference, whose sprite has one
 * size): level k in [0, 32] is the scale s_k = 0.25 * 2^(k/8), its entries the
 * offsets (row, column) from the centre within ceil(max(1, r) s_k) + 1 (r =
 * the largest offset of a non-zero sprite entry) whose bilinear sample of
 * the sprite at centre + offset / s_k, divided by s_k^2, is non-zero: 2 int16
 * offsets and 3 float values per entry, row-major.  *count = the level's
 * entries; nothing is written when capacity is smaller (or arrays NULL). */
int bt_psf_levels(const uint8_t* psf_rgb, int psf_size, int level, int16_t* offsets,
                  float* values, int capacity, int* count);

/* Diagnostic: the capacities of the star pass's deferred-pixel units (no
 * counterpart in the reference).  Pixels whose stars exceed the per-pixel
 * budget of the main star pass are cut into units of candidate kd-tree
 * leaves that all SMs share; `nodes` (default max(2^18, W*H)) bounds the
 * kd-tree nodes of those pixels' searches held at once, `units` (default
 * max(2^15, W*H/8), at least 2) the units, whose size grows to fit.
 * Pixels past either bound are rendered one block per pixel instead.  0
 * keeps a default.  Synchronises the device; no frame of m may be in
 * flight. */
int bt_map_set_star_capacity(bt_map* m, size_t nodes, size_t units);

/* Diagnostic: the number of those pixels (up to 32768) whose first tree
 * search keeps its emitted nodes (1024 at most each) for the second pass to
 * copy; the others are searched twice.  Negative: the default
 * (clamp(W*H/512, 1024, 32768)); 0: none.  Frames are the same either way.
 * Synchronises the device; no frame of m may be in flight. */
int bt_map_set_star_slab(bt_map* m, int pixels);

/* addDiffraction (BT/MakeImageKernel.cu:775-800) on a caller's star-light
 * buffer: light and out are DEVICE arrays of width*height*3 floats (the
 * renderer's size; the summed star light sumStarLight produces), different
 * buffers; the sprite is the star set's psf.  A pixel whose brightest
 * channel exceeds 65025 adds min(65025, (light / (10000 max^0.6) * sprite)^2)
 * per channel around itself, rows clipped at the image's edges, columns
 * wrapped.  As the reference's thread reads its own pixel for every sprite
 * entry, the entries after the centre (row-major) see the centre's term
 * added to it; terms of other bright pixels are not seen (in the reference
 * that depends on thread timing).  Deterministic; uses m's scratch. */
int bt_map_diffract(bt_map* m, const bt_stars* stars, const float* light, float* out,
                    void* stream);
/* Renders one frame on `stream`.  A frame that draws both the environment and
 * stars draws the environment on a second stream owned by `m` (created at the
 * priority of `stream`) while the star passes run on `stream`; `stream` waits
 * for it before compositing, so all work of the call is done when the work
 * queued on `stream` is. */
int bt_map_render(bt_map* m, const bt_frame* f, void* stream);

/* Device pointers into a renderer's scratch after a frame (for tests and
 * tools): corner (theta, phi), block gaps, black-hole mask, smoothed area,
 * summed star light (3 floats), star image and environment image. */
typedef struct bt_map_buffers {
  const float* thphi;
  const int32_t* gap;
  const uint8_t* bh;
  const float* area;
  const float* light;
  const uint8_t* stars_img;
  const uint8_t* env_img;
  const float* light_diffracted;  /* star light after diffraction (3 floats) */
} bt_map_buffers;
int bt_map_scratch(const bt_map* m, bt_map_buffers* b);

/* Work census of the last frame a renderer drew (f: that frame's
 * description): the environment columns the pixels span (distortEnvironment
 * Map's pixNum, BT/MakeImageKernel.cu:650-657; two summed-area reads each)
 * and the star candidates per pixel, those of the kd-tree nodes the search
 * emits (the reference tests them all, its starsToCheck :265-275) and those
 * left after this build's node-box pruning, and the stars that pass the quad
 * test (each placed in the pixel and splatted).  Synchronises `stream`.  For
 * rooflines and reports; no counterpart in the reference. */
typedef struct bt_map_census_t {
  uint64_t env_columns;          /* sum over coloured pixels of pixNum + 1     */
  uint64_t env_pixels;           /* pixels coloured from the environment       */
  uint64_t star_pixels;          /* pixels outside the shadow                  */
  uint64_t star_candidates_ref;  /* sum of starsToCheck                        */
  uint64_t star_candidates;      /* sum of stars in the leaves tested here     */
  uint64_t star_hits;            /* stars that pass the quad test (splatted)   */
  uint64_t heavy_candidates;     /* candidates of pixels with more than 2048   */
  uint64_t heavy_hits;           /* hits of those pixels                       */
} bt_map_census_t;
int bt_map_census(bt_map* m, const bt_frame* f, bt_map_census_t* out, void* stream);

/* ----------------------------------------------------------- cache files */

/* The reference's grid and star cache files (cereal binary archives,
 * written by write / writeStars, BT/BlackTracer.cpp:26-46, and loaded at
 * :226-258 and :306-335), read and written without cereal:
 * little-endian, each vector as a uint64 element count followed by its
 * elements, each int as 4 bytes.
 *   .grid  Grid::serialize (BT/Grid.h:36-39): int MAXLEVEL, N, M, then the
 *          PSHOffsetTable (BT/PSHOffsetTable.h:46-48): vector<float>
 *          hashTable (2 per slot), vector<int> offsetTable (2 per entry),
 *          vector<int> hashPosTag (2 per slot), int hashTableWidth,
 *          int offsetTableWidth.
 *   .star  StarProcessor::serialize (BT/StarProcessor.h:21-23):
 *          vector<int> binaryStarTree, vector<float> starPos,
 *          vector<float> starMag, int starSize, treeSize, treeLevel. */

/* A perfect spatial hash of lattice keys (i, j) -> (theta, phi): the
 * reference's PSHOffsetTable (BT/PSHOffsetTable.h), as the reference's
 * renderer consumes it (hashLookup, BT/kernel.cuh:713-733).  Buffers are
 * the caller's (HOST); a call whose capacities are too small returns
 * BT_ERR_ARG with the widths set, so the caller can size and call again. */
typedef struct bt_psh {
  float* hash_table;      /* 2 * hash_width^2: (theta, phi) per slot        */
  int32_t* pos_tag;       /* 2 * hash_width^2: key (i, j) per slot          */
  int32_t* offset_table;  /* 2 * offset_width^2                             */
  size_t cap_hash;        /* capacity of hash_table and pos_tag, elements   */
  size_t cap_offset;      /* capacity of offset_table, elements             */
  int32_t hash_width;     /* out (in, for bt_grid_file_write)               */
  int32_t offset_width;   /* out (in, for bt_grid_file_write)               */
} bt_psh;

/* Builds a table for n keys (2n ints, (i, j) >= 0, distinct) and values (2n
 * floats): replaces saveAsGpuHash + PSHOffsetTable::PSHOffsetTable
 * (BT/Grid.h:642-654, BT/PSHOffsetTable.h:350-370, widths :59-79).  Same table widths as
 * the reference (hash width (int)(sqrt(1.1 n) + 1.1), offset width
 * (int)(sqrt(n / 4) + 1.1) raised to be coprime with it) unless those fail
 * a few times -- regular key sets such as a uniform lattice -- after which
 * both widths grow.  Offsets are found by a deterministic search (the
 * reference seeds rand() with the time), so the table is reproducible.
 * HOST only.  BT_ERR_NUMERIC if no table was found after the bounded
 * retries. */
int bt_psh_build(const int32_t* keys, const float* values, size_t n, bt_psh* out);

/* The float2 map grid of a PSH table: makeGrid (BT/MakeImageKernel.cu
 * :369-384) -- every lattice vertex (i < N, j < M) looked up, (-2,-2) where
 * absent; with sym (M / N > 3) the lower hemisphere is mirrored into rows
 * 2N-1-i (rows = 2N-1).  Tables are DEVICE arrays; grid is a DEVICE array
 * of rows * M float2.  Offsets outside the table wrap (the reference reads
 * out of bounds there). */
int bt_grid_map_from_psh(const float* hash_table, const int32_t* pos_tag,
                         const int32_t* offset_table, int hash_width,
                         int offset_width, int N, int M, float* grid, int rows,
                         void* stream);

/* Writes / reads a .grid file.  maxlevel, N and M as the reference's Grid
 * holds them; tables as bt_psh (hash_width and offset_width are inputs for
 * writing).  Reading checks every count against the file's size and the
 * lattice shape against maxlevel; HOST only. */
int bt_grid_file_write(const char* path, int maxlevel, int N, int M, const bt_psh* t);
int bt_grid_file_read(const char* path, int32_t* maxlevel, int32_t* N, int32_t* M,
                      bt_psh* t);

/* A built grid to a .grid file the reference loads (BT/BlackTracer.cpp
 * :236-242): compact export, bt_psh_build, bt_grid_file_write.  Synchronises
 * `stream`.  The reference writes an empty table when startlevel ==
 * maxlevel (BT/Grid.h:623); here the table always holds the vertices. */
int bt_grid_save(bt_grid* g, const char* path, void* stream);

/* Shape of a .grid file's map grid: rows (2N-1 when mirrored, else N),
 * cols (M), sym (1 when mirrored); and the file's maxlevel (the map's grid
 * level).  Any output may be NULL. */
int bt_grid_file_map_shape(const char* path, int32_t* maxlevel, int32_t* rows,
                           int32_t* cols, int32_t* sym);
/* A .grid file straight to a DEVICE map grid (rows x cols float2, as
 * bt_grid_map_export returns): read, upload (stream-ordered allocation,
 * released on `stream`), bt_grid_map_from_psh. */
int bt_grid_file_load_map(const char* path, float* grid, int rows, int cols,
                          void* stream);

/* .star files.  Write: the arrays of bt_stars_build_tree / bt_stars_create
 * (star_pos, star_mag 2n each, tree bt_stars_tree_size(treeLevel)).  Read:
 * bt_stars_file_info for the counts, then bt_stars_file_read into HOST
 * arrays of those sizes. */
int bt_stars_file_write(const char* path, const float* star_pos, const float* star_mag,
                        int n, const int* tree, int treeLevel);
int bt_stars_file_info(const char* path, int* n, int* treeLevel);
int bt_stars_file_read(const char* path, float* star_pos, float* star_mag, int n_cap,
                       int* tree, int tree_cap);

/* ---------------------------------------------------------- camera view */

/* Camera-sky corner directions of a perspective W x H view looking along
 * the camera's forward direction, turned by offset_ver (up) and offset_hor
 * (right): Viewer::makeCameraView (BT/Viewer.h:109-133), with the
 * horizontal field of view view_angle (radians; the vertical one is
 * H / W of it).  |offset_ver| must not exceed (pi - vertical angle) / 2
 * (the reference prints an error and leaves the view unset).  view: DEVICE
 * float2 array of (H+1)*(W+1) (theta, phi). */
int bt_view_camera(float* view, int width, int height, double view_angle,
                   double offset_ver, double offset_hor, void* stream);

/* --------------------------------------------------------------- serving */

/* A frame server: requests of any resolution, camera and spin are rendered
 * (grid + per-pixel map, equirectangular sphere view) by a worker thread
 * with continuous batching -- admission by HBM budget and in-flight slots,
 * grids resident in a cache keyed by the exact camera and spin and reused,
 * the grids missing at an admission round built together as one grid set,
 * frames of different requests on their own streams, overlapping each other
 * and the next grid build.  Grid builds run on the highest-priority stream
 * and frames on lower ones, smaller frames first; the grid cache's memory is
 * reserved once, so that serving allocates no device memory for new poses.
 * No counterpart in the reference (a single-scene host program,
 * BT/BlackTracer.cpp). */
typedef struct bt_server bt_server;

typedef struct bt_server_config {
  int32_t maxlevel, startlevel, angle;  /* grids built for requests         */
  int32_t precision;                    /* BT_PRECISION_* of grid builds    */
  size_t grid_cache_bytes;              /* HBM budget of resident grids,
                                           reserved when the server is
                                           created                          */
  size_t render_bytes;                  /* HBM budget of render slots       */
  int32_t max_inflight;                 /* frames admitted at once          */
  int32_t max_build_batch;              /* grids built together (set size)  */
  const bt_env* env;                    /* environment map, or NULL         */
  const bt_stars* stars;                /* resident star set, or NULL       */
  int32_t step, lr;                     /* splat radius, lensing + redshift */
} bt_server_config;

/* Defaults: L6 -> L11 full-sphere grids, fast FP64, 40 GB grid cache,
 * 40 GB render slots, 16 frames in flight, sets of 8, step 1, lr on. */
void bt_server_config_default(bt_server_config* c);

typedef struct bt_request {
  uint64_t id;            /* caller's tag, returned in the completion     */
  int32_t width, height;
  bt_camera cam;
  double a;               /* spin                                         */
  uint8_t* out;           /* width*height*4 BGRA8: pinned host or device  */
} bt_request;

typedef struct bt_completion {
  uint64_t id;
  int32_t status;         /* BT_OK or the error code                      */
  int32_t grid_reused;    /* 1: the grid was resident                     */
  double t_submit, t_admit, t_done;  /* seconds, steady clock             */
} bt_completion;

typedef struct bt_server_stats {
  int64_t submitted, completed, failed;
  int64_t grid_hits, grid_misses, grids_built, build_sets, evictions;
  int64_t grids_resident;
  size_t grid_cache_bytes_used, render_bytes_used;
} bt_server_stats;

/* The server uses the device current at creation; env and stars must
 * outlive it. */
int bt_server_create(const bt_server_config* cfg, bt_server** out);
/* Thread-safe, non-blocking.  r->out must stay valid until completion.  A
 * request whose frame needs more device memory than the whole render budget
 * (render_bytes) completes with status BT_ERR_NOMEM instead of waiting. */
int bt_server_submit(bt_server* s, const bt_request* r);
/* Up to cap completions; waits up to wait_ms for the first one. */
int bt_server_poll(bt_server* s, bt_completion* out, int cap, int* n, int wait_ms);
int bt_server_stats_get(bt_server* s, bt_server_stats* st);
/* Finishes every submitted request, then releases the server. */
void bt_server_destroy(bt_server* s);

/* FP64 FMA throughput of the current device, TFLOP/s (2 flops per FMA),
 * from an independent-chain DFMA kernel timed with CUDA events: the peak
 * the FP64 integrator's roofline is reported against. */
int bt_probe_fp64_tflops(double* tflops, void* stream);

/* The fast form's reciprocal (approximate reciprocal refined by one
 * Newton-Raphson step: relative error ~1e-12) on n DEVICE values: for tests
 * that check it against 1/x.  No counterpart in the reference. */
int bt_probe_fast_rcp(const double* x, double* out, size_t n, void* stream);

/* Message for the last error on this thread ("" when none). */
const char* bt_last_error(void);

/* Library build/version string. */
const char* bt_version(void);

#ifdef __cplusplus
}
#endif
#endif /* BLACKTRACER_H */
