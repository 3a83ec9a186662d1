// map_internal.h -- shared declarations of the per-pixel map.
#pragma once

#include "bt_internal.h"

namespace bt {

struct Cam7 {
  float v[7];  // Camera::getParamArray, BT/Camera.h:67-78
};

// Resident environment map: its summed-area table in HBM.
struct EnvMap {
  int rows, cols;
  float4* sat;  // rows*cols
};

// Per-resolution scratch of the renderer (the reference's dev_in, dev_gap,
// dev_bh, dev_area, dev_areaSmooth, star buffers).
struct MapScratch {
  int M, N;             // output width, height
  float2* thphi;        // (N+1)(M+1) celestial corners
  int* gap;             // (N+1)(M+1) block size at each corner
  uint8_t* bh;          // N*M black-hole mask
  float* area;          // N*M solid angle (smoothed in place)
  float* area_tmp;      // N*M
  float* light;         // N*M*3 summed star light
  float* light2;        // N*M*3 star light after diffraction
  uint8_t* stars_img;   // N*M*4 star image (BGRA8)
  uint8_t* flag;        // N*M: pixel holds at least one star
  float3* cells;        // N*M*(2s+1)^2 splat cells (lazy)
  int cells_fw;         // 2s+1 the cells were sized for
  uint32_t* diff_list;  // bright pixels (diffraction)
  uint32_t* diff_count;
  uint32_t* env_wide;   // pixels spanning many environment columns
  uint32_t* env_wide_count;
  uint32_t* heavy_list; // pixels deferred to the block-per-pixel star path
  uint32_t* heavy_order;// the same, queued giant-first
  uint32_t* heavy_count;// 4 counters (deferred, giant, other, next item)
  // deferred pixels in units of candidate leaves (stars.cu, lazy): per
  // deferred pixel its nodes and leaves, node and unit offsets; the node
  // pool with the leaves up to each node; per unit its cell sums and whether
  // it splatted a star; control words
  uint32_t *hv_nn, *hv_nl, *hv_noff, *hv_uoff;
  int* hv_pool;
  uint32_t* hv_pend;
  float* hv_partial;
  uint8_t* hv_uany;
  uint32_t* hv_ctl;
  // the first pass's emitted nodes, kHvSlab per deferred pixel for the first
  // hv_slab_pixels pixels, so that the second pass copies instead of
  // searching again
  int* hv_slab;
  uint32_t hv_slab_pixels;
  int hv_slab_req;  // pixels the slab holds; < 0: the default for the frame size
  size_t hv_node_cap, hv_unit_cap;  // 0: the defaults
  int hv_fw;
};

struct StarSet;
const StarSet* stars_internal(const bt_stars* s);

// Device bytes of the star unit path's scratch of an np-pixel frame with a
// (fw x fw) splat (reserved at the first frame with stars).
size_t map_star_scratch_bytes(size_t np, int fw);

// One frame's inputs.
struct MapFrame {
  const float2* grid;   // map grid GN x GM (rows = GN1 for half grids)
  int GN, GM, gridlvl;
  const float2* view;   // (N+1)(M+1)
  float hor, ver;
  Cam7 cam;
  const EnvMap* env;
  const bt_stars* stars;
  int map, star, lr, step, diffraction;
  const float2* grid2;  // second grid (G = 2 blending) or NULL
  const float2* blend_border;  // bhBorder of the blend
  int blend_angles;
  float alpha;
  int bb_table;         // 0: the reference's 391-entry table, 1: 1024-entry FP32
  int psf_scale;        // diffraction footprint scaled by sqrt(pixel magnification)
  uint8_t* out_bg;      // N*M*4 environment (or final) image
  uint8_t* out;         // N*M*4 final image
  bt_trails* trails;    // star trails between frames, or NULL
  // Set when the environment image is drawn on another stream: compositing
  // onto out_bg waits for it.
  cudaEvent_t bg_ready = nullptr;
};

int map_run_env(MapScratch& S, const MapFrame& F, cudaStream_t s);
// The two parts of map_run_env: the per-pixel corners, shadow mask and
// smoothed solid angles, then the environment image (which reads only those).
int map_run_prep(MapScratch& S, const MapFrame& F, cudaStream_t s);
int map_run_envmap(MapScratch& S, const MapFrame& F, cudaStream_t s);
int blend_prepare(const float2* ga, const float2* gb, int GN, int GM, float2* border,
                  float2* border2, int nang, uint32_t* edge, cudaStream_t s);
int map_run_stars(MapScratch& S, const MapFrame& F, cudaStream_t s);
// addDiffraction of a star-light buffer (N*M*3 floats) into out (stars.cu).
int map_diffract(MapScratch& S, const StarSet& SS, const float* light, float* out,
                 int psf_scale, const float2* view, const float* area, cudaStream_t s);
// Capacities of the star pass's unit path (stars.cu; 0 = the defaults).
int map_set_star_capacity(MapScratch& S, size_t nodes, size_t units);
int map_set_star_slab(MapScratch& S, int pixels);
// The same for a caller's light buffer with a star set's sprite, unscaled.
int map_diffract_light(MapScratch& S, const bt_stars* stars, const float* light, float* out,
                       cudaStream_t s);
StarSet stars_for_frame(const bt_stars* s, int bb_table);
// Star trails of this frame into the trail buffer (trails.cu).
int trails_run(bt_trails* t, MapScratch& Sc, const MapFrame& F, const StarSet& SS,
               cudaStream_t s);
const float* trails_buffer(const bt_trails* t);
// Census of the last frame's environment and star passes (bt_map_census).
int map_env_census(const MapScratch& S, int env_rows, unsigned long long* out, cudaStream_t s);
int map_star_census(const MapScratch& Sc, const MapFrame& F, unsigned long long* out,
                    cudaStream_t s);
int launch_view_sphere(float2* view, int W, int H, cudaStream_t s);
// Summed-area table from a device BGR8 image; sin_t / cos_t: the host's
// sinf / cosf of pxsz * k for k = 0..max(rows, cols) (pxsz = 2 pi / cols),
// pow_t: the host's powf(v, 2.2f) for v = 0..255 (device copies).
int launch_sat(const uint8_t* bgr, int rows, int cols, const float* sin_t, const float* cos_t,
               const float* pow_t, float4* sat, cudaStream_t s);

}  // namespace bt
