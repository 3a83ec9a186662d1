// map_api.cu -- C ABI of the per-pixel map: resident environment maps,
// renderers (per-resolution scratch) and the frame call that replaces
// makeImage / cudaPrep (annemiekie/BlackTracer BT/MakeImageKernel.cu:1206-1559).
#include <cstring>
#include <new>
#include <vector>
#include <cmath>

#include "bt_internal.h"
#include "map_internal.h"

struct bt_env {
  bt::EnvMap e;
};

struct bt_blend {
  float2* border;   // 2 + 2 * nang: the box, then (grid a, grid b) per direction
  float2* border2;
  uint32_t* edge;
  uint32_t* edge_host;
  int nang;
  int rows, cols;
  int ready;
};

struct bt_map {
  bt::MapScratch S;
  uint8_t* tmp_img;  // env image when stars are composited on top
  // The environment image of a frame with stars is drawn on a second stream
  // (the caller's priority) while the star passes run: it needs only the
  // pixel set-up and the stars need it only when compositing.
  cudaStream_t side;
  int side_prio;
  cudaEvent_t ev_prep, ev_bg;
};

using namespace bt;

namespace {

void map_free(bt_map* m) {
  void* ptrs[] = {m->S.thphi, m->S.gap,   m->S.bh,        m->S.area,
                  m->S.area_tmp, m->S.light, m->S.light2, m->S.stars_img,
                  m->S.flag, m->S.cells, m->S.diff_list, m->S.diff_count,
                  m->S.heavy_list, m->S.heavy_order, m->S.heavy_count, m->S.env_wide,
                  m->S.env_wide_count, m->tmp_img, m->S.hv_nn, m->S.hv_nl, m->S.hv_noff,
                  m->S.hv_uoff, m->S.hv_pool, m->S.hv_pend, m->S.hv_partial, m->S.hv_uany,
                  m->S.hv_ctl, m->S.hv_slab};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (m->side) {
    cudaStreamSynchronize(m->side);
    cudaStreamDestroy(m->side);
  }
  if (m->ev_prep) cudaEventDestroy(m->ev_prep);
  if (m->ev_bg) cudaEventDestroy(m->ev_bg);
}

// The side stream at the priority of the caller's stream s.
int side_stream(bt_map* m, cudaStream_t s) {
  int prio = 0;
  BT_CUDA_TRY(cudaStreamGetPriority(s, &prio));
  if (m->side && prio == m->side_prio) return BT_OK;
  if (m->side) {
    BT_CUDA_TRY(cudaStreamSynchronize(m->side));
    BT_CUDA_TRY(cudaStreamDestroy(m->side));
    m->side = nullptr;
  }
  BT_CUDA_TRY(cudaStreamCreateWithPriority(&m->side, cudaStreamNonBlocking, prio));
  m->side_prio = prio;
  return BT_OK;
}

}  // namespace

namespace {
// The frame description of bt_frame for the map passes.
MapFrame frame_of(const bt_frame* f) {
  MapFrame F;
  F.grid = (const float2*)f->grid;
  F.GN = f->grid_rows;
  F.GM = f->grid_cols;
  F.gridlvl = f->grid_level;
  F.view = (const float2*)f->view;
  F.hor = f->hor;
  F.ver = f->ver;
  for (int q = 0; q < 7; q++) F.cam.v[q] = f->cam[q];
  F.env = f->env ? &f->env->e : nullptr;
  F.stars = f->stars;
  F.bb_table = f->bb_table;
  F.psf_scale = f->psf_scale;
  F.grid2 = (const float2*)f->grid2;
  F.blend_border = nullptr;
  F.blend_angles = 0;
  F.alpha = f->alpha;
  if (f->grid2) {
    // camUpdate (BT/MakeImageKernel.cu:386-389): the camera between the two
    for (int q = 0; q < 7; q++) F.cam.v[q] = (1.f - f->alpha) * f->cam[q] + f->alpha * f->cam2[q];
    F.blend_border = f->blend->border;
    F.blend_angles = f->blend->nang;
  }
  F.map = f->map;
  F.star = f->star;
  F.lr = f->lr;
  F.step = f->step;
  F.diffraction = f->diffraction;
  F.out = f->out;
  F.trails = f->trails;
  return F;
}
}  // namespace

extern "C" {

int bt_env_create(const uint8_t* bgr, int rows, int cols, int bgr_on_device,
                  bt_env** out, void* stream) {
  clear_error();
  BT_ARG_CHECK(out && bgr, "NULL pointer");
  BT_ARG_CHECK(rows > 0 && cols > 0 && (size_t)rows * cols <= ((size_t)1 << 31),
               "environment size out of range");
  *out = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  bt_env* e = new (std::nothrow) bt_env;
  if (!e) return BT_ERR_NOMEM;
  e->e.rows = rows;
  e->e.cols = cols;
  e->e.sat = nullptr;
  const size_t n = (size_t)rows * cols;
  cudaError_t err = cudaMalloc((void**)&e->e.sat, n * sizeof(float4));
  if (err != cudaSuccess) {
    delete e;
    set_error("summed-area table allocation failed: %s", cudaGetErrorString(err));
    return BT_ERR_NOMEM;
  }
  // The host's sinf / cosf of the grid angles and powf of the byte values
  // (the reference computes the table on the host: its values are those).
  const int kmax = rows > cols ? rows : cols;
  const float pxsz = kPi2F / (1.f * cols);
  std::vector<float> tabs((size_t)2 * (kmax + 1) + 256);
  for (int k = 0; k <= kmax; k++) {
    tabs[k] = sinf(pxsz * k);
    tabs[(size_t)kmax + 1 + k] = cosf(pxsz * k);
  }
  for (int v = 0; v < 256; v++) tabs[(size_t)2 * (kmax + 1) + v] = powf((float)v, 2.2f);
  const uint8_t* src = bgr;
  uint8_t* staged = nullptr;
  float* dtabs = nullptr;
  err = cudaMalloc((void**)&dtabs, tabs.size() * sizeof(float));
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(dtabs, tabs.data(), tabs.size() * sizeof(float),
                          cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess && !bgr_on_device) {
    err = cudaMalloc((void**)&staged, n * 3);
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(staged, bgr, n * 3, cudaMemcpyHostToDevice, s);
    src = staged;
  }
  if (err != cudaSuccess) {
    if (staged) cudaFree(staged);
    if (dtabs) cudaFree(dtabs);
    cudaFree(e->e.sat);
    delete e;
    set_error("environment upload failed: %s", cudaGetErrorString(err));
    return BT_ERR_CUDA;
  }
  int rc = launch_sat(src, rows, cols, dtabs, dtabs + kmax + 1, dtabs + 2 * (kmax + 1),
                      e->e.sat, s);
  // the host tables and staging must outlive the copies and the kernels
  cudaStreamSynchronize(s);
  if (staged) cudaFree(staged);
  cudaFree(dtabs);
  if (rc) {
    cudaFree(e->e.sat);
    delete e;
    return rc;
  }
  *out = e;
  return BT_OK;
}

void bt_env_destroy(bt_env* e) {
  if (!e) return;
  if (e->e.sat) cudaFree(e->e.sat);
  delete e;
}

int bt_env_sat(const bt_env* e, const float** sat, int32_t* rows, int32_t* cols) {
  BT_ARG_CHECK(e && sat, "NULL pointer");
  *sat = (const float*)e->e.sat;
  if (rows) *rows = e->e.rows;
  if (cols) *cols = e->e.cols;
  return BT_OK;
}

int bt_blend_create(bt_blend** out) {
  clear_error();
  BT_ARG_CHECK(out != nullptr, "NULL pointer");
  *out = nullptr;
  bt_blend* b = new (std::nothrow) bt_blend;
  if (!b) return BT_ERR_NOMEM;
  std::memset(b, 0, sizeof(*b));
  b->nang = 1000;  // angleNum, BT/MakeImageKernel.cu:1257
  const size_t bytes = (size_t)(2 + 2 * b->nang) * sizeof(float2);
  cudaError_t e = cudaMalloc((void**)&b->border, bytes);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->border2, bytes);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->edge, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&b->edge_host, sizeof(uint32_t));
  if (e != cudaSuccess) {
    cudaFree(b->border); cudaFree(b->border2); cudaFree(b->edge);
    delete b;
    set_error("blend allocation failed: %s", cudaGetErrorString(e));
    return BT_ERR_NOMEM;
  }
  *out = b;
  return BT_OK;
}

void bt_blend_destroy(bt_blend* b) {
  if (!b) return;
  cudaFree(b->border);
  cudaFree(b->border2);
  cudaFree(b->edge);
  if (b->edge_host) cudaFreeHost(b->edge_host);
  delete b;
}

int bt_blend_prepare(bt_blend* b, const float* grid_a, const float* grid_b, int rows, int cols,
                     void* stream) {
  clear_error();
  BT_ARG_CHECK(b && grid_a && grid_b, "NULL pointer");
  BT_ARG_CHECK(rows > 1 && cols > 1, "invalid grid shape");
  cudaStream_t s = (cudaStream_t)stream;
  if (int rc = blend_prepare((const float2*)grid_a, (const float2*)grid_b, rows, cols,
                             b->border, b->border2, b->nang, b->edge, s))
    return rc;
  BT_CUDA_TRY(cudaMemcpyAsync(b->edge_host, b->edge, sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, s));
  b->rows = rows;
  b->cols = cols;
  b->ready = 1;
  return BT_OK;
}

int bt_blend_info(const bt_blend* b, const float** border, int32_t* angles,
                  uint32_t* walks_at_edge) {
  BT_ARG_CHECK(b != nullptr, "NULL pointer");
  if (border) *border = (const float*)b->border;
  if (angles) *angles = b->nang;
  if (walks_at_edge) *walks_at_edge = b->edge_host ? *b->edge_host : 0;
  return BT_OK;
}

int bt_map_create(int width, int height, bt_map** out) {
  clear_error();
  BT_ARG_CHECK(out != nullptr, "NULL pointer");
  BT_ARG_CHECK(width > 0 && height > 0 && (size_t)width * height <= ((size_t)1 << 28),
               "image size out of range");
  *out = nullptr;
  bt_map* m = new (std::nothrow) bt_map;
  if (!m) return BT_ERR_NOMEM;
  std::memset(m, 0, sizeof(*m));
  MapScratch& S = m->S;
  S.M = width;
  S.N = height;
  S.hv_slab_req = -1;  // the default slab for the frame size
  const size_t np = (size_t)width * height;
  const size_t nc = (size_t)(width + 1) * (height + 1);
  cudaError_t e = cudaSuccess;
#define MALLOC(p, bytes) \
  if (e == cudaSuccess) e = cudaMalloc((void**)&(p), (bytes));
  MALLOC(S.thphi, nc * sizeof(float2));
  MALLOC(S.gap, nc * sizeof(int));
  MALLOC(S.bh, np);
  MALLOC(S.area, np * sizeof(float));
  MALLOC(S.area_tmp, np * sizeof(float));
  MALLOC(S.light, np * 3 * sizeof(float));
  MALLOC(S.light2, np * 3 * sizeof(float));
  MALLOC(S.stars_img, np * 4);
  MALLOC(S.flag, np);
  MALLOC(S.diff_list, np * sizeof(uint32_t));
  MALLOC(S.diff_count, sizeof(uint32_t));
  MALLOC(S.heavy_list, np * sizeof(uint32_t));
  MALLOC(S.heavy_order, np * sizeof(uint32_t));
  MALLOC(S.env_wide, np * sizeof(uint32_t));
  MALLOC(S.env_wide_count, sizeof(uint32_t));
  MALLOC(S.heavy_count, 4 * sizeof(uint32_t));
  MALLOC(m->tmp_img, np * 4);
#undef MALLOC
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->ev_prep, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->ev_bg, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    map_free(m);
    delete m;
    set_error("renderer allocation (%dx%d) failed: %s", width, height,
              cudaGetErrorString(e));
    return BT_ERR_NOMEM;
  }
  *out = m;
  return BT_OK;
}

void bt_map_destroy(bt_map* m) {
  if (!m) return;
  map_free(m);
  delete m;
}

int bt_view_sphere(float* view, int width, int height, void* stream) {
  clear_error();
  BT_ARG_CHECK(view && width > 0 && height > 0, "invalid view arguments");
  return launch_view_sphere((float2*)view, width, height, (cudaStream_t)stream);
}

int bt_map_render(bt_map* m, const bt_frame* f, void* stream) {
  clear_error();
  BT_ARG_CHECK(m && f, "NULL pointer");
  BT_ARG_CHECK(f->grid && f->view && f->out, "grid, view and out are required");
  BT_ARG_CHECK(f->grid_rows > 1 && f->grid_cols > 1 && f->grid_level >= 1,
               "invalid grid description");
  BT_ARG_CHECK(!f->map || f->env, "map requested without an environment");
  BT_ARG_CHECK(!f->star || f->stars, "stars requested without a star set");
  BT_ARG_CHECK(f->step >= 0 && f->step <= 2, "step out of [0, 2]");
  BT_ARG_CHECK(f->bb_table == 0 || f->bb_table == 1, "bb_table must be 0 or 1");
  BT_ARG_CHECK(!f->grid2 || (f->blend && f->blend->ready && f->blend->rows == f->grid_rows &&
                             f->blend->cols == f->grid_cols),
               "a second grid needs a blend prepared on grids of the same shape");
  cudaStream_t s = (cudaStream_t)stream;
  MapFrame F = frame_of(f);
  // environment into the output directly, or into a temporary when stars
  // are composited on top (addStarsAndBackground)
  F.out_bg = (f->star && f->map) ? m->tmp_img : f->out;
  if (f->star && f->map) {
    if (int rc = side_stream(m, s)) return rc;
    if (int rc = map_run_prep(m->S, F, s)) return rc;
    BT_CUDA_TRY(cudaEventRecord(m->ev_prep, s));
    BT_CUDA_TRY(cudaStreamWaitEvent(m->side, m->ev_prep, 0));
    if (int rc = map_run_envmap(m->S, F, m->side)) return rc;
    BT_CUDA_TRY(cudaEventRecord(m->ev_bg, m->side));
    F.bg_ready = m->ev_bg;
    const int rc = map_run_stars(m->S, F, s);
    if (rc) cudaStreamWaitEvent(s, m->ev_bg, 0);  // the caller's stream still joins
    return rc;
  }
  int rc = map_run_env(m->S, F, s);
  if (rc) return rc;
  if (f->star) {
    rc = map_run_stars(m->S, F, s);
    if (rc) return rc;
  }
  return BT_OK;
}

int bt_map_set_star_capacity(bt_map* m, size_t nodes, size_t units) {
  clear_error();
  BT_ARG_CHECK(m != nullptr, "NULL renderer");
  BT_ARG_CHECK(units == 0 || units >= 2, "units must be 0 (default) or at least 2");
  BT_ARG_CHECK(nodes <= 0xffffffffu && units <= 0xffffffffu, "capacity above 2^32 - 1");
  return map_set_star_capacity(m->S, nodes, units);
}

int bt_map_set_star_slab(bt_map* m, int pixels) {
  clear_error();
  BT_ARG_CHECK(m != nullptr, "NULL renderer");
  BT_ARG_CHECK(pixels <= 32768, "slab above 32768 pixels");
  return map_set_star_slab(m->S, pixels);
}

int bt_map_diffract(bt_map* m, const bt_stars* stars, const float* light, float* out,
                    void* stream) {
  clear_error();
  BT_ARG_CHECK(m && stars && light && out, "NULL pointer");
  BT_ARG_CHECK(light != out, "light and out must be different buffers");
  return map_diffract_light(m->S, stars, light, out, (cudaStream_t)stream);
}

int bt_map_census(bt_map* m, const bt_frame* f, bt_map_census_t* out, void* stream) {
  clear_error();
  BT_ARG_CHECK(m && f && out, "NULL pointer");
  BT_ARG_CHECK(f->view && (!f->map || f->env) && (!f->star || f->stars),
               "the frame description of the last render is needed");
  cudaStream_t s = (cudaStream_t)stream;
  const MapFrame F = frame_of(f);
  unsigned long long* dev = nullptr;
  BT_CUDA_TRY(cudaMallocAsync((void**)&dev, 8 * sizeof(unsigned long long), s));
  unsigned long long host[8] = {0};
  cudaError_t e = cudaMemsetAsync(dev, 0, 8 * sizeof(unsigned long long), s);
  // out[0..1]: environment; out[2..7]: stars
  int rc = BT_OK;
  if (e == cudaSuccess && f->map) rc = map_env_census(m->S, f->env->e.rows, dev, s);
  if (e == cudaSuccess && rc == BT_OK && f->star) rc = map_star_census(m->S, F, dev + 2, s);
  if (e == cudaSuccess && rc == BT_OK)
    e = cudaMemcpyAsync(host, dev, sizeof(host), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(dev, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_error("census: %s", cudaGetErrorString(e));
    return BT_ERR_CUDA;
  }
  if (rc) return rc;
  out->env_columns = host[0];
  out->env_pixels = host[1];
  out->star_pixels = host[2];
  out->star_candidates_ref = host[3];
  out->star_candidates = host[4];
  out->star_hits = host[5];
  out->heavy_candidates = host[6];
  out->heavy_hits = host[7];
  return BT_OK;
}

int bt_map_scratch(const bt_map* m, bt_map_buffers* b) {
  BT_ARG_CHECK(m && b, "NULL pointer");
  b->thphi = (const float*)m->S.thphi;
  b->gap = m->S.gap;
  b->bh = m->S.bh;
  b->area = m->S.area;
  b->light = m->S.light;
  b->stars_img = m->S.stars_img;
  b->env_img = m->tmp_img;
  b->light_diffracted = m->S.light2;
  return BT_OK;
}

}  // extern "C"
