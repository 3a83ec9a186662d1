// blacktracer.hpp -- C++ host mirror of the reference's hot-path interfaces,
// over the C ABI of blacktracer.h (link with libblacktracer_b200.so and
// libcudart).  Header-only.
//
// Same class names, constructor signatures and meaning as the reference
// (annemiekie/BlackTracer, "BT/" = BlackTracer2/BlackTracer/):
//   BlackHole(afactor)                                 BT/BlackHole.h:7-21
//   Camera(theta, phi, r, speed)                       BT/Camera.h:27-38
//   Camera(theta, phi, r, br, btheta, bphi)            BT/Camera.h:40-52
//   Grid(maxLevelPrec, startLevel, angle, camera, bh)  BT/Grid.h:605-624
//   Viewer(viewangle, offUp, offRight, pixw, pixh, sphere)   BT/Viewer.h:20-33
//   StarProcessor(stars, treeLevel, magnitudeCut)      BT/StarProcessor.h:34-64
//   Distorter(grids, viewer, stars, cams)              BT/Distorter.h:166-176
// Differences, all deliberate:
//   * No OpenCV: celestial points are Point2d {x = theta, y = phi}; images
//     are BGR8 / BGRA8 byte buffers in cv::Mat's channel order.
//   * No image files: the star list and the environment image are passed in
//     memory; Distorter renders into a caller buffer instead of a PNG.  The
//     grid and star cache files are the reference's (Grid::save / load,
//     StarProcessor(file) / save).
//   * Errors throw blacktracer::Error (the reference printed and carried on).
//   * Grid keeps its lattice on the device; CamToCel / steps / blockLevels
//     are host copies made on first access.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "blacktracer.h"

namespace blacktracer {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
  if (rc != BT_OK) throw Error(rc, std::string("blacktracer: ") + bt_last_error());
}

// metric::a / metric::asq (BT/Metric.h:36-39): the spin that Camera
// constructors read, set by BlackHole.
inline double& current_spin() {
  static double a = 0.0;
  return a;
}

class BlackHole {
 public:
  double a;
  explicit BlackHole(double afactor) { setA(afactor); }
  void setA(double afactor) {
    a = afactor;
    current_spin() = afactor;
  }
  double getAngVel(double mass) const { return mass * a; }
};

class Camera {
 public:
  double theta = 0, phi = 0, r = 0;
  double speed = 0, br = 0, btheta = 0, bphi = 0;
  double alpha = 0, w = 0, wbar = 0, Delta = 0, ro = 0;
  double a = 0;  // spin the frame scalars were computed for

  Camera() {}
  Camera(double theCam, double phiCam, double radfactor, double speedCam) {
    a = current_spin();
    bt_camera c;
    check(bt_camera_static(a, theCam, phiCam, radfactor, speedCam, &c));
    from(c);
  }
  Camera(double theCam, double phiCam, double radfactor, double _br,
         double _btheta, double _bphi) {
    a = current_spin();
    bt_camera c;
    check(bt_camera_orbit(a, theCam, phiCam, radfactor, _br, _btheta, _bphi, &c));
    from(c);
  }
  bt_camera raw() const {
    bt_camera c{theta, phi, r, speed, br, btheta, bphi, alpha, w, wbar, Delta, ro};
    return c;
  }
  std::vector<float> getParamArray() const {
    std::vector<float> v(7);
    bt_camera c = raw();
    check(bt_camera_params(&c, v.data()));
    return v;
  }
  double getDistFromBH(float mass) const { return mass * r; }

 private:
  void from(const bt_camera& c) {
    theta = c.theta; phi = c.phi; r = c.r; speed = c.speed; br = c.br;
    btheta = c.btheta; bphi = c.bphi; alpha = c.alpha; w = c.w; wbar = c.wbar;
    Delta = c.Delta; ro = c.ro;
  }
};

// Device memory owned by the mirror classes.
template <class T>
class DeviceArray {
 public:
  DeviceArray() {}
  explicit DeviceArray(size_t n) { resize(n); }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  ~DeviceArray() {
    if (p_) cudaFree(p_);
  }
  void resize(size_t n) {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = n;
    if (n && cudaMalloc((void**)&p_, n * sizeof(T)) != cudaSuccess)
      throw Error(BT_ERR_NOMEM, "device allocation failed");
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }
  void swap(DeviceArray& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
  }

 private:
  T* p_ = nullptr;
  size_t n_ = 0;
};

struct Point2d {
  double x, y;  // theta, phi
};

class Grid {
 public:
  int equafactor = 0, MAXLEVEL = 0, N = 0, M = 0, STARTN = 0, STARTM = 0, STARTLVL = 0;

  Grid() {}
  Grid(int maxLevelPrec, int startLevel, bool angle, const Camera* camera,
       const BlackHole* bh, const bt_integ_opts* opts = nullptr,
       cudaStream_t stream = nullptr)
      : stream_(stream) {
    MAXLEVEL = maxLevelPrec;
    STARTLVL = startLevel;
    equafactor = angle ? 1 : 0;
    int32_t n, m, sn, sm;
    check(bt_grid_dims(MAXLEVEL, equafactor, &n, &m));
    check(bt_grid_dims(STARTLVL, equafactor, &sn, &sm));
    N = n; M = m; STARTN = sn; STARTM = sm;
    check(bt_grid_create(MAXLEVEL, equafactor, &g_));
    bt_camera c = camera->raw();
    const double a = bh ? bh->a : camera->a;
    int rc = bt_grid_build(g_, &c, a, STARTLVL, opts, stream_);
    if (rc == BT_OK) rc = bt_grid_query(g_, &info_, stream_);
    if (rc != BT_OK) {
      bt_grid_destroy(g_);
      g_ = nullptr;
      check(rc);
    }
  }
  Grid(const Grid&) = delete;
  Grid& operator=(const Grid&) = delete;
  Grid(Grid&& o) noexcept { *this = std::move(o); }
  Grid& operator=(Grid&& o) noexcept {
    std::swap(g_, o.g_);
    std::swap(stream_, o.stream_);
    std::swap(info_, o.info_);
    equafactor = o.equafactor; MAXLEVEL = o.MAXLEVEL; N = o.N; M = o.M;
    STARTN = o.STARTN; STARTM = o.STARTM; STARTLVL = o.STARTLVL;
    cam_to_cel_.swap(o.cam_to_cel_);
    block_levels_.swap(o.block_levels_);
    steps_.swap(o.steps_);
    exported_ = o.exported_;
    file_map_.swap(o.file_map_);
    std::swap(file_rows_, o.file_rows_);
    std::swap(file_cols_, o.file_cols_);
    return *this;
  }

  // write(filename, grid), BT/BlackTracer.cpp:26-33: the reference's .grid
  // cache file (MAXLEVEL, N, M and the vertices' perfect spatial hash).
  void save(const std::string& path) {
    if (!g_) throw Error(BT_ERR_STATE, "a grid loaded from a file is already a file");
    check(bt_grid_save(g_, path.c_str(), stream_));
  }

  // The cereal load of BT/BlackTracer.cpp:236-242.  Like the reference's
  // loaded Grid it holds MAXLEVEL, N and M and renders, but its CamToCel,
  // steps and blockLevels are empty (they are not in the file).
  static Grid load(const std::string& path, cudaStream_t stream = nullptr) {
    Grid g;
    g.stream_ = stream;
    int32_t ml = 0, rows = 0, cols = 0, sym = 0;
    check(bt_grid_file_map_shape(path.c_str(), &ml, &rows, &cols, &sym));
    g.MAXLEVEL = ml;
    g.M = cols;
    g.N = sym ? (rows + 1) / 2 : rows;
    g.equafactor = sym ? 0 : 1;
    g.file_map_.resize((size_t)2 * rows * cols);
    g.file_rows_ = rows;
    g.file_cols_ = cols;
    check(bt_grid_file_load_map(path.c_str(), g.file_map_.get(), rows, cols, stream));
    g.exported_ = true;
    return g;
  }

  // The float2 map grid the renderer reads (makeGrid's output).
  void mapGrid(const float** grid, int32_t* rows, int32_t* cols) const {
    if (!g_) {
      *grid = file_map_.get();
      *rows = file_rows_;
      *cols = file_cols_;
      return;
    }
    int32_t sym = 0;
    check(bt_grid_map_export(g_, grid, rows, cols, &sym, stream_));
  }
  ~Grid() {
    if (g_) bt_grid_destroy(g_);
  }

  bt_grid* handle() const { return g_; }
  const bt_grid_info& info() const { return info_; }
  int64_t traced() const { return info_.traced; }

  // Build this grid again for another camera at the same MAXLEVEL, start level
  // and view, reusing its device buffers and its tuned trace configuration.
  // The reference makes a new Grid per camera (BT/BlackTracer.cpp:252); this
  // gives the same grid without the allocations.  Host copies (CamToCel,
  // steps, blockLevels) are taken again on their next use.
  void rebuild(const Camera* camera, const BlackHole* bh = nullptr,
               const bt_integ_opts* opts = nullptr) {
    if (!g_) throw Error(BT_ERR_STATE, "a grid loaded from a file cannot be built");
    bt_camera c = camera->raw();
    const double a = bh ? bh->a : camera->a;
    check(bt_grid_build(g_, &c, a, STARTLVL, opts, stream_));
    check(bt_grid_query(g_, &info_, stream_));
    exported_ = false;
    cam_to_cel_.clear();
    block_levels_.clear();
    steps_.clear();
  }

  // The autotuner on this grid's last build (bt_grid_tune): later builds and
  // rebuild() use the fastest trace shape, refill size and build form found.
  // For the MIXED form it also picks fp64_band for p99_target_rad; pass the
  // result's fp64_band in the options of later MIXED builds.
  bt_tune_result tune(const bt_integ_opts* opts = nullptr, double p99_target_rad = 1e-6,
                      int repeats = 2) {
    if (!g_) throw Error(BT_ERR_STATE, "a grid loaded from a file cannot be tuned");
    bt_tune_result r;
    std::memset(&r, 0, sizeof(r));
    check(bt_grid_tune(g_, opts, p99_target_rad, repeats, &r, stream_));
    return r;
  }

  // CUDA-graph replay of the level builds (bt_grid_set_graph) and the
  // one-launch build at blocksPerSm blocks per SM, 0 for off (bt_grid_set_flow).
  void setGraph(bool on) {
    if (!g_) throw Error(BT_ERR_STATE, "a grid loaded from a file is not built");
    check(bt_grid_set_graph(g_, on ? 1 : 0));
  }
  void setFlow(int blocksPerSm) {
    if (!g_) throw Error(BT_ERR_STATE, "a grid loaded from a file is not built");
    check(bt_grid_set_flow(g_, blocksPerSm));
  }

  // BT/Grid.h:575, 577, 588 -- host copies, keyed i<<32|j like the reference.
  const std::unordered_map<uint64_t, Point2d>& CamToCel() { exportHost(); return cam_to_cel_; }
  const std::vector<int>& steps() { exportHost(); return steps_; }
  const std::unordered_map<uint64_t, int>& blockLevels() { exportHost(); return block_levels_; }

 private:
  void exportHost() {
    if (exported_) return;
    const size_t cap = (size_t)info_.traced + 2 * (size_t)M + 16;
    std::vector<uint32_t> vi(cap), vj(cap), bi(cap), bj(cap);
    std::vector<double> th(cap), ph(cap);
    std::vector<int32_t> st(cap);
    std::vector<int8_t> lv(cap);
    bt_grid_export_t e;
    std::memset(&e, 0, sizeof(e));
    e.vi = vi.data(); e.vj = vj.data(); e.theta = th.data(); e.phi = ph.data();
    e.steps = st.data(); e.cap_vertices = cap;
    e.bi = bi.data(); e.bj = bj.data(); e.level = lv.data(); e.cap_blocks = cap;
    check(bt_grid_export(g_, &e, stream_));
    if (cudaStreamSynchronize(stream_) != cudaSuccess) throw Error(BT_ERR_CUDA, "sync failed");
    steps_.assign((size_t)M * N, 0);
    cam_to_cel_.reserve(e.n_vertices);
    for (size_t k = 0; k < e.n_vertices; k++) {
      const uint64_t key = (uint64_t)vi[k] << 32 | vj[k];
      cam_to_cel_[key] = Point2d{th[k], ph[k]};
      steps_[(size_t)vi[k] * M + vj[k]] = st[k];
    }
    for (size_t k = 0; k < e.n_blocks; k++)
      block_levels_[(uint64_t)bi[k] << 32 | bj[k]] = lv[k];
    exported_ = true;
  }

  bt_grid* g_ = nullptr;
  cudaStream_t stream_ = nullptr;
  bt_grid_info info_{};
  std::unordered_map<uint64_t, Point2d> cam_to_cel_;
  std::unordered_map<uint64_t, int> block_levels_;
  std::vector<int> steps_;
  bool exported_ = false;
  DeviceArray<float> file_map_;  // a grid loaded from a file
  int32_t file_rows_ = 0, file_cols_ = 0;
};

class Viewer {
 public:
  DeviceArray<float> viewMatrix;  // (pixh+1)*(pixw+1) (theta, phi) pairs
  double viewAngleUp = 0, viewAngleWide = 0;
  int pixelwidth = 0, pixelheight = 0;

  Viewer(double viewangle, double offUp, double offRight, int pixw, int pixh,
         bool sphere, cudaStream_t stream = nullptr) {
    pixelwidth = pixw;
    pixelheight = pixh;
    viewMatrix.resize((size_t)2 * (pixh + 1) * (pixw + 1));
    if (sphere) {
      check(bt_view_sphere(viewMatrix.get(), pixw, pixh, stream));
    } else {  // makeCameraView(offUp, offRight), BT/Viewer.h:109-133
      viewAngleWide = viewangle;
      viewAngleUp = 1. * pixh * viewAngleWide / (1. * pixw);
      check(bt_view_camera(viewMatrix.get(), pixw, pixh, viewangle, offUp, offRight, stream));
    }
  }
};

// One star of the input list: theta = pi/2 - dec, phi = ra (already wrapped,
// as readStars2 leaves them), magnitude, B-V colour index.
struct Star {
  float theta, phi, mag, bv;
};

class StarProcessor {
 public:
  std::vector<int> binaryStarTree;
  std::vector<float> starPos;
  std::vector<float> starMag;
  int starSize = 0;
  int treeSize = 0;
  int treeLevel = 0;

  StarProcessor(const std::vector<Star>& stars, int _treeLevel, float magnitudeCut,
                const uint8_t* psf_rgb = nullptr, int psf_size = 0,
                cudaStream_t stream = nullptr) {
    treeLevel = _treeLevel;
    treeSize = bt_stars_tree_size(treeLevel);
    const int n = (int)stars.size();
    std::vector<float> th(n), ph(n), mg(n), bv(n);
    for (int k = 0; k < n; k++) {
      th[k] = stars[k].theta; ph[k] = stars[k].phi; mg[k] = stars[k].mag; bv[k] = stars[k].bv;
    }
    starPos.resize((size_t)2 * n);
    starMag.resize((size_t)2 * n);
    binaryStarTree.resize(treeSize);
    check(bt_stars_build_tree(th.data(), ph.data(), mg.data(), bv.data(), n, treeLevel,
                              magnitudeCut, starPos.data(), starMag.data(),
                              binaryStarTree.data(), &starSize));
    starPos.resize((size_t)2 * starSize);
    starMag.resize((size_t)2 * starSize);
    check(bt_stars_create(starPos.data(), starMag.data(), starSize, binaryStarTree.data(),
                          treeLevel, psf_rgb, psf_size, &s_, stream));
  }
  // The cereal load of a star cache file (BT/BlackTracer.cpp:326-331).
  explicit StarProcessor(const std::string& starFile, const uint8_t* psf_rgb = nullptr,
                         int psf_size = 0, cudaStream_t stream = nullptr) {
    check(bt_stars_file_info(starFile.c_str(), &starSize, &treeLevel));
    treeSize = bt_stars_tree_size(treeLevel);
    starPos.resize((size_t)2 * starSize);
    starMag.resize((size_t)2 * starSize);
    binaryStarTree.resize(treeSize);
    check(bt_stars_file_read(starFile.c_str(), starPos.data(), starMag.data(), starSize,
                             binaryStarTree.data(), treeSize));
    check(bt_stars_create(starPos.data(), starMag.data(), starSize, binaryStarTree.data(),
                          treeLevel, psf_rgb, psf_size, &s_, stream));
  }
  // writeStars, BT/BlackTracer.cpp:40-46.
  void save(const std::string& path) const {
    check(bt_stars_file_write(path.c_str(), starPos.data(), starMag.data(), starSize,
                              binaryStarTree.data(), treeLevel));
  }
  StarProcessor(const StarProcessor&) = delete;
  StarProcessor& operator=(const StarProcessor&) = delete;
  ~StarProcessor() {
    if (s_) bt_stars_destroy(s_);
  }
  const bt_stars* handle() const { return s_; }

 private:
  bt_stars* s_ = nullptr;
};

// Distorter (BT/Distorter.h:166) + makeImage (BT/MakeImageKernel.cu:1206):
// renders grids[0] through the viewer with the stars and the environment.
class Distorter {
 public:
  bool star = true, map = true, lr = true, diffraction = false;
  bool trails = false;  // star trails from the previous frame (addTrails)
  int step = 1;

  Distorter(std::vector<Grid>* grids, Viewer* viewer, StarProcessor* stars,
            std::vector<Camera>* cams, const uint8_t* env_bgr, int env_rows,
            int env_cols, cudaStream_t stream = nullptr)
      : grids_(grids), view_(viewer), stars_(stars), cams_(cams), stream_(stream) {
    if (grids->empty() || cams->size() != grids->size())
      throw Error(BT_ERR_ARG, "one camera per grid is needed");
    check(bt_map_create(viewer->pixelwidth, viewer->pixelheight, &m_));
    if (grids->size() > 1) {
      int rc = bt_blend_create(&blend_);
      if (rc) {
        bt_map_destroy(m_);
        m_ = nullptr;
        check(rc);
      }
    }
    if (env_bgr) {
      int rc = bt_env_create(env_bgr, env_rows, env_cols, 0, &env_, stream_);
      if (rc) {
        bt_map_destroy(m_);
        m_ = nullptr;
        check(rc);
      }
    }
  }
  Distorter(const Distorter&) = delete;
  Distorter& operator=(const Distorter&) = delete;
  ~Distorter() {
    if (trails_) bt_trails_destroy(trails_);
    if (blend_) bt_blend_destroy(blend_);
    if (env_) bt_env_destroy(env_);
    if (m_) bt_map_destroy(m_);
  }

  // One frame into a device BGRA8 buffer of width*height*4 bytes.  hor / ver
  // are the look-around offsets the reference's arrow keys change
  // (BT/MakeImageKernel.cu:1081-1102).  With several grids, prec selects the
  // pair blended as the reference's '=' / '-' keys do (:990-1008): grids
  // (int)p and (int)p + 1 with weight fmod(p, 1) of the second, p = fmod(prec,
  // G - 1).
  void renderDevice(uint8_t* out_bgra, float hor = 0.f, float ver = 0.f, float prec = 0.f) {
    const int G = (int)grids_->size();
    int gnr = 0;
    float alpha = 0.f;
    if (G > 1) {
      const float p = std::fmod(prec, (float)G - 1.f);
      alpha = std::fmod(p, 1.f);
      gnr = (int)p;
      if (gnr < 0 || gnr > G - 2) throw Error(BT_ERR_ARG, "prec must not be negative");
    }
    Grid& g = (*grids_)[gnr];
    const float* grid = nullptr;
    int32_t rows = 0, cols = 0;
    g.mapGrid(&grid, &rows, &cols);
    bt_frame f;
    std::memset(&f, 0, sizeof(f));
    f.grid = grid;
    f.grid_rows = rows;
    f.grid_cols = cols;
    f.grid_level = g.MAXLEVEL;
    f.view = view_->viewMatrix.get();
    f.hor = hor;
    f.ver = ver;
    const std::vector<float> c = (*cams_)[gnr].getParamArray();
    for (int q = 0; q < 7; q++) f.cam[q] = c[q];
    f.env = env_;
    f.stars = stars_ ? stars_->handle() : nullptr;
    f.map = map && env_ ? 1 : 0;
    f.star = star && stars_ ? 1 : 0;
    f.lr = lr ? 1 : 0;
    f.step = step;
    f.diffraction = diffraction ? 1 : 0;
    f.out = out_bgra;
    if (trails && f.star) {
      if (!trails_)
        check(bt_trails_create(stars_->starSize, view_->pixelwidth, view_->pixelheight, 30, 0,
                               &trails_));
      f.trails = trails_;
    }
    if (G > 1) {
      const float* grid2 = nullptr;
      int32_t rows2 = 0, cols2 = 0;
      (*grids_)[gnr + 1].mapGrid(&grid2, &rows2, &cols2);
      if (rows2 != rows || cols2 != cols) throw Error(BT_ERR_ARG, "grids of different shapes");
      if (gnr != prepared_) {  // findBhCenter / findBhBorders / smoothBorder
        check(bt_blend_prepare(blend_, grid, grid2, rows, cols, stream_));
        prepared_ = gnr;
      }
      const std::vector<float> c2 = (*cams_)[gnr + 1].getParamArray();
      for (int q = 0; q < 7; q++) f.cam2[q] = c2[q];
      f.grid2 = grid2;
      f.alpha = alpha;
      f.blend = blend_;
    }
    check(bt_map_render(m_, &f, stream_));
  }

  // One frame into a host BGRA8 buffer (the reference wrote it to a PNG).
  void render(uint8_t* host_bgra, float hor = 0.f, float ver = 0.f, float prec = 0.f) {
    const size_t bytes = (size_t)view_->pixelwidth * view_->pixelheight * 4;
    if (out_.size() != bytes) out_.resize(bytes);
    renderDevice(out_.get(), hor, ver, prec);
    if (cudaMemcpyAsync(host_bgra, out_.get(), bytes, cudaMemcpyDeviceToHost, stream_) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
      throw Error(BT_ERR_CUDA, "frame download failed");
  }

 private:
  std::vector<Grid>* grids_;
  Viewer* view_;
  StarProcessor* stars_;
  std::vector<Camera>* cams_;
  cudaStream_t stream_;
  bt_map* m_ = nullptr;
  bt_env* env_ = nullptr;
  bt_blend* blend_ = nullptr;
  bt_trails* trails_ = nullptr;
  int prepared_ = -1;  // grid pair the blend was prepared for
  DeviceArray<uint8_t> out_;
};

}  // namespace blacktracer
