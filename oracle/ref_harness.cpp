// ref_harness.cpp -- drives the REFERENCE's own code, compiled in place.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file against the
// reference headers where they lie (BlackTracer2/BlackTracer/ of the reference
// tree) into oracle/_ref/libbtref.so.  No reference source is copied into this
// repository; this file only calls the reference's classes:
//   Camera (BT/Camera.h:27,40), BlackHole (BT/BlackHole.h:7),
//   Grid::integration_wrapper (BT/Grid.h:514), Grid::raytrace (BT/Grid.h:291),
//   Grid::fixTvertices (BT/Grid.h:103), Grid::Grid (BT/Grid.h:605-624),
//   PSHOffsetTable (BT/PSHOffsetTable.h), StarProcessor::makeTree and the
//   cereal archives of Grid and StarProcessor (BT/Grid.h:36-39,
//   BT/StarProcessor.h:21-23; cereal 1.2.2 as vendored with the reference),
//   Viewer::makeCameraView (BT/Viewer.h:109-133).
// It exposes them through a small extern "C" surface that oracle/__init__.py
// loads with ctypes, so the plain-C restatement (oracle/bt_oracle.c) and the
// GPU library can be pinned to the reference's own outputs.
#include <algorithm>
#include <cstdlib>
#include <chrono>
#include <cstdio>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <numeric>
#include <set>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include "opencv2/imgcodecs/imgcodecs.hpp"
#include "opencv2/highgui/highgui.hpp"
#include "opencv2/imgproc/imgproc.hpp"
#include <cereal/archives/binary.hpp>
#include <cereal/types/vector.hpp>
#include <cereal/types/memory.hpp>
#include <cereal/types/unordered_map.hpp>
#include "cuda_runtime.h"
// The grid's work routines are private; the harness needs to call them one by
// one (raytrace, then fixTvertices in a chosen order).
#define private public
#include "Grid.h"
#include "StarProcessor.h"
#include "Viewer.h"
#undef private

// StarProcessor holds an (always empty) cv::Mat; its inline destructor
// references two OpenCV library functions that an empty Mat never calls.  No
// OpenCV library is linked, so the harness supplies stand-ins that stop the
// process if they are ever reached.
namespace cv {
void fastFree(void*) { std::abort(); }
void Mat::deallocate() { std::abort(); }
}  // namespace cv

namespace {

struct NullBuf : std::streambuf {
  int overflow(int c) override { return c; }
};

// Silences the reference's progress printing on std::cout during a call.
struct Quiet {
  NullBuf nb;
  std::streambuf* old;
  Quiet() : old(std::cout.rdbuf(&nb)) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

// Packs/unpacks Camera's public fields (BT/Camera.h:8-11) as 12 doubles.
void cam_to_array(const Camera& c, double* o) {
  double v[12] = {c.theta, c.phi, c.r, c.speed, c.br, c.btheta, c.bphi,
                  c.alpha, c.w, c.wbar, c.Delta, c.ro};
  std::copy(v, v + 12, o);
}
Camera cam_from_array(const double* v) {
  Camera c;
  c.theta = v[0]; c.phi = v[1]; c.r = v[2]; c.speed = v[3]; c.br = v[4];
  c.btheta = v[5]; c.bphi = v[6]; c.alpha = v[7]; c.w = v[8]; c.wbar = v[9];
  c.Delta = v[10]; c.ro = v[11];
  return c;
}

void export_grid(Grid& g, double* theta, double* phi, uint8_t* exists,
                 int32_t* steps, int8_t* blevel) {
  const size_t NM = (size_t)g.N * g.M;
  for (size_t q = 0; q < NM; q++) { theta[q] = -2; phi[q] = -2; }
  std::fill(exists, exists + NM, 0);
  std::fill(blevel, blevel + NM, (int8_t)-1);
  for (auto& e : g.CamToCel) {
    uint32_t i = (uint32_t)(e.first >> 32), j = (uint32_t)e.first;
    size_t id = (size_t)i * g.M + j;
    theta[id] = e.second.x;
    phi[id] = e.second.y;
    exists[id] = 1;
  }
  for (size_t q = 0; q < NM; q++) steps[q] = g.steps[q];
  for (auto& e : g.blockLevels) {
    uint32_t i = (uint32_t)(e.first >> 32), j = (uint32_t)e.first;
    blevel[(size_t)i * g.M + j] = (int8_t)e.second;
  }
}

}  // namespace

extern "C" {

// kind 0: Camera(theta, phi, r, speed)            BT/Camera.h:27
// kind 1: Camera(theta, phi, r, br, btheta, bphi)  BT/Camera.h:40
void btref_camera(int kind, double a, double theta, double phi, double r,
                  double p0, double p1, double p2, double* out12) {
  BlackHole bh(a);
  Camera c = kind == 0 ? Camera(theta, phi, r, p0)
                       : Camera(theta, phi, r, p0, p1, p2);
  cam_to_array(c, out12);
}

// Grid::integration_wrapper over n rays, split into nthreads disjoint slices
// (each slice on its own Grid object; the wrapper only reads the camera and
// the spin globals).
void btref_integrate_rays(const double* cam12, double a, const double* theta,
                          const double* phi, long n, double* theta_out,
                          double* phi_out, int32_t* steps, int nthreads) {
  Quiet q;
  BlackHole bh(a);
  Camera cam = cam_from_array(cam12);
  if (nthreads < 1) nthreads = 1;
  if (n < nthreads * 4) nthreads = 1;
  auto work = [&](long lo, long hi) {
    Grid g;
    g.cam = &cam;
    g.black = &bh;
    int m = (int)(hi - lo);
    std::vector<double> th(theta + lo, theta + hi), ph(phi + lo, phi + hi);
    std::vector<int> st(m);
    g.integration_wrapper(th, ph, m, st);
    for (int k = 0; k < m; k++) {
      theta_out[lo + k] = th[k];
      phi_out[lo + k] = ph[k];
      steps[lo + k] = st[k];
    }
  };
  if (nthreads == 1) { work(0, n); return; }
  std::vector<std::thread> ts;
  for (int t = 0; t < nthreads; t++) {
    long lo = n * t / nthreads, hi = n * (t + 1) / nthreads;
    ts.emplace_back(work, lo, hi);
  }
  for (auto& t : ts) t.join();
}

// Adaptive grid.
//   order 0: raytrace only (no T-vertex fix)
//   order 1: raytrace, then fixTvertices over blockLevels sorted by
//            (level ascending, key ascending)
//   order 2: raytrace, then fixTvertices in the unordered_map's own
//            iteration order, exactly as the constructor does (BT/Grid.h:620)
// Returns the number of CamToCel entries; the hash table of :623 is skipped.
long btref_grid_build(int maxlevel, int startlevel, int angle,
                      const double* cam12, double a, int order, double* theta,
                      double* phi, uint8_t* exists, int32_t* steps,
                      int8_t* blevel) {
  Quiet q;
  BlackHole bh(a);
  Camera cam = cam_from_array(cam12);
  Grid g;
  // Field set-up of Grid::Grid, BT/Grid.h:606-616
  g.MAXLEVEL = maxlevel;
  g.STARTLVL = startlevel;
  g.cam = &cam;
  g.black = &bh;
  g.equafactor = angle ? 1 : 0;
  g.N = (uint32_t)round(pow(2, g.MAXLEVEL) / (2 - g.equafactor) + 1);
  g.STARTN = (uint32_t)round(pow(2, startlevel) / (2 - g.equafactor) + 1);
  g.M = (2 - g.equafactor) * 2 * (g.N - 1);
  g.STARTM = (2 - g.equafactor) * 2 * (g.STARTN - 1);
  g.steps = std::vector<int>(g.M * g.N);
  g.raytrace();
  if (order == 1) {
    std::vector<std::pair<uint64_t, int>> bl(g.blockLevels.begin(),
                                             g.blockLevels.end());
    std::sort(bl.begin(), bl.end(), [](const std::pair<uint64_t, int>& x,
                                       const std::pair<uint64_t, int>& y) {
      return x.second != y.second ? x.second < y.second : x.first < y.first;
    });
    for (auto& b : bl) g.fixTvertices(b);
  } else if (order == 2) {
    for (auto block : g.blockLevels) g.fixTvertices(block);
  }
  export_grid(g, theta, phi, exists, steps, blevel);
  return (long)g.CamToCel.size();
}

// The full reference constructor (incl. the perfect hash), timed: the
// faithful single-thread CPU baseline.  Returns wall seconds; *nrays = number
// of CamToCel entries.
double btref_grid_time(int maxlevel, int startlevel, int angle,
                       const double* cam12, double a, long* nentries) {
  Quiet q;
  BlackHole bh(a);
  Camera cam = cam_from_array(cam12);
  auto t0 = std::chrono::steady_clock::now();
  Grid g(maxlevel, startlevel, angle != 0, &cam, &bh);
  auto t1 = std::chrono::steady_clock::now();
  if (nentries) *nentries = (long)g.CamToCel.size();
  return std::chrono::duration<double>(t1 - t0).count();
}

// StarProcessor::makeTree (BT/StarProcessor.h:172-212) on a star list
// {theta, phi, mag, bv}, with the set-up of the constructor (:263-271).
void btref_star_tree(const float* theta, const float* phi, const float* mag,
                     const float* bv, int n, int treeLevel, float* star_pos,
                     float* star_mag, int* tree) {
  std::vector<std::vector<float>> stars(n);
  for (int k = 0; k < n; k++) stars[k] = {theta[k], phi[k], mag[k], bv[k]};
  StarProcessor sp;
  sp.starSize = n;
  sp.starMag.resize(n * 2);
  sp.starPos.resize(n * 2);
  sp.treeLevel = treeLevel;
  sp.treeSize = (1 << (treeLevel + 1)) - 1;
  sp.binaryStarTree.resize(sp.treeSize);
  float thphi[2] = {0, 0};
  float size[2] = {PI, PI2};
  sp.makeTree(stars, 0, thphi, size, 0);
  std::copy(sp.starPos.begin(), sp.starPos.end(), star_pos);
  std::copy(sp.starMag.begin(), sp.starMag.end(), star_mag);
  std::copy(sp.binaryStarTree.begin(), sp.binaryStarTree.end(), tree);
}

// ---- cache files, through cereal (the reference's own archive code) ----

// The reference's Grid constructor (with its perfect hash, BT/Grid.h:605-624)
// written as BT/BlackTracer.cpp:26-33 writes it.  Returns CamToCel's size.
long btref_grid_file_write(const char* path, int maxlevel, int startlevel, int angle,
                           const double* cam12, double a) {
  Quiet q;
  BlackHole bh(a);
  Camera cam = cam_from_array(cam12);
  Grid g(maxlevel, startlevel, angle != 0, &cam, &bh);
  {
    std::ofstream ofs(path, std::ios::out | std::ios::binary);
    cereal::BinaryOutputArchive oarch(ofs);
    oarch(g);
  }
  return (long)g.CamToCel.size();
}

// A .grid file read as BT/BlackTracer.cpp:236-242 reads it; dims first.
int btref_grid_file_dims(const char* path, int* maxlevel, int* N, int* M, int* hw, int* ow) {
  Grid g;
  std::ifstream ifs(path, std::ios::in | std::ios::binary);
  if (!ifs.good()) return -1;
  {
    cereal::BinaryInputArchive iarch(ifs);
    iarch(g);
  }
  *maxlevel = g.MAXLEVEL;
  *N = g.N;
  *M = g.M;
  *hw = g.hasher.hashTableWidth;
  *ow = g.hasher.offsetTableWidth;
  return 0;
}

// The file's tables as the reference holds them, and every lattice vertex
// looked up with the reference's hash (PSHOffsetTable::hashFunc plus the tag
// test of hashLookup): dense N*M float2, (-2,-2) where absent.
int btref_grid_file_decode(const char* path, float* hash_table, int* offset_table,
                           int* pos_tag, float* dense) {
  Grid g;
  std::ifstream ifs(path, std::ios::in | std::ios::binary);
  if (!ifs.good()) return -1;
  {
    cereal::BinaryInputArchive iarch(ifs);
    iarch(g);
  }
  PSHOffsetTable& h = g.hasher;
  std::copy(h.hashTable.begin(), h.hashTable.end(), hash_table);
  std::copy(h.offsetTable.begin(), h.offsetTable.end(), offset_table);
  std::copy(h.hashPosTag.begin(), h.hashPosTag.end(), pos_tag);
  const int hw = h.hashTableWidth;
  for (int i = 0; i < g.N; i++)
    for (int j = 0; j < g.M; j++) {
      int2 key = {i, j};
      int2 s = h.hashFunc(key);
      const int id = s.x * hw + s.y;
      float* o = dense + 2 * ((size_t)i * g.M + j);
      if (h.hashPosTag[2 * id] != i || h.hashPosTag[2 * id + 1] != j) {
        o[0] = -2.f;
        o[1] = -2.f;
      } else {
        o[0] = h.hashTable[2 * id];
        o[1] = h.hashTable[2 * id + 1];
      }
    }
  return 0;
}

// The reference's PSHOffsetTable built from keys / values (BT/PSHOffsetTable.h
// :350-370); its widths, then its tables.
void btref_psh_build(const int* keys, const float* vals, int n, int* hw, int* ow,
                     float* hash_table, int* offset_table, int* pos_tag, long cap_hash,
                     long cap_offset) {
  Quiet q;
  std::vector<int2> el(n);
  std::vector<float2> dt(n);
  for (int k = 0; k < n; k++) {
    el[k] = {keys[2 * k], keys[2 * k + 1]};
    dt[k] = {vals[2 * k], vals[2 * k + 1]};
  }
  PSHOffsetTable t(el, dt);
  *hw = t.hashTableWidth;
  *ow = t.offsetTableWidth;
  if ((long)t.hashTable.size() <= cap_hash && (long)t.offsetTable.size() <= cap_offset) {
    std::copy(t.hashTable.begin(), t.hashTable.end(), hash_table);
    std::copy(t.offsetTable.begin(), t.offsetTable.end(), offset_table);
    std::copy(t.hashPosTag.begin(), t.hashPosTag.end(), pos_tag);
  }
}

// A StarProcessor with the given tree written / read through cereal
// (BT/BlackTracer.cpp:40-46, :326-331).
void btref_stars_file_write(const char* path, const float* pos, const float* mag, int n,
                            const int* tree, int treeLevel) {
  StarProcessor sp;
  sp.starSize = n;
  sp.treeLevel = treeLevel;
  sp.treeSize = (1 << (treeLevel + 1)) - 1;
  sp.starPos.assign(pos, pos + 2 * n);
  sp.starMag.assign(mag, mag + 2 * n);
  sp.binaryStarTree.assign(tree, tree + sp.treeSize);
  std::ofstream ofs(path, std::ios::out | std::ios::binary);
  cereal::BinaryOutputArchive oarch(ofs);
  oarch(sp);
}

int btref_stars_file_read(const char* path, int* n, int* treeLevel, float* pos, float* mag,
                          int* tree, int cap_n, int cap_tree) {
  StarProcessor sp;
  std::ifstream ifs(path, std::ios::in | std::ios::binary);
  if (!ifs.good()) return -1;
  {
    cereal::BinaryInputArchive iarch(ifs);
    iarch(sp);
  }
  *n = sp.starSize;
  *treeLevel = sp.treeLevel;
  if (sp.starSize <= cap_n && (int)sp.binaryStarTree.size() <= cap_tree) {
    std::copy(sp.starPos.begin(), sp.starPos.end(), pos);
    std::copy(sp.starMag.begin(), sp.starMag.end(), mag);
    std::copy(sp.binaryStarTree.begin(), sp.binaryStarTree.end(), tree);
  }
  return 0;
}

// Viewer(viewangle, offUp, offRight, pixw, pixh, sphere = false): the
// perspective view of BT/Viewer.h:20-33, 109-133.
void btref_view_camera(double angle, double offUp, double offRight, int w, int h, float* out) {
  Quiet q;
  Viewer v(angle, offUp, offRight, w, h, false);
  for (size_t k = 0; k < v.viewMatrix.size(); k++) {
    out[2 * k] = v.viewMatrix[k].x;
    out[2 * k + 1] = v.viewMatrix[k].y;
  }
}

}  // extern "C"
