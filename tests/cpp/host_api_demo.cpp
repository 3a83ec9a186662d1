// Drives the C++ host mirror (include/blacktracer.hpp) the way the
// reference's main() drives its classes (BT/BlackTracer.cpp:192-343), and
// prints results for tests/test_cpp_host.py to check against the oracle.
//   host_api_demo camera           (no GPU needed)
//   host_api_demo grid             (GPU)
//   host_api_demo frame            (GPU)
//   host_api_demo files <dir>      (GPU: cache files, perspective view, G = 2)
//   host_api_demo rebuild          (GPU: tune, graph replay, rebuild vs new Grid)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "blacktracer.hpp"

using namespace blacktracer;

int main(int argc, char** argv) {
  const char* mode = argc > 1 ? argv[1] : "camera";
  BlackHole black(0.999);
  Camera cam(M_PI / 2, 0.0, 5.0, 0.0, 0.0, 1.0);
  if (!std::strcmp(mode, "camera")) {
    printf("%.17g %.17g %.17g %.17g %.17g %.17g\n", cam.speed, cam.alpha, cam.w, cam.wbar,
           cam.Delta, cam.ro);
    BlackHole b2(0.6);
    Camera c2(M_PI / 2, 0.0, 30.0, 0.0);
    printf("%.17g %.17g %.17g %.17g %.17g %.17g\n", c2.speed, c2.alpha, c2.w, c2.wbar,
           c2.Delta, c2.ro);
    try {
      Camera bad(M_PI / 2, 0.0, -1.0, 0.0);
      printf("no error\n");
    } catch (const Error& e) {
      printf("error %d\n", e.code);
    }
    return 0;
  }
  if (!std::strcmp(mode, "grid")) {
    Grid g(8, 5, true, &cam, &black);
    auto& cc = g.CamToCel();
    auto& bl = g.blockLevels();
    long maxlvl = 0;
    for (auto& e : bl) maxlvl = e.second > maxlvl ? e.second : maxlvl;
    double sum = 0;
    for (auto& e : cc) sum += e.second.x + e.second.y;
    printf("%d %d %zu %zu %ld %.10f %lld\n", g.N, g.M, cc.size(), bl.size(), maxlvl, sum,
           (long long)g.traced());
    return 0;
  }
  if (!std::strcmp(mode, "frame")) {
    std::vector<Grid> grids;
    grids.emplace_back(8, 5, true, &cam, &black);
    std::vector<Camera> cams{cam};
    Viewer view(M_PI / 2, 0, 0, 256, 128, true);
    std::vector<Star> stars;
    for (int k = 0; k < 2000; k++) {
      const float u = (k * 0.618034f) - std::floor(k * 0.618034f);
      const float v = (k * 0.381966f * 1.7f) - std::floor(k * 0.381966f * 1.7f);
      stars.push_back(Star{std::acos(1 - 2 * u), 2.f * (float)M_PI * v, 1.5f, 0.3f});
    }
    StarProcessor sp(stars, 6, 1000.f);
    std::vector<uint8_t> env(128 * 256 * 3);
    for (size_t q = 0; q < env.size(); q++) env[q] = (uint8_t)((q * 37) % 251);
    Distorter d(&grids, &view, &sp, &cams, env.data(), 128, 256);
    std::vector<uint8_t> img(256 * 128 * 4);
    d.render(img.data());
    long s = 0;
    for (auto b : img) s += b;
    printf("%ld %d\n", s, sp.starSize);
    return 0;
  }
  if (!std::strcmp(mode, "files") && argc > 2) {
    // cache files, the perspective view and blending between two grids
    const std::string dir = argv[2];
    std::vector<Grid> grids;
    grids.emplace_back(7, 4, true, &cam, &black);
    Camera cam2(M_PI / 2, 0.0, 6.0, 0.0, 0.0, 1.0);
    grids.emplace_back(7, 4, true, &cam2, &black);
    std::vector<Star> stars;
    for (int k = 0; k < 1500; k++) {
      const float u = (k * 0.618034f) - std::floor(k * 0.618034f);
      const float v = (k * 0.381966f * 1.3f) - std::floor(k * 0.381966f * 1.3f);
      stars.push_back(Star{std::acos(1 - 2 * u), 2.f * (float)M_PI * v, 2.0f, 0.5f});
    }
    StarProcessor sp(stars, 6, 1000.f);
    grids[0].save(dir + "/a.grid");
    sp.save(dir + "/s.star");
    std::vector<Grid> loaded;
    loaded.push_back(Grid::load(dir + "/a.grid"));
    StarProcessor sp2(dir + "/s.star");
    std::vector<uint8_t> env(128 * 256 * 3);
    for (size_t q = 0; q < env.size(); q++) env[q] = (uint8_t)((q * 53) % 241);
    Viewer persp(1.2, 0.1, 0.4, 160, 96, false);
    std::vector<Grid> one;
    one.push_back(std::move(grids[0]));
    grids.erase(grids.begin());
    std::vector<Camera> cams1{cam};
    std::vector<uint8_t> a(160 * 96 * 4), b(160 * 96 * 4);
    {
      Distorter d(&one, &persp, &sp, &cams1, env.data(), 128, 256);
      d.render(a.data());
    }
    {
      Distorter d(&loaded, &persp, &sp2, &cams1, env.data(), 128, 256);
      d.render(b.data());
    }
    const bool same = a == b;
    // two grids, blended half way
    std::vector<Grid> pair;
    pair.push_back(std::move(one[0]));
    pair.push_back(std::move(grids[0]));
    std::vector<Camera> cams2{cam, cam2};
    Viewer sphere(M_PI / 2, 0, 0, 160, 80, true);
    std::vector<uint8_t> c0(160 * 80 * 4), c5(160 * 80 * 4), c0b(160 * 80 * 4);
    Distorter d2(&pair, &sphere, &sp, &cams2, env.data(), 128, 256);
    d2.render(c0.data(), 0.f, 0.f, 0.f);
    d2.render(c5.data(), 0.f, 0.f, 0.5f);
    d2.render(c0b.data(), 0.f, 0.f, 0.f);
    printf("%d %d %d %d %d\n", same ? 1 : 0, loaded[0].MAXLEVEL, sp2.starSize,
           c0 == c0b ? 1 : 0, c0 != c5 ? 1 : 0);
    return 0;
  }
  if (!std::strcmp(mode, "rebuild")) {
    // One grid tuned, switched to graph replay and built again for a second
    // camera (twice: capture, then replay) must equal a new Grid of that camera.
    Grid g(8, 5, true, &cam, &black);
    const bt_tune_result t = g.tune(nullptr, 1e-6, 1);
    g.setGraph(true);
    Camera cam2(M_PI / 2, 0.3, 7.0, 0.0, 0.0, 1.0);
    g.rebuild(&cam2, &black);
    g.rebuild(&cam2, &black);
    Grid fresh(8, 5, true, &cam2, &black);
    const auto& a = g.CamToCel();
    const auto& b = fresh.CamToCel();
    bool same = a.size() == b.size();
    for (const auto& e : a) {
      auto it = b.find(e.first);
      if (it == b.end() || std::memcmp(&it->second, &e.second, sizeof(Point2d))) {
        same = false;
        break;
      }
    }
    same = same && g.steps() == fresh.steps() && g.blockLevels() == fresh.blockLevels();
    printf("%d %d %lld %lld\n", same ? 1 : 0, t.candidates, (long long)g.traced(),
           (long long)fresh.traced());
    return 0;
  }
  return 2;
}
