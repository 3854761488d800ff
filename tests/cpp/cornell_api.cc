// The Cornell-style box built and rendered through the reference-shaped C++
// API (include/snogray_b200.hpp), the way a snogray program builds it with
// SurfaceGroup / Mesh / Sphere / Tripar / materials / Camera / RenderMgr.
//
//   cornell_api host            build on the host only, print scene info
//   cornell_api render W H SPP OUT.f32 [SEED]
//                               render; raw RGB floats to OUT.f32
//   cornell_api limit W H SPP LX LY LW LH OUT.f32 [SEED]
//                               a --limit render of the LW x LH pixels at
//                               (LX, LY) of the W x H film, set up as the
//                               reference's driver does (snogray.lua:442-454,
//                               543-560): an output of the limit's size with
//                               its sample base, a pattern of the limit plus
//                               the filter margin, the 5-argument
//                               RenderMgr::render
// Prints one JSON line: scene info, or the render's statistics and the camera
// as the C ABI receives it.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "snogray_b200.hpp"

using namespace snogray_b200;

// Records what the render reports (util/progress.h's interface).
struct NullProgress : Progress {
  unsigned size = 0;
  bool ended = false;
  void set_size(unsigned n) override { size = n; }
  void end() override { ended = true; }
};

static SurfaceGroup cornell() {
  auto white = std::make_shared<Lambert>(Color(0.73f, 0.73f, 0.73f));
  auto red = std::make_shared<Lambert>(Color(0.65f, 0.05f, 0.05f));
  auto green = std::make_shared<Lambert>(Color(0.12f, 0.45f, 0.15f));
  auto glass = std::make_shared<Glass>(Medium(1.5f));
  auto light = std::make_shared<Glow>(Color(15.f));

  auto room = std::make_shared<Mesh>();
  const float v[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}, {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}};
  for (auto &p : v) room->add_vertex(Pos(p[0], p[1], p[2]));
  const Mesh::part_index_t pw = room->add_part(white), pr = room->add_part(red), pg = room->add_part(green);
  room->add_triangles(pw, {0, 1, 2, 0, 2, 3, 4, 6, 5, 4, 7, 6, 3, 2, 6, 3, 6, 7});   // floor, ceiling, back
  room->add_triangles(pr, {0, 3, 7, 0, 7, 4});                                      // left wall x=0
  room->add_triangles(pg, {1, 5, 6, 1, 6, 2});                                      // right wall x=1

  SurfaceGroup g;
  g.add(room);
  g.add(std::make_shared<Sphere>(white, Pos(0.3f, 0.3f, 0.65f), 0.3f));
  g.add(std::make_shared<Sphere>(glass, Pos(0.7f, 0.6f, 0.3f), 0.3f));
  // normal = e2 x e1 points down, into the room
  g.add(std::make_shared<Tripar>(light, Pos(0.375f, 0.999f, 0.375f), Vec(0, 0, 0.25f), Vec(0.25f, 0, 0), true));
  return g;
}

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: cornell_api host | render W H SPP OUT.f32 [SEED] | "
                         "limit W H SPP LX LY LW LH OUT.f32 [SEED]\n");
    return 2;
  }
  try {
    const std::string mode = argv[1];
    RenderParams params;
    params.min_path_len = 3;
    params.max_path_len = 8;
    params.direct_samples = 1;
    if (mode == "host") {
      GlobalRenderState state(cornell(), params, false);
      const SnogSceneInfo i = state.info();
      std::printf("{\"n_nodes\": %u, \"n_plist\": %u, \"max_depth\": %u, \"n_triangles\": %u, "
                  "\"n_spheres\": %u, \"n_tripars\": %u, \"n_lights\": %u}\n",
                  i.n_nodes, i.n_plist, i.max_depth, i.n_triangles, i.n_spheres, i.n_tripars, i.n_lights);
      return 0;
    }
    const bool limit = mode == "limit";
    if (!((mode == "render" && argc >= 6) || (limit && argc >= 10))) throw std::runtime_error("bad arguments");
    const unsigned w = unsigned(std::atoi(argv[2])), h = unsigned(std::atoi(argv[3]));
    params.samples = unsigned(std::atoi(argv[4]));
    const int seed_arg = limit ? 10 : 6;
    params.seed = argc > seed_arg ? std::strtoull(argv[seed_arg], nullptr, 10) : 0;
    const char *out_path = argv[limit ? 9 : 5];
    check(snog_init(0), "snog_init");
    GlobalRenderState state(cornell(), params);
    Camera cam;
    cam.move(Pos(0.5f, 0.5f, -1.2f));
    cam.point(Pos(0.5f, 0.5f, 0.5f), Vec(0, 1, 0));
    cam.set_vert_fov(40.f * 3.14159265358979f / 180.f, float(w) / float(h));
    RenderStats stats;
    std::vector<float> rgb;
    if (limit) {
      const int lx = std::atoi(argv[5]), ly = std::atoi(argv[6]), lw = std::atoi(argv[7]), lh = std::atoi(argv[8]);
      ImageSampledOutput out(unsigned(lw), unsigned(lh), lx, ly);
      const int xm = out.filter_x_radius(), ym = out.filter_y_radius();
      RenderPattern pattern(lx - xm, ly - ym, lw + 2 * xm, lh + 2 * ym);
      NullProgress prog;
      RenderMgr(state, cam, w, h).render(8, pattern, out, prog, stats);
      if (prog.size != unsigned((lw + 2 * xm) * (lh + 2 * ym)) || !prog.ended)
        throw std::runtime_error("progress not reported");
      rgb = out.rgb;
    } else {
      ImageSampledOutput out(w, h);
      RenderMgr(state, cam, w, h).render(out, stats);
      rgb = out.rgb;
    }
    FILE *f = std::fopen(out_path, "wb");
    if (!f) throw std::runtime_error("cannot write output");
    std::fwrite(rgb.data(), sizeof(float), rgb.size(), f);
    std::fclose(f);
    const SnogCamera c = cam.c_struct();
    std::printf("{\"paths\": %llu, \"closest_rays\": %llu, \"scene_intersect_calls\": %llu, "
                "\"scene_shadow_tests\": %llu, \"illum_calls\": %llu, \"intersect_nodes\": %llu, "
                "\"intersect_tests\": %llu, \"shadow_nodes\": %llu, \"shadow_tests\": %llu, \"camera\": [",
                (unsigned long long)stats.paths, (unsigned long long)stats.closest_rays,
                stats.scene_intersect_calls, stats.scene_shadow_tests, stats.illum_calls,
                stats.intersect.space_node_intersect_calls, stats.intersect.surface_intersects_tests,
                stats.shadow.space_node_intersect_calls, stats.shadow.surface_intersects_tests);
    const float *vals[4] = {c.pos, c.forward, c.right, c.up};
    for (int k = 0; k < 4; k++)
      for (int a = 0; a < 3; a++) std::printf("%.9g, ", double(vals[k][a]));
    std::printf("%.9g, %.9g]}\n", double(c.tan_half_fov_x), double(c.tan_half_fov_y));
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
