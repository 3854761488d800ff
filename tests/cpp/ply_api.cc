// A PLY mesh loaded and rendered through the reference-shaped C++ API
// (include/snogray_b200.hpp), as a snogray program does with load_ply_file:
// the mesh (one Cook-Torrance part, vertex normals from the file) under a
// 0.5 x 0.5 area light.
//
//   ply_api host FILE                      host-only build, print scene info
//   ply_api render FILE W H SPP OUT.f32 [SEED]
// Prints one JSON line: scene info, or paths and the camera as the C ABI
// receives it.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>

#include "snogray_b200.hpp"

using namespace snogray_b200;

static SurfaceGroup scene(const std::string &file) {
  auto ct = std::make_shared<CookTorrance>(Color(0.7f, 0.3f, 0.2f), Color(1.f), 0.2f, Ior(1.5f));
  auto light = std::make_shared<Glow>(Color(10.f));
  auto mesh = std::make_shared<Mesh>();
  load_ply_file(file, *mesh, mesh->add_part(ct));
  SurfaceGroup g;
  g.add(mesh);
  // normal = e2 x e1 points down
  g.add(std::make_shared<Tripar>(light, Pos(0.25f, 1.2f, 0.25f), Vec(0, 0, 0.5f), Vec(0.5f, 0, 0), true));
  return g;
}

int main(int argc, char **argv) {
  try {
    if (argc < 3) throw std::runtime_error("usage: ply_api host FILE | render FILE W H SPP OUT.f32 [SEED]");
    const std::string mode = argv[1];
    RenderParams params;
    params.min_path_len = 3;
    params.max_path_len = 8;
    params.direct_samples = 1;
    if (mode == "host") {
      GlobalRenderState state(scene(argv[2]), params, false);
      const SnogSceneInfo i = state.info();
      std::printf("{\"n_nodes\": %u, \"n_plist\": %u, \"max_depth\": %u, \"n_triangles\": %u}\n", i.n_nodes,
                  i.n_plist, i.max_depth, i.n_triangles);
      return 0;
    }
    if (mode != "render" || argc < 7) throw std::runtime_error("bad arguments");
    const unsigned w = unsigned(std::atoi(argv[3])), h = unsigned(std::atoi(argv[4]));
    params.samples = unsigned(std::atoi(argv[5]));
    params.seed = argc > 7 ? std::strtoull(argv[7], nullptr, 10) : 0;
    check(snog_init(0), "snog_init");
    GlobalRenderState state(scene(argv[2]), params);
    Camera cam;
    cam.move(Pos(0.5f, 0.55f, -1.3f));
    cam.point(Pos(0.5f, 0.3f, 0.5f), Vec(0, 1, 0));
    cam.set_vert_fov(45.f * 3.14159265358979f / 180.f, float(w) / float(h));
    ImageSampledOutput out(w, h);
    RenderStats stats;
    RenderMgr(state, cam, w, h).render(out, stats);
    FILE *f = std::fopen(argv[6], "wb");
    if (!f) throw std::runtime_error("cannot write output");
    std::fwrite(out.rgb.data(), sizeof(float), out.rgb.size(), f);
    std::fclose(f);
    const SnogCamera c = cam.c_struct();
    std::printf("{\"paths\": %llu, \"camera\": [", (unsigned long long)stats.paths);
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
