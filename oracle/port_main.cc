// port_main.cc -- command-line driver of the restatement (port.cc), with the
// same modes and output files as ref_harness.cc so one parser serves both.
// TEST INFRASTRUCTURE (the oracle).
//
//   snog_port octree SPEC OUT
//   snog_port trace SPEC RAYS OUT [threads]

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "port.h"
#include "scene_spec.h"

using namespace snogport;

static int mode_octree(const std::string &spec_path, const std::string &out) {
  snogspec::Scene spec = snogspec::load(spec_path);
  Scene s = build(spec);
  FILE *f = fopen(out.c_str(), "wb");
  if (!f) return 1;
  float hdr[4] = {s.oct.origin.x, s.oct.origin.y, s.oct.origin.z, s.oct.size};
  uint32_t n_nodes = uint32_t(s.oct.heads.size()), n_list = uint32_t(s.oct.list.size());
  fwrite(hdr, 4, 4, f);
  fwrite(&n_nodes, 4, 1, f);
  fwrite(&n_list, 4, 1, f);
  for (uint32_t i = 0; i < n_nodes; i++) {
    fwrite(&s.oct.children[8 * size_t(i)], 4, 8, f);
    fwrite(&s.oct.heads[i], 4, 1, f);
  }
  fwrite(s.oct.list.data(), 4, n_list, f);
  fclose(f);
  printf("{\"nodes\": %u, \"list\": %u}\n", n_nodes, n_list);
  return 0;
}

static int mode_trace(const std::string &spec_path, const std::string &rays_path, const std::string &out,
                      unsigned threads) {
  snogspec::Scene spec = snogspec::load(spec_path);
  Scene s = build(spec);
  snogspec::RayBatch rb = snogspec::load_rays(rays_path);
  const uint32_t n = rb.n;
  std::vector<int32_t> prim(n, -1);
  std::vector<float> tout(n, 0.f), nrm(size_t(n) * 3, 0.f);
  std::vector<unsigned long long> nodes(2 * threads, 0), tests(2 * threads, 0), hits(2 * threads, 0);
  std::atomic<uint32_t> next(0);
  auto t0 = std::chrono::steady_clock::now();
  auto work = [&](unsigned tid) {
    for (;;) {
      uint32_t b = next.fetch_add(4096);
      if (b >= n) break;
      for (uint32_t i = b; i < std::min(n, b + 4096); i++) {
        const bool any = i >= rb.n_closest;
        Hit h = trace(s, V{rb.ox()[i], rb.oy()[i], rb.oz()[i]}, V{rb.dx()[i], rb.dy()[i], rb.dz()[i]},
                      rb.tmax()[i], any);
        prim[i] = h.prim;
        if (!any && h.prim >= 0) tout[i] = h.t;
        nodes[2 * tid + any] += h.nodes;
        tests[2 * tid + any] += h.tests;
        hits[2 * tid + any] += h.prim >= 0;
      }
    }
  };
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; t++) pool.emplace_back(work, t);
  for (auto &th : pool) th.join();
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  FILE *f = fopen(out.c_str(), "wb");
  if (!f) return 1;
  fwrite(prim.data(), 4, n, f);
  fwrite(tout.data(), 4, n, f);
  fwrite(nrm.data(), 4, size_t(n) * 3, f);
  for (int k = 0; k < 2; k++) {
    unsigned long long v[5] = {0, 0, 0, 0, 0};
    for (unsigned t = 0; t < threads; t++) {
      v[0] += tests[2 * t + k];
      v[1] += hits[2 * t + k];
      v[4] += nodes[2 * t + k];
    }
    fwrite(v, 8, 5, f);
  }
  fclose(f);
  printf("{\"rays\": %u, \"seconds\": %.6f, \"threads\": %u, \"mrays_per_s\": %.4f}\n", n, secs, threads,
         n / secs * 1e-6);
  return 0;
}

int main(int argc, char **argv) {
  try {
    if (argc >= 4 && std::string(argv[1]) == "octree") return mode_octree(argv[2], argv[3]);
    if (argc >= 5 && std::string(argv[1]) == "trace")
      return mode_trace(argv[2], argv[3], argv[4], argc > 5 ? unsigned(atoi(argv[5])) : 1u);
    fprintf(stderr, "usage: snog_port octree SPEC OUT | trace SPEC RAYS OUT [threads]\n");
    return 2;
  } catch (std::exception &e) {
    fprintf(stderr, "snog_port: %s\n", e.what());
    return 1;
  }
}
