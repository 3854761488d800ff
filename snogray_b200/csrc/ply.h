// ply.h -- PLY mesh reader (ply.cc).

#ifndef SNOG_PLY_H
#define SNOG_PLY_H

#include <cstdint>
#include <string>
#include <vector>

namespace snog {

struct PlyMeshHost {
  std::vector<float> vertices;    // 3 per vertex
  std::vector<float> normals;     // 3 per vertex, or empty
  std::vector<uint32_t> triangles;
};

// Throws std::runtime_error with the reason on any error.
PlyMeshHost read_ply(const std::string &path);

}  // namespace snog

#endif
