// Wavefront OBJ ingestion: Mesh::LoadFromFile (mesh/Mesh.cpp:7-90) over the
// reference's vendored tinyobjloader (external/tinyobjloader, v2.0.0-rc),
// restated: the same number parsing, face-index rules and polygon
// triangulation, and the same per-triangle vertex records.
#pragma once
#include <stdint.h>
#include <string>
#include <vector>

namespace gyt {

// One record per triangle, as Mesh::untransformedTriangles holds them:
// positions p0 p1 p2 (9 floats), shading normals n0 n1 n2 (9 floats, from
// the file or the normalised face normal), texture coordinates (6 floats).
struct ObjMesh {
  std::vector<float> pos, nrm, uv;
  uint32_t triangles() const { return (uint32_t)(pos.size() / 9); }
};

// reverse_vertices: Mesh::LoadFromFile's flag (second and third vertex of
// every triangle swapped). Returns false with a message on malformed input
// (the reference exits on those, or reads out of bounds).
bool load_obj(const std::string& path, bool reverse_vertices, ObjMesh* out, std::string* err);

}  // namespace gyt
