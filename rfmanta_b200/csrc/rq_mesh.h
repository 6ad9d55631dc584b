// The rq_mesh object behind the mesh-file readers' handle (host code).
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/rfmanta_b200.h"

// One entry of a mesh's material table (OBJ files; PLY meshes have none).
struct rq_mesh_material {
  int32_t kind = RQ_MAT_LAMBERTIAN;
  float diffuse[3] = {0.8f, 0.8f, 0.8f};
  float specular[3] = {0.f, 0.f, 0.f};
  float filter[3] = {1.f, 1.f, 1.f};
  int32_t exponent = 0;
  float reflectivity = 0.f;
  float refraction = 1.f;
  float alpha = 1.f;
};

struct rq_mesh {
  std::vector<float> vertices;     // 3 per vertex
  std::vector<uint32_t> indices;   // 3 per triangle
  std::vector<uint32_t> face_material;
  std::vector<rq_mesh_material> materials;
};

// Mesh::removeDegenerateTriangles (Model/Groups/Mesh.cc:315-359).
void rq_mesh_remove_degenerate(rq_mesh* m);
