// sc_mesh.cuh -- triangle mesh -> signed distance grid on the GPU
// (manifold2SDF, FluidSim/src/cpu/util.cc:203-310), the collider set-up of
// FluidSimulator::setCollider (FluidSim/include/FluidSim/cpu/fluid-simulator.h:62-71).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace sc {

struct MeshSdfArgs {
  int nx, ny, nz;           // grid cells; cell (x, y, z) centre at ((x + 0.5) h + origin.x, ...)
  double h;
  double ox, oy, oz;
  const double* vertices;   // device, nvertices x 3
  int64_t nvertices;
  const int32_t* triangles; // device, ntriangles x 3 vertex indices
  int64_t ntriangles;
  int exact_band;           // cells around each triangle's box with exact distances (3 in setCollider)
  int exact_distance;       // 0: the reference's point-triangle arithmetic; 1: true distances
  int wait_limit;           // polls before a sweep barrier wait gives up (0: the default)
};

// Device scratch mesh_to_sdf needs (crossing counts, closest triangles when the
// caller passes none, status words, packed triangle vertices).
size_t mesh_to_sdf_scratch_bytes(const MeshSdfArgs& a, bool need_closest);

// Writes the signed distance (reference layout, z fastest) to `sdf` and, when
// `closest` is not null, the triangle each cell's distance was taken from (-1:
// none).  Uses `scratch` (at least mesh_to_sdf_scratch_bytes bytes, 256-byte
// aligned) when given, else allocates its scratch on the stream.  Returns 0,
// -1 with `msg` set for a triangle index outside [0, nvertices), -3 when an
// allocation fails, -6 when a sweep barrier wait timed out.  Synchronises the
// stream.
int mesh_to_sdf(cudaStream_t st, const MeshSdfArgs& a, double* sdf, int32_t* closest, void* scratch,
                size_t scratch_bytes, std::string* msg);

}  // namespace sc
