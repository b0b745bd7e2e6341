// sc_surface.cuh -- marching-cubes surface export on the GPU: rebuildSurface
// (FluidSim/src/cpu/rebuild-surface.cc:686-741), the mesh the simulator's fluid
// SDF is turned into for export (FluidSim/disabled/fluid-sim.cc:230-238).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace sc {

struct SurfaceArgs {
  int nx, ny, nz;      // SDF samples; sample (x, y, z) sits at ((x + 0.5) hx + ox, ...)
  double hx, hy, hz;   // spacing per axis
  double ox, oy, oz;   // origin
  const double* sdf;   // device, reference layout (z fastest)
};

// Device scratch the two calls below share (per-cube case masks and first
// vertex numbers, per-block counts, the totals and a status word).
size_t surface_scratch_bytes(const SurfaceArgs& a);

// Counts the mesh: vertices and index entries (3 per triangle).  Synchronises
// the stream.  Returns 0, or -2 on a CUDA error.
int surface_count(cudaStream_t st, const SurfaceArgs& a, void* scratch, int64_t* nvertices,
                  int64_t* nindices);

// Writes the mesh counted by the surface_count call just made on the same
// scratch and arguments: vertices and normals (3 doubles each) numbered as the
// reference numbers them, and the index entries (uint32) in its order.
// Synchronises the stream.  Returns 0, -2 on a CUDA error, -1 with `msg` set if
// an index entry found no vertex (a broken case table).
int surface_fill(cudaStream_t st, const SurfaceArgs& a, void* scratch, double* vertices, double* normals,
                 uint32_t* indices, std::string* msg);

}  // namespace sc
