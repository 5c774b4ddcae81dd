// Trilinear coarse-lattice shape functions shared by the coarse-space kernels
// (assembly, restriction, prolongation) and the fused CG step.
#pragma once
#include <cuda_runtime.h>

#include "fem_internal.h"

namespace femb200 {

__device__ __forceinline__ float tri_weight(float tx, float ty, float tz, int corner) {
  const float wx = (corner & 4) ? tx : 1.f - tx;
  const float wy = (corner & 2) ? ty : 1.f - ty;
  const float wz = (corner & 1) ? tz : 1.f - tz;
  return wx * wy * wz;
}

// Local coordinate of a point along one lattice axis, clamped to [0, 1] and
// snapped to the cell face within 1e-4: a mesh node on a face gets exactly 0
// or 1, so a coarse node whose support holds only such nodes assembles an
// exactly-zero row (decoupled) instead of a rounding-sized one.
__device__ __forceinline__ float lattice_coord(float x, float lo, float inv_H, int i) {
  float t = fminf(fmaxf((x - lo) * inv_H - (float)i, 0.f), 1.f);
  if (t < 1e-4f) t = 0.f;
  if (t > 1.f - 1e-4f) t = 1.f;
  return t;
}

// local coordinates of a point in lattice cell ijk
__device__ __forceinline__ void cell_local(const CoarseDev& c, int3 ijk, float x, float y, float z,
                                           float t[3]) {
  t[0] = lattice_coord(x, c.lo.x, c.inv_H, ijk.x);
  t[1] = lattice_coord(y, c.lo.y, c.inv_H, ijk.y);
  t[2] = lattice_coord(z, c.lo.z, c.inv_H, ijk.z);
}

// The lattice cell of mesh node i and its local coordinates there, from the
// per-node table built with the lattice (the same values cell_local gives).
__device__ __forceinline__ int node_lattice(const CoarseDev& c, int i, float t[3]) {
  const float4 v = __ldg(c.node_lat + i);
  t[0] = v.x;
  t[1] = v.y;
  t[2] = v.z;
  return __float_as_int(v.w);
}

}  // namespace femb200
