// wf_scene.h -- the scene format parsed into raster operations, shared by the
// host voxelizer (wf_host.cpp) and the device voxelizer (wf_scene.cu).
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

namespace wf {

// One primitive of a scene in file order (Scene::voxelize, src/scene.rs:
// 149-230): a sphere filled where the cell centre satisfies
// (x+0.5-cx)^2 + (y+0.5-cy)^2 + (z+0.5-cz)^2 <= r2 in f32, evaluated left to
// right, or a box filling [x0,x1) x [y0,y1) x [z0,z1).  For a sphere the
// integer bounds are a conservative box around it (the test decides).
struct RasterOp {
  int sphere;
  float cx, cy, cz, r2;
  long long x0, x1, y0, y1, z0, z1;
  uint8_t id;
};

// Scene::parse + the material registration of Scene::voxelize: ops in file
// order with material ids (de-duplicated by the bit pattern of eps_r, mu_r,
// sigma; at most 255), and table[id] = the Q16.16 coefficients of each
// registered material.  Returns false with the reference's message in err.
bool scene_parse(const char *text, int nx, int ny, int nz, float dt, float dx,
                 std::vector<RasterOp> *ops, int32_t (*table)[4], int *n_materials,
                 std::string *err);

// Device voxelizer: ids (pitch bytes per row, nz*ny rows) set to `fill`, then
// every op applied in order on `stream`.  The ids hold the planes
// [z_lo, z_lo + nz) of the scene's grid (ops carry that grid's coordinates).
int launch_voxelize(const std::vector<RasterOp> &ops, uint8_t *ids, int nx, int ny, int nz,
                    int pitch, uint8_t fill, void *stream, int z_lo = 0);

}  // namespace wf
